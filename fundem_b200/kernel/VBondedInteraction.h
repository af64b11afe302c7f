// VBondedInteraction view of the bonds of a simulation in libfundem_b200,
// with host getters for the state the reference keeps per bond
// (kernel/VBondedInteraction.h:448-494).
#pragma once
#include <vector>

#include "LSParticle.h"

class VBondedInteraction {
public:
    void bind(fundem_sim* sim) { sim_ = sim; }

    size_t numPair_device() const
    {
        if (!sim_) return 0;
        int n = 0;
        fundem_detail::check(fundem_num_bonds(sim_, &n), "num_bonds");
        return (size_t)n;
    }

    void download()
    {
        const size_t n = numPair_device();
        activated_.resize(n); point_.resize(n); energy_.resize(6 * n);
        if (n == 0) return;
        fundem_detail::check(fundem_get_bonds(sim_, activated_.data(), &point_[0].x, energy_.data()), "get_bonds");
    }
    const std::vector<int> activatedHostRef() { download(); return activated_; }
    const std::vector<double3> centerPointHostRef() { download(); return point_; }
    // per bond: Un, Us, Ub, Ut, maximum normal stress, maximum shear stress
    const std::vector<double> energyAndStressHostRef() { download(); return energy_; }

    // device pointers (kernel/VBondedInteraction.h:452-480 of the reference):
    // ids, activation, centre point, radius and initial length are the
    // library's own arrays; the other fields are per-field copies, a
    // snapshot refreshed by each call, valid until the next step
    int* masterObjectID() { return view().master; }
    int* slaveObjectID() { return view().slave; }
    int* activated() { return view().activated; }
    double3* centerPoint() { return reinterpret_cast<double3*>(view().center_point); }
    double* radius() { return view().radius; }
    double* initialLength() { return view().initial_length; }
    double* B1() { return view().B1; }
    double* B2() { return view().B2; }
    double* B3() { return view().B3; }
    double* B4() { return view().B4; }
    double* Un() { return view().Un; }
    double* Us() { return view().Us; }
    double* Ub() { return view().Ub; }
    double* Ut() { return view().Ut; }
    double* maxNormalStress() { return view().max_normal_stress; }
    double* maxShearStress() { return view().max_shear_stress; }
    double* tensileStrength() { return view().tensile_strength; }
    double* cohesion() { return view().cohesion; }
    double* frictionCoefficient() { return view().friction; }
    double3* masterVBondPointLocalVectorN1() { return frame(0); }
    double3* masterVBondPointLocalVectorN2() { return frame(1); }
    double3* masterVBondPointLocalVectorN3() { return frame(2); }
    double3* masterVBondPointLocalPosition() { return frame(3); }
    double3* slaveVBondPointLocalVectorN1() { return frame(4); }
    double3* slaveVBondPointLocalVectorN2() { return frame(5); }
    double3* slaveVBondPointLocalVectorN3() { return frame(6); }
    double3* slaveVBondPointLocalPosition() { return frame(7); }

private:
    fundem_bond_view view()
    {
        fundem_bond_view v{};
        if (sim_) fundem_detail::check(fundem_bond_view_get(sim_, &v), "bond_view_get");
        return v;
    }
    double3* frame(int k) { return reinterpret_cast<double3*>(view().frames[k]); }

    fundem_sim* sim_ = nullptr;
    std::vector<int> activated_;
    std::vector<double3> point_;
    std::vector<double> energy_;
};
