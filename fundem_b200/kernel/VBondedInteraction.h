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

private:
    fundem_sim* sim_ = nullptr;
    std::vector<int> activated_;
    std::vector<double3> point_;
    std::vector<double> energy_;
};
