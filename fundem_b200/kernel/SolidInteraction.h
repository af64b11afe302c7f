// SolidInteraction view of one contact list (particle-particle or
// particle-wall) of a simulation in libfundem_b200, with the host getters of
// the reference (kernel/SolidInteraction.h:346-372).  Contacts come in
// canonical (node, partner) order; the reference's order follows its cell
// loop, and the set is the same.
#pragma once
#include <vector>

#include "LSParticle.h"

class SolidInteraction {
public:
    explicit SolidInteraction(int kind) : kind_(kind) {}
    void bind(fundem_sim* sim) { sim_ = sim; }

    size_t numPair_device() const
    {
        if (!sim_) return 0;
        long long n = 0;
        fundem_detail::check(fundem_num_contacts(sim_, kind_, &n), "num_contacts");
        return (size_t)n;
    }

    // host copies of the current list: master = global boundary-node index,
    // slave = partner object
    void download()
    {
        const size_t n = numPair_device();
        master_.resize(n); slave_.resize(n); point_.resize(n); normal_.resize(n); overlap_.resize(n);
        spring_.resize(n); en_.resize(n); es_.resize(n);
        if (n == 0) return;
        fundem_detail::check(fundem_get_contacts(sim_, kind_, master_.data(), slave_.data(), &point_[0].x,
                                                 &normal_[0].x, overlap_.data(), &spring_[0].x, en_.data(),
                                                 es_.data()), "get_contacts");
    }
    const std::vector<int> masterIDHostRef() { download(); return master_; }
    const std::vector<int> slaveIDHostRef() { download(); return slave_; }
    const std::vector<double3> contactPointHostRef() { download(); return point_; }
    const std::vector<double3> contactNormalHostRef() { download(); return normal_; }
    const std::vector<double> contactOverlapHostRef() { download(); return overlap_; }
    const std::vector<double3> slidingSpringHostRef() { download(); return spring_; }

    // device pointers (kernel/SolidInteraction.h:323-330 of the reference):
    // contiguous copies of the list's contacts in (node, partner) order, a
    // read-only snapshot refreshed by each call, valid until the next step
    double3* contactPoint() { return reinterpret_cast<double3*>(view().point); }
    double3* contactNormal() { return reinterpret_cast<double3*>(view().normal); }
    double* contactOverlap() { return view().overlap; }
    double* normalElasticEnergy() { return view().normal_energy; }
    double* slidingElasticEnergy() { return view().sliding_energy; }
    double3* slidingSpring() { return reinterpret_cast<double3*>(view().spring); }
    int* masterID() { return view().master; }
    int* slaveID() { return view().slave; }

private:
    fundem_contact_view view()
    {
        fundem_contact_view v{};
        if (sim_) fundem_detail::check(fundem_contact_view_get(sim_, kind_, &v), "contact_view_get");
        return v;
    }

    fundem_sim* sim_ = nullptr;
    int kind_;
    std::vector<int> master_, slave_;
    std::vector<double3> point_, normal_, spring_;
    std::vector<double> overlap_, en_, es_;
};
