// fd_adjoint.cuh -- launch interface of the reverse sweep (fd_adjoint.cu).
#pragma once
#include "fd_kernels.cuh"

namespace fd {

// particle adjoints of one reverse step (device arrays, 3 per particle)
struct AdjParticles {
    int n;
    const int* geo;
    const int* mat;
    const double3* angvel;  // constant over the run: the bodies do not turn
    GeoSetDev G;
    double* xb;     // adjoint of the positions
    double* vb;     // adjoint of the velocities at the step's end
    double* vhb;    // adjoint of the velocities at force time
    double* Fb;     // adjoint of the step's forces
    double* Feb;    // adjoint of the forces reaching the next step's first half-kick
    double* pgrad;  // 4 per particle material: kn, ks, damping ratio, mu
};

struct AdjContactArgs {
    AdjRec rec;            // the list at this step
    const int* nslots;     // slots of the list at this step
    MatDev M;              // particle materials
    MatDev MW;             // wall materials
    GeoSetDev GW;          // wall geometries
    const double3* wall_angvel;  // prescribed wall angular velocities
    const double* Sb_cur;  // spring adjoints of this step's slots
    double* Sb_prev;       // spring adjoints of the previous step's slots (accumulated)
    int sb_prev_cap;
    double dt;
};

struct AdjBondArgs {
    int n;
    const int* master;
    const int* slave;
    const int* active;     // recorded at the step
    const double* rij;     // recorded at the step
    const double* B;       // 4 per bond
    const double* L0;
    const double* dn;      // 3 per bond: n1j - n1i in the world frame, recorded at the step
};

void adj_force(const AdjParticles& a, double dt, cudaStream_t s);
void adj_contacts(const AdjParticles& a, const AdjContactArgs& c, cudaStream_t s);
void adj_bonds(const AdjParticles& a, const AdjBondArgs& b, cudaStream_t s);
void adj_particles(const AdjParticles& a, double dt, cudaStream_t s);

}  // namespace fd
