// fd_adjoint.cuh -- launch interface of the reverse sweep (fd_adjoint.cu).
#pragma once
#include "fd_kernels.cuh"

namespace fd {

// particle adjoints of one reverse step (device arrays, 3 per particle)
struct AdjParticles {
    int n;
    const int* geo;
    const int* mat;
    const double3* angvel;  // without turning bodies: constant over the run
    GeoSetDev G;
    double* xb;     // adjoint of the positions
    double* vb;     // adjoint of the velocities at the step's end
    double* vhb;    // adjoint of the velocities at force time
    double* Fb;     // adjoint of the step's forces
    double* Feb;    // adjoint of the forces reaching the next step's first half-kick
    double* pgrad;  // 4 per particle material: kn, ks, damping ratio, mu
    // turning bodies (rot = 1: some particle geometry has a nonzero inverse
    // inertia).  Per particle and step the record holds 10 doubles:
    // orientation (4), angular velocity (3), torque (3); pr_prev at the step's
    // start (the previous step's end), pr_cur after the step's drift
    // (orientation), first half-kick (angular velocity at force time) and
    // forces (torque)
    int rot;
    const double* pr_prev;
    const double* pr_cur;
    double* qb;     // 4 per particle: adjoint of the orientation
    double* wb;     // adjoint of the angular velocity at the step's end
    double* whb;    // adjoint of the angular velocity at force time
    double* Tb;     // adjoint of the step's torques
    double* Teb;    // adjoint of the torques reaching the next step's first half-kick
};
// doubles per particle and step in the record: orientation after the drift
// (4), angular velocity at force time (3), torque (3), angular velocity at the
// step's end, after the second half kick (3)
constexpr int ADJ_PREC = 13;

struct AdjContactArgs {
    AdjRec rec;            // the list at this step
    double3 period;        // domain lengths in x and y (periodic wrap codes)
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
// the record of turning bodies: orientation and angular velocity (after a
// drift), torque and angular velocity at the end of the step (after the
// second half kick), or all (a segment's start)
void adj_record_rot(const ObjDev& P, double* dst, int what, cudaStream_t s);
enum { ADJ_REC_QW = 1, ADJ_REC_T = 2 };

}  // namespace fd
