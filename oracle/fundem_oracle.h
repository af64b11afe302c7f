/*
 * fundem_oracle.h -- CPU restatement of FunDEM's level-set DEM timestep.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * fundem_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it.  The product never links or calls it.
 *
 * It restates, in plain C with OpenMP, the reference algorithm step by step:
 *   - LSSolver::compute* loops                      kernel/LSSolver.h:1091-1229
 *   - hashing / stable sort / cell start-end        myUtility/mySpatialGrid.cu:4-26,
 *                                                   myUtility/buildHashStartEnd.cu:18-137
 *   - node-vs-SDF count/write detection             LSParticleContactDetectionKernel.cu:4-607
 *   - linear spring-dashpot contact + friction      contactKernel.cuh:4-77, contactKernel.cu:46-291
 *   - V-model bonds                                 contactKernel.cuh:138-199, contactKernel.cu:293-371
 *   - half-kick / drift integration                 particleIntegrationKernel.cu:3-48
 *   - periodic X/Y ghosts                           PeriodicBoundary.h:7-317, mySpatialGrid.cu:28-152,214-240
 *   - host setup (materials, geometry, mass
 *     properties, bond stiffness and frames)        LSParticle.h:221-342, LSSolver.h:470-586,
 *                                                   VBondedInteraction.h:10-195, myMat.h:163-194
 *
 * Parity is pinned against dumps of the reference's own CUDA build run on a
 * B200 (oracle/ref_driver.cu, fixtures under tests/golden/).
 */
#ifndef FUNDEM_ORACLE_H
#define FUNDEM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_world orc_world;

/* contact list kinds */
enum { ORC_PP = 0, ORC_PW = 1, ORC_GX = 2, ORC_GY = 3, ORC_GXY = 4, ORC_GR90 = 5, ORC_GR180 = 6, ORC_GR270 = 7 };

orc_world* orc_create(void);
void orc_destroy(orc_world* w);
void orc_set_threads(int n);
/* 1: emulate nvcc's default mul+add contraction in the contact-membership
   arithmetic (default); 0: plain IEEE mul and add. */
void orc_set_fma_mode(int mode);
int orc_get_fma_mode(void);
/* choose, per contracted difference of products, which product is fused */
void orc_set_fma_pattern(int pattern);

int orc_add_material(orc_world* w, int wall, double kn, double ks, double mu, double e);
int orc_add_geometry(orc_world* w, int wall, double mass, const double inertia[6],
                     const double origin[3], double spacing, const int size[3],
                     const double* sdf, int n_nodes, const double* nodes);
int orc_mass_properties(double density, const double origin[3], double spacing,
                        const int size[3], const double* sdf,
                        double* mass, double centroid[3], double inertia[6]);
void orc_inverse_sym(const double in[6], double out[6]);
int orc_add_object(orc_world* w, int wall, const double pos[3], const double vel[3],
                   const double angvel[3], const double q[4], int mat, int geo);
int orc_add_bond(orc_world* w, int master, int slave, const double point[3],
                 const double normal[3], double radius, double L0, double E, double nu,
                 double tensile, double cohesion, double mu);
void orc_set_periodic(orc_world* w, int x, int y);
/* addPeriodicBoundarySector / removePeriodicBoundary, LSSolver.h:410-424 */
void orc_set_sector(orc_world* w, int on);
void orc_set_inertia_mode(orc_world* w, int physical);
/* damping square roots: 0 single precision as the reference, 1 double (test use) */
void orc_set_damping_sqrt64(int on);
int orc_setup(orc_world* w, const double minb[3], const double maxb[3]);

/* pre-loop detection (LSSolver.h:1093-1096 and the periodic variants) */
int orc_initial_detect(orc_world* w);
/* one in-loop step without output */
int orc_step(orc_world* w, const double g[3], double dt);
/* pieces of a step */
int orc_half_kick(orc_world* w, const double g[3], double dt);            /* K12 with h = dt/2 */
int orc_front(orc_world* w, const double g[3], double dt);                /* kick, drift particles, drift walls */
int orc_detect_and_force(orc_world* w, double dt);                        /* hash .. bonded forces */

int orc_num_objects(orc_world* w, int wall);
void orc_get_state(orc_world* w, int wall, double* pos, double* vel, double* angvel,
                   double* q, double* force, double* torque);
void orc_set_state(orc_world* w, int wall, const double* pos, const double* vel,
                   const double* angvel, const double* q, const double* force,
                   const double* torque);
long long orc_num_nodes(orc_world* w);
void orc_get_geometry(orc_world* w, int wall, int geo, double* radius, double* inv_mass,
                      double inertia[6], double inv_inertia[6]);
void orc_get_grid(orc_world* w, int wall, double minb[3], double maxb[3], double inv_cell[3],
                  int size[3]);

long long orc_num_contacts(orc_world* w, int kind);
void orc_get_contacts(orc_world* w, int kind, int* master, int* slave, double* point,
                      double* normal, double* overlap, double* spring, double* en, double* es);
/* Replace a contact list (history for the next detection).  Entries must be
   grouped by master node in ascending node order. */
int orc_set_contacts(orc_world* w, int kind, long long n, const int* master,
                     const int* slave, const double* spring);

int orc_num_bonds(orc_world* w);
void orc_get_bonds(orc_world* w, int* activated, double* point, double* un, double* us,
                   double* ub, double* ut, double* sn, double* ss);
void orc_set_bond_activation(orc_world* w, const int* activated);
void orc_get_bond_params(orc_world* w, double* b1234, double* local_frames);

#ifdef __cplusplus
}
#endif
#endif
