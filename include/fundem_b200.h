/*
 * fundem_b200.h -- C ABI of the B200 level-set DEM timestep (libfundem_b200.so).
 *
 * Plain C: opaque handle, caller-owned host arrays (or device pointers where
 * stated), status codes, no exceptions across the boundary.  All device work
 * is stream-ordered on the simulation's stream.  Arrays of 3-vectors are
 * packed xyz doubles; quaternions are scalar-first (q0, q1, q2, q3).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the reference project).  The reference's own boundary is a set of
 * extern "C" kernel launchers driven by header-only C++ classes; here the
 * launch sequence of one step is owned by the library, and the
 * header-compatible C++ classes (the headers in fundem_b200/kernel/) sit on top of these
 * functions.
 */
#ifndef FUNDEM_B200_H
#define FUNDEM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fundem_sim fundem_sim;

typedef enum {
    FUNDEM_OK = 0,
    FUNDEM_ERR_ARG = 1,       /* invalid argument (the reference prints to stderr and skips) */
    FUNDEM_ERR_CUDA = 2,      /* a CUDA call failed */
    FUNDEM_ERR_CAPACITY = 3,  /* a pair/contact/candidate list overflowed during a step */
    FUNDEM_ERR_STATE = 4,     /* call out of order (e.g. step before setup) */
    FUNDEM_ERR_NUMERIC = 5    /* non-finite particle state detected */
} fundem_status;

enum { FUNDEM_FP64 = 0, FUNDEM_FP32_MIXED = 1 };
/* inverse-inertia rule of the particle geometries */
enum { FUNDEM_INERTIA_REFERENCE = 0, FUNDEM_INERTIA_PHYSICAL = 1 };
/* contact list kinds */
enum { FUNDEM_PP = 0, FUNDEM_PW = 1, FUNDEM_GX = 2, FUNDEM_GY = 3, FUNDEM_GXY = 4,
       FUNDEM_GR90 = 5, FUNDEM_GR180 = 6, FUNDEM_GR270 = 7 /* sector images */ };

const char* fundem_version(void);
const char* fundem_status_string(int status);

/* LSSolver(dir, stream, maxGPUThread, device), kernel/LSSolver.h:14-21, and
   activateGPUDevice, LSSolver.h:601-613 (which calls exit(1) on failure;
   this returns FUNDEM_ERR_CUDA).  stream may be NULL (the legacy stream).
   Every call's work is ordered on that stream; inside a step the simulation
   forks the particle-wall and image detection onto two streams of its own
   and joins them back before the force sums, so a call's work still ends on
   the given stream. */
int fundem_create(fundem_sim** out, int device, void* stream);
int fundem_destroy(fundem_sim* sim);
/* precision of the contact path.  FUNDEM_FP64 reproduces the reference.
   FUNDEM_FP32_MIXED evaluates the node predicate, the SDF gradient, the
   contact and bond laws and the force sums in single precision; positions,
   orientations, their integration and the tangential-spring history stay in
   double precision.  No counterpart in the reference.  May be changed
   between steps. */
int fundem_set_precision(fundem_sim* sim, int mode);
/* neighbour list of the particle-particle broad phase: -1 (default) keeps
   one from 8192 particles on, 0 searches the cell table every step, 1 keeps
   one; both give the same pairs.  Takes effect at the next detection.
   No counterpart in the reference. */
int fundem_set_neighbour_list(fundem_sim* sim, int mode);
/* Pair cache of the particle-particle list.  The reference detects every
   step from scratch (count and write passes, LSParticleContactDetectionKernel.cu:4-305,
   after a fresh hash and sort).  With the cache, the candidate pairs and the
   nodes that may pass the node predicate (the contact slots) are built with
   every culling margin widened by a positional skin, and kept while no
   particle has drifted by more than half the skin since that build (drift:
   centre displacement plus twice the largest bounding radius times the
   chord of its rotation); a particle that changes visibility, a periodic
   wrap, a list growth or a state change through this API rebuilds them.
   Every step still evaluates the exact double-precision predicate on every
   slot, so the contacts are those a full detection gives.  mode -1 (default)
   keeps the cache from 8192 particles on, 0 never, 1 always; skin <= 0
   picks 0.01 times the largest particle bounding radius.  The adjoint's
   recording runs full detections.  Takes effect at the next step.
   No counterpart in the reference. */
int fundem_set_pair_cache(fundem_sim* sim, int mode, double skin);
/* rebuilds of the pair cache and steps run with it since setup, and the skin
   in use (zeros when the cache is off) */
int fundem_pair_cache_stats(fundem_sim* sim, long long* rebuilds, long long* steps, double* skin);
/* Wall groups for a batch of independent simulations tiled into one: for each
   particle (n = the particle count), the first wall and the number of walls
   it may meet; the particle-wall broad phase then tests only those walls
   instead of every wall (the reference tests every wall in the particle's
   wall-cell neighbourhood, LSParticleContactDetectionKernel.cu:307-429).
   n = 0 removes the groups.  No counterpart in the reference. */
int fundem_set_wall_groups(fundem_sim* sim, int n, const int* first, const int* count);
/* when nonzero every step writes full contact records (point, normal,
   overlap, energies); otherwise only node, partner and sliding spring */
int fundem_set_records(fundem_sim* sim, int full_records);

/* LSSolver::addParticleMaterial / addWallMaterial, LSSolver.h:33-42, 175-183
   (clamps of LSParticle::addMaterial, LSParticle.h:221-231) */
int fundem_add_material(fundem_sim* sim, int wall, double kn, double ks, double mu, double e, int* id_out);
/* LSSolver::addParticleGeometry / addWallGeometry, LSSolver.h:58-76, 196-213
   (LSParticle::addGeometry, LSParticle.h:233-267).  sdf is x-fastest,
   size[0]*size[1]*size[2] values; nodes are n_nodes xyz triples. */
int fundem_add_geometry(fundem_sim* sim, int wall, double mass, const double inertia[6], const double origin[3],
                        double spacing, const int size[3], const double* sdf, int n_nodes, const double* nodes,
                        int* id_out);
/* mass, centroid and inertia from a density (LSSolver.h:470-586; host) */
int fundem_mass_properties(double density, const double origin[3], double spacing, const int size[3],
                           const double* sdf, double* mass, double centroid[3], double inertia[6]);

/* Shapes whose signed-distance grid fundem_levelset_grid evaluates on the GPU
   (the implicit functions of kernel/helper/LevelSetObjectGenerator.h). */
enum fundem_shape_kind {
    FUNDEM_SHAPE_SUPERELLIPSOID = 0, /* param: rx, ry, rz, ee, en                    (:1264-1354) */
    FUNDEM_SHAPE_SPHERE = 1,         /* param: radius                                (:1628-1661) */
    FUNDEM_SHAPE_BOX = 2,            /* param: lx, ly, lz, centred on the origin      (:1781-1867) */
    FUNDEM_SHAPE_CYLINDER = 3,       /* param: A xyz, B xyz, radius                  (:2050-2131) */
    FUNDEM_SHAPE_MESH = 4            /* closed triangle mesh: vertices, triangles    (:888-953) */
};
typedef struct fundem_shape {
    int kind;               /* fundem_shape_kind */
    int positive_inside;    /* 1: value and gradient negated (the walls' convention) */
    double param[8];
    int n_vertices;         /* FUNDEM_SHAPE_MESH: host arrays, xyz per vertex ... */
    const double* vertices;
    int n_triangles;        /* ... and three vertex indices per triangle */
    const int* triangles;
} fundem_shape;
/* Base::buildGrid, LevelSetObjectGenerator.h:122-224, evaluated on the GPU:
   sdf[i + nx (j + ny k)] at origin + (i, j, k) * spacing holds f / |grad f|
   where |grad f| > 1e-12, else -spacing/2 (f <= 0) or +spacing/2.  sdf is a
   host array of nx*ny*nz doubles; the call returns when it is filled.
   device < 0 uses the current device; stream may be NULL. */
int fundem_levelset_grid(int device, void* stream, const fundem_shape* shape, const double origin[3],
                         double spacing, const int size[3], double* sdf);
/* LSSolver::addParticle / addWall, LSSolver.h:88-104, 225-238 (host arrays) */
int fundem_add_objects(fundem_sim* sim, int wall, int n, const double* pos, const double* vel, const double* angvel,
                       const double* quat, const int* mat, const int* geo);
/* setFixedVelocityToWall / setFixedAngularVelocityToWall, LSSolver.h:266-282;
   moveLSParticle / moveWall, LSSolver.h:244-258 */
int fundem_set_wall_motion(fundem_sim* sim, int index, const double vel[3], const double angvel[3]);
int fundem_move(fundem_sim* sim, int wall, int index, const double offset[3]);
/* addBondedInteraction, LSSolver.h:296-317 (VBondedInteraction::add,
   VBondedInteraction.h:74-195); uses the current host-side state */
int fundem_add_bonds(fundem_sim* sim, int n, const int* master, const int* slave, const double* point,
                     const double* normal, const double* radius, const double* length, const double* young,
                     const double* poisson, const double* tensile, const double* cohesion, const double* friction);
/* addPeriodicBoundaryXD / YD / removePeriodicBoundary, LSSolver.h:384-414 */
int fundem_set_periodic(fundem_sim* sim, int x, int y);
/* addPeriodicBoundarySector / removePeriodicBoundary, LSSolver.h:410-424
   (PeriodicBoundary.h:319-425): the quarter sector x >= min.x, y >= min.y
   of the domain repeats under quarter turns about the z axis through the
   domain's min corner.  A body leaving through one face comes back through
   the other, turned; bodies next to the faces meet images turned by +90, 180
   and -90 degrees (contact kinds 5, 6, 7).  As in the reference, an image's
   angular velocity is its body's, not turned, and a contact's reaction goes
   to the body unturned.  Takes effect at the next fundem_setup. */
int fundem_set_periodic_sector(fundem_sim* sim, int on);
/* inverse inertia of the particle geometries.  FUNDEM_INERTIA_REFERENCE
   (default) keeps inverse() of myMat.h:163-194, which gives zero when
   |det I| < 1e-30: bodies of millimetre scale (det of order 1e-34) then
   never change their angular velocity.  FUNDEM_INERTIA_PHYSICAL inverts
   every matrix that is not singular relative to its own scale
   (|det I| > 1e-12 max(|Ixx|, |Iyy|, |Izz|)^3), so such bodies turn under
   contact torques.  No counterpart in the reference.  Takes effect at the
   next fundem_setup. */
int fundem_set_inertia_mode(fundem_sim* sim, int mode);

/* LSSolver::upload, LSSolver.h:692-703: domain and grids, template tables,
   device state.  May be called again (multi-phase runs): state already on
   the device is kept, contact history is kept when the node count is
   unchanged (SolidInteraction.h:23-49). */
int fundem_setup(fundem_sim* sim, const double domain_min[3], const double domain_max[3]);
/* the pre-loop detection (LSSolver.h:1093-1094 and the periodic variants) */
int fundem_detect(fundem_sim* sim);
/* detection without forces that also lists node-partner pairs separated by
   a gap up to `gap` (overlap >= -gap); for building packings and placing
   bonds.  No counterpart in the reference. */
int fundem_detect_proximity(fundem_sim* sim, double gap);
/* nsteps iterations of the loop body of LSSolver::compute* (LSSolver.h:1097-1107):
   kick, drift, detection, forces, bonds, kick.  The host waits for the
   stream once every 64 steps, to grow the contact lists ahead of their
   counts; the reference synchronises every step. */
int fundem_step(fundem_sim* sim, int nsteps, const double gravity[3], double dt);
/* nsteps iterations as fundem_step, recorded once into a CUDA graph and
   replayed on later calls with the same nsteps, gravity, time step and
   settings; the graph is recorded again after any list growth or
   re-setup.  Each call first grows the contact lists ahead of their counts
   (one stream synchronisation).  For many small simulations on separate
   streams, whose steps are launch-bound.  No counterpart in the reference. */
int fundem_step_graph(fundem_sim* sim, int nsteps, const double gravity[3], double dt);
/* one step split at the addExternalForceTorque hook (LSSolver.h:588): after
   step_begin the force/torque arrays hold the step's contact and bond sums;
   the caller may add to them (stream-ordered) before step_end. */
int fundem_step_begin(fundem_sim* sim, const double gravity[3], double dt);
int fundem_step_end(fundem_sim* sim, const double gravity[3], double dt);
/* wait for the stream and grow the contact lists ahead of their counts;
   returns the accumulated device error status */
int fundem_sync(fundem_sim* sim);
/* record one status word per step into a host ring without stalling */
int fundem_status_word(fundem_sim* sim, unsigned int* flags);

/* state transfer (host arrays; any pointer may be NULL) */
int fundem_num_objects(fundem_sim* sim, int wall, int* n);
int fundem_get_objects(fundem_sim* sim, int wall, double* pos, double* vel, double* angvel, double* quat,
                       double* force, double* torque);
int fundem_set_objects(fundem_sim* sim, int wall, const double* pos, const double* vel, const double* angvel,
                       const double* quat, const double* force, const double* torque);
/* raw device pointers of the state (LSParticle::position() ... , LSParticle.h:768-777) */
typedef struct {
    double* pos;
    double* vel;
    double* angvel;
    double* force;
    double* torque;
    double* quat;
    int* mat;
    int* geo;
    int n;
} fundem_device_view;
int fundem_device_view_get(fundem_sim* sim, int wall, fundem_device_view* out);

/* contact lists in canonical (node, partner) order; records are valid only
   for steps run with full records (the pre-loop detection always writes them) */
int fundem_num_contacts(fundem_sim* sim, int kind, long long* n);
int fundem_get_contacts(fundem_sim* sim, int kind, int* node, int* partner, double* point, double* normal,
                        double* overlap, double* spring, double* en, double* es);
/* Device pointers of one list's contacts, as SolidInteraction's getters hand
   them out (contactPoint(), contactNormal(), contactOverlap(),
   normalElasticEnergy(), slidingElasticEnergy(), slidingSpring(),
   masterID(), slaveID(), numPair_device(): kernel/SolidInteraction.h:323-334):
   the contacts are copied into contiguous arrays owned by the simulation, in
   (node, partner) order, n of them.  A read-only snapshot: valid until the
   next step or view call on the simulation; point, normal, overlap and the
   energies are filled for steps run with full records. */
typedef struct {
    double* point;           /* 3 per contact */
    double* normal;          /* 3 per contact */
    double* overlap;
    double* normal_energy;
    double* sliding_energy;
    double* spring;          /* 3 per contact */
    int* master;             /* global boundary-node index */
    int* slave;              /* partner object */
    long long n;
} fundem_contact_view;
int fundem_contact_view_get(fundem_sim* sim, int kind, fundem_contact_view* out);
/* Device pointers of the bonds, as VBondedInteraction's getters hand them out
   (kernel/VBondedInteraction.h:452-485): ids, activation, centre point,
   radius and initial length point at the library's own arrays; the
   beam stiffnesses, energies, stresses and body-frame vectors are copied
   into one array per field.  The copies are a snapshot, valid until the
   next step or view call. */
typedef struct {
    int* master;
    int* slave;
    int* activated;
    double* center_point;    /* 3 per bond */
    double* radius;
    double* initial_length;
    double *B1, *B2, *B3, *B4;
    double *Un, *Us, *Ub, *Ut, *max_normal_stress, *max_shear_stress;
    double *tensile_strength, *cohesion, *friction;
    double* frames[8];       /* 3 per bond: master n1 n2 n3 point, slave n1 n2 n3 point (body frames) */
    int n;
} fundem_bond_view;
int fundem_bond_view_get(fundem_sim* sim, fundem_bond_view* out);
/* replace the history (previous step's list) of one kind */
int fundem_set_contacts(fundem_sim* sim, int kind, long long n, const int* node, const int* partner,
                        const double* spring);
/* candidate pairs of the last detection */
int fundem_num_pairs(fundem_sim* sim, int kind, long long* n);

/* bond state (VBondedInteraction getters, VBondedInteraction.h:448-494) */
int fundem_num_bonds(fundem_sim* sim, int* n);
int fundem_get_bonds(fundem_sim* sim, int* activated, double* point, double* energy6);
int fundem_set_bond_activation(fundem_sim* sim, const int* activated);

/* derived template data (geometryInfo, LSParticle.h:53-173) */
int fundem_get_geometry(fundem_sim* sim, int wall, int geo, double* radius, double* inv_mass, double inertia[6],
                        double inv_inertia[6]);
int fundem_get_grid(fundem_sim* sim, int wall, double minb[3], double maxb[3], double inv_cell[3], int size[3]);
/* Inclusive prefix sum of n ints in device memory, stream-ordered:
   d_prefix[i] = d_count[0] + ... + d_count[i].  Replaces buildPrefixSum,
   kernel/CUDAKernelFunction/myUtility/buildHashStartEnd.cu:139-177 (which
   runs thrust::inclusive_scan); scratch is taken with cudaMallocAsync on the
   stream and released after the scan.  stream may be NULL. */
int fundem_prefix_sum(int* d_prefix, const int* d_count, long long n, void* stream);

/* Stable sort of object cell hashes, device arrays, stream-ordered:
   d_sorted receives the permutation that orders d_hash ascending, objects of
   equal hash in ascending index, and hashes outside [0, num_cells) (the
   reference's -1 for objects outside the grid) last; d_sorted_hash (may be
   NULL) receives the sorted hashes, -1 for those.  Replaces the sort of
   buildHashStartEnd, kernel/CUDAKernelFunction/myUtility/buildHashStartEnd.cu:69-137
   (thrust::sort_by_key on int32 hashes); here the hashes are 64-bit, so grids
   of more than 2^31 cells work.  An LSD radix sort, 8 bits per pass over the
   bits num_cells needs; scratch is taken with cudaMallocAsync on the stream
   and released after the sort.  stream may be NULL. */
int fundem_hash_sort(const long long* d_hash, int n, long long num_cells, int* d_sorted, long long* d_sorted_hash,
                     void* stream);

/* The same inclusive prefix sum without any device allocation.  No
   counterpart in the reference.  For callers that cannot allocate device
   memory at the point of the call: code working inside a memory budget that
   another allocator has already reserved (a cudaMalloc there can fail), and
   code that cannot accept cudaMalloc's implicit device synchronisation.  The
   scratch is a fixed 16 KiB device array inside this library, held on every
   GPU that loads it until the process exits, which limits n to
   FUNDEM_NOALLOC_SCAN_MAX; larger n returns FUNDEM_ERR_ARG.  The first call
   on a device looks up the array's device address (once per device, on the
   current device), so make that first call before any stream capture.  The
   array is shared by all calls on a device: calls that overlap on the GPU
   race. */
#define FUNDEM_NOALLOC_SCAN_MAX 16777216LL
int fundem_prefix_sum_noalloc(int* d_prefix, const int* d_count, long long n, void* stream);

/* Reverse-mode gradients (the adjoint of the step, in the precision set when
   the recording begins: FP64, or FP32_MIXED, whose recorded single-precision
   run is swept with double-precision contact and bond Jacobians; the
   precision may not change while recording).  No counterpart in the reference.  Loss gradients on the final state are carried back to the
   initial velocities and to each particle material's normal stiffness,
   shear stiffness, damping ratio and friction coefficient.  Contact topology
   is frozen at each step, as the forward run had it (including each
   contact's stick or slip and each bond's breakage); orientations are
   differentiated when a particle geometry has a nonzero inverse inertia
   (fundem_adjoint_backward_rot takes loss gradients on them); otherwise
   they are fixed, and constant angular velocities of particles and
   prescribed ones of walls enter the contact velocities.  Bonds are
   differentiated between bodies that do not turn.  Sector periodicity is not
   differentiated.
   begin: start recording from the current state (after fundem_detect),
     with a checkpoint every checkpoint_interval steps;
   forward: run steps (one gravity and time step for the whole recording);
   backward: dl_dpos, dl_dvel (n*3, the loss gradient on the final positions
     and velocities) -> dl_dvel0 (n*3) and dl_dparams (4 per particle
     material: kn, ks, damping ratio, mu).  Each checkpoint segment is re-run
     once with recording, then swept in reverse; the final state is restored
     afterwards.
   end: drop the recording. */
int fundem_adjoint_begin(fundem_sim* sim, int checkpoint_interval);
int fundem_adjoint_forward(fundem_sim* sim, int nsteps, const double gravity[3], double dt);
int fundem_adjoint_backward(fundem_sim* sim, const double* dl_dpos, const double* dl_dvel, double* dl_dvel0,
                            double* dl_dparams);
int fundem_adjoint_end(fundem_sim* sim);
/* fundem_adjoint_backward with turning bodies: dl_dquat (n*4) and dl_dangvel
   (n*3) carry the loss gradient on the final orientations and angular
   velocities (either may be NULL: zero), dl_dangvel0 (n*3, may be NULL)
   receives the gradient with respect to the initial angular velocities.
   The reverse sweep differentiates the world-frame inertia of the half
   kick (particleIntegrationKernel.cu:3-32), the quaternion Euler step with
   its normalisation (myQua.h:77-93), the lever arms of the contact torques
   and the contact velocity (contactKernel.cu:104, 120-123) and the partner's
   orientation in the SDF lookup and the normal.  Runs with bonds between
   turning bodies are refused at fundem_adjoint_begin.  No counterpart in
   the reference. */
int fundem_adjoint_backward_rot(fundem_sim* sim, const double* dl_dpos, const double* dl_dvel,
                                const double* dl_dquat, const double* dl_dangvel, double* dl_dvel0,
                                double* dl_dangvel0, double* dl_dparams);

/* Checkpoint files (FP64 binary): object state, the contact history of every
   list and bond activation, which is all a restart needs besides the setup
   calls.  read expects a simulation set up with the same materials,
   geometries, objects and bonds (the counts are checked); a run continued
   from a checkpoint repeats the uninterrupted run bit for bit.  The
   reference keeps no restart files (its VTU output is not reloadable). */
int fundem_checkpoint_write(fundem_sim* sim, const char* path);
int fundem_checkpoint_read(fundem_sim* sim, const char* path);

/* text of the last error a call on this simulation returned (empty when
   none); valid until the next call on it.  The reference prints such
   messages to std::cerr instead. */
const char* fundem_last_error(fundem_sim* sim);

/* kernel launches issued by this simulation so far */
int fundem_launch_count(fundem_sim* sim, long long* n);
/* CUDA-event timing of kernel groups on the simulation's stream (off by
   default).  fundem_kernel_time returns the summed device time and the
   number of timed intervals since the last query, then resets. */
enum {
    FUNDEM_T_INTEGRATE = 0, FUNDEM_T_HASH = 1, FUNDEM_T_BROAD = 2, FUNDEM_T_NARROW_PP = 3,
    FUNDEM_T_NARROW_PW = 4, FUNDEM_T_GHOST = 5, FUNDEM_T_REDUCE = 6, FUNDEM_NTIMERS = 7
};
/* on: FUNDEM_PROF_TIMERS times the kernel groups (plain steps then run every
   stage on the simulation's stream, so that each timer sees its own stage;
   the results are the same bit for bit); FUNDEM_PROF_COUNTERS also counts
   narrow-phase work (one shared-memory atomic per pair and a few global
   atomics per block, so keep it out of timed runs); 0 turns both off */
enum { FUNDEM_PROF_TIMERS = 1, FUNDEM_PROF_COUNTERS = 2 };
int fundem_set_profiling(fundem_sim* sim, int on);
int fundem_kernel_time(fundem_sim* sim, int group, double* ms_total, long long* count);
/* narrow-phase work since the last call while the counters are on:
   candidate pairs, node clusters examined, clusters that survived culling,
   node contacts, nodes given the exact double-precision predicate */
int fundem_work_counters(fundem_sim* sim, unsigned long long out[5]);
/* pair-cache work of the particle-particle predicate pass since the last
   fundem_work_counters call (which resets these too): slots given the exact
   predicate, and slots of carried steps skipped because the node was outside
   the partner at the last rebuild by more than the SDF's Lipschitz bound
   times both bodies' drift since (such a slot cannot hold a contact) */
int fundem_slot_counters(fundem_sim* sim, unsigned long long out[2]);
/* launch shape of the narrow phase, in blocks per SM, for the selection, the
   predicate pass, the contact-law pass and the per-pair sums (grid-stride
   kernels: results do not depend on it); 0 keeps a kernel's default, each
   value 0..64.  The reference takes a caller-chosen grid per launcher
   (gridD, blockD of every launcher, e.g. LSParticleContactDetectionKernel.cu:609).
   fundem_get_launch_shape returns the shape in use, defaults resolved. */
int fundem_set_launch_shape(fundem_sim* sim, const int blocks_per_sm[4]);
int fundem_get_launch_shape(fundem_sim* sim, int blocks_per_sm[4]);

#ifdef __cplusplus
}
#endif
#endif
