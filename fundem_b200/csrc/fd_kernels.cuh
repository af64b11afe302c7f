// fd_kernels.cuh -- launch interface of the timestep kernels (fd_kernels.cu).
#pragma once
#include "fd_internal.cuh"

// resident blocks per SM the narrow-phase kernels are compiled for (their
// default grids fill one wave of them)
#ifndef FD_SELECT_MIN_BLOCKS
#define FD_SELECT_MIN_BLOCKS 4
#endif
#ifndef FD_CONTACT_MIN_BLOCKS
#define FD_CONTACT_MIN_BLOCKS 2
#endif
// the predicate pass of the contact kernels: latency-bound gathers, so as
// many resident warps as fit without spilling
#ifndef FD_PROBE_MIN_BLOCKS
#define FD_PROBE_MIN_BLOCKS 4
#endif

namespace fd {

// Everything one simulation keeps on the device.  Plain pointers; ownership
// and sizes live in the host-side Sim object (fd_api.cu).
struct PairListDev {
    // pairs of the current step (A-major segments, partners ascending)
    int* pairA;
    int* pairB;
    int* seg_off;      // per particle A: first pair
    int* seg_cnt;      // per particle A: number of pairs
    int* c_off;        // per pair: first contact
    int* c_cnt;        // per pair: number of contacts
    double* pf;        // per pair: F (3), torque on A (3), torque on B (3)
    int* n_pairs;      // device counter
    int cap_pairs;
    // previous step (history source)
    int* o_pairA;
    int* o_counters;   // previous step's counters: pairs, slots, contacts
    int* o_pairB;
    int* o_seg_off;
    int* o_seg_cnt;
    int* o_c_off;
    int* o_c_cnt;
    // contact slots of the current step: the nodes that passed the
    // single-precision filter, contiguous per pair; c_node is the global
    // boundary-node id of a contact and -1 for a slot that is none
    int* c_node;
    int* c_slave;
    int* c_pair;       // pair of each slot
    int* c_hit;        // slots holding a contact, listed by the predicate pass
                       // for the contact-law pass (n_hits of them)
    int* c_k;          // node key of each slot: cluster-order index relative to
                       // the geometry (ascending within a pair)
    double* c_force;   // 9 per slot: F, torque on A, torque on B (contacts only)
    int4* p_aux;       // per pair: cell of B (x, y, z), first history slot
    int* p_hist_cnt;   // per pair: history slots
    double* c_spring;  // 3 per contact
    double* c_point;   // 3 per contact (records)
    double* c_normal;  // 3 per contact (records)
    double* c_overlap; // records
    double* c_en;      // records
    double* c_es;      // records
    int* n_slots;      // device counter: slots used
    int* n_hits;       // device counter: contacts (n_slots + 1)
    int cap_contacts;  // slot capacity
    int* carry_n;      // pair cache: carried steps since the layout was built
    int* c_test;       // pair cache, carried steps: the slots the bound does not
                       // skip, listed for the predicate pass (n_test of them)
    int* n_test;
    float* p_bound;    // pair cache, carried steps: per pair, how far the SDF can
                       // have moved at a node since the rebuild (k_pc_carry)
    float* c_phi0;     // pair cache: per slot, the node's signed distance to the
                       // partner at the last rebuild (rounded down; -inf when
                       // the predicate stopped before the distance)
    // previous contacts
    int* o_c_node;
    int* o_c_k;
    double* o_c_spring;
};

// Reverse index over the particle-particle and ghost lists together: for each
// particle, the pairs in which it is the partner, as codes pair * 8 + kind,
// sorted by (owner, kind).
struct RevDev {
    int* cnt;
    int* off;
    int* fill;
    int* code;
    int cap;
};

struct ObjDev {
    int n;
    double3* pos;
    double3* vel;
    double3* angvel;
    double3* force;
    double3* torque;
    fd_quat* q;
    int* mat;
    int* geo;
    long long* hash;   // cell hash of the current step (-1 when not hashed)
    int* node_base;    // first global boundary node of each object
    float4* rot;       // 3 per object: rows of the rotation matrix, single
                       // precision, refreshed at every hashing (culling only)
};

struct GeoSetDev {
    int n;
    const FdGeo* geo;
    const double* sdf;
    const float* sdf32;
    const float* dist;
    const float* cellmin;
    const double3* nodes;     // cluster order
    const int* node_lid;      // original local index of each node (cluster order)
    const FdCluster* clusters;
    const float4* nodes32;      // cluster order, single precision (culling only)
    const float4* clus_sphere;  // per cluster: centre, radius (single precision)
    const int2* clus_range;     // per cluster: first node, node count
    double rmax;              // largest bounding radius over the set
    double grid_rmax;         // largest grid radius over the set
};

struct MatDev {
    const double* kn;
    const double* ks;
    const double* mu;
    const double* e;
};

// Cell table of one object set (hashGrid of buildHashStartEnd.cu:69-137).
// The objects' 64-bit cell keys are sorted by a stable LSD radix sort (so
// each cell lists its objects in ascending index, as the reference's stable
// thrust::sort_by_key does); the runs of equal keys are the cells.  A grid of
// few cells keeps a dense start/count table over all cells; a grid of many
// cells (dense would be large next to the object count) keeps an
// open-addressing hash table of its occupied cells instead.
struct CellTableDev {
    FdGrid g;
    int hashed;                 // 0: dense table, 1: hash table of occupied cells
    int* count;                 // dense: objects per cell
    int* start;                 // dense: first slot of each cell (valid where count > 0)
    int* fill;                  // dense: scatter counters
    unsigned long long* hkey;   // hashed: cell key per table slot (~0: empty)
    int2* hval;                 // hashed: (first slot, objects) per table slot
    unsigned long long hmask;   // hashed: table size - 1 (a power of two)
    int* sorted;                // object index per slot, by cell key
    unsigned long long* skey;   // cell key per slot (~0 for objects in no cell, last)
    // sort scratch: the second key/index buffers, per-block digit counts and
    // their scan's temporary
    unsigned long long* key_b;
    int* idx_b;
    int* bcount;
    int* bscan_tmp;
    int nobj_cap;               // objects the scratch holds
};

struct GhostDev {
    double3* pos;
    long long* hash;
    CellTableDev cells;
    int* occ;  // box of the cells holding ghost images: min x, y, z, max x, y, z
    int* searchers;  // particles whose search box reaches a ghost image
    int* nsearch;    // their count
    // sector images only (null for the translated X/Y images, which share the
    // particle's orientation and velocity): orientation, velocity and the
    // single-precision rotation rows of each image
    fd_quat* q;
    double3* vel;
    float4* rot;
    // translated images under the pair cache: 1 where the particle has an
    // image this step (the images of a rebuild also cover the particles
    // within the skin of the image band, whose pairs the cache keeps)
    unsigned char* live;
};

struct BondDev {
    int n;
    const int* master;
    const int* slave;
    int* active;
    double3* point;
    const double* B;      // 4 per bond
    const double* radius;
    const double* L0;
    const double* ts;
    const double* coh;
    const double* mu;
    const double3* frames; // 8 per bond: mn1 mn2 mn3 mp sn1 sn2 sn3 sp
    double* energy;        // 6 per bond: Un Us Ub Ut sn ss
    double* out;           // 9 per bond: F, Ti, Tj
    const int* plist_off;  // per particle (n+1): bonds touching it
    const int* plist;      // bond id * 2 + side
    int* rec_active;       // adjoint recording (null when off): bond active at the step
    double* rec_rij;       // 3 per bond: bond vector rb_i - rb_j at the step
    double* rec_dn;        // 3 per bond: frame difference n1j - n1i at the step
};

// Adjoint recording of one list at one step, one entry per contact slot
// (null pointers when not recording).  The partner index Bp is the particle
// that takes the reaction (the image's particle for ghosts, -1 for walls).
struct AdjRec {
    int* hit;        // 1 when the slot holds a contact
    int* A;
    int* Bp;
    int* B;          // partner as listed (wall index for walls)
    int* geoB;       // partner geometry (in the wall set for walls)
    int* matB;       // partner material (a wall material for walls)
    int* nid;        // global boundary-node id of the contact
    int* hist;       // slot of the same contact in the previous step, -1 when none
    double* rel;     // 3 per slot: contact node minus partner centre, world frame
    double* vc;      // 3 per slot: relative velocity of A against the partner
    double* sprev;   // 3 per slot: sliding spring before this step's update
    double* qB;      // 4 per slot: partner orientation
    double* arm;     // 3 per slot: contact node minus A's centre, world frame
    int* wrap;       // per slot: periodic shifts of the force-side centres,
                     // (sAx + 1) + 3 (sAy + 1) + 9 (sBx + 1) + 27 (sBy + 1)
    int cap;         // slots the record holds
};

// Verlet neighbour list of the particle-particle broad phase: per particle A,
// up to NL_MAX partners B > A whose centre lay within rA + rB + skin at the
// last build, ascending, by minimum-image distance in periodic directions
// (so a particle that wraps keeps the partners it meets on the other side).
// Rebuilt when a particle moved more than skin / 2 since then (minimum image)
// or changed visibility (inside or outside the domain).  The per-step filter
// applies the raw-position tests of the cell search.
constexpr int NL_MAX = 64;
struct NlDev {
    double3* ref;   // positions at the last build
    int* vis;       // visibility (cell hash >= 0) at the last build
    int* cnt;       // partners per particle
    int* list;      // NL_MAX per particle
    int* ctrl;      // [0]: rebuild requested
    double skin;
    int periodic_x, periodic_y;  // distances and displacements by minimum image
    double pair_skin;   // positional skin of the pair cache (0 without it): the
                        // list is rebuilt once a particle moved (skin - pair_skin) / 2
};

// Pair cache of the particle-particle list.  The candidate pairs and the
// nodes that may pass the node predicate (the contact slots) are built with
// every culling margin widened by a positional skin, and kept while no
// particle has drifted by more than skin / 2 since that build: the drift of
// particle i is |c_i - c_i0| + 2 r_max * 2 sin(theta_i / 2), theta_i its
// rotation since the build, which bounds how far any node of a pair can move
// in its partner's body frame (pairs stay listed, nodes stay slotted, while
// the two drifts sum to less than the skin).  Every step still runs the
// exact double-precision predicate on every slot, so the contacts are the
// ones a full detection gives.  ctrl[0]: rebuild this step (set by the check
// or by the host), ctrl[1]: rebuilds so far, ctrl[2]: the last build
// overflowed its lists (the next step builds again).
struct PairCacheDev {
    double3* ref_pos;   // positions at the last build
    fd_quat* ref_q;     // orientations at the last build
    int* ref_vis;       // visibility (hashed) at the last build
    // ctrl: [0] rebuild this step, [1] rebuilds so far, [2] the last build
    // overflowed the particle-particle lists, [3] rebuild at the next step,
    // [4] the translated ghost lists of this step are built without the
    // cache (a particle wrapped, or an image outside the domain's other
    // directions), [5] the ghost lists' gate this step ([0] or [4]), [6]
    // [4] again, as the ghost kernels' skin switch, [7] rebuild requests of
    // this step, moved to [3] at its end
    int* ctrl;
    float* drift;       // per particle: the drift bound since the last build (rounded up)
    float4* disp;       // per particle: displacement since the last build (x, y, z) and
                        // the rotation part of the drift bound (rounded up)
    double skin;
    double reach;       // largest lever arm of a rotation in the drift bound:
                        // 2 r_max, or a larger SDF-grid radius
    // walls (the particle-wall list): state and cell at the last build, and
    // their drift bounds and displacements as for the particles (rotation
    // lever arm: the wall's SDF-grid radius)
    double3* wref_pos;
    fd_quat* wref_q;
    long long* wref_hash;
    float* wdrift;
    float4* wdisp;
};

struct StepArgs {
    AdjRec rec;      // recording of the list being launched (rec.hit null: off)
    double dt;
    double probe;      // contact when overlap >= -probe (0 in a timestep)
    double3 gravity;
    int periodic_x, periodic_y;
    int sector;      // sector periodicity (the force side of particle and wall contacts folds bodies)
    int records;
    double skin;       // positional skin of the culling stages (the pair cache; 0 without it)
    const int* gate;   // pair cache: the selection runs only when *gate != 0 (null: always)
    const float* drift;  // pair cache: per-particle drift bounds (see PairCacheDev)
    const float4* disp;  // pair cache: per-particle displacements (see PairCacheDev)
    const float* driftB; // the partners' drift bounds and displacements when they
    const float4* dispB; // are walls (null: the particles')
    const int* noskin;   // non-null and nonzero: this step's selection takes no skin
    // launch shape of the narrow phase, in blocks per SM (0: the default):
    // selection, predicate pass, contact-law pass, pair sums
    int shape[4];
    unsigned int* flags;
    unsigned long long* stats;  // optional: pairs, clusters, clusters kept, contacts (narrow kernels)
};

// contiguous copy of a list's contacts, in (node, partner) order
struct ContactViewDev {
    double* point;     // 3 per contact
    double* normal;    // 3 per contact
    double* overlap;
    double* en;
    double* es;
    double* spring;    // 3 per contact
    int* master;       // global boundary node
    int* slave;        // partner
};
// the bonds' interleaved per-bond parameters and state as one array per field
struct BondViewDev {
    double* B[4];       // B1 .. B4
    double* energy[6];  // Un, Us, Ub, Ut, maximum normal stress, maximum shear stress
    double3* frames[8]; // master n1 n2 n3 point, slave n1 n2 n3 point (body frames)
};

// integration and hashing
void launch_kick(const ObjDev& P, const GeoSetDev& G, double3 gravity, double h, cudaStream_t s);
void launch_drift(const ObjDev& O, double dt, cudaStream_t s);
// launch_kick(h), launch_kick(h) and launch_drift(dt) of the particles in one
// pass: the end of one step and the start of the next
void launch_kick_drift(const ObjDev& P, const GeoSetDev& G, double3 gravity, double h, double dt, cudaStream_t s);
// cell hash of each object (-1 outside the grid) and its single-precision
// rotation rows
void launch_hash(const ObjDev& O, const FdGrid& g, cudaStream_t s);
// the cell table from the objects' hashes (O.hash); with gate non-null a
// hash-table build runs only when *gate != 0 (the pair cache's rebuild flag)
void launch_cell_table(ObjDev& O, CellTableDev& T, int* scan_tmp, size_t scan_tmp_ints, cudaStream_t s,
                       const int* gate = nullptr);
// stable sort of n 64-bit keys (key 0 .. num_keys - 1, or negative: last) on
// the stream: out_idx gets the permutation, out_key the sorted keys (~0 for
// the negative ones).  Scratch: key_b (n), idx_b (n), bcount and bscan_tmp
// sized by radix_sort_scratch.
void radix_sort_keys(const long long* keys, int n, long long num_keys, unsigned long long* out_key, int* out_idx,
                     unsigned long long* key_b, int* idx_b, int* bcount, int* bscan_tmp, cudaStream_t s,
                     const int* gate = nullptr);
// ints needed for bcount and bscan_tmp for n keys
void radix_sort_scratch(int n, size_t& bcount_ints, size_t& bscan_ints);
// ctrl (the pair cache's, or null): a wrap requests the uncached ghost
// stage this step and a rebuild at the next
// src: positions to wrap into P.pos (null: P.pos in place)
void launch_wrap(ObjDev& P, const FdGrid& g, int dim, cudaStream_t s, int* ctrl = nullptr,
                 const double3* src = nullptr);
// ext_skin > 0 (the pair cache, ctrl non-null): particles within ext_skin of
// the image band get images too (Gh.live marks the true ones); an image
// outside the domain in a direction it is not translated along (the
// reference hashes it into a clamped cell) makes this step's ghost stage
// uncached
void launch_ghost_build(const ObjDev& P, GhostDev& Gh, int kind, cudaStream_t s, double ext_skin = 0.0,
                        int* ctrl = nullptr);
// the ghost lists' gate and skin switch of this step (ctrl[5], ctrl[6])
void launch_ghost_gate(int* ctrl, cudaStream_t s);
// sector periodicity: turn bodies that left the quarter sector back in, then
// build the three turned image sets (R90, R180, R270)
void launch_sector_wrap(ObjDev& P, const FdGrid& g, cudaStream_t s);
void launch_sector_images(const ObjDev& P, GhostDev* R, cudaStream_t s);

// pair lists.  skin widens the sphere tests and the body-level cull (the pair
// cache); with gate non-null the kernels run only when *gate != 0
void launch_broad_pp(const ObjDev& P, const GeoSetDev& G, const CellTableDev& T, PairListDev& L,
                     unsigned int* flags, double probe, cudaStream_t s, double skin = 0.0,
                     const int* gate = nullptr);
// the same pairs through the neighbour list (check, conditional rebuild, filter)
void launch_broad_pp_nl(const ObjDev& P, const GeoSetDev& G, const CellTableDev& T, PairListDev& L, NlDev& nl,
                        unsigned int* flags, double probe, cudaStream_t s, const int* gate = nullptr);
// pair cache: flag a rebuild when a particle drifted by more than skin / 2
// (or changed visibility); after the particle-particle narrow phase, keep
// the state of a rebuild step as the new reference and clear the flag
void launch_pair_cache_check(const ObjDev& P, const PairCacheDev& c, cudaStream_t s);
void launch_pair_cache_commit(const ObjDev& P, const PairCacheDev& c, const PairListDev& L, cudaStream_t s);
// walls: flag a rebuild when a wall drifted by more than skin / 2 or changed
// cell; after the particle-wall narrow phase of a rebuild, keep their state
void launch_pair_cache_check_walls(const ObjDev& W, const GeoSetDev& GW, const PairCacheDev& c, cudaStream_t s);
void launch_pair_cache_commit_walls(const ObjDev& W, const PairCacheDev& c, cudaStream_t s);
// end of a cached step: a list (particle-wall, ghosts) that overflowed asks
// for a rebuild, this step's requests become the next step's rebuild, the
// flags clear
void launch_pair_cache_end(const PairCacheDev& c, const PairListDev* lists, int n_lists, cudaStream_t s);
// wall_range (null: every wall): per particle, the first wall and the wall
// count it may meet (a batch of simulations tiled into one)
void launch_broad_pw(const ObjDev& P, const GeoSetDev& G, const ObjDev& W, const GeoSetDev& GW,
                     const FdGrid& wg, PairListDev& L, unsigned int* flags, double probe, cudaStream_t s,
                     const int2* wall_range = nullptr, double skin = 0.0, const int* gate = nullptr);
// skin, gate and noskin: the pair cache (ctrl[5], ctrl[6]), as for the
// particle-particle list
void launch_broad_ghost(const ObjDev& P, const GeoSetDev& G, const GhostDev& Gh, PairListDev& L,
                        unsigned int* flags, double probe, cudaStream_t s, double skin = 0.0,
                        const int* gate = nullptr, const int* noskin = nullptr);
// a.gate non-null (particle-particle and translated ghost lists under the
// pair cache): on steps without a rebuild the selection is skipped and the
// previous step's pairs and slots are carried into this step's list
void launch_narrow(int kind, const ObjDev& P, const GeoSetDev& G, const MatDev& M, const ObjDev& W,
                   const GeoSetDev& GW, const MatDev& MW, const FdGrid& pgrid, const FdGrid& wgrid,
                   const GhostDev* gh, PairListDev& L, const StepArgs& a, int with_force, bool mixed, cudaStream_t s);
// gate (non-null): the index is rebuilt only when *gate != 0 (a step whose
// lists keep their pairs keeps the index of the step that built them)
void launch_reverse(const ObjDev& P, PairListDev* lists, const int* active, RevDev& R, int* scan_tmp,
                    size_t scan_tmp_ints, cudaStream_t s, const int* gate = nullptr);
// mixed: single-precision contact law, bond law and force sums
void launch_bonds(const ObjDev& P, BondDev& B, bool mixed, cudaStream_t s);
void launch_reduce(ObjDev& P, PairListDev* lists, const int* active, const RevDev& R, const BondDev& B, bool mixed,
                   cudaStream_t s);
// the n contacts of a list (keys and sort scratch of the list's slot
// capacity; max_key bounds node << 32 | partner) into the view
void launch_contact_view(const PairListDev& L, long long* keys, int* order, unsigned long long* skey,
                         unsigned long long* key_b, int* idx_b, int* bcount, int* bscan, long long n,
                         long long max_key, const ContactViewDev& v, cudaStream_t s);
void launch_bond_view(const BondDev& B, const BondViewDev& v, cudaStream_t s);

// Kernel launches of the calling thread are counted into *c (null: not
// counted); the library points it at the calling simulation's counter for
// the duration of each call.  count_launch() counts one launch made
// elsewhere (the adjoint kernels).
void set_launch_counter(long long* c);
void count_launch();

// exclusive scan of n ints (out may alias in); returns needed tmp ints when tmp == nullptr
size_t scan_tmp_size(long long n);
void scan_exclusive(const int* in, int* out, long long n, int* tmp, cudaStream_t s, const int* gate = nullptr);
// inclusive scan of n ints; tmp as for scan_exclusive
void scan_inclusive(const int* in, int* out, long long n, int* tmp, cudaStream_t s);

}  // namespace fd
