// fd_kernels.cu -- sm_100a kernels of the level-set DEM timestep.
//
// Per step (one CUDA stream, no host synchronisation):
//   kick + drift (+ wall drift)            particleIntegrationKernel.cu:3-48
//   hash + counting sort into a dense cell table
//                                          mySpatialGrid.cu:4-26, buildHashStartEnd.cu:47-137
//   broad phase: one thread per particle lists candidate partners (bounding
//                spheres, or SDF-grid spheres for walls and ghosts), sorted
//                by partner id, into an A-major pair list
//   narrow phase + contact force, fused: one warp per candidate pair streams
//                A's surface nodes cluster by cluster through B's SDF,
//                culls whole clusters with exact-conservative bounds, applies
//                the reference's node predicate bit for bit
//                (LSParticleContactDetectionKernel.cu:4-607), carries the
//                sliding spring from the previous step, evaluates the linear
//                spring-dashpot law (contactKernel.cuh:4-77) and reduces the
//                pair's force and torques with warp shuffles
//   reverse index of the pair list (pairs grouped by partner)
//   bonds (contactKernel.cu:293-371), one thread per bond
//   per-particle reduction in a fixed order (no atomics on forces)
#include "fd_kernels.cuh"
#include "../../include/fundem_b200.h"

#include <algorithm>
#include <cstdio>
#include <mutex>

namespace fd {

namespace {

constexpr int TPB = 256;
constexpr int MAX_CAND = 64;        // candidate partners per particle and kind
constexpr int MAX_CLUSTERS = 64;    // clusters per template (two warp-wide batches)
constexpr int MAX_NODE_QUEUE = 32 * MAX_CLUSTERS;  // per-warp queue of nodes for the exact test
constexpr int NARROW_WARPS = 8;     // warps per block in the narrow kernel
constexpr double PI_D = 3.14159265358979323846;

inline int nblocks(long long n, int tpb = TPB) { return (int)((n + tpb - 1) / tpb); }

__device__ __forceinline__ void set_flag(unsigned int* flags, unsigned int f)
{
    if (flags) atomicOr(flags, f);
}

// ---------------------------------------------------------------------------
// scan (exclusive, int), three-phase: tile scan, scan of tile sums, add
// ---------------------------------------------------------------------------
constexpr int SCAN_TPB = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_TPB * SCAN_ITEMS;

__device__ __forceinline__ int block_excl_scan(int v, int* total)
{
    __shared__ int warp_sum[SCAN_TPB / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = (lane < SCAN_TPB / 32) ? warp_sum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < SCAN_TPB / 32) warp_sum[lane] = s;
    }
    __syncthreads();
    const int before = (wid > 0) ? warp_sum[wid - 1] : 0;
    if (total) *total = warp_sum[SCAN_TPB / 32 - 1];
    const int r = before + x - v;
    __syncthreads();
    return r;
}

template <bool INCLUSIVE>
__global__ void k_scan_tile(const int* in, int* out, long long n, int* tile_sums, const int* gate)
{
    if (gate && *gate == 0) return;
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    int s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + k;
        v[k] = (i < n) ? in[i] : 0;
        s += v[k];
    }
    int total;
    int run = block_excl_scan(s, &total);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long i = base + k;
        if (INCLUSIVE) run += v[k];
        if (i < n) out[i] = run;
        if (!INCLUSIVE) run += v[k];
    }
    if (tile_sums && threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int* out, long long n, const int* tile_off, const int* gate)
{
    if (gate && *gate == 0) return;
    const long long i = (long long)blockIdx.x * SCAN_TILE + threadIdx.x;
    const int add = tile_off[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const long long j = i + (long long)k * SCAN_TPB;
        if (j < n && j < (long long)(blockIdx.x + 1) * SCAN_TILE) out[j] += add;
    }
}

// ---------------------------------------------------------------------------
// integration, particleIntegrationKernel.cu:3-48 and myQua.h:77-93
// ---------------------------------------------------------------------------
__device__ __forceinline__ void kick_one(ObjDev& P, const GeoSetDev& G, double3 g, double h, int i)
{
    const int gi = P.geo[i];
    const FdGeo& geo = G.geo[gi];
    const double invM = geo.inv_mass;
    if (fd_is_zero(invM)) return;
    P.vel[i] = P.vel[i] + (P.force[i] * invM + g) * h;
    const double3 w = P.angvel[i];
    const fd_quat q = P.q[i];
    const double3 Iw = fd_smv(fd_rot_tensor(q, geo.inertia), w);
    P.angvel[i] = w + fd_smv(fd_rot_tensor(q, geo.inv_inertia), P.torque[i] - cross3(w, Iw)) * h;
}

__global__ void k_kick(ObjDev P, GeoSetDev G, double3 g, double h)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    kick_one(P, G, g, h, i);
}

__device__ __forceinline__ fd_quat quat_integrate(fd_quat q, double3 w, double dt)
{
    const double3 v = w * (0.5 * dt);
    fd_quat d;
    d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
    d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
    d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
    d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
    fd_quat s = {q.q0 + d.q0, q.q1 + d.q1, q.q2 + d.q2, q.q3 + d.q3};
    return fd_normalize_q(s);
}

__device__ __forceinline__ void drift_one(ObjDev& O, double dt, int i)
{
    O.pos[i] = O.pos[i] + dt * O.vel[i];
    O.q[i] = quat_integrate(O.q[i], O.angvel[i], dt);
}

__global__ void k_drift(ObjDev O, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O.n) return;
    drift_one(O, dt, i);
}

// the second half kick of one step, then the first half kick and the drift
// of the next (no force is computed between them): one pass over the state
// instead of three, each half kick the same arithmetic as k_kick's
__global__ void k_kick_drift(ObjDev P, GeoSetDev G, double3 g, double h, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    kick_one(P, G, g, h, i);
    kick_one(P, G, g, h, i);
    drift_one(P, dt, i);
}

// ---------------------------------------------------------------------------
// hashing and the dense cell table (counting sort)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void quat_matrix(const fd_quat q, double R[9])
{
    const double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
    R[0] = 1.0 - 2.0 * (q2 * q2 + q3 * q3); R[1] = 2.0 * (q1 * q2 - q0 * q3); R[2] = 2.0 * (q1 * q3 + q0 * q2);
    R[3] = 2.0 * (q1 * q2 + q0 * q3); R[4] = 1.0 - 2.0 * (q1 * q1 + q3 * q3); R[5] = 2.0 * (q2 * q3 - q0 * q1);
    R[6] = 2.0 * (q1 * q3 - q0 * q2); R[7] = 2.0 * (q2 * q3 + q0 * q1); R[8] = 1.0 - 2.0 * (q1 * q1 + q2 * q2);
}

__global__ void k_hash(ObjDev O, FdGrid g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= O.n) return;
    const long long h = fd_hash(O.pos[i], g);
    O.hash[i] = h;
    if (O.rot) {
        double R[9];
        quat_matrix(O.q[i], R);
        O.rot[3 * i + 0] = make_float4((float)R[0], (float)R[1], (float)R[2], 0.f);
        O.rot[3 * i + 1] = make_float4((float)R[3], (float)R[4], (float)R[5], 0.f);
        O.rot[3 * i + 2] = make_float4((float)R[6], (float)R[7], (float)R[8], 0.f);
    }
}

// ---------------------------------------------------------------------------
// stable LSD radix sort of 64-bit cell keys, 8 bits per pass over the bits a
// key can use: per block a digit histogram, an exclusive scan of the counts
// (digit-major, so equal digits keep block order), then a scatter that ranks
// each key within its block by warp (match of equal digits) and by lane
// ---------------------------------------------------------------------------
constexpr int RS_TPB = 256;
constexpr int RS_RADIX = 256;
constexpr unsigned long long RS_NONE = ~0ull;  // key of an object in no cell

__global__ void k_rs_keys(const long long* hash, int n, long long num, unsigned long long* key, int* idx,
                          const int* gate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    const long long h = hash[i];
    key[i] = (h >= 0 && h < num) ? (unsigned long long)h : RS_NONE;
    idx[i] = i;
}

__global__ void __launch_bounds__(RS_TPB) k_rs_hist(const unsigned long long* key, int n, int shift, int* bcount,
                                                   int nblk, const int* gate)
{
    if (gate && *gate == 0) return;
    __shared__ int h[RS_RADIX];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * RS_TPB + threadIdx.x;
    if (i < n) atomicAdd(&h[(key[i] >> shift) & (RS_RADIX - 1)], 1);
    __syncthreads();
    bcount[(long long)threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(RS_TPB) k_rs_scatter(const unsigned long long* key, const int* idx, int n, int shift,
                                                      const int* boff, int nblk, unsigned long long* okey, int* oidx,
                                                      const int* gate)
{
    if (gate && *gate == 0) return;
    constexpr int NW = RS_TPB / 32;
    __shared__ int wcnt[NW][RS_RADIX];
    for (int d = threadIdx.x; d < NW * RS_RADIX; d += RS_TPB) (&wcnt[0][0])[d] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.x * RS_TPB + threadIdx.x;
    const bool valid = i < n;
    const unsigned long long k = valid ? key[i] : 0ull;
    const int digit = valid ? (int)((k >> shift) & (RS_RADIX - 1)) : RS_RADIX;
    const unsigned int peers = __match_any_sync(0xffffffffu, digit);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && lane == __ffs(peers) - 1) wcnt[w][digit] = __popc(peers);
    __syncthreads();
    if (valid) {
        int pos = boff[(long long)digit * nblk + blockIdx.x] + rank;
        for (int v = 0; v < w; ++v) pos += wcnt[v][digit];
        okey[pos] = k;
        oidx[pos] = idx[i];
    }
}

// dense table: objects per cell (atomic count), slots by an atomic scatter,
// then each cell's slots put in ascending object index, so the table equals
// the one a stable sort of the hashes gives
__global__ void k_clear_cells(int* a, int* b, long long n, const int* gate)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    a[i] = 0;
    b[i] = 0;
}
__global__ void k_cell_count(const long long* hash, int n, long long num, int* count, const int* gate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    const long long h = hash[i];
    if (h >= 0 && h < num) atomicAdd(&count[h], 1);
}
__global__ void k_cell_scatter(const long long* hash, int n, long long num, const int* start, int* fill, int* sorted,
                               const int* gate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    const long long h = hash[i];
    if (h < 0 || h >= num) return;
    sorted[start[h] + atomicAdd(&fill[h], 1)] = i;
}
__global__ void k_cell_order(long long num, const int* count, const int* start, int* sorted, const int* gate)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= num || (gate && *gate == 0)) return;
    const int m = count[c];
    if (m < 2) return;
    int* seg = sorted + start[c];
    for (int a = 1; a < m; ++a) {
        const int v = seg[a];
        int b = a - 1;
        while (b >= 0 && seg[b] > v) {
            seg[b + 1] = seg[b];
            --b;
        }
        seg[b + 1] = v;
    }
}

__global__ void k_hkey_clear(unsigned long long* hkey, unsigned long long n, const int* gate)
{
    const unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    hkey[i] = RS_NONE;
}

__device__ __forceinline__ unsigned long long cell_slot_hash(unsigned long long k)
{
    // splitmix64 finaliser
    k ^= k >> 30;
    k *= 0xbf58476d1ce4e5b9ull;
    k ^= k >> 27;
    k *= 0x94d049bb133111ebull;
    k ^= k >> 31;
    return k;
}

__global__ void k_cells_hashed(const unsigned long long* key, int n, long long num, unsigned long long* hkey,
                               int2* hval, unsigned long long hmask, unsigned int* flags, const int* gate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (gate && *gate == 0)) return;
    const unsigned long long k = key[i];
    if (k >= (unsigned long long)num || (i > 0 && key[i - 1] == k)) return;
    int e = i + 1;
    while (e < n && key[e] == k) ++e;
    unsigned long long slot = cell_slot_hash(k) & hmask;
    // the table holds at least twice as many slots as there are objects, so
    // an empty slot is always found; the probe count is bounded all the same
    for (unsigned long long probe = 0; probe <= hmask; ++probe) {
        const unsigned long long prev = atomicCAS(&hkey[slot], RS_NONE, k);
        if (prev == RS_NONE || prev == k) {
            hval[slot] = make_int2(i, e - i);
            return;
        }
        slot = (slot + 1) & hmask;
    }
    set_flag(flags, FD_FLAG_INDEX);
}

// objects in cell h: their count, and the first of their slots in *first
__device__ __forceinline__ int cell_lookup(const CellTableDev& T, long long h, int& first)
{
    if (!T.hashed) {
        const int c = T.count[h];
        if (c) first = T.start[h];
        return c;
    }
    const unsigned long long k = (unsigned long long)h;
    unsigned long long slot = cell_slot_hash(k) & T.hmask;
    for (unsigned long long probe = 0; probe <= T.hmask; ++probe) {
        const unsigned long long kk = T.hkey[slot];
        if (kk == k) {
            const int2 v = T.hval[slot];
            first = v.x;
            return v.y;
        }
        if (kk == RS_NONE) return 0;
        slot = (slot + 1) & T.hmask;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// periodic wrap and ghosts, mySpatialGrid.cu:28-56, 87-152, 214-240
// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 wrap_x(double3 p, const FdGrid& g)
{
    const double3 off = mk3(g.maxb.x - g.minb.x, 0., 0.);
    if (p.x < g.minb.x) p = p + off;
    else if (p.x >= g.maxb.x) p = p - off;
    return p;
}
__device__ __forceinline__ double3 wrap_y(double3 p, const FdGrid& g)
{
    const double3 off = mk3(0., g.maxb.y - g.minb.y, 0.);
    if (p.y < g.minb.y) p = p + off;
    else if (p.y >= g.maxb.y) p = p - off;
    return p;
}

// periodic shifts of the force-side centres ri, rj against the detection-side
// cA, cB (-1, 0 or 1 period per axis), as one code for the adjoint's record
__device__ __forceinline__ int wrap_code(double3 cA, double3 ri, double3 cB, double3 rj, const FdGrid& g)
{
    const double Lx = g.maxb.x - g.minb.x, Ly = g.maxb.y - g.minb.y;
    auto sh = [](double d, double L) { return d > 0.5 * L ? 1 : (d < -0.5 * L ? -1 : 0); };
    return (sh(ri.x - cA.x, Lx) + 1) + 3 * (sh(ri.y - cA.y, Ly) + 1) + 9 * (sh(rj.x - cB.x, Lx) + 1) +
           27 * (sh(rj.y - cB.y, Ly) + 1);
}

__global__ void k_wrap(ObjDev P, FdGrid g, int dim, int* ctrl, const double3* src)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const double3 p0 = src ? src[i] : P.pos[i];
    const double3 p1 = dim == 0 ? wrap_x(p0, g) : wrap_y(p0, g);
    P.pos[i] = p1;
    // under the pair cache a wrap changes which particles have images: the
    // ghost lists of this step are built afresh, and every list at the next
    if (ctrl && (p1.x != p0.x || p1.y != p0.y)) {
        ctrl[4] = 1;
        ctrl[7] = 1;
    }
}

// calculateGhostHashKernel, including its z test against maxBound.y (:236):
// an image outside the domain is hashed into the clamped boundary cell, an
// image inside it is not a ghost
// Returns the directions (bit 0 x, 1 y, 2 z) in which the image lies
// outside the domain.
__device__ __forceinline__ int image_hash(GhostDev& Gh, int i, double3 r)
{
    const FdGrid& g = Gh.cells.g;
    int3 gc = fd_cell_of(r, g);
    int outm = 0;
    if (r.x < g.minb.x) { gc.x = 0; outm |= 1; }
    else if (r.x >= g.maxb.x) { gc.x = g.size.x - 1; outm |= 1; }
    if (r.y < g.minb.y) { gc.y = 0; outm |= 2; }
    else if (r.y >= g.maxb.y) { gc.y = g.size.y - 1; outm |= 2; }
    if (r.z < g.minb.z) { gc.z = 0; outm |= 4; }
    else if (r.z >= g.maxb.y) { gc.z = g.size.z - 1; outm |= 4; }
    const bool out = outm != 0;
    const long long h = out ? fd_lin3(gc.x, gc.y, gc.z, g.size) : -1;
    Gh.hash[i] = h;
    if (h >= 0 && h < g.num) {
        atomicMin(&Gh.occ[0], gc.x); atomicMin(&Gh.occ[1], gc.y); atomicMin(&Gh.occ[2], gc.z);
        atomicMax(&Gh.occ[3], gc.x); atomicMax(&Gh.occ[4], gc.y); atomicMax(&Gh.occ[5], gc.z);
    }
    return outm;
}

// The image of a particle in the first cell column (row, or both) sits one
// period beyond the domain; every other particle keeps its own position.  A
// particle enters the image table when that position lies outside the
// domain, tested as the reference tests it (z against max y): the shifted
// ones, and unshifted ones above max y.  Gh.live marks these entries.
// Under the pair cache (ctrl non-null) particles without an entry that lie
// within ext_skin of the image band get a shifted entry too, so that a
// rebuild lists the pairs of every particle that can gain an image before
// the next rebuild.
__device__ __forceinline__ int image_out_mask(double3 r, const FdGrid& g)
{
    int m = 0;
    if (r.x < g.minb.x || r.x >= g.maxb.x) m |= 1;
    if (r.y < g.minb.y || r.y >= g.maxb.y) m |= 2;
    if (r.z < g.minb.z || r.z >= g.maxb.y) m |= 4;
    return m;
}
__global__ void k_ghost_build(ObjDev P, GhostDev Gh, int kind, double ext_skin, int* ctrl)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const FdGrid& g = Gh.cells.g;
    const double3 p = P.pos[i];
    const double3 ox = mk3(g.maxb.x - g.minb.x, 0., 0.), oy = mk3(0., g.maxb.y - g.minb.y, 0.);
    const double3 shift = kind == FD_GX ? ox : kind == FD_GY ? oy : ox + oy;
    const int3 c = fd_cell_of(p, g);
    bool shifted = false;
    if (kind == FD_GX) shifted = c.x == 0;
    if (kind == FD_GY) shifted = c.y == 0;
    if (kind == FD_GXY) shifted = c.x == 0 && c.y == 0;
    const double3 ru = shifted ? p + shift : p;
    const bool live = image_out_mask(ru, g) != 0;
    bool band = false;
    if (ctrl && !live) {
        const bool bx = (p.x - g.minb.x) * g.inv.x < 1.0 + ext_skin * g.inv.x * 1.01;
        const bool by = (p.y - g.minb.y) * g.inv.y < 1.0 + ext_skin * g.inv.y * 1.01;
        if (kind == FD_GX) band = bx;
        if (kind == FD_GY) band = by;
        if (kind == FD_GXY) band = bx && by;
    }
    const double3 r = live ? ru : band ? p + shift : p;
    Gh.pos[i] = r;
    if (Gh.live) Gh.live[i] = live ? 1 : 0;
    const int outm = image_hash(Gh, i, r);
    if (ctrl && (live || band)) {
        // outside the domain across the translation only: its cell is the
        // natural one in the other directions, and candidacy follows the
        // geometry; otherwise (a clamped cell) this step is built uncached
        const int along = kind == FD_GX ? 1 : kind == FD_GY ? 2 : 3;
        if (outm & ~along) {
            ctrl[4] = 1;
            ctrl[7] = 1;
        }
    }
}

__global__ void k_ghost_gate(int* ctrl)
{
    ctrl[5] = (ctrl[0] != 0 || ctrl[4] != 0) ? 1 : 0;
    ctrl[6] = ctrl[4];
}

// end of a cached step
struct CachedCounts {
    int* n_pairs[4];
    int* n_slots[4];
    int cap_pairs[4];
    int cap_contacts[4];
    int n;
};
// a build of the particle-wall or ghost lists that overflowed is not kept
__global__ void k_pc_end(int* ctrl, CachedCounts gc)
{
    for (int k = 0; k < gc.n; ++k)
        if (*gc.n_pairs[k] > gc.cap_pairs[k] || *gc.n_slots[k] > gc.cap_contacts[k]) ctrl[7] = 1;
    ctrl[3] = ctrl[7];
    ctrl[7] = 0;
    ctrl[0] = 0;
    ctrl[4] = 0;
    ctrl[5] = 0;
    ctrl[6] = 0;
}

// ---------------------------------------------------------------------------
// sector periodicity, mySpatialGrid.cu:58-85, 154-213 (PeriodicBoundary.h:
// 319-425): the quarter sector x >= min.x, y >= min.y repeats under quarter
// turns about the z axis through the domain's min corner
// ---------------------------------------------------------------------------
// rotateVector, myVec.h:143-182 (device branch): v turned by the angle |om|
// about om, v + (sin t / t) om x v + ((1 - cos t) / t^2) om x (om x v)
__device__ __forceinline__ double3 turn_vec(double3 v, double3 om)
{
    const double th2 = dot3(om, om);
    if (fd_is_zero(th2)) {
        const double3 oxv = cross3(om, v), oo = cross3(om, oxv);
        return v + oxv + 0.5 * oo;
    }
    const double inv = rsqrt(th2);
    const double th = th2 * inv;
    double sn, cs;
    sincos(th, &sn, &cs);
    const double A = sn * inv, B = (1.0 - cs) * (inv * inv);
    const double3 oxv = cross3(om, v), oo = cross3(om, oxv);
    return v + A * oxv + B * oo;
}
// rotateQuaternion, myQua.h:131-180: the turn about om times q, normalised
__device__ __forceinline__ fd_quat turn_quat(fd_quat q, double3 om)
{
    const double th2 = om.x * om.x + om.y * om.y + om.z * om.z;
    if (fd_is_zero(th2)) return q;
    const double th = sqrt(th2);
    const double inv = 1.0 / th;
    const double ux = om.x * inv, uy = om.y * inv, uz = om.z * inv;
    const double half = 0.5 * th;
    const double c = cos(half), sn = sin(half);
    const double r0 = c, r1 = sn * ux, r2 = sn * uy, r3 = sn * uz;
    fd_quat o;
    o.q0 = r0 * q.q0 - r1 * q.q1 - r2 * q.q2 - r3 * q.q3;
    o.q1 = r0 * q.q1 + r1 * q.q0 + r2 * q.q3 - r3 * q.q2;
    o.q2 = r0 * q.q2 - r1 * q.q3 + r2 * q.q0 + r3 * q.q1;
    o.q3 = r0 * q.q3 + r1 * q.q2 - r2 * q.q1 + r3 * q.q0;
    return fd_normalize_q(o);
}
// velocity, position about the min corner and orientation turned by a about z
__device__ __forceinline__ void sector_turn(double3& v, double3& p, fd_quat& q, double3 mn, double a)
{
    const double3 om = mk3(0., 0., a);
    v = turn_vec(v, om);
    p = mn + turn_vec(p - mn, om);
    q = turn_quat(q, om);
}

// position and velocity of a body as the sector wrap of this step leaves
// them: the reference computes particle and wall contact forces after that
// wrap from contacts detected before it, so the force side of those contacts
// sees the turned body
__device__ __forceinline__ void sector_fold(double3& p, double3& v, double3 mn)
{
    if (p.x < mn.x && p.y >= mn.y) {
        const double3 om = mk3(0., 0., -0.5 * PI_D);
        v = turn_vec(v, om);
        p = mn + turn_vec(p - mn, om);
    }
    if (p.y < mn.y && p.x >= mn.x) {
        const double3 om = mk3(0., 0., 0.5 * PI_D);
        v = turn_vec(v, om);
        p = mn + turn_vec(p - mn, om);
    }
}

// a body that left through the x face comes back through the y face turned
// by -90 degrees, and one that left through the y face by +90 degrees
__global__ void k_sector_wrap(ObjDev P, double3 mn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    double3 v = P.vel[i], p = P.pos[i];
    fd_quat q = P.q[i];
    bool turned = false;
    if (p.x < mn.x && p.y >= mn.y) { sector_turn(v, p, q, mn, -0.5 * PI_D); turned = true; }
    if (p.y < mn.y && p.x >= mn.x) { sector_turn(v, p, q, mn, 0.5 * PI_D); turned = true; }
    P.vel[i] = v;
    P.pos[i] = p;
    P.q[i] = q;
    if (turned && P.rot) {
        // the single-precision rotation rows of this step follow the turn
        double R[9];
        quat_matrix(q, R);
        P.rot[3 * i + 0] = make_float4((float)R[0], (float)R[1], (float)R[2], 0.f);
        P.rot[3 * i + 1] = make_float4((float)R[3], (float)R[4], (float)R[5], 0.f);
        P.rot[3 * i + 2] = make_float4((float)R[6], (float)R[7], (float)R[8], 0.f);
    }
}

__device__ __forceinline__ void image_store(GhostDev& Gh, int i, double3 p, double3 v, fd_quat q)
{
    Gh.pos[i] = p;
    Gh.vel[i] = v;
    Gh.q[i] = q;
    double R[9];
    quat_matrix(q, R);
    Gh.rot[3 * i + 0] = make_float4((float)R[0], (float)R[1], (float)R[2], 0.f);
    Gh.rot[3 * i + 1] = make_float4((float)R[3], (float)R[4], (float)R[5], 0.f);
    Gh.rot[3 * i + 2] = make_float4((float)R[6], (float)R[7], (float)R[8], 0.f);
    image_hash(Gh, i, p);
}

// images turned by +90 degrees (bodies in the first cell row in y), -90
// degrees (first cell column in x) and 180 degrees (the corner cell); every
// other image is a copy of its body
__global__ void k_sector_images(ObjDev P, GhostDev R90, GhostDev R180, GhostDev R270)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const FdGrid& g = R90.cells.g;
    const double3 p = P.pos[i], v = P.vel[i];
    const fd_quat q = P.q[i];
    const int3 c = fd_cell_of(p, g);
    const bool row0 = c.y == 0, col0 = c.x == 0;
    double3 pa = p, va = v;
    fd_quat qa = q;
    if (row0) sector_turn(va, pa, qa, g.minb, 0.5 * PI_D);
    image_store(R90, i, pa, va, qa);
    pa = p; va = v; qa = q;
    if (row0 && col0) sector_turn(va, pa, qa, g.minb, PI_D);
    image_store(R180, i, pa, va, qa);
    pa = p; va = v; qa = q;
    if (col0) sector_turn(va, pa, qa, g.minb, -0.5 * PI_D);
    image_store(R270, i, pa, va, qa);
}

// ---------------------------------------------------------------------------
// broad phase
// ---------------------------------------------------------------------------
__device__ __forceinline__ int cell_index_clamped(double x, double mn, double inv, int size)
{
    double v = (x - mn) * inv;
    v = fmin(fmax(v, -1.0), (double)size);
    int c = (int)v;
    return c < 0 ? 0 : (c > size - 1 ? size - 1 : c);
}

// cells the nodes of a body of radius r centred at c can search, in grid g
__device__ __forceinline__ void body_search_range(double3 c, double r, const FdGrid& g, int3& lo, int3& hi)
{
    lo.x = max(cell_index_clamped(c.x - r, g.minb.x, g.inv.x, g.size.x) - 1, 0);
    lo.y = max(cell_index_clamped(c.y - r, g.minb.y, g.inv.y, g.size.y) - 1, 0);
    lo.z = max(cell_index_clamped(c.z - r, g.minb.z, g.inv.z, g.size.z) - 1, 0);
    hi.x = min(cell_index_clamped(c.x + r, g.minb.x, g.inv.x, g.size.x) + 1, g.size.x - 1);
    hi.y = min(cell_index_clamped(c.y + r, g.minb.y, g.inv.y, g.size.y) + 1, g.size.y - 1);
    hi.z = min(cell_index_clamped(c.z + r, g.minb.z, g.inv.z, g.size.z) + 1, g.size.z - 1);
}

__device__ __forceinline__ void decode_cell(long long h, int3 s, int3& c)
{
    c.x = (int)(h % s.x);
    c.y = (int)((h / s.x) % s.y);
    c.z = (int)(h / ((long long)s.x * s.y));
}

__device__ void emit_pairs(int A, int* buf, int cnt, int total, PairListDev& L, unsigned int* flags)
{
    if (total > MAX_CAND) set_flag(flags, FD_FLAG_NEIGHBOR_OVERFLOW);
    // insertion sort by partner id: deterministic pair order
    for (int a = 1; a < cnt; ++a) {
        const int v = buf[a];
        int b = a - 1;
        while (b >= 0 && buf[b] > v) { buf[b + 1] = buf[b]; --b; }
        buf[b + 1] = v;
    }
    int base = 0;
    if (cnt > 0) base = atomicAdd(L.n_pairs, cnt);
    if (cnt > 0 && base + cnt > L.cap_pairs) {
        set_flag(flags, FD_FLAG_PAIR_OVERFLOW);
        L.seg_off[A] = 0;
        L.seg_cnt[A] = 0;
        return;
    }
    L.seg_off[A] = base;
    L.seg_cnt[A] = cnt;
    for (int k = 0; k < cnt; ++k) {
        L.pairA[base + k] = A;
        L.pairB[base + k] = buf[k];
    }
}

constexpr double BOUND_REL = 1e-9;

// True when no point within `radius` of p (a position in B's body frame, in
// single precision) can pass the node predicate against B (or, with probe >
// 0, come within `probe` of B).  Conservative: single-precision evaluation
// with relative margins far above its rounding (about 1e-7 relative), bounds
// that hold in exact arithmetic:
//   * B's bounding sphere (particle pairs: the reference's radius test),
//   * B's SDF grid box (nodes outside it are never contacts),
//   * D(v): lower bound on the distance from grid node v to any cell whose
//     corner minimum is <= 0, 1-Lipschitz in the position,
//   * the Lipschitz bound of the trilinear SDF (distance-like fields).
__device__ __forceinline__ bool sphere_culled(float px, float py, float pz, float radius, bool radius_test,
                                              const FdGeo& GB, const GeoSetDev& SB, double rB, double probe)
{
    const float scale = (float)rB + radius + (float)GB.spacing;
    const float margin = 2e-5f * scale;
    const float rho = radius + margin;
    if (radius_test) {
        const float lim = (float)rB + rho;
        if (px * px + py * py + pz * pz > lim * lim) return true;
    }
    const float is = (float)GB.inv_spacing;
    const float gx = (px - (float)GB.origin.x) * is, gy = (py - (float)GB.origin.y) * is,
                gz = (pz - (float)GB.origin.z) * is;
    const float rg = rho * is + 1e-4f;
    if (gx < -rg || gy < -rg || gz < -rg) return true;
    if (gx > GB.size.x - 1 + rg || gy > GB.size.y - 1 + rg || gz > GB.size.z - 1 + rg) return true;
    if (probe == 0.0) {
        const int vx = min(max(__float2int_rn(gx), 0), GB.size.x - 1);
        const int vy = min(max(__float2int_rn(gy), 0), GB.size.y - 1);
        const int vz = min(max(__float2int_rn(gz), 0), GB.size.z - 1);
        const float D = __ldg(SB.dist + GB.dist_off + fd_lin3(vx, vy, vz, GB.size));
        const float sp = (float)GB.spacing;
        const float dx = (gx - vx) * sp, dy = (gy - vy) * sp, dz = (gz - vz) * sp;
        if (D - sqrtf(dx * dx + dy * dy + dz * dz) > rho) return true;
    }
    // the Lipschitz bound only helps where the field is distance-like
    if (GB.lip < 4.0 && gx >= 0.f && gy >= 0.f && gz >= 0.f && gx < GB.size.x - 1 && gy < GB.size.y - 1 &&
        gz < GB.size.z - 1) {
        const int i0 = (int)gx, j0 = (int)gy, k0 = (int)gz;
        const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
        const float* S = SB.sdf32 + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
        const float fx = gx - i0, fy = gy - j0, fz = gz - k0;
        const float c00 = __ldg(S) * (1.f - fx) + __ldg(S + 1) * fx;
        const float c10 = __ldg(S + sx) * (1.f - fx) + __ldg(S + sx + 1) * fx;
        const float c01 = __ldg(S + sxy) * (1.f - fx) + __ldg(S + sxy + 1) * fx;
        const float c11 = __ldg(S + sxy + sx) * (1.f - fx) + __ldg(S + sxy + sx + 1) * fx;
        const float phi = (c00 * (1.f - fy) + c10 * fy) * (1.f - fz) + (c01 * (1.f - fy) + c11 * fy) * fz;
        const float bound = (float)GB.lip * rho + (float)probe;
        if (phi - bound > 1e-5f * (fabsf(phi) + bound + (float)GB.spacing)) return true;
    }
    return false;
}

// Body-level cull of a candidate pair in single precision: A's bounding
// sphere (radius rA about cA) against B, through B's rotation rows
__device__ __forceinline__ bool body_culled32(const double3 cA, double rA, const double3 cB, const float4* RB,
                                              bool radius_test, const FdGeo& GB, const GeoSetDev& SB, double probe)
{
    const float4 b0 = RB[0], b1 = RB[1], b2 = RB[2];
    const float dx = (float)(cA.x - cB.x), dy = (float)(cA.y - cB.y), dz = (float)(cA.z - cB.z);
    const float px = fmaf(b0.x, dx, fmaf(b1.x, dy, b2.x * dz));
    const float py = fmaf(b0.y, dx, fmaf(b1.y, dy, b2.y * dz));
    const float pz = fmaf(b0.z, dx, fmaf(b1.z, dy, b2.z * dz));
    return sphere_culled(px, py, pz, (float)rA, radius_test, GB, SB, GB.radius, probe);
}

// cells that can hold the centre of a partner of a body of radius r centred
// at c, when partners have radius at most rp: every partner centre within
// r + rp of c lies in a cell overlapping [c - r - rp, c + r + rp]
__device__ __forceinline__ void partner_search_range(double3 c, double reach, const FdGrid& g, int3& lo, int3& hi)
{
    lo.x = cell_index_clamped(c.x - reach, g.minb.x, g.inv.x, g.size.x);
    lo.y = cell_index_clamped(c.y - reach, g.minb.y, g.inv.y, g.size.y);
    lo.z = cell_index_clamped(c.z - reach, g.minb.z, g.inv.z, g.size.z);
    hi.x = cell_index_clamped(c.x + reach, g.minb.x, g.inv.x, g.size.x);
    hi.y = cell_index_clamped(c.y + reach, g.minb.y, g.inv.y, g.size.y);
    hi.z = cell_index_clamped(c.z + reach, g.minb.z, g.inv.z, g.size.z);
}

// The cells a body's ghost search covers: those within `reach` of its
// centre, and every cell next to a cell its nodes (within rA of the centre)
// can occupy.  The predicate takes an image as a candidate of a node when the
// image's cell is next to the node's (LSParticleContactDetectionKernel.cu:
// 431-607); an image outside the domain in y or z sits in a clamped cell
// (mySpatialGrid.cu:214-240) that its position does not reach, and only the
// node neighbourhoods find it.
__device__ __forceinline__ void ghost_search_range(double3 c, double rA, double reach, const FdGrid& g, int3& lo,
                                                   int3& hi)
{
    partner_search_range(c, reach, g, lo, hi);
    int3 blo, bhi;
    body_search_range(c, rA, g, blo, bhi);
    lo = make_int3(min(lo.x, blo.x), min(lo.y, blo.y), min(lo.z, blo.z));
    hi = make_int3(max(hi.x, bhi.x), max(hi.y, bhi.y), max(hi.z, bhi.z));
}

#ifndef FD_BROAD_LANES
#define FD_BROAD_LANES 8
#endif
constexpr int BROAD_LANES = FD_BROAD_LANES;  // lanes per particle in the cell-table broad phases
constexpr int BROAD_CAND = 128;              // candidate slots staged per lane group and pass

// d with its periodic components taken to the nearest image
__device__ __forceinline__ double3 nl_min_image(double3 d, const NlDev& nl, const FdGrid& g)
{
    if (nl.periodic_x) {
        const double L = g.maxb.x - g.minb.x;
        d.x -= L * rint(d.x / L);
    }
    if (nl.periodic_y) {
        const double L = g.maxb.y - g.minb.y;
        d.y -= L * rint(d.y / L);
    }
    return d;
}

// Cell-table broad phase, BROAD_LANES lanes per particle A: the lanes read
// the cells around A, share out the objects in them, test each (partner
// order B > A for particle pairs, bounding spheres, body-level cull) and
// emit A's pairs sorted by partner id.  GHOST: partners are the ghost images
// of a cell table built from ghost positions (no B > A rule; the reach is the
// partner's SDF grid radius, since ghost pairs have no radius test).
//
// LIST: only the particles in alist[0 .. *acount) search (the ghost phases
// list the particles whose search box reaches a ghost image; the others
// were given empty segments by k_ghost_searchers).
//
// NLB: build the neighbour list instead of the pairs (only when a rebuild
// was requested): the sphere test is widened by the skin, the body-level
// cull is left to the per-step filter, and each particle's partners go to its
// fixed slice of the list.
//
// skin (pair cache): partners within rA + rB + skin are listed and the
// body-level cull treats A's sphere as skin larger; gate: the kernel runs
// only when *gate != 0 (null: always).
template <bool GHOST, bool LIST, bool NLB>
__global__ void __launch_bounds__(TPB) k_broad_cells(ObjDev P, GeoSetDev G, CellTableDev T, const double3* gpos,
                                                     const float4* grot, const int* occ, const int* alist, const int* acount,
                                                     PairListDev L, NlDev nl, unsigned int* flags, double probe,
                                                     double skin, const int* gate, const int* noskin)
{
    if (gate && *gate == 0) return;
    if (noskin && *noskin) skin = 0.0;
    if (NLB && nl.ctrl[0] == 0) return;
    __shared__ int s_list[TPB / BROAD_LANES][MAX_CAND];
    __shared__ int s_cand[TPB / BROAD_LANES][BROAD_CAND];
    const unsigned int full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int gl = lane & (BROAD_LANES - 1);
    const int gbase = lane & ~(BROAD_LANES - 1);
    const int gb = threadIdx.x / BROAD_LANES;
    constexpr int GPW = 32 / BROAD_LANES;           // lane groups per warp
    constexpr int GPB = TPB / BROAD_LANES;          // lane groups per block
    const int total = LIST ? *acount : P.n;
    // warp-uniform loop over the warp's groups
    for (int gw = blockIdx.x * GPB + (gb & ~(GPW - 1)); gw < total; gw += gridDim.x * GPB) {
    const int gidx = gw + (gb & (GPW - 1));
    const bool valid = gidx < total;
    const int A = valid ? (LIST ? alist[gidx] : gidx) : 0;
    double3 cA = mk3(0., 0., 0.);
    double rA = 0.;
    int3 lo = make_int3(0, 0, 0), hi = make_int3(-1, -1, -1);
    if (valid) {
        cA = P.pos[A];
        rA = G.geo[P.geo[A]].radius;
        // above the sphere test's own tolerance (rs * (1 + 2 BOUND_REL))
        const double reach = (rA + (GHOST ? G.grid_rmax : G.rmax)) * (1.0 + 8.0 * BOUND_REL) + (NLB ? nl.skin : skin);
        if (NLB && gl == 0) {
            nl.ref[A] = cA;
            nl.vis[A] = P.hash[A] >= 0;
        }
        if (GHOST) {
            ghost_search_range(cA, rA * (1.0 + 8.0 * BOUND_REL) + skin, reach, T.g, lo, hi);
        } else {
            partner_search_range(cA, reach, T.g, lo, hi);
        }
        if (occ) {
            // only the cells that hold ghost images
            lo.x = max(lo.x, occ[0]); lo.y = max(lo.y, occ[1]); lo.z = max(lo.z, occ[2]);
            hi.x = min(hi.x, occ[3]); hi.y = min(hi.y, occ[4]); hi.z = min(hi.z, occ[5]);
        }
    }
    const int nx = max(hi.x - lo.x + 1, 0), ny = max(hi.y - lo.y + 1, 0), nz = max(hi.z - lo.z + 1, 0);
    const int ncell = nx * ny * nz;
    const int ncell_max = __reduce_max_sync(full, ncell);
    int cnt = 0;  // partners that passed (uniform over the lane group)
    for (int c0 = 0; c0 < ncell_max; c0 += BROAD_LANES) {
        int cc = 0, cs = 0;
        const int ci = c0 + gl;
        if (ci < ncell) {
            const int x = lo.x + ci % nx, y = lo.y + (ci / nx) % ny;
            const int z = lo.z + ci / (nx * ny);
            const long long h = fd_lin3(x, y, z, T.g.size);
            cc = cell_lookup(T, h, cs);
        }
        // exclusive scan of the cell counts over the lane group
        int incl = cc;
#pragma unroll
        for (int d = 1; d < BROAD_LANES; d <<= 1) {
            const int y = __shfl_up_sync(full, incl, d, BROAD_LANES);
            if (gl >= d) incl += y;
        }
        const int ex = incl - cc;
        const int tot = __shfl_sync(full, incl, BROAD_LANES - 1, BROAD_LANES);
        const int tot_max = __reduce_max_sync(full, tot);
        for (int f0 = 0; f0 < tot_max; f0 += BROAD_LANES) {
            // stage the table slots of the next BROAD_CAND candidates
            if (f0 % BROAD_CAND == 0) {
                __syncwarp();
                for (int t = max(ex, f0); t < min(ex + cc, f0 + BROAD_CAND); ++t) s_cand[gb][t - f0] = cs + (t - ex);
                __syncwarp();
            }
            const int f = f0 + gl;
            bool pass = false;
            int B = -1;
            if (valid && f < tot) {
                B = T.sorted[s_cand[gb][f % BROAD_CAND]];
                if (GHOST || B > A) {
                    const FdGeo& GB = G.geo[P.geo[B]];
                    const double3 cB = GHOST ? gpos[B] : P.pos[B];
                    if (NLB) {
                        const double rs = (rA + GB.radius) * (1.0 + 8.0 * BOUND_REL) + nl.skin;
                        pass = lengthSq3(nl_min_image(cA - cB, nl, T.g)) <= rs * rs;
                    } else {
                        const double rs = rA + (GHOST ? GB.grid_radius : GB.radius) + skin;
                        if (lengthSq3(cA - cB) <= rs * rs * (1.0 + 4.0 * BOUND_REL))
                            pass = !body_culled32(cA, rA + skin, cB, (GHOST && grot ? grot : P.rot) + 3ll * B,
                                                  !GHOST, GB, G, probe);
                    }
                }
            }
            const unsigned int gm = (__ballot_sync(full, pass) >> gbase) & ((1u << BROAD_LANES) - 1u);
            if (pass) {
                const int pos = cnt + __popc(gm & ((1u << gl) - 1u));
                if (pos < MAX_CAND) s_list[gb][pos] = B;
            }
            cnt += __popc(gm);
        }
    }
    __syncwarp();
    if (valid && cnt > MAX_CAND && gl == 0) set_flag(flags, FD_FLAG_NEIGHBOR_OVERFLOW);
    const int n = min(cnt, MAX_CAND);
    if (NLB) {
        static_assert(NL_MAX >= MAX_CAND, "a list slice holds every partner");
        if (valid) {
            for (int e = gl; e < n; e += BROAD_LANES) {
                const int v = s_list[gb][e];
                int r = 0;
                for (int j = 0; j < n; ++j) r += (s_list[gb][j] < v);
                nl.list[(long long)A * NL_MAX + r] = v;
            }
            if (gl == 0) nl.cnt[A] = n;
        }
        __syncwarp();
        continue;
    }
    int base = 0;
    if (valid && gl == 0 && n > 0) base = atomicAdd(L.n_pairs, n);
    base = __shfl_sync(full, base, 0, BROAD_LANES);
    const bool ok = base + n <= L.cap_pairs;
    if (valid && n > 0 && !ok && gl == 0) set_flag(flags, FD_FLAG_PAIR_OVERFLOW);
    if (valid && gl == 0) {
        L.seg_off[A] = (ok && n > 0) ? base : 0;
        L.seg_cnt[A] = ok ? n : 0;
    }
    // pairs of A in ascending partner order (partners are distinct)
    if (valid && ok) {
        for (int e = gl; e < n; e += BROAD_LANES) {
            const int v = s_list[gb][e];
            int r = 0;
            for (int j = 0; j < n; ++j) r += (s_list[gb][j] < v);
            L.pairA[base + r] = A;
            L.pairB[base + r] = v;
        }
    }
    __syncwarp();
    }
}

// neighbour list: request a rebuild when a particle moved more than skin / 2
// since the last build or changed visibility
__global__ void k_nl_check(ObjDev P, NlDev nl, FdGrid g, const int* gate)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || (gate && *gate == 0)) return;
    // with the pair cache, partners within rA + rB + pair_skin must stay
    // listed: the list is rebuilt before any particle moves (skin - pair_skin) / 2
    const double h = 0.5 * (nl.skin - nl.pair_skin);
    const bool moved = lengthSq3(nl_min_image(P.pos[i] - nl.ref[i], nl, g)) > h * h;
    const bool vis = P.hash[i] >= 0;
    if (moved || vis != (nl.vis[i] != 0)) nl.ctrl[0] = 1;
}

// the pairs from the neighbour list: the exact sphere test and the
// body-level cull of the cell search, on the listed partners (ascending, so
// each particle's pairs come out in partner order)
__global__ void __launch_bounds__(TPB) k_nl_filter(ObjDev P, GeoSetDev G, PairListDev L, NlDev nl,
                                                   unsigned int* flags, double probe, const int* gate)
{
    if (gate && *gate == 0) return;
    constexpr int LN = 8;  // lanes per particle
    const unsigned int full = 0xffffffffu;
    const int lane = threadIdx.x & 31, gl = lane & (LN - 1), gbase = lane & ~(LN - 1);
    const int A = (blockIdx.x * blockDim.x + threadIdx.x) / LN;
    const bool valid = A < P.n;
    double3 cA = mk3(0., 0., 0.);
    double rA = 0.;
    int cnt = 0;
    if (valid) {
        cA = P.pos[A];
        rA = G.geo[P.geo[A]].radius;
        cnt = nl.cnt[A];
    }
    const int cmax = __reduce_max_sync(full, cnt);
    // two passes: count the partners that pass, then write them in order
    unsigned long long passed = 0ull;  // bit e: entry e passed (entries < NL_MAX)
    for (int e0 = 0; e0 < cmax; e0 += LN) {
        const int e = e0 + gl;
        bool pass = false;
        if (valid && e < cnt) {
            const int B = nl.list[(long long)A * NL_MAX + e];
            if (P.hash[B] >= 0) {
                const FdGeo& GB = G.geo[P.geo[B]];
                const double3 cB = P.pos[B];
                const double rs = rA + GB.radius + nl.pair_skin;
                if (lengthSq3(cA - cB) <= rs * rs * (1.0 + 4.0 * BOUND_REL))
                    pass = !body_culled32(cA, rA + nl.pair_skin, cB, P.rot + 3ll * B, true, GB, G, probe);
            }
        }
        const unsigned int gm = (__ballot_sync(full, pass) >> gbase) & ((1u << LN) - 1u);
        passed |= (unsigned long long)gm << e0;
    }
    const int n = __popcll(passed);
    int base = 0;
    if (valid && gl == 0 && n > 0) base = atomicAdd(L.n_pairs, n);
    base = __shfl_sync(full, base, 0, LN);
    const bool ok = base + n <= L.cap_pairs;
    if (valid && n > 0 && !ok && gl == 0) set_flag(flags, FD_FLAG_PAIR_OVERFLOW);
    if (valid && gl == 0) {
        L.seg_off[A] = (ok && n > 0) ? base : 0;
        L.seg_cnt[A] = ok ? n : 0;
    }
    if (valid && ok) {
        for (int e = gl; e < cnt; e += LN) {
            if (!((passed >> e) & 1ull)) continue;
            const int r = __popcll(passed & ((1ull << e) - 1ull));
            L.pairA[base + r] = A;
            L.pairB[base + r] = nl.list[(long long)A * NL_MAX + e];
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) nl.ctrl[0] = 0;
}

// ---------------------------------------------------------------------------
// pair cache of the particle-particle list (see PairCacheDev)
// ---------------------------------------------------------------------------
// flag a rebuild when a particle drifted by more than skin / 2 since the last
// build or changed visibility
__global__ void k_pc_check(ObjDev P, PairCacheDev c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const double3 d = P.pos[i] - c.ref_pos[i];
    // 2 sin(theta / 2) = 2 |vector part of q conj(q0)|: the chord a unit
    // lever arm sweeps under the rotation since the build
    const fd_quat q = P.q[i], r = c.ref_q[i];
    const double vx = r.q0 * q.q1 - q.q0 * r.q1 - (q.q2 * r.q3 - q.q3 * r.q2);
    const double vy = r.q0 * q.q2 - q.q0 * r.q2 - (q.q3 * r.q1 - q.q1 * r.q3);
    const double vz = r.q0 * q.q3 - q.q0 * r.q3 - (q.q1 * r.q2 - q.q2 * r.q1);
    const double chord = 2.0 * sqrt(vx * vx + vy * vy + vz * vz);
    const double drift = sqrt(lengthSq3(d)) + c.reach * chord;
    // every particle's bound, for the slot test of the predicate pass
    c.drift[i] = __double2float_ru(drift);
    c.disp[i] = make_float4((float)d.x, (float)d.y, (float)d.z, __double2float_ru(c.reach * chord));
    if (c.ctrl[0] != 0) return;
    if (c.ctrl[2] != 0 || c.ctrl[3] != 0) {
        // the last build overflowed its lists, or the last step asked for a
        // rebuild: build again
        c.ctrl[0] = 1;
        return;
    }
    // a little below skin / 2, so that the two drifts of a pair stay below
    // the single-precision skin the culling stages use
    const bool vis = P.hash[i] >= 0;
    if (!(drift <= 0.5 * c.skin * (1.0 - 1e-6)) || vis != (c.ref_vis[i] != 0)) c.ctrl[0] = 1;
}

// a step without a rebuild: this step's pairs and slots are the previous
// step's, carried over; each pair's history is its own slots of the previous
// step, and its partner's cell is taken from this step's hash
__global__ void k_pc_carry(PairListDev L, int n_obj, const long long* hash, FdGrid g, const int* gate,
                           const float* drift, const float4* disp, const float* driftB, const float4* dispB,
                           const int* geo_of, const FdGeo* geos, float spacing_margin)
{
    if (*gate != 0) return;
    const int npairs = min(L.o_counters[0], L.cap_pairs);
    const int nslots = min(L.o_counters[1], L.cap_contacts);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    // the layout (segments, pairs, slot keys) is copied into the other
    // generation on the first carried step after a build; from the second on
    // both generations hold it already
    const bool copy = L.carry_n == nullptr || *L.carry_n == 0;
    if (t0 == 0) {
        *L.n_pairs = L.o_counters[0];
        *L.n_slots = L.o_counters[1];
    }
    if (copy)
        for (long long i = t0; i < n_obj; i += stride) {
            L.seg_off[i] = L.o_seg_off[i];
            L.seg_cnt[i] = L.o_seg_cnt[i];
        }
    for (long long p = t0; p < npairs; p += stride) {
        const int A = L.o_pairA[p];
        const int B = L.o_pairB[p];
        const int off = L.o_c_off[p], cnt = L.o_c_cnt[p];
        if (copy) {
            L.pairA[p] = A;
            L.pairB[p] = B;
            L.c_off[p] = off;
            L.c_cnt[p] = cnt;
        }
        if (drift && disp && L.p_bound) {
            // the slot bound's right-hand side for the pair (see k_contact):
            // lip_B times how far a node can have moved in B's frame, plus a
            // margin in units of B's grid spacing (the single-precision
            // predicate's rounding).  The node's offset from B's centre moved
            // by at most |dc_A - dc_B| + the two rotation parts (lever arms up
            // to the reach); the displacements are stored in single
            // precision, whose rounding (1e-7 of each) the term
            // 1e-6 (drift_A + drift_B) covers; never more than the sum of
            // the two drift bounds.
            const FdGeo& GB = geos[geo_of[B]];
            const float lip = __double2float_ru(GB.lip);
            const float4 a = disp[A], b = dispB[B];
            const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
            const float dab = __fadd_ru(drift[A], driftB[B]);
            const float rel = __fadd_ru(__fadd_ru(__fsqrt_ru(__fadd_ru(__fadd_ru(__fmul_ru(dx, dx), __fmul_ru(dy, dy)),
                                                                       __fmul_ru(dz, dz))),
                                                  __fadd_ru(a.w, b.w)),
                                        __fmul_ru(1e-6f, dab));
            float bound = __fmul_ru(lip, fminf(rel, dab));
            if (spacing_margin > 0.f)
                bound = __fadd_ru(__fmul_ru(bound, 1.000001f), __fmul_ru(spacing_margin, __double2float_ru(GB.spacing)));
            L.p_bound[p] = bound;
        }
        if (cnt > 0) {
            int3 bc;
            decode_cell(hash[B], g.size, bc);
            L.p_aux[p] = make_int4(bc.x, bc.y, bc.z, off);
            L.p_hist_cnt[p] = cnt;
        }
    }
    if (copy)
        for (long long k = t0; k < nslots; k += stride) L.c_k[k] = L.o_c_k[k];
}

// after the particle-particle narrow phase of a rebuild step: its state is the
// new reference; the flag is cleared for the next step
__global__ void k_pc_commit(ObjDev P, PairCacheDev c, PairListDev L)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n || c.ctrl[0] == 0) return;
    c.ref_pos[i] = P.pos[i];
    c.ref_q[i] = P.q[i];
    c.ref_vis[i] = P.hash[i] >= 0;
    if (i == 0) {
        c.ctrl[1] += 1;
        // a build whose pairs or slots did not fit is not kept: the next
        // step builds again (the host grows the lists at its next check)
        c.ctrl[2] = (*L.n_pairs > L.cap_pairs || *L.n_slots > L.cap_contacts) ? 1 : 0;
    }
}

// walls: the drift bound of each wall since the last build (rotation lever
// arm: its SDF-grid radius, the farthest a node inside its grid can be), and
// a rebuild when it exceeds skin / 2 or the wall's cell changed (the
// particle-wall candidates follow the wall's cell)
__global__ void k_pc_check_walls(ObjDev W, GeoSetDev GW, PairCacheDev c)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= W.n) return;
    const double3 d = W.pos[w] - c.wref_pos[w];
    const fd_quat q = W.q[w], r = c.wref_q[w];
    const double vx = r.q0 * q.q1 - q.q0 * r.q1 - (q.q2 * r.q3 - q.q3 * r.q2);
    const double vy = r.q0 * q.q2 - q.q0 * r.q2 - (q.q3 * r.q1 - q.q1 * r.q3);
    const double vz = r.q0 * q.q3 - q.q0 * r.q3 - (q.q1 * r.q2 - q.q2 * r.q1);
    const double rot = GW.geo[W.geo[w]].grid_radius * 2.0 * sqrt(vx * vx + vy * vy + vz * vz);
    const double drift = sqrt(lengthSq3(d)) + rot;
    c.wdrift[w] = __double2float_ru(drift);
    c.wdisp[w] = make_float4((float)d.x, (float)d.y, (float)d.z, __double2float_ru(rot));
    if (c.ctrl[0] != 0) return;
    if (!(drift <= 0.5 * c.skin * (1.0 - 1e-6)) || W.hash[w] != c.wref_hash[w]) c.ctrl[0] = 1;
}
__global__ void k_pc_commit_walls(ObjDev W, PairCacheDev c)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= W.n || c.ctrl[0] == 0) return;
    c.wref_pos[w] = W.pos[w];
    c.wref_q[w] = W.q[w];
    c.wref_hash[w] = W.hash[w];
}

// ghost phases: particles whose search box reaches the cells holding ghost
// images are listed for k_broad_cells<true, true>; the others get empty
// segments here
__global__ void k_ghost_searchers(ObjDev P, GeoSetDev G, FdGrid g, const int* occ, PairListDev L, int* alist,
                                  int* acount, double skin, const int* gate, const int* noskin)
{
    const int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= P.n || (gate && *gate == 0)) return;
    if (noskin && *noskin) skin = 0.0;
    const double rA = G.geo[P.geo[A]].radius;
    const double reach = (rA + G.grid_rmax) * (1.0 + 8.0 * BOUND_REL) + skin;
    int3 lo, hi;
    ghost_search_range(P.pos[A], rA * (1.0 + 8.0 * BOUND_REL) + skin, reach, g, lo, hi);
    const bool any = max(lo.x, occ[0]) <= min(hi.x, occ[3]) && max(lo.y, occ[1]) <= min(hi.y, occ[4]) &&
                     max(lo.z, occ[2]) <= min(hi.z, occ[5]);
    if (any) {
        alist[atomicAdd(acount, 1)] = A;
    } else {
        L.seg_off[A] = 0;
        L.seg_cnt[A] = 0;
    }
}

// wall_range (null: every wall): per particle, the first wall and the number
// of walls it can meet (the walls of its own simulation in a batch of
// simulations tiled into one)
__global__ void k_broad_pw(ObjDev P, GeoSetDev G, ObjDev W, GeoSetDev GW, FdGrid wg, PairListDev L,
                           unsigned int* flags, double probe, const int2* wall_range, double skin, const int* gate)
{
    const int A = blockIdx.x * blockDim.x + threadIdx.x;
    if (A >= P.n || (gate && *gate == 0)) return;
    const double3 cA = P.pos[A];
    const double rA = G.geo[P.geo[A]].radius;
    int3 lo, hi;
    body_search_range(cA, rA * (1.0 + BOUND_REL) + skin, wg, lo, hi);
    int buf[MAX_CAND];
    int cnt = 0, total = 0;
    const int2 wr = wall_range ? wall_range[A] : make_int2(0, W.n);
    const int wend = min(wr.x + wr.y, W.n);
    for (int w = max(wr.x, 0); w < wend; ++w) {
        const long long h = W.hash[w];
        if (h < 0 || h >= wg.num) continue;
        int3 c;
        decode_cell(h, wg.size, c);
        if (c.x < lo.x || c.x > hi.x || c.y < lo.y || c.y > hi.y || c.z < lo.z || c.z > hi.z) continue;
        const FdGeo& GB = GW.geo[W.geo[w]];
        const double rs = rA + GB.grid_radius + skin;
        const double3 cW = W.pos[w];
        if (lengthSq3(cA - cW) > rs * rs * (1.0 + 4.0 * BOUND_REL)) continue;
        if (body_culled32(cA, rA + skin, cW, W.rot + 3ll * w, false, GB, GW, probe)) continue;
        if (cnt < MAX_CAND) buf[cnt++] = w;
        ++total;
    }
    emit_pairs(A, buf, cnt, total, L, flags);
}

// ---------------------------------------------------------------------------
// contact law, contactKernel.cuh:4-77
// ---------------------------------------------------------------------------
__device__ __forceinline__ double3 sliding_spring(double3 prev, double3 sv, double3 n, double3 fn, double mu,
                                                  double k, double c, double dt)
{
    double3 spring = mk3(0., 0., 0.);
    if (mu > 0. && k > 0.) {
        double3 p1 = prev - dot3(prev, n) * n;
        const double ap1 = length3(p1);
        if (!fd_is_zero(ap1)) p1 = p1 * (length3(prev) / ap1);
        spring = p1 + sv * dt;
        double3 sf = -k * spring - c * sv;
        const double asf = length3(sf);
        const double afn = length3(fn);
        if (!fd_is_zero(asf) && asf > mu * afn) {
            sf = sf * (mu * afn / asf);
            spring = -(sf + c * sv) * (1.0 / k);
        }
    }
    return spring;
}

__device__ __forceinline__ void linear_contact(double3& F, double3& spring, double3 vc, double3 n, double delta,
                                               double dt, double kn, double ks, double mu, double res, double m)
{
    if (delta > 0.) {
        const double lr = log(res);
        const double diss = -lr / (double)sqrtf((float)(lr * lr + PI_D * PI_D));
        const double cn = 2. * diss * (double)sqrtf((float)(m * kn));
        const double3 vn = dot3(vc, n) * n;
        const double3 fn = (kn * delta) * n - cn * vn;
        const double cs = 2. * diss * (double)sqrtf((float)(m * ks));
        const double3 vs = vc - vn;
        spring = sliding_spring(spring, vs, n, fn, mu, ks, cs, dt);
        const double3 fs = -ks * spring - cs * vs;
        F = fn + fs;
    } else {
        spring = mk3(0., 0., 0.);
    }
}

// ---------------------------------------------------------------------------
// narrow phase + force, one warp per candidate pair
// ---------------------------------------------------------------------------
struct NarrowArgs {
    ObjDev P;
    GeoSetDev G;
    MatDev M;
    ObjDev W;
    GeoSetDev GW;
    MatDev MW;
    FdGrid pgrid;
    FdGrid wgrid;
    GhostDev gh;
    PairListDev L;
    StepArgs a;
    int with_force;
};

// the slave side of a pair, by kind
template <int KIND> struct Slave;
template <> struct Slave<FD_PP> {
    __device__ static double3 pos(const NarrowArgs& n, int j) { return n.P.pos[j]; }
    __device__ static double3 vel(const NarrowArgs& n, int j) { return n.P.vel[j]; }
    __device__ static fd_quat q(const NarrowArgs& n, int j) { return n.P.q[j]; }
    __device__ static const float4* rot(const NarrowArgs& n, int j) { return n.P.rot + 3ll * j; }
    __device__ static const FdGeo& geo(const NarrowArgs& n, int j) { return n.G.geo[n.P.geo[j]]; }
    __device__ static const GeoSetDev& set(const NarrowArgs& n) { return n.G; }
    __device__ static long long hash(const NarrowArgs& n, int j) { return n.P.hash[j]; }
    __device__ static const FdGrid& grid(const NarrowArgs& n) { return n.pgrid; }
    static constexpr bool radius_test = true;
};
template <> struct Slave<FD_PW> {
    __device__ static double3 pos(const NarrowArgs& n, int j) { return n.W.pos[j]; }
    __device__ static double3 vel(const NarrowArgs& n, int j) { return n.W.vel[j]; }
    __device__ static fd_quat q(const NarrowArgs& n, int j) { return n.W.q[j]; }
    __device__ static const float4* rot(const NarrowArgs& n, int j) { return n.W.rot + 3ll * j; }
    __device__ static const FdGeo& geo(const NarrowArgs& n, int j) { return n.GW.geo[n.W.geo[j]]; }
    __device__ static const GeoSetDev& set(const NarrowArgs& n) { return n.GW; }
    __device__ static long long hash(const NarrowArgs& n, int j) { return n.W.hash[j]; }
    __device__ static const FdGrid& grid(const NarrowArgs& n) { return n.wgrid; }
    static constexpr bool radius_test = false;
};
// ghost images: translated images share their body's orientation and
// velocity; sector images carry their own.  The angular velocity is always
// the body's own, as in addGhostLevelSetParticleContactForceTorqueKernel
// (contactKernel.cu:262), which does not turn it with the image.
struct SlaveGhost {
    __device__ static double3 pos(const NarrowArgs& n, int j) { return n.gh.pos[j]; }
    __device__ static double3 vel(const NarrowArgs& n, int j) { return n.gh.vel ? n.gh.vel[j] : n.P.vel[j]; }
    __device__ static fd_quat q(const NarrowArgs& n, int j) { return n.gh.q ? n.gh.q[j] : n.P.q[j]; }
    __device__ static const float4* rot(const NarrowArgs& n, int j)
    {
        return (n.gh.rot ? n.gh.rot : n.P.rot) + 3ll * j;
    }
    __device__ static const FdGeo& geo(const NarrowArgs& n, int j) { return n.G.geo[n.P.geo[j]]; }
    __device__ static const GeoSetDev& set(const NarrowArgs& n) { return n.G; }
    __device__ static long long hash(const NarrowArgs& n, int j) { return n.gh.hash[j]; }
    __device__ static const FdGrid& grid(const NarrowArgs& n) { return n.pgrid; }
    static constexpr bool radius_test = false;
};
template <> struct Slave<FD_GX> : SlaveGhost {};
template <> struct Slave<FD_GY> : SlaveGhost {};
template <> struct Slave<FD_GXY> : SlaveGhost {};

// Evaluate node predicate for one node.  Returns true when overlap >= 0 and
// fills the grid fraction and the eight corner values.
template <int KIND>
__device__ __forceinline__ bool node_predicate(const double3 gp, const int3 bcell, const FdGrid& sg, const double3 cB,
                                               const fd_quat qB, const FdGeo& GB, const double* sdf, double rB2,
                                               double probe, double& overlap, double& fx, double& fy, double& fz,
                                               double p[8])
{
    int3 lo, hi;
    fd_node_range(gp, sg, lo, hi);
    if (bcell.x < lo.x || bcell.x > hi.x || bcell.y < lo.y || bcell.y > hi.y || bcell.z < lo.z || bcell.z > hi.z)
        return false;
    const double3 rel = mk3(gp.x - cB.x, gp.y - cB.y, gp.z - cB.z);
    if (Slave<KIND>::radius_test) {
        if (xm_len2(rel) > rB2) return false;
    }
    const double3 lp = xm_rrot(rel, qB);
    const double gx = (lp.x - GB.origin.x) * GB.inv_spacing;
    const double gy = (lp.y - GB.origin.y) * GB.inv_spacing;
    const double gz = (lp.z - GB.origin.z) * GB.inv_spacing;
    const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
    if (i0 < 0 || j0 < 0 || k0 < 0) return false;
    if (i0 >= GB.size.x - 1 || j0 >= GB.size.y - 1 || k0 >= GB.size.z - 1) return false;
    fx = gx - (double)i0;
    fy = gy - (double)j0;
    fz = gz - (double)k0;
    const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
    const double* S = sdf + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
    p[0] = __ldg(S);
    p[1] = __ldg(S + 1);
    p[2] = __ldg(S + sx);
    p[3] = __ldg(S + sx + 1);
    p[4] = __ldg(S + sxy);
    p[5] = __ldg(S + sxy + 1);
    p[6] = __ldg(S + sxy + sx);
    p[7] = __ldg(S + sxy + sx + 1);
    overlap = -xm_trilinear(fx, fy, fz, p);
    return overlap >= -probe;
}

// Per-pair rigid transform from A's body frame into B's body frame, in
// FP32, for culling only (the exact predicate stays in FP64):
// p_B = M p_A + t with M = R(qB)^T R(qA), t = R(qB)^T (cA - cB).
struct CullXf {
    float m[9];
    float t[3];
};

// from the single-precision rotation rows of A and B; the product's
// relative error (a few 1e-7) is far below the cull margins
__device__ __forceinline__ CullXf cull_transform(const float4* RA, const float4* RB, const double3 cA,
                                                 const double3 cB)
{
    const float4 a0 = RA[0], a1 = RA[1], a2 = RA[2];
    const float4 b0 = RB[0], b1 = RB[1], b2 = RB[2];
    CullXf x;
    // M = RB^T RA
    x.m[0] = fmaf(b0.x, a0.x, fmaf(b1.x, a1.x, b2.x * a2.x));
    x.m[1] = fmaf(b0.x, a0.y, fmaf(b1.x, a1.y, b2.x * a2.y));
    x.m[2] = fmaf(b0.x, a0.z, fmaf(b1.x, a1.z, b2.x * a2.z));
    x.m[3] = fmaf(b0.y, a0.x, fmaf(b1.y, a1.x, b2.y * a2.x));
    x.m[4] = fmaf(b0.y, a0.y, fmaf(b1.y, a1.y, b2.y * a2.y));
    x.m[5] = fmaf(b0.y, a0.z, fmaf(b1.y, a1.z, b2.y * a2.z));
    x.m[6] = fmaf(b0.z, a0.x, fmaf(b1.z, a1.x, b2.z * a2.x));
    x.m[7] = fmaf(b0.z, a0.y, fmaf(b1.z, a1.y, b2.z * a2.y));
    x.m[8] = fmaf(b0.z, a0.z, fmaf(b1.z, a1.z, b2.z * a2.z));
    const float dx = (float)(cA.x - cB.x), dy = (float)(cA.y - cB.y), dz = (float)(cA.z - cB.z);
    x.t[0] = fmaf(b0.x, dx, fmaf(b1.x, dy, b2.x * dz));
    x.t[1] = fmaf(b0.y, dx, fmaf(b1.y, dy, b2.y * dz));
    x.t[2] = fmaf(b0.z, dx, fmaf(b1.z, dy, b2.z * dz));
    return x;
}

// Cluster culling: true when no node of the cluster can pass the node
// predicate (or, with probe > 0, come within `probe` of B).  Conservative:
// single-precision evaluation with relative margins far above its rounding
// (about 1e-7 relative), bounds that hold in exact arithmetic:
//   * B's bounding sphere (particle pairs: the reference's radius test),
//   * B's SDF grid box (nodes outside it are never contacts),
//   * D(v): lower bound on the distance from grid node v to any cell whose
//     corner minimum is <= 0, 1-Lipschitz in the position,
//   * the Lipschitz bound of the trilinear SDF (coarse grids such as plane
//     walls, where it is tight).
template <int KIND>
__device__ __forceinline__ bool cluster_culled(const float4 cl, const CullXf& x, const FdGeo& GB,
                                               const GeoSetDev& SB, double rB, double probe)
{
    const float cx = cl.x, cy = cl.y, cz = cl.z;
    const float px = fmaf(x.m[0], cx, fmaf(x.m[1], cy, fmaf(x.m[2], cz, x.t[0])));
    const float py = fmaf(x.m[3], cx, fmaf(x.m[4], cy, fmaf(x.m[5], cz, x.t[1])));
    const float pz = fmaf(x.m[6], cx, fmaf(x.m[7], cy, fmaf(x.m[8], cz, x.t[2])));
    return sphere_culled(px, py, pz, cl.w, Slave<KIND>::radius_test, GB, SB, rB, probe);
}

// Node filter: true when a node certainly fails the node predicate.  The
// node is mapped into B's frame in single precision (position error below
// perr); it is dropped only when
//   * it lies farther than rB + perr from B's centre (particle pairs), or
//   * it lies outside B's grid box by more than the error, or
//   * (distance-like fields) the single-precision trilinear value exceeds the
//     probe by more than the field's Lipschitz bound times the error, or
//   * it sits inside one cell, away from the cell faces by more than the
//     error, whose eight corner values all exceed the probe (the trilinear
//     value is a convex combination of them).
// Nodes that pass go to the exact double-precision predicate.
template <int KIND>
__device__ __forceinline__ bool node_filtered(const float4 p, const CullXf& x, const FdGeo& GB, const GeoSetDev& SB,
                                              float rB, float perr, double probe)
{
    const float cx = p.x, cy = p.y, cz = p.z;
    const float px = fmaf(x.m[0], cx, fmaf(x.m[1], cy, fmaf(x.m[2], cz, x.t[0])));
    const float py = fmaf(x.m[3], cx, fmaf(x.m[4], cy, fmaf(x.m[5], cz, x.t[1])));
    const float pz = fmaf(x.m[6], cx, fmaf(x.m[7], cy, fmaf(x.m[8], cz, x.t[2])));
    if (Slave<KIND>::radius_test) {
        const float lim = rB + perr;
        if (px * px + py * py + pz * pz > lim * lim) return true;
    }
    const float is = (float)GB.inv_spacing;
    const float gx = (px - (float)GB.origin.x) * is, gy = (py - (float)GB.origin.y) * is,
                gz = (pz - (float)GB.origin.z) * is;
    const float ge = perr * is + 1e-4f;
    const float hx = (float)(GB.size.x - 1), hy = (float)(GB.size.y - 1), hz = (float)(GB.size.z - 1);
    if (gx < -ge || gy < -ge || gz < -ge || gx > hx + ge || gy > hy + ge || gz > hz + ge) return true;
    if (gx < ge || gy < ge || gz < ge || gx > hx - ge || gy > hy - ge || gz > hz - ge) return false;
    const int i0 = (int)gx, j0 = (int)gy, k0 = (int)gz;
    const float fx = gx - i0, fy = gy - j0, fz = gz - k0;
    if (GB.lip < 4.0) {
        const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
        const float* S = SB.sdf32 + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
        const float c00 = __ldg(S) * (1.f - fx) + __ldg(S + 1) * fx;
        const float c10 = __ldg(S + sx) * (1.f - fx) + __ldg(S + sx + 1) * fx;
        const float c01 = __ldg(S + sxy) * (1.f - fx) + __ldg(S + sxy + 1) * fx;
        const float c11 = __ldg(S + sxy + sx) * (1.f - fx) + __ldg(S + sxy + sx + 1) * fx;
        const float phi = (c00 * (1.f - fy) + c10 * fy) * (1.f - fz) + (c01 * (1.f - fy) + c11 * fy) * fz;
        const float slack = (float)GB.lip * perr + 1e-5f * (fabsf(phi) + (float)GB.spacing);
        return phi - (float)probe > slack;
    }
    // the trilinear value anywhere the node can be (within ge of its
    // single-precision position, in grid units) is at least the smallest
    // corner minimum over the cells that box touches (one to a few cells:
    // two per axis where the node is within ge of a cell face)
    const int ilo = max((int)floorf(gx - ge), 0), ihi = min((int)floorf(gx + ge), GB.size.x - 2);
    const int jlo = max((int)floorf(gy - ge), 0), jhi = min((int)floorf(gy + ge), GB.size.y - 2);
    const int klo = max((int)floorf(gz - ge), 0), khi = min((int)floorf(gz + ge), GB.size.z - 2);
    if (ihi - ilo > 2 || jhi - jlo > 2 || khi - klo > 2) return false;  // a margin of more than a cell: keep
    const long long rx = GB.size.x - 1, rxy = (long long)(GB.size.y - 1) * (GB.size.x - 1);
    const float* CM = SB.cellmin + GB.cellmin_off;
    for (int k = klo; k <= khi; ++k)
        for (int j = jlo; j <= jhi; ++j)
            for (int i = ilo; i <= ihi; ++i)
                if (__ldg(CM + k * rxy + j * rx + i) <= (float)probe) return false;
    return true;
}

// ---------------------------------------------------------------------------
// narrow phase, stage 1: one warp per candidate pair.  The clusters of A's
// surface nodes are culled against B, the nodes of the surviving clusters are
// filtered in single precision, and the nodes that may pass the exact
// predicate become the pair's contact slots (contiguous, in cluster order).
// The warp also finds the pair in the previous step's list, the history
// source of its contacts.
// ---------------------------------------------------------------------------
//
// With the pair cache (n.a.gate non-null) the kernel runs only on rebuild
// steps, and every culling margin is widened by the skin n.a.skin: a cluster
// is kept when it may come within reach of B after moves of up to the skin,
// a node is slotted when it may pass the predicate after such moves.
template <int KIND>
__global__ void __launch_bounds__(NARROW_WARPS * 32, FD_SELECT_MIN_BLOCKS) k_select(NarrowArgs n)
{
    if (n.a.gate && *n.a.gate == 0) return;
    // a new layout: the next carried step copies it (k_pc_carry)
    if (blockIdx.x == 0 && threadIdx.x == 0 && n.L.carry_n) *n.L.carry_n = 0;
    __shared__ unsigned short s_node[NARROW_WARPS][MAX_NODE_QUEUE];
    // work counters, summed per block and added to the global ones once
    __shared__ unsigned long long s_stats[4];
    if (n.a.stats && threadIdx.x < 4) s_stats[threadIdx.x] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const unsigned int lt_mask = (1u << lane) - 1u;
    PairListDev& L = n.L;
    const int npairs = min(*L.n_pairs, L.cap_pairs);
    const int nwarps = gridDim.x * NARROW_WARPS;
    const double skin = (n.a.noskin && *n.a.noskin) ? 0.0 : n.a.skin;
    for (int p = blockIdx.x * NARROW_WARPS + wib; p < npairs; p += nwarps) {
        const int A = L.pairA[p];
        const int B = L.pairB[p];
        const FdGeo& GA = n.G.geo[n.P.geo[A]];
        const double3 cA = n.P.pos[A];
        const double3 cB = Slave<KIND>::pos(n, B);
        const FdGeo& GB = Slave<KIND>::geo(n, B);
        const GeoSetDev& SB = Slave<KIND>::set(n);
        const double rB = GB.radius;
        const int ncl = GA.clus_count;
        if (ncl > MAX_CLUSTERS) set_flag(n.a.flags, FD_FLAG_CLUSTER_OVERFLOW);
        // ---- cluster culling, one cluster per lane
        unsigned long long keep = 0ull;
        const CullXf xf = cull_transform(n.P.rot + 3ll * A, Slave<KIND>::rot(n, B), cA, cB);
        for (int c0 = 0; c0 < min(ncl, MAX_CLUSTERS); c0 += 32) {
            const int c = c0 + lane;
            bool k = false;
            if (c < ncl) {
                float4 cl = n.G.clus_sphere[GA.clus_off + c];
                cl.w += (float)skin;
                k = !cluster_culled<KIND>(cl, xf, GB, SB, rB, n.a.probe);
            }
            keep |= ((unsigned long long)__ballot_sync(0xffffffffu, k)) << c0;
        }
        const int kept = __popcll(keep);
        // ---- single-precision filter over the nodes of the surviving
        // clusters; nodes that may pass the predicate are queued in cluster
        // order
        const float perr = 4e-6f * (float)(length3(cA - cB) + GA.radius + rB + GB.spacing) + (float)skin;
        int ncand = 0;
        while (keep) {
            const int c = __ffsll((long long)keep) - 1;
            keep &= keep - 1ull;
            const int2 cr = n.G.clus_range[GA.clus_off + c];
            const int k = cr.x + lane;
            bool cand = false;
            if (lane < cr.y)
                cand = !node_filtered<KIND>(n.G.nodes32[GA.node_off + k], xf, GB, SB, (float)rB, perr, n.a.probe);
            const unsigned int m = __ballot_sync(0xffffffffu, cand);
            if (cand) s_node[wib][ncand + __popc(m & lt_mask)] = (unsigned short)k;
            ncand += __popc(m);
        }
        __syncwarp();
        if (n.a.stats && lane == 0) {
            atomicAdd(&s_stats[0], 1ull);
            atomicAdd(&s_stats[1], (unsigned long long)min(ncl, MAX_CLUSTERS));
            atomicAdd(&s_stats[2], (unsigned long long)kept);
            atomicAdd(&s_stats[3], (unsigned long long)ncand);
        }
        // ---- contact slots of the pair
        int base = 0;
        if (ncand > 0) {
            if (lane == 0) base = atomicAdd(L.n_slots, ncand);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + ncand > L.cap_contacts) {
                if (lane == 0) set_flag(n.a.flags, FD_FLAG_CONTACT_OVERFLOW);
                base = 0;
                ncand = 0;
            }
        }
        if (ncand > 0) {
            // history: the same pair in the previous step's list
            int oc_off = 0, oc_cnt = 0;
            {
                const int os = L.o_seg_off[A], on = L.o_seg_cnt[A];
                int found = -1;
                for (int k0 = 0; k0 < on && found < 0; k0 += 32) {
                    const int k = k0 + lane;
                    const bool eq = (k < on) && (L.o_pairB[os + k] == B);
                    const unsigned int m = __ballot_sync(0xffffffffu, eq);
                    if (m) found = os + k0 + __ffs(m) - 1;
                }
                if (found >= 0) { oc_off = L.o_c_off[found]; oc_cnt = L.o_c_cnt[found]; }
            }
            for (int i = lane; i < ncand; i += 32) {
                L.c_pair[base + i] = p;
                L.c_k[base + i] = s_node[wib][i];
            }
            if (lane == 0) {
                int3 bcell;
                decode_cell(Slave<KIND>::hash(n, B), Slave<KIND>::grid(n).size, bcell);
                L.p_aux[p] = make_int4(bcell.x, bcell.y, bcell.z, oc_off);
                L.p_hist_cnt[p] = oc_cnt;
            }
        }
        if (lane == 0) {
            L.c_off[p] = base;
            L.c_cnt[p] = ncand;
        }
        __syncwarp();
    }
    if (n.a.stats) {
        __syncthreads();
        if (threadIdx.x < 4 && s_stats[threadIdx.x]) {
            // pairs, clusters, clusters kept, nodes given the exact predicate
            const int slot[4] = {0, 1, 2, 4};
            atomicAdd(&n.a.stats[slot[threadIdx.x]], s_stats[threadIdx.x]);
        }
    }
}

// ---------------------------------------------------------------------------
// narrow phase, stage 2: one thread per contact slot.  The exact
// double-precision node predicate (LSParticleContactDetectionKernel.cu:37-119);
// for a contact, the normal, the contact point and the history carried over
// from the previous step (first match on the node, :288-297), then the
// contact law (contactKernel.cu:46-291).  A slot whose node is not in contact
// keeps node id -1.  Force and torques go to the slot; stage 3 sums them per
// pair.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// pair cache, particle-particle list, carried steps: the slots the predicate
// pass must test.  A slot is skipped when its node was outside B at the
// rebuild by more than the SDF can change under the pair's relative motion
// since (|grad phi| <= lip, the trilinear bound; k_pc_carry stored the pair's
// bound); the others are listed, so that the predicate pass runs full warps.
// The wall and image lists are short: there the extra pass cost more than
// the idle lanes, and the predicate pass tests the bound itself.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_slot_filter(NarrowArgs n)
{
    PairListDev& L = n.L;
    if (n.a.gate == nullptr || *n.a.gate != 0 || L.c_test == nullptr) return;
    const int nitems = min(*L.n_slots, L.cap_contacts);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // a block's pass covers SF_UNROLL * TPB slots (slot s0 + u * TPB + tid
    // for u = 0 .. SF_UNROLL - 1), listed in slot order with one atomic: one
    // slot per thread and pass spent a third of its issue slots waiting at
    // the pass's barriers
    constexpr int SF_UNROLL = 4;
    constexpr int NW = TPB / 32;
    const long long stride = (long long)gridDim.x * blockDim.x * SF_UNROLL;
    __shared__ int w_count[SF_UNROLL * NW];
    __shared__ int b_base;
    int tested = 0, skipped = 0;
    for (long long s0 = (long long)blockIdx.x * blockDim.x * SF_UNROLL; s0 < nitems; s0 += stride) {
        int sl[SF_UNROLL], pr[SF_UNROLL];
        bool in[SF_UNROLL];
        float phi0[SF_UNROLL];
#pragma unroll
        for (int u = 0; u < SF_UNROLL; ++u) {
            const long long t = s0 + u * TPB + threadIdx.x;
            in[u] = t < nitems;
            sl[u] = in[u] ? (int)t : 0;
            pr[u] = in[u] ? L.c_pair[sl[u]] : 0;
            phi0[u] = in[u] ? L.c_phi0[sl[u]] : 0.f;
        }
        unsigned int m[SF_UNROLL];
#pragma unroll
        for (int u = 0; u < SF_UNROLL; ++u) {
            bool keep = false;
            if (in[u]) {
                keep = !(phi0[u] > __fadd_ru(L.p_bound[pr[u]], 1e-12f));
                if (!keep) L.c_node[sl[u]] = -1;
            }
            m[u] = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) w_count[u * NW + warp] = __popc(m[u]);
            tested += __popc(m[u]);
            skipped += __popc(__ballot_sync(0xffffffffu, in[u])) - __popc(m[u]);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int total = 0;
            for (int w = 0; w < SF_UNROLL * NW; ++w) {
                const int c = w_count[w];
                w_count[w] = total;
                total += c;
            }
            b_base = total ? atomicAdd(L.n_test, total) : 0;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < SF_UNROLL; ++u)
            if ((m[u] >> lane) & 1u)
                L.c_test[b_base + w_count[u * NW + warp] + __popc(m[u] & ((1u << lane) - 1u))] = sl[u];
        __syncthreads();
    }
    if (n.a.stats && lane == 0) {
        if (tested) atomicAdd(&n.a.stats[5], (unsigned long long)tested);
        if (skipped) atomicAdd(&n.a.stats[6], (unsigned long long)skipped);
    }
}

template <int KIND, int PASS>
__global__ void __launch_bounds__(TPB, PASS == 0 ? FD_PROBE_MIN_BLOCKS : FD_CONTACT_MIN_BLOCKS) k_contact(NarrowArgs n)
{
    PairListDev& L = n.L;
    // pair cache (particle-particle, particle-wall and translated image
    // lists, predicate pass): a rebuild step tests every slot and stores its
    // bound; a carried step tests the slots k_slot_filter listed (the
    // particle-particle list) or tests the slot bound here (the others).  An
    // image list under the cache also holds the pairs of particles that have
    // no image entry this step: their slots hold no contact.
    constexpr bool TRANSLATED = KIND == FD_GX || KIND == FD_GY || KIND == FD_GXY;
    const bool cache = (KIND == FD_PP || KIND == FD_PW || TRANSLATED) && PASS == 0 && n.a.gate != nullptr &&
                       L.c_phi0 != nullptr && n.a.drift != nullptr;
    const bool carried = cache && *n.a.gate == 0;
    const bool listed = KIND == FD_PP && carried && L.c_test != nullptr;
    const bool slot_test = carried && !listed;
    const bool phi0_store = cache && !carried;
    const bool live_test = TRANSLATED && PASS == 0 && n.gh.live != nullptr;
    // pass 0: every slot (or the listed ones); pass 1: the slots pass 0
    // listed as contacts
    const int nitems = PASS == 0 ? min(listed ? *L.n_test : *L.n_slots, L.cap_contacts)
                                 : min(*L.n_hits, L.cap_contacts);
    const int lane = threadIdx.x & 31;
    const bool periodic = (KIND == FD_PP || KIND == FD_PW) && (n.a.periodic_x || n.a.periodic_y);
    const int stride = gridDim.x * blockDim.x;
    if (carried && blockIdx.x == 0 && threadIdx.x == 0 && L.carry_n) atomicAdd(L.carry_n, 1);
    int hits = 0;
    for (int s0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); s0 < nitems; s0 += stride) {
        const int t = s0 + lane;
        bool continue_slot = false;
        const int s = t < nitems ? (PASS == 1 ? L.c_hit[t] : listed ? L.c_test[t] : t) : t;
        bool hit = false;
        if ((slot_test || live_test) && t < nitems) {
            const int p = L.c_pair[s];
            if (live_test && !n.gh.live[L.pairB[p]]) {
                L.c_node[s] = -1;
                if (phi0_store) L.c_phi0[s] = __int_as_float(0xff800000);  // -inf: never skipped
                continue_slot = true;
            } else if (slot_test && L.c_phi0[s] > __fadd_ru(L.p_bound[p], 1e-12f)) {
                // the bound k_slot_filter tests for the particle-particle list
                L.c_node[s] = -1;
                continue_slot = true;
            }
        }
        if (t < nitems && !continue_slot) {
            const int p = L.c_pair[s];
            const int k = L.c_k[s];
            const int A = L.pairA[p];
            const int B = L.pairB[p];
            const int4 aux = L.p_aux[p];
            const int3 bcell = make_int3(aux.x, aux.y, aux.z);
            const FdGeo& GA = n.G.geo[n.P.geo[A]];
            const double3 cA = n.P.pos[A];
            const fd_quat qA = n.P.q[A];
            const double3 cB = Slave<KIND>::pos(n, B);
            const fd_quat qB = Slave<KIND>::q(n, B);
            const FdGeo& GB = Slave<KIND>::geo(n, B);
            const GeoSetDev& SB = Slave<KIND>::set(n);
            const FdGrid& sg = Slave<KIND>::grid(n);
            const double rB2 = GB.radius * GB.radius;
            const int pool = GA.node_off + k;
            const double3 node = n.G.nodes[pool];
            const double3 r = xm_rot(qA, node);
            const double3 gp = mk3(r.x + cA.x, r.y + cA.y, r.z + cA.z);
            // an overlap the predicate did not reach stays +inf (a slot that
            // is never skipped)
            double ov = PASS == 0 ? __longlong_as_double(0x7ff0000000000000ll) : 0., fx = 0., fy = 0., fz = 0., pv[8];
            hit = node_predicate<KIND>(gp, bcell, sg, cB, qB, GB, SB.sdf, rB2, n.a.probe, ov, fx, fy, fz, pv);
            if (phi0_store) L.c_phi0[s] = __double2float_rd(-ov);
            int nid = -1;
            if (PASS == 1 && hit) {
                double3 nrm = fd_gradient_q(fx, fy, fz, pv);
                nrm = fd_rot(qB, nrm);
                nrm = fd_normalize(nrm);
                const double3 pt = gp + (0.5 * ov) * nrm;
                nid = n.P.node_base[A] + n.G.node_lid[pool];
                double3 spring = mk3(0., 0., 0.);
                int hist = -1;
                {
                    // the previous slots of the pair are ascending in node
                    // key; a node appears at most once per pair.  A carried
                    // layout keeps each slot's previous self at its index.
                    const int oc_off = aux.w, oc_end = aux.w + L.p_hist_cnt[p];
                    int lo = oc_off, hi = oc_end;
                    if (s >= oc_off && s < oc_end && L.o_c_k[s] == k) lo = hi = s;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (L.o_c_k[mid] < k) lo = mid + 1; else hi = mid;
                    }
                    if (lo < oc_end && L.o_c_k[lo] == k && L.o_c_node[lo] == nid) {
                        const double* sp = L.o_c_spring + 3ll * lo;
                        spring = mk3(sp[0], sp[1], sp[2]);
                        hist = lo;
                    }
                }
                const AdjRec& R = n.a.rec;
                if (R.hit && s < R.cap) {
                    R.A[s] = A;
                    R.B[s] = B;
                    R.Bp[s] = KIND == FD_PW ? -1 : B;
                    R.geoB[s] = KIND == FD_PW ? n.W.geo[B] : n.P.geo[B];
                    R.matB[s] = KIND == FD_PW ? n.W.mat[B] : n.P.mat[B];
                    R.nid[s] = nid;
                    R.hist[s] = hist;
                    R.rel[3 * s + 0] = gp.x - cB.x;
                    R.rel[3 * s + 1] = gp.y - cB.y;
                    R.rel[3 * s + 2] = gp.z - cB.z;
                    R.sprev[3 * s + 0] = spring.x;
                    R.sprev[3 * s + 1] = spring.y;
                    R.sprev[3 * s + 2] = spring.z;
                    R.qB[4 * s + 0] = qB.q0;
                    R.qB[4 * s + 1] = qB.q1;
                    R.qB[4 * s + 2] = qB.q2;
                    R.qB[4 * s + 3] = qB.q3;
                    R.arm[3 * s + 0] = r.x;
                    R.arm[3 * s + 1] = r.y;
                    R.arm[3 * s + 2] = r.z;
                    R.wrap[s] = 13 + 27;  // no shift unless the force side records one
                }
                double kn = 0., ks = 0.;
                if (n.with_force) {
                    // force-side state (positions after the periodic wrap,
                    // LSSolver.h:1175-1190)
                    double3 ri = cA, rj = cB;
                    if (periodic) {
                        if (n.a.periodic_x) { ri = wrap_x(ri, n.pgrid); if (KIND == FD_PP) rj = wrap_x(rj, n.pgrid); }
                        if (n.a.periodic_y) { ri = wrap_y(ri, n.pgrid); if (KIND == FD_PP) rj = wrap_y(rj, n.pgrid); }
                    }
                    double3 vi = n.P.vel[A], vjs = Slave<KIND>::vel(n, B);
                    const double3 wi = n.P.angvel[A];
                    if ((KIND == FD_PP || KIND == FD_PW) && n.a.sector) {
                        sector_fold(ri, vi, n.pgrid.minb);
                        if (KIND == FD_PP) sector_fold(rj, vjs, n.pgrid.minb);
                    }
                    const int mi = n.P.mat[A];
                    const double invMi = GA.inv_mass;
                    const double kni = n.M.kn[mi], ksi = n.M.ks[mi], mui = n.M.mu[mi], ei = n.M.e[mi];
                    double3 vj, wj;
                    double effM = 0., mu, res;
                    if (KIND == FD_PW) {
                        vj = vjs;
                        wj = n.W.angvel[B];
                        const int mj = n.W.mat[B];
                        mu = fmin(mui, n.MW.mu[mj]);
                        res = fmin(ei, n.MW.e[mj]);
                        if (invMi > 0.) effM = 1. / invMi;
                        kn = kni;
                        ks = ksi;
                    } else {
                        vj = vjs;
                        wj = n.P.angvel[B];
                        const double invMj = GB.inv_mass;
                        const int mj = n.P.mat[B];
                        const double knj = n.M.kn[mj], ksj = n.M.ks[mj];
                        if (kni > 0. && knj > 0.) kn = kni * knj / (kni + knj);
                        if (ksi > 0. && ksj > 0.) ks = ksi * ksj / (ksi + ksj);
                        if (invMi > 0. || invMj > 0.) effM = 1. / (invMi + invMj);
                        res = fmin(ei, n.M.e[mj]);
                        mu = fmin(mui, n.M.mu[mj]);
                    }
                    const double3 vc = (vi + cross3(wi, pt - ri)) - (vj + cross3(wj, pt - rj));
                    if (R.hit && s < R.cap) {
                        R.vc[3 * s + 0] = vc.x;
                        R.vc[3 * s + 1] = vc.y;
                        R.vc[3 * s + 2] = vc.z;
                        R.wrap[s] = wrap_code(cA, ri, cB, rj, n.pgrid);
                    }
                    double3 F = mk3(0., 0., 0.);
                    linear_contact(F, spring, vc, nrm, ov, n.a.dt, kn, ks, mu, res, effM);
                    const double3 TA = cross3(pt - ri, F);
                    const double3 TB = cross3(pt - rj, -F);
                    double* o = L.c_force + 9ll * s;
                    o[0] = F.x; o[1] = F.y; o[2] = F.z;
                    o[3] = TA.x; o[4] = TA.y; o[5] = TA.z;
                    o[6] = TB.x; o[7] = TB.y; o[8] = TB.z;
                }
                L.c_slave[s] = B;
                L.c_spring[3 * s + 0] = spring.x;
                L.c_spring[3 * s + 1] = spring.y;
                L.c_spring[3 * s + 2] = spring.z;
                if (n.a.records) {
                    if (!n.with_force) {
                        const int mi = n.P.mat[A];
                        kn = n.M.kn[mi];
                        ks = n.M.ks[mi];
                        if (KIND != FD_PW) {
                            const int mj = n.P.mat[B];
                            const double knj = n.M.kn[mj], ksj = n.M.ks[mj];
                            kn = (kn > 0. && knj > 0.) ? kn * knj / (kn + knj) : 0.;
                            ks = (ks > 0. && ksj > 0.) ? ks * ksj / (ks + ksj) : 0.;
                        }
                    }
                    L.c_point[3 * s + 0] = pt.x;
                    L.c_point[3 * s + 1] = pt.y;
                    L.c_point[3 * s + 2] = pt.z;
                    L.c_normal[3 * s + 0] = nrm.x;
                    L.c_normal[3 * s + 1] = nrm.y;
                    L.c_normal[3 * s + 2] = nrm.z;
                    L.c_overlap[s] = ov;
                    L.c_en[s] = 0.5 * ov * ov * kn;
                    L.c_es[s] = 0.5 * lengthSq3(spring) * ks;
                }
            }
            if (PASS == 1) {
                L.c_node[s] = nid;
            } else {
                if (!hit) L.c_node[s] = -1;
                if (n.a.rec.hit && s < n.a.rec.cap) n.a.rec.hit[s] = hit ? 1 : 0;
            }
        }
        if (cache && !listed && n.a.stats) {
            // slots given the exact predicate, slots skipped (k_slot_filter
            // counts the listed steps)
            const unsigned int tested = __ballot_sync(0xffffffffu, t < nitems && !continue_slot);
            const unsigned int skipped = __ballot_sync(0xffffffffu, continue_slot);
            if (lane == 0 && tested) atomicAdd(&n.a.stats[5], (unsigned long long)__popc(tested));
            if (lane == 0 && skipped) atomicAdd(&n.a.stats[6], (unsigned long long)__popc(skipped));
        }
        if (PASS == 0) {
            // contacts are listed for pass 1, one atomic per warp
            const unsigned int m = __ballot_sync(0xffffffffu, hit);
            if (m) {
                int base = 0;
                if (lane == 0) base = atomicAdd(L.n_hits, __popc(m));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (hit) L.c_hit[base + __popc(m & ((1u << lane) - 1u))] = s;
                hits += __popc(m);
            }
        }
    }
    if (PASS == 0 && n.a.stats && lane == 0 && hits) atomicAdd(&n.a.stats[3], (unsigned long long)hits);
}

// ---------------------------------------------------------------------------
// narrow phase, stage 3: the pair's force and torques summed over its contact
// slots.  Eight lanes per pair: lane l sums slots l, l + 8, ... in order, then
// a fixed butterfly combines the lanes, so the result does not depend on
// where the pair's slots lie.
// ---------------------------------------------------------------------------
__global__ void k_pair_sum(PairListDev L, int with_force)
{
    const int npairs = min(*L.n_pairs, L.cap_pairs);
    const int lane = threadIdx.x & 31, grp = lane >> 3, l = lane & 7;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int p0 = warp * 4; p0 < npairs; p0 += nwarps * 4) {
        const int p = p0 + grp;
        double acc[9] = {0., 0., 0., 0., 0., 0., 0., 0., 0.};
        int o = 0, c = 0;
        if (p < npairs && with_force) {
            o = L.c_off[p];
            c = L.c_cnt[p];
        }
        // slots l, l + 8, l + 16, ... in order; four node ids loaded ahead
        for (int j0 = l; j0 < c; j0 += 32) {
            int nd[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) nd[u] = j0 + 8 * u < c ? L.c_node[o + j0 + 8 * u] : -1;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (nd[u] < 0) continue;
                const double* f = L.c_force + 9ll * (o + j0 + 8 * u);
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[t] += f[t];
            }
        }
        // pairs without contact slots keep no sum: k_reduce skips them by
        // their slot count
        if (__any_sync(0xffffffffu, c > 0)) {
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 4);
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 2);
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 1);
            }
        }
        if (p < npairs && c > 0) {
            double* out = L.pf + 9ll * p;
#pragma unroll
            for (int t = 0; t < 8; ++t)
                if (l == t) out[t] = acc[t];
            if (l == 0) out[8] = acc[8];
        }
    }
}

// ---------------------------------------------------------------------------
// Mixed precision (FUNDEM_FP32_MIXED).  The node predicate, the SDF
// gradient, the contact law, the bond law and the force sums run in single
// precision with single-precision accumulation; positions, orientations and
// their integration, and the tangential-spring history, stay in double
// precision.  Node positions are formed relative to the body centres, so the
// single-precision quantities are millimetre-scale offsets, never absolute
// coordinates.
// ---------------------------------------------------------------------------
struct v3f {
    float x, y, z;
};
__device__ __forceinline__ v3f mkf(float x, float y, float z) { return v3f{x, y, z}; }
__device__ __forceinline__ v3f tof(double3 a) { return v3f{(float)a.x, (float)a.y, (float)a.z}; }
__device__ __forceinline__ double3 tod(v3f a) { return mk3((double)a.x, (double)a.y, (double)a.z); }
__device__ __forceinline__ v3f operator+(v3f a, v3f b) { return v3f{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3f operator-(v3f a, v3f b) { return v3f{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3f operator-(v3f a) { return v3f{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ v3f operator*(float s, v3f a) { return v3f{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ float dotf(v3f a, v3f b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float lenf(v3f a) { return sqrtf(dotf(a, a)); }
__device__ __forceinline__ v3f crossf(v3f a, v3f b)
{
    return v3f{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// R v and R^T v from the rotation rows
__device__ __forceinline__ v3f rowsf(float4 r0, float4 r1, float4 r2, v3f v)
{
    return v3f{fmaf(r0.x, v.x, fmaf(r0.y, v.y, r0.z * v.z)), fmaf(r1.x, v.x, fmaf(r1.y, v.y, r1.z * v.z)),
               fmaf(r2.x, v.x, fmaf(r2.y, v.y, r2.z * v.z))};
}
constexpr float PI_F = 3.14159265358979f;

// the linear contact law (contactKernel.cuh:4-77) in single precision, with
// the spring history accumulated in double precision
__device__ __forceinline__ v3f linear_contact32(double3& spring, v3f vc, v3f n, float delta, float dt, float kn,
                                                float ks, float mu, float res, float m)
{
    if (!(delta > 0.f)) {
        spring = mk3(0., 0., 0.);
        return mkf(0.f, 0.f, 0.f);
    }
    const float lr = logf(res);
    const float diss = -lr / sqrtf(lr * lr + PI_F * PI_F);
    const float cn = 2.f * diss * sqrtf(m * kn);
    const v3f vn = dotf(vc, n) * n;
    const v3f fn = (kn * delta) * n - cn * vn;
    const float cs = 2.f * diss * sqrtf(m * ks);
    const v3f vs = vc - vn;
    if (mu > 0.f && ks > 0.f) {
        // the history itself is kept in double precision: projection onto
        // the tangent plane, accumulation and the Coulomb rescaling
        const double3 nd = tod(n), vsd = tod(vs);
        double3 p1 = spring - dot3(spring, nd) * nd;
        const double ap1 = length3(p1);
        if (!fd_is_zero(ap1)) p1 = p1 * (length3(spring) / ap1);
        spring = p1 + (double)dt * vsd;
        const v3f sf = -ks * tof(spring) - cs * vs;
        const float asf = lenf(sf), afn = lenf(fn);
        if (asf > 1e-20f && asf > mu * afn) {
            const double scale = (double)(mu * afn) / (double)asf;
            const double3 sfd = -(double)ks * spring - (double)cs * vsd;
            spring = (-1.0 / (double)ks) * (scale * sfd + (double)cs * vsd);
        }
    } else {
        spring = mk3(0., 0., 0.);
    }
    return fn + (-ks * tof(spring) - cs * vs);
}

template <int KIND, int PASS>
__global__ void __launch_bounds__(TPB, PASS == 0 ? FD_PROBE_MIN_BLOCKS : FD_CONTACT_MIN_BLOCKS) k_contact32(NarrowArgs n)
{
    PairListDev& L = n.L;
    float* cf = reinterpret_cast<float*>(L.c_force);
    // pass 0: every slot; pass 1: the slots pass 0 listed as contacts
    const int nitems = PASS == 0 ? min(*L.n_slots, L.cap_contacts) : min(*L.n_hits, L.cap_contacts);
    const int lane = threadIdx.x & 31;
    const bool periodic = (KIND == FD_PP || KIND == FD_PW) && (n.a.periodic_x || n.a.periodic_y);
    const int stride = gridDim.x * blockDim.x;
    // pair cache, as in k_contact; the single-precision predicate's own
    // rounding (a few 1e-7 of the SDF values) is covered by a margin of
    // 1e-4 of B's grid spacing in the pair bound
    constexpr bool TRANSLATED = KIND == FD_GX || KIND == FD_GY || KIND == FD_GXY;
    const bool cache = (KIND == FD_PP || KIND == FD_PW || TRANSLATED) && PASS == 0 && n.a.gate != nullptr &&
                       L.c_phi0 != nullptr && n.a.drift != nullptr;
    const bool carried = cache && *n.a.gate == 0;
    const bool listed = KIND == FD_PP && carried && L.c_test != nullptr;
    const bool slot_test = carried && !listed;
    const bool phi0_store = cache && !carried;
    const bool live_test = TRANSLATED && PASS == 0 && n.gh.live != nullptr;
    const int nitems_c = PASS == 0 && listed ? min(*L.n_test, L.cap_contacts) : nitems;
    if (carried && blockIdx.x == 0 && threadIdx.x == 0 && L.carry_n) atomicAdd(L.carry_n, 1);
    int hits = 0;
    for (int s0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31); s0 < nitems_c; s0 += stride) {
        const int t = s0 + lane;
        const int s = t < nitems_c ? (PASS == 1 ? L.c_hit[t] : listed ? L.c_test[t] : t) : t;
        bool hit = false;
        bool continue_slot = false;
        if ((slot_test || live_test) && t < nitems_c) {
            const int p = L.c_pair[s];
            if (live_test && !n.gh.live[L.pairB[p]]) {
                L.c_node[s] = -1;
                if (phi0_store) L.c_phi0[s] = __int_as_float(0xff800000);  // -inf: never skipped
                continue_slot = true;
            } else if (slot_test && L.c_phi0[s] > __fadd_ru(L.p_bound[p], 1e-12f)) {
                // k_pc_carry's pair bound carries the margin of 1e-4 of B's
                // grid spacing in this precision
                L.c_node[s] = -1;
                continue_slot = true;
            }
        }
        if (t < nitems_c && !continue_slot) {
            const int p = L.c_pair[s];
            const int k = L.c_k[s];
            const int A = L.pairA[p];
            const int B = L.pairB[p];
            const int4 aux = L.p_aux[p];
            const FdGeo& GA = n.G.geo[n.P.geo[A]];
            const double3 cA = n.P.pos[A];
            const double3 cB = Slave<KIND>::pos(n, B);
            const FdGeo& GB = Slave<KIND>::geo(n, B);
            const GeoSetDev& SB = Slave<KIND>::set(n);
            const FdGrid& sg = Slave<KIND>::grid(n);
            const float4* RB = Slave<KIND>::rot(n, B);
            const float4 b0 = RB[0], b1 = RB[1], b2 = RB[2];
            // the rigid transforms in double precision (as in FP64 mode), the
            // position inside the cell and the SDF interpolation in single
            const int pool = GA.node_off + k;
            const double3 rd = xm_rot(n.P.q[A], n.G.nodes[pool]);
            const double3 gp = mk3(rd.x + cA.x, rd.y + cA.y, rd.z + cA.z);
            const v3f r = tof(rd);  // node offset from A's centre
            int3 lo, hi;
            fd_node_range(gp, sg, lo, hi);
            // an overlap the predicate did not reach stays +inf (a slot that
            // is never skipped)
            float ov = PASS == 0 ? __int_as_float(0x7f800000) : 0.f, fx = 0.f, fy = 0.f, fz = 0.f, pv[8];
            float phi0v = __int_as_float(0xff800000);  // the slot bound to store (-inf: never skipped)
            if (aux.x >= lo.x && aux.x <= hi.x && aux.y >= lo.y && aux.y <= hi.y && aux.z >= lo.z && aux.z <= hi.z) {
                const double3 rel = mk3(gp.x - cB.x, gp.y - cB.y, gp.z - cB.z);
                if (!Slave<KIND>::radius_test || xm_len2(rel) <= GB.radius * GB.radius) {
                    const double3 lp = xm_rrot(rel, Slave<KIND>::q(n, B));
                    const double gx = (lp.x - GB.origin.x) * GB.inv_spacing;
                    const double gy = (lp.y - GB.origin.y) * GB.inv_spacing;
                    const double gz = (lp.z - GB.origin.z) * GB.inv_spacing;
                    const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
                    if (i0 >= 0 && j0 >= 0 && k0 >= 0 && i0 < GB.size.x - 1 && j0 < GB.size.y - 1 &&
                        k0 < GB.size.z - 1) {
                        fx = (float)(gx - (double)i0);
                        fy = (float)(gy - (double)j0);
                        fz = (float)(gz - (double)k0);
                        const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
                        const long long c0 = GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
                        if (KIND == FD_PW) {
                            // wall grids are coarse (a plane wall is one cell
                            // the size of the domain, corner values of tenths
                            // of a metre): single-precision interpolation
                            // there would carry errors of 1e-8 m, so the
                            // (few) wall contacts interpolate in double
                            const double* S = SB.sdf + c0;
                            double pd[8] = {__ldg(S), __ldg(S + 1), __ldg(S + sx), __ldg(S + sx + 1), __ldg(S + sxy),
                                            __ldg(S + sxy + 1), __ldg(S + sxy + sx), __ldg(S + sxy + sx + 1)};
                            const double ovd = -xm_trilinear(gx - (double)i0, gy - (double)j0, gz - (double)k0, pd);
#pragma unroll
                            for (int c = 0; c < 8; ++c) pv[c] = (float)pd[c];
                            ov = (float)ovd;
                            phi0v = __double2float_rd(-ovd);
                            hit = ovd >= -n.a.probe;
                        } else {
                            const float* S = SB.sdf32 + c0;
                            pv[0] = __ldg(S); pv[1] = __ldg(S + 1); pv[2] = __ldg(S + sx); pv[3] = __ldg(S + sx + 1);
                            pv[4] = __ldg(S + sxy); pv[5] = __ldg(S + sxy + 1); pv[6] = __ldg(S + sxy + sx);
                            pv[7] = __ldg(S + sxy + sx + 1);
                            const float c00 = pv[0] * (1.f - fx) + pv[1] * fx, c10 = pv[2] * (1.f - fx) + pv[3] * fx;
                            const float c01 = pv[4] * (1.f - fx) + pv[5] * fx, c11 = pv[6] * (1.f - fx) + pv[7] * fx;
                            ov = -((c00 * (1.f - fy) + c10 * fy) * (1.f - fz) + (c01 * (1.f - fy) + c11 * fy) * fz);
                            phi0v = -ov;
                            hit = ov >= -(float)n.a.probe;
                        }
                    }
                }
            }
            if (phi0_store) L.c_phi0[s] = phi0v;
            int nid = -1;
            if (PASS == 1 && hit) {
                // gradient with the x weight truncated as the reference does
                // (LSParticleContactDetectionKernel.cuh:34)
                const float wy0 = 1.f - fy, wy1 = fy, wz0 = 1.f - fz, wz1 = fz;
                const v3f gB = mkf((pv[1] - pv[0]) * wy0 * wz0 + (pv[3] - pv[2]) * wy1 * wz0 +
                                       (pv[5] - pv[4]) * wy0 * wz1 + (pv[7] - pv[6]) * wy1 * wz1,
                                   (pv[2] - pv[0]) * wz0 + (pv[6] - pv[4]) * wz1,
                                   (pv[4] - pv[0]) * wy0 + (pv[6] - pv[2]) * wy1);
                v3f nrm = rowsf(b0, b1, b2, gB);
                const float l2 = dotf(nrm, nrm);
                nrm = l2 > 1e-20f ? rsqrtf(l2) * nrm : mkf(0.f, 0.f, 0.f);
                const v3f arm = r + (0.5f * ov) * nrm;  // contact point relative to A's centre
                nid = n.P.node_base[A] + n.G.node_lid[pool];
                double3 spring = mk3(0., 0., 0.);
                int hist = -1;
                {
                    const int oc_off = aux.w, oc_end = aux.w + L.p_hist_cnt[p];
                    int lo2 = oc_off, hi2 = oc_end;
                    if (s >= oc_off && s < oc_end && L.o_c_k[s] == k) lo2 = hi2 = s;
                    while (lo2 < hi2) {
                        const int mid = (lo2 + hi2) >> 1;
                        if (L.o_c_k[mid] < k) lo2 = mid + 1; else hi2 = mid;
                    }
                    if (lo2 < oc_end && L.o_c_k[lo2] == k && L.o_c_node[lo2] == nid) {
                        const double* sp = L.o_c_spring + 3ll * lo2;
                        spring = mk3(sp[0], sp[1], sp[2]);
                        hist = lo2;
                    }
                }
                const AdjRec& R = n.a.rec;
                if (R.hit && s < R.cap) {
                    const fd_quat qB = Slave<KIND>::q(n, B);
                    R.A[s] = A;
                    R.B[s] = B;
                    R.Bp[s] = KIND == FD_PW ? -1 : B;
                    R.geoB[s] = KIND == FD_PW ? n.W.geo[B] : n.P.geo[B];
                    R.matB[s] = KIND == FD_PW ? n.W.mat[B] : n.P.mat[B];
                    R.nid[s] = nid;
                    R.hist[s] = hist;
                    R.rel[3 * s + 0] = gp.x - cB.x;
                    R.rel[3 * s + 1] = gp.y - cB.y;
                    R.rel[3 * s + 2] = gp.z - cB.z;
                    R.sprev[3 * s + 0] = spring.x;
                    R.sprev[3 * s + 1] = spring.y;
                    R.sprev[3 * s + 2] = spring.z;
                    R.qB[4 * s + 0] = qB.q0;
                    R.qB[4 * s + 1] = qB.q1;
                    R.qB[4 * s + 2] = qB.q2;
                    R.qB[4 * s + 3] = qB.q3;
                    R.arm[3 * s + 0] = rd.x;
                    R.arm[3 * s + 1] = rd.y;
                    R.arm[3 * s + 2] = rd.z;
                    R.wrap[s] = 13 + 27;  // no shift unless the force side records one
                }
                const int mi = n.P.mat[A];
                float kn = 0.f, ks = 0.f;
                float mu, res, effM = 0.f;
                const double kni = n.M.kn[mi], ksi = n.M.ks[mi];
                const double invMi = GA.inv_mass;
                if (KIND == FD_PW) {
                    const int mj = n.W.mat[B];
                    mu = (float)fmin(n.M.mu[mi], n.MW.mu[mj]);
                    res = (float)fmin(n.M.e[mi], n.MW.e[mj]);
                    if (invMi > 0.) effM = (float)(1. / invMi);
                    kn = (float)kni;
                    ks = (float)ksi;
                } else {
                    const int mj = n.P.mat[B];
                    const double knj = n.M.kn[mj], ksj = n.M.ks[mj], invMj = GB.inv_mass;
                    if (kni > 0. && knj > 0.) kn = (float)(kni * knj / (kni + knj));
                    if (ksi > 0. && ksj > 0.) ks = (float)(ksi * ksj / (ksi + ksj));
                    if (invMi > 0. || invMj > 0.) effM = (float)(1. / (invMi + invMj));
                    res = (float)fmin(n.M.e[mi], n.M.e[mj]);
                    mu = (float)fmin(n.M.mu[mi], n.M.mu[mj]);
                }
                if (n.with_force) {
                    double3 ri = cA, rj = cB;
                    if (periodic) {
                        if (n.a.periodic_x) { ri = wrap_x(ri, n.pgrid); if (KIND == FD_PP) rj = wrap_x(rj, n.pgrid); }
                        if (n.a.periodic_y) { ri = wrap_y(ri, n.pgrid); if (KIND == FD_PP) rj = wrap_y(rj, n.pgrid); }
                    }
                    double3 vid = n.P.vel[A], vjd = Slave<KIND>::vel(n, B);
                    if ((KIND == FD_PP || KIND == FD_PW) && n.a.sector) {
                        sector_fold(ri, vid, n.pgrid.minb);
                        if (KIND == FD_PP) sector_fold(rj, vjd, n.pgrid.minb);
                    }
                    const v3f armA = tof(cA - ri) + arm;
                    const v3f armB = tof(cA - rj) + arm;
                    const v3f vi = tof(vid), wi = tof(n.P.angvel[A]);
                    const v3f vj = tof(vjd);
                    const v3f wj = tof(KIND == FD_PW ? n.W.angvel[B] : n.P.angvel[B]);
                    const v3f vc = (vi + crossf(wi, armA)) - (vj + crossf(wj, armB));
                    if (R.hit && s < R.cap) {
                        R.vc[3 * s + 0] = vc.x;
                        R.vc[3 * s + 1] = vc.y;
                        R.vc[3 * s + 2] = vc.z;
                        R.wrap[s] = wrap_code(cA, ri, cB, rj, n.pgrid);
                    }
                    const v3f F = linear_contact32(spring, vc, nrm, ov, (float)n.a.dt, kn, ks, mu, res, effM);
                    const v3f TA = crossf(armA, F);
                    const v3f TB = crossf(armB, -F);
                    float* o = cf + 9ll * s;
                    o[0] = F.x; o[1] = F.y; o[2] = F.z;
                    o[3] = TA.x; o[4] = TA.y; o[5] = TA.z;
                    o[6] = TB.x; o[7] = TB.y; o[8] = TB.z;
                }
                L.c_slave[s] = B;
                L.c_spring[3 * s + 0] = spring.x;
                L.c_spring[3 * s + 1] = spring.y;
                L.c_spring[3 * s + 2] = spring.z;
                if (n.a.records) {
                    L.c_point[3 * s + 0] = cA.x + arm.x;
                    L.c_point[3 * s + 1] = cA.y + arm.y;
                    L.c_point[3 * s + 2] = cA.z + arm.z;
                    L.c_normal[3 * s + 0] = nrm.x;
                    L.c_normal[3 * s + 1] = nrm.y;
                    L.c_normal[3 * s + 2] = nrm.z;
                    L.c_overlap[s] = ov;
                    L.c_en[s] = 0.5 * (double)ov * (double)ov * (double)kn;
                    L.c_es[s] = 0.5 * lengthSq3(spring) * (double)ks;
                }
            }
            if (PASS == 1) {
                L.c_node[s] = nid;
            } else {
                if (!hit) L.c_node[s] = -1;
                if (n.a.rec.hit && s < n.a.rec.cap) n.a.rec.hit[s] = hit ? 1 : 0;
            }
        }
        if (PASS == 0) {
            // contacts are listed for pass 1, one atomic per warp
            const unsigned int m = __ballot_sync(0xffffffffu, hit);
            if (m) {
                int base = 0;
                if (lane == 0) base = atomicAdd(L.n_hits, __popc(m));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (hit) L.c_hit[base + __popc(m & ((1u << lane) - 1u))] = s;
                hits += __popc(m);
            }
        }
    }
    if (PASS == 0 && n.a.stats && lane == 0 && hits) atomicAdd(&n.a.stats[3], (unsigned long long)hits);
}

// stage 3 in single precision: eight lanes per pair, as k_pair_sum
__global__ void k_pair_sum32(PairListDev L, int with_force)
{
    const float* cf = reinterpret_cast<const float*>(L.c_force);
    float* pf = reinterpret_cast<float*>(L.pf);
    const int npairs = min(*L.n_pairs, L.cap_pairs);
    const int lane = threadIdx.x & 31, grp = lane >> 3, l = lane & 7;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int p0 = warp * 4; p0 < npairs; p0 += nwarps * 4) {
        const int p = p0 + grp;
        float acc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        int o = 0, c = 0;
        if (p < npairs && with_force) {
            o = L.c_off[p];
            c = L.c_cnt[p];
        }
        for (int j0 = l; j0 < c; j0 += 32) {
            int nd[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) nd[u] = j0 + 8 * u < c ? L.c_node[o + j0 + 8 * u] : -1;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (nd[u] < 0) continue;
                const float* f = cf + 9ll * (o + j0 + 8 * u);
#pragma unroll
                for (int t = 0; t < 9; ++t) acc[t] += f[t];
            }
        }
        if (__any_sync(0xffffffffu, c > 0)) {
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 4);
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 2);
                acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 1);
            }
        }
        if (p < npairs && c > 0) {
            float* out = pf + 9ll * p;
#pragma unroll
            for (int t = 0; t < 8; ++t)
                if (l == t) out[t] = acc[t];
            if (l == 0) out[8] = acc[8];
        }
    }
}

// ---------------------------------------------------------------------------
// reverse index: pairs grouped by partner B, sorted by A
// ---------------------------------------------------------------------------
// kinds that have a partner side: particle pairs and the six ghost lists
// (FD_GX .. FD_GR270 are consecutive)
constexpr int REV_LISTS = 7;
__host__ __device__ constexpr int rev_kind(int k) { return k == 0 ? FD_PP : FD_GX + k - 1; }
static_assert(FD_GR270 == FD_GX + 5 && FD_NKIND == FD_GR270 + 1, "ghost kinds are consecutive and last");
static_assert(FD_NKIND <= 8, "a reverse-index code keeps the kind in 3 bits");

struct RevArgs {
    PairListDev L[REV_LISTS];
    int active[REV_LISTS];
    RevDev R;
    int n_obj;
    const int* gate;  // non-null: build only when *gate != 0
};

// the pair behind a flat index over the active lists
__device__ __forceinline__ bool rev_locate(const RevArgs& r, int idx, int& k, int& p)
{
#pragma unroll
    for (k = 0; k < REV_LISTS; ++k) {
        if (!r.active[k]) continue;
        const int np = min(*r.L[k].n_pairs, r.L[k].cap_pairs);
        if (idx < np) { p = idx; return true; }
        idx -= np;
    }
    return false;
}

__global__ void k_rev_count(RevArgs r)
{
    if (r.gate && *r.gate == 0) return;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x;; idx += gridDim.x * blockDim.x) {
        int k, p;
        if (!rev_locate(r, idx, k, p)) return;
        const int B = r.L[k].pairB[p];
        // only pairs with contact slots carry a force to the partner
        if (B >= 0 && B < r.n_obj && r.L[k].c_cnt[p] > 0) atomicAdd(&r.R.cnt[B], 1);
    }
}
__global__ void k_rev_fill(RevArgs r)
{
    if (r.gate && *r.gate == 0) return;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x;; idx += gridDim.x * blockDim.x) {
        int k, p;
        if (!rev_locate(r, idx, k, p)) return;
        const int B = r.L[k].pairB[p];
        if (B >= 0 && B < r.n_obj && r.L[k].c_cnt[p] > 0) {
            const int slot = r.R.off[B] + atomicAdd(&r.R.fill[B], 1);
            if (slot < r.R.cap) r.R.code[slot] = p * 8 + rev_kind(k);  // pair counts stay below 2^28
        }
    }
}
// deterministic order: by owner, then kind (an owner has one pair per kind
// with a given partner)
__global__ void k_rev_sort(RevArgs r)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.n_obj || (r.gate && *r.gate == 0)) return;
    const int o = r.R.off[i];
    const int cnt = min(r.R.cnt[i], r.R.cap - o);
    int* seg = r.R.code + o;
    auto key = [&](int code) {
        const int kind = code & 7;
        const int k = kind == FD_PP ? 0 : kind - FD_GX + 1;
        return (long long)r.L[k].pairA[code >> 3] * 8 + kind;
    };
    for (int a = 1; a < cnt; ++a) {
        const int v = seg[a];
        const long long kv = key(v);
        int b = a - 1;
        while (b >= 0 && key(seg[b]) > kv) { seg[b + 1] = seg[b]; --b; }
        seg[b + 1] = v;
    }
}

// ---------------------------------------------------------------------------
// bonds, contactKernel.cuh:138-199 and contactKernel.cu:293-371
// ---------------------------------------------------------------------------
__global__ void k_bonds(ObjDev P, BondDev Bd)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Bd.n) return;
    double* E = Bd.energy + 6ll * k;
    double* O = Bd.out + 9ll * k;
    for (int t = 0; t < 9; ++t) O[t] = 0.;
    if (Bd.rec_active) Bd.rec_active[k] = Bd.active[k] != 0;
    if (Bd.active[k] == 0) {
        for (int t = 0; t < 6; ++t) E[t] = 0.;
        return;
    }
    const int i = Bd.master[k], j = Bd.slave[k];
    const fd_quat qi = P.q[i], qj = P.q[j];
    const double3* f = Bd.frames + 8ll * k;
    const double3 n1i = fd_rot(qi, f[0]), n2i = fd_rot(qi, f[1]), n3i = fd_rot(qi, f[2]);
    const double3 n1j = fd_rot(qj, f[4]), n2j = fd_rot(qj, f[5]), n3j = fd_rot(qj, f[6]);
    const double3 ri = P.pos[i], rj = P.pos[j];
    const double3 rbi = fd_rot(qi, f[3]) + ri;
    const double3 rbj = fd_rot(qj, f[7]) + rj;
    Bd.point[k] = 0.5 * (rbi + rbj);
    double3 F = mk3(0., 0., 0.), Mij = mk3(0., 0., 0.), Mji = mk3(0., 0., 0.);
    int act = 1;
    const double3 rij = rbi - rbj;
    if (Bd.rec_rij) {
        Bd.rec_rij[3 * k + 0] = rij.x;
        Bd.rec_rij[3 * k + 1] = rij.y;
        Bd.rec_rij[3 * k + 2] = rij.z;
        Bd.rec_dn[3 * k + 0] = n1j.x - n1i.x;
        Bd.rec_dn[3 * k + 1] = n1j.y - n1i.y;
        Bd.rec_dn[3 * k + 2] = n1j.z - n1i.z;
    }
    const double D = length3(rij);
    if (!fd_is_zero(D)) {
        const double B1 = Bd.B[4 * k], B2 = Bd.B[4 * k + 1], B3 = Bd.B[4 * k + 2], B4 = Bd.B[4 * k + 3];
        const double R = Bd.radius[k], D0 = Bd.L0[k];
        const double3 nij = fd_normalize(rij);
        const double3 e = -nij;
        E[0] = 0.5 * B1 * (D - D0) * (D - D0);
        E[1] = B2 * (0.5 * dot3(n1j - n1i, e) - 0.25 * dot3(n1i, n1j) + 0.75);
        E[2] = (0.25 * B2 + B3 + 0.5 * B4) * (dot3(n1i, n1j) + 1.);
        E[3] = -0.5 * B4 * (dot3(n1i, n1j) + dot3(n2i, n2j) + dot3(n3i, n3j) - 1);
        const double3 dn = n1j - n1i;
        F = B1 * (D - D0) * e + B2 / (2 * D) * (dn - dot3(dn, e) * e);
        const double3 MTB = B3 * cross3(n1j, n1i) - 0.5 * B4 * (cross3(n2j, n2i) + cross3(n3j, n3i));
        Mij = -0.5 * B2 * cross3(e, n1i) + MTB;
        Mji = 0.5 * B2 * cross3(e, n1j) - MTB;
        const double bnf = dot3(F, nij);
        const double3 bsf = F - bnf * nij;
        const double btt = dot3(MTB, nij);
        const double3 bbt = MTB - btt * nij;
        const double Ab = R * R * PI_D;
        const double Ib = Ab * R * R / 4.;
        const double Jb = 2 * Ib;
        E[4] = -bnf / Ab + length3(bbt) / Ib * R;
        E[5] = length3(bsf) / Ab + fabs(btt) / Jb * R;
        if (Bd.ts[k] > 0. && E[4] > Bd.ts[k]) act = 0;
        else if (Bd.coh[k] > 0. && E[5] > Bd.coh[k] - Bd.mu[k] * E[4]) act = 0;
    }
    Bd.active[k] = act;
    const double3 Ti = Mij + cross3(rbi - ri, F);
    const double3 Tj = Mji + cross3(rbj - rj, -F);
    O[0] = F.x; O[1] = F.y; O[2] = F.z;
    O[3] = Ti.x; O[4] = Ti.y; O[5] = Ti.z;
    O[6] = Tj.x; O[7] = Tj.y; O[8] = Tj.z;
}

// the V-bond (contactKernel.cuh:138-199) in single precision; the frames are
// rotated with the single-precision rotation rows, the bond vector is formed
// from the double-precision centre difference plus the rotated offsets
__global__ void k_bonds32(ObjDev P, BondDev Bd)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= Bd.n) return;
    double* E = Bd.energy + 6ll * k;
    float* O = reinterpret_cast<float*>(Bd.out) + 9ll * k;
    for (int t = 0; t < 9; ++t) O[t] = 0.f;
    if (Bd.rec_active) Bd.rec_active[k] = Bd.active[k] != 0;
    if (Bd.active[k] == 0) {
        for (int t = 0; t < 6; ++t) E[t] = 0.;
        return;
    }
    const int i = Bd.master[k], j = Bd.slave[k];
    const float4 a0 = P.rot[3ll * i], a1 = P.rot[3ll * i + 1], a2 = P.rot[3ll * i + 2];
    const float4 b0 = P.rot[3ll * j], b1 = P.rot[3ll * j + 1], b2 = P.rot[3ll * j + 2];
    const double3* f = Bd.frames + 8ll * k;
    const v3f n1i = rowsf(a0, a1, a2, tof(f[0])), n2i = rowsf(a0, a1, a2, tof(f[1])), n3i = rowsf(a0, a1, a2, tof(f[2]));
    const v3f n1j = rowsf(b0, b1, b2, tof(f[4])), n2j = rowsf(b0, b1, b2, tof(f[5])), n3j = rowsf(b0, b1, b2, tof(f[6]));
    const double3 ri = P.pos[i], rj = P.pos[j];
    const v3f oi = rowsf(a0, a1, a2, tof(f[3])), oj = rowsf(b0, b1, b2, tof(f[7]));
    Bd.point[k] = 0.5 * (ri + rj) + 0.5 * tod(oi + oj);
    v3f F = mkf(0.f, 0.f, 0.f), Mij = mkf(0.f, 0.f, 0.f), Mji = mkf(0.f, 0.f, 0.f);
    int act = 1;
    const v3f rij = tof(ri - rj) + (oi - oj);
    if (Bd.rec_rij) {
        Bd.rec_rij[3 * k + 0] = rij.x;
        Bd.rec_rij[3 * k + 1] = rij.y;
        Bd.rec_rij[3 * k + 2] = rij.z;
        Bd.rec_dn[3 * k + 0] = n1j.x - n1i.x;
        Bd.rec_dn[3 * k + 1] = n1j.y - n1i.y;
        Bd.rec_dn[3 * k + 2] = n1j.z - n1i.z;
    }
    const float D = lenf(rij);
    if (D > 1e-20f) {
        const float B1 = (float)Bd.B[4 * k], B2 = (float)Bd.B[4 * k + 1], B3 = (float)Bd.B[4 * k + 2],
                    B4 = (float)Bd.B[4 * k + 3];
        const float R = (float)Bd.radius[k], D0 = (float)Bd.L0[k];
        const v3f nij = rsqrtf(dotf(rij, rij)) * rij;
        const v3f e = -nij;
        const float c11 = dotf(n1i, n1j);
        E[0] = 0.5 * (double)B1 * (double)(D - D0) * (double)(D - D0);
        E[1] = (double)(B2 * (0.5f * dotf(n1j - n1i, e) - 0.25f * c11 + 0.75f));
        E[2] = (double)((0.25f * B2 + B3 + 0.5f * B4) * (c11 + 1.f));
        E[3] = (double)(-0.5f * B4 * (c11 + dotf(n2i, n2j) + dotf(n3i, n3j) - 1.f));
        const v3f dn = n1j - n1i;
        F = (B1 * (D - D0)) * e + (B2 / (2.f * D)) * (dn - dotf(dn, e) * e);
        const v3f MTB = B3 * crossf(n1j, n1i) - (0.5f * B4) * (crossf(n2j, n2i) + crossf(n3j, n3i));
        Mij = (-0.5f * B2) * crossf(e, n1i) + MTB;
        Mji = (0.5f * B2) * crossf(e, n1j) - MTB;
        const float bnf = dotf(F, nij);
        const v3f bsf = F - bnf * nij;
        const float btt = dotf(MTB, nij);
        const v3f bbt = MTB - btt * nij;
        const float Ab = R * R * PI_F;
        const float Ib = Ab * R * R / 4.f;
        const float Jb = 2.f * Ib;
        const float sn = -bnf / Ab + lenf(bbt) / Ib * R;
        const float ss = lenf(bsf) / Ab + fabsf(btt) / Jb * R;
        E[4] = sn;
        E[5] = ss;
        if (Bd.ts[k] > 0. && sn > (float)Bd.ts[k]) act = 0;
        else if (Bd.coh[k] > 0. && ss > (float)(Bd.coh[k] - Bd.mu[k] * (double)sn)) act = 0;
    }
    Bd.active[k] = act;
    const v3f Ti = Mij + crossf(oi, F);
    const v3f Tj = Mji + crossf(oj, -F);
    O[0] = F.x; O[1] = F.y; O[2] = F.z;
    O[3] = Ti.x; O[4] = Ti.y; O[5] = Ti.z;
    O[6] = Tj.x; O[7] = Tj.y; O[8] = Tj.z;
}

// ---------------------------------------------------------------------------
// per-particle reduction, fixed order
// ---------------------------------------------------------------------------
struct ReduceArgs {
    ObjDev P;
    PairListDev L[FD_NKIND];
    int active[FD_NKIND];
    RevDev R;
    BondDev B;
};

// Real = double: FP64 mode; Real = float: mixed mode (pair and bond results
// stored and summed in single precision)
template <typename Real>
__global__ void k_reduce(ReduceArgs r)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= r.P.n) return;
    Real F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    auto add = [](Real* acc, const Real* v, Real sgn) {
        acc[0] += sgn * v[0];
        acc[1] += sgn * v[1];
        acc[2] += sgn * v[2];
    };
    // pairs the particle owns, kind by kind
    for (int kind = 0; kind < FD_NKIND; ++kind) {
        if (!r.active[kind]) continue;
        const PairListDev& L = r.L[kind];
        const Real* pfa = reinterpret_cast<const Real*>(L.pf);
        const int s = L.seg_off[i], c = L.seg_cnt[i];
        for (int k = s; k < s + c; ++k) {
            if (L.c_cnt[k] == 0) continue;  // no contact slot, no sum kept
            const Real* pf = pfa + 9ll * k;
            add(F, pf, Real(1));
            add(T, pf + 3, Real(1));
        }
    }
    // pairs in which it is the partner, by owner
    {
        const int rs = r.R.off[i], rc = min(r.R.cnt[i], r.R.cap - rs);
        for (int e = rs; e < rs + rc; ++e) {
            const int code = r.R.code[e];
            const int kind = code & 7, k = code >> 3;
            const PairListDev& L = r.L[kind];
            if (kind != FD_PP && L.pairA[k] == i) continue;  // a particle against its own ghost
            if (L.c_cnt[k] == 0) continue;
            const Real* pf = reinterpret_cast<const Real*>(L.pf) + 9ll * k;
            add(F, pf, Real(-1));
            add(T, pf + 6, Real(1));
        }
    }
    if (r.B.n > 0) {
        const Real* out = reinterpret_cast<const Real*>(r.B.out);
        for (int e = r.B.plist_off[i]; e < r.B.plist_off[i + 1]; ++e) {
            const int code = r.B.plist[e];
            const int b = code >> 1, side = code & 1;
            const Real* o = out + 9ll * b;
            if (side == 0) { add(F, o, Real(1)); add(T, o + 3, Real(1)); }
            else { add(F, o, Real(-1)); add(T, o + 6, Real(1)); }
        }
    }
    r.P.force[i] = mk3((double)F[0], (double)F[1], (double)F[2]);
    r.P.torque[i] = mk3((double)T[0], (double)T[1], (double)T[2]);
}

}  // namespace

// kernel launches are counted into the counter the calling thread set
// (fundem_launch_count); none when it set none
thread_local long long* t_launch_counter = nullptr;
void set_launch_counter(long long* c) { t_launch_counter = c; }
void count_launch()
{
    if (t_launch_counter) ++*t_launch_counter;
}
static inline void note_launch()
{
    if (t_launch_counter) ++*t_launch_counter;
}

// ---------------------------------------------------------------------------
// contiguous views of a contact list and of the bonds (the device arrays the
// reference's SolidInteraction and VBondedInteraction getters return)
// ---------------------------------------------------------------------------
__global__ void k_view_keys(PairListDev L, long long* key)
{
    const int nslots = min(*L.n_slots, L.cap_contacts);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < L.cap_contacts; s += gridDim.x * blockDim.x) {
        const int node = s < nslots ? L.c_node[s] : -1;
        key[s] = node >= 0 ? ((long long)node << 32) | (unsigned int)L.c_slave[s] : -1ll;
    }
}
__global__ void k_view_gather(PairListDev L, const int* order, long long n, ContactViewDev v)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int s = order[i];
        v.master[i] = L.c_node[s];
        v.slave[i] = L.c_slave[s];
        for (int d = 0; d < 3; ++d) {
            v.point[3 * i + d] = L.c_point[3 * s + d];
            v.normal[3 * i + d] = L.c_normal[3 * s + d];
            v.spring[3 * i + d] = L.c_spring[3 * s + d];
        }
        v.overlap[i] = L.c_overlap[s];
        v.en[i] = L.c_en[s];
        v.es[i] = L.c_es[s];
    }
}
__global__ void k_bond_view(BondDev B, BondViewDev v)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B.n) return;
    for (int t = 0; t < 4; ++t) v.B[t][k] = B.B[4 * k + t];
    for (int t = 0; t < 6; ++t) v.energy[t][k] = B.energy[6 * k + t];
    for (int t = 0; t < 8; ++t) v.frames[t][k] = B.frames[8 * k + t];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
size_t scan_tmp_size(long long n)
{
    size_t total = 0;
    long long m = n;
    while (m > SCAN_TILE) {
        m = (m + SCAN_TILE - 1) / SCAN_TILE;
        total += (size_t)m;
    }
    return total + 1;
}

void scan_exclusive(const int* in, int* out, long long n, int* tmp, cudaStream_t s, const int* gate)
{
    if (n <= 0) return;
    if (n <= SCAN_TILE) {
        k_scan_tile<false><<<1, SCAN_TPB, 0, s>>>(in, out, n, nullptr, gate); note_launch();
        return;
    }
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    int* sums = tmp;
    k_scan_tile<false><<<(unsigned)tiles, SCAN_TPB, 0, s>>>(in, out, n, sums, gate); note_launch();
    scan_exclusive(sums, sums, tiles, tmp + tiles, s, gate);
    k_scan_add<<<(unsigned)tiles, SCAN_TPB, 0, s>>>(out, n, sums, gate); note_launch();
}

void scan_inclusive(const int* in, int* out, long long n, int* tmp, cudaStream_t s)
{
    if (n <= 0) return;
    if (n <= SCAN_TILE) {
        k_scan_tile<true><<<1, SCAN_TPB, 0, s>>>(in, out, n, nullptr, nullptr); note_launch();
        return;
    }
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    int* sums = tmp;
    k_scan_tile<true><<<(unsigned)tiles, SCAN_TPB, 0, s>>>(in, out, n, sums, nullptr); note_launch();
    scan_exclusive(sums, sums, tiles, tmp + tiles, s);
    k_scan_add<<<(unsigned)tiles, SCAN_TPB, 0, s>>>(out, n, sums, nullptr); note_launch();
}

void launch_kick(const ObjDev& P, const GeoSetDev& G, double3 gravity, double h, cudaStream_t s)
{
    if (P.n > 0) { k_kick<<<nblocks(P.n), TPB, 0, s>>>(P, G, gravity, h); note_launch(); }
}
void launch_drift(const ObjDev& O, double dt, cudaStream_t s)
{
    if (O.n > 0) { k_drift<<<nblocks(O.n), TPB, 0, s>>>(O, dt); note_launch(); }
}
void launch_kick_drift(const ObjDev& P, const GeoSetDev& G, double3 gravity, double h, double dt, cudaStream_t s)
{
    if (P.n > 0) { k_kick_drift<<<nblocks(P.n), TPB, 0, s>>>(P, G, gravity, h, dt); note_launch(); }
}
void launch_hash(const ObjDev& O, const FdGrid& g, cudaStream_t s)
{
    if (O.n > 0) { k_hash<<<nblocks(O.n), TPB, 0, s>>>(O, g); note_launch(); }
}
void radix_sort_scratch(int n, size_t& bcount_ints, size_t& bscan_ints)
{
    const long long nblk = std::max<long long>((n + RS_TPB - 1) / RS_TPB, 1);
    bcount_ints = (size_t)(RS_RADIX * nblk);
    bscan_ints = scan_tmp_size((long long)bcount_ints);
}
void radix_sort_keys(const long long* keys, int n, long long num_keys, unsigned long long* out_key, int* out_idx,
                     unsigned long long* key_b, int* idx_b, int* bcount, int* bscan_tmp, cudaStream_t s,
                     const int* gate)
{
    if (n <= 0) return;
    // bits a key can use; keys of objects in no cell sort after every cell
    int bits = 1;
    while (bits < 64 && ((unsigned long long)num_keys >> bits) != 0ull) ++bits;
    const int passes = (bits + 7) / 8;
    const int nblk = (n + RS_TPB - 1) / RS_TPB;
    // the last pass writes (out_key, out_idx)
    unsigned long long* kb[2] = {out_key, key_b};
    int* ib[2] = {out_idx, idx_b};
    int src = passes & 1;
    k_rs_keys<<<nblocks(n), TPB, 0, s>>>(keys, n, num_keys, kb[src], ib[src], gate); note_launch();
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        k_rs_hist<<<nblk, RS_TPB, 0, s>>>(kb[src], n, shift, bcount, nblk, gate); note_launch();
        scan_exclusive(bcount, bcount, (long long)RS_RADIX * nblk, bscan_tmp, s, gate);
        k_rs_scatter<<<nblk, RS_TPB, 0, s>>>(kb[src], ib[src], n, shift, bcount, nblk, kb[src ^ 1], ib[src ^ 1], gate);
        note_launch();
        src ^= 1;
    }
}
void launch_cell_table(ObjDev& O, CellTableDev& T, int* scan_tmp, size_t, cudaStream_t s, const int* gate)
{
    if (O.n <= 0) return;
    if (T.hashed) {
        // sparse grids: radix sort of the keys, runs into a hash table
        radix_sort_keys(O.hash, O.n, T.g.num, T.skey, T.sorted, T.key_b, T.idx_b, T.bcount, T.bscan_tmp, s, gate);
        if (gate) {
            k_hkey_clear<<<nblocks((long long)T.hmask + 1), TPB, 0, s>>>(T.hkey, T.hmask + 1, gate); note_launch();
        } else {
            cudaMemsetAsync(T.hkey, 0xff, sizeof(unsigned long long) * (T.hmask + 1), s);
        }
        k_cells_hashed<<<nblocks(O.n), TPB, 0, s>>>(T.skey, O.n, T.g.num, T.hkey, T.hval, T.hmask, nullptr, gate);
        note_launch();
        return;
    }
    // dense grids: count, scan, scatter, then each cell in object order
    if (gate) {
        k_clear_cells<<<nblocks(T.g.num), TPB, 0, s>>>(T.count, T.fill, T.g.num, gate);
        note_launch();
    } else {
        cudaMemsetAsync(T.count, 0, sizeof(int) * T.g.num, s);
        cudaMemsetAsync(T.fill, 0, sizeof(int) * T.g.num, s);
    }
    k_cell_count<<<nblocks(O.n), TPB, 0, s>>>(O.hash, O.n, T.g.num, T.count, gate); note_launch();
    scan_exclusive(T.count, T.start, T.g.num, scan_tmp, s, gate);
    k_cell_scatter<<<nblocks(O.n), TPB, 0, s>>>(O.hash, O.n, T.g.num, T.start, T.fill, T.sorted, gate);
    note_launch();
    k_cell_order<<<nblocks(T.g.num), TPB, 0, s>>>(T.g.num, T.count, T.start, T.sorted, gate); note_launch();
}
void launch_wrap(ObjDev& P, const FdGrid& g, int dim, cudaStream_t s, int* ctrl, const double3* src)
{
    if (P.n > 0) { k_wrap<<<nblocks(P.n), TPB, 0, s>>>(P, g, dim, ctrl, src); note_launch(); }
}
void launch_ghost_build(const ObjDev& P, GhostDev& Gh, int kind, cudaStream_t s, double ext_skin, int* ctrl)
{
    // occupied-cell box of the ghost images: empty until the build fills it
    cudaMemsetAsync(Gh.occ, 0x7f, 3 * sizeof(int), s);
    cudaMemsetAsync(Gh.occ + 3, 0xff, 3 * sizeof(int), s);
    if (P.n > 0) { k_ghost_build<<<nblocks(P.n), TPB, 0, s>>>(P, Gh, kind, ext_skin, ctrl); note_launch(); }
}
void launch_ghost_gate(int* ctrl, cudaStream_t s)
{
    k_ghost_gate<<<1, 1, 0, s>>>(ctrl);
    note_launch();
}
void launch_sector_wrap(ObjDev& P, const FdGrid& g, cudaStream_t s)
{
    if (P.n > 0) { k_sector_wrap<<<nblocks(P.n), TPB, 0, s>>>(P, g.minb); note_launch(); }
}
void launch_sector_images(const ObjDev& P, GhostDev* R, cudaStream_t s)
{
    for (int d = 0; d < 3; ++d) {
        cudaMemsetAsync(R[d].occ, 0x7f, 3 * sizeof(int), s);
        cudaMemsetAsync(R[d].occ + 3, 0xff, 3 * sizeof(int), s);
    }
    if (P.n > 0) { k_sector_images<<<nblocks(P.n), TPB, 0, s>>>(P, R[0], R[1], R[2]); note_launch(); }
}

void launch_broad_pp(const ObjDev& P, const GeoSetDev& G, const CellTableDev& T, PairListDev& L,
                     unsigned int* flags, double probe, cudaStream_t s, double skin, const int* gate)
{
    cudaMemsetAsync(L.n_pairs, 0, sizeof(int), s);
    if (P.n > 0) {
        k_broad_cells<false, false, false><<<nblocks((long long)P.n * BROAD_LANES), TPB, 0, s>>>(
            P, G, T, nullptr, nullptr, nullptr, nullptr, nullptr, L, NlDev{}, flags, probe, skin, gate, nullptr);
        note_launch();
    }
}
void launch_broad_pp_nl(const ObjDev& P, const GeoSetDev& G, const CellTableDev& T, PairListDev& L, NlDev& nl,
                        unsigned int* flags, double probe, cudaStream_t s, const int* gate)
{
    cudaMemsetAsync(L.n_pairs, 0, sizeof(int), s);
    if (P.n <= 0) return;
    k_nl_check<<<nblocks(P.n), TPB, 0, s>>>(P, nl, T.g, gate); note_launch();
    k_broad_cells<false, false, true><<<nblocks((long long)P.n * BROAD_LANES), TPB, 0, s>>>(
        P, G, T, nullptr, nullptr, nullptr, nullptr, nullptr, L, nl, flags, probe, 0.0, gate, nullptr);
    note_launch();
    k_nl_filter<<<nblocks((long long)P.n * 8), TPB, 0, s>>>(P, G, L, nl, flags, probe, gate); note_launch();
}
void launch_pair_cache_check(const ObjDev& P, const PairCacheDev& c, cudaStream_t s)
{
    if (P.n > 0) { k_pc_check<<<nblocks(P.n), TPB, 0, s>>>(P, c); note_launch(); }
}
void launch_pair_cache_commit(const ObjDev& P, const PairCacheDev& c, const PairListDev& L, cudaStream_t s)
{
    if (P.n > 0) { k_pc_commit<<<nblocks(P.n), TPB, 0, s>>>(P, c, L); note_launch(); }
}
void launch_pair_cache_end(const PairCacheDev& c, const PairListDev* lists, int n_lists, cudaStream_t s)
{
    CachedCounts gc{};
    gc.n = std::min(n_lists, 4);
    for (int k = 0; k < gc.n; ++k) {
        gc.n_pairs[k] = lists[k].n_pairs;
        gc.n_slots[k] = lists[k].n_slots;
        gc.cap_pairs[k] = lists[k].cap_pairs;
        gc.cap_contacts[k] = lists[k].cap_contacts;
    }
    k_pc_end<<<1, 1, 0, s>>>(c.ctrl, gc);
    note_launch();
}

void launch_broad_pw(const ObjDev& P, const GeoSetDev& G, const ObjDev& W, const GeoSetDev& GW,
                     const FdGrid& wg, PairListDev& L, unsigned int* flags, double probe, cudaStream_t s,
                     const int2* wall_range, double skin, const int* gate)
{
    cudaMemsetAsync(L.n_pairs, 0, sizeof(int), s);
    if (P.n > 0) {
        k_broad_pw<<<nblocks(P.n), TPB, 0, s>>>(P, G, W, GW, wg, L, flags, probe, wall_range, skin, gate);
        note_launch();
    }
}
void launch_pair_cache_check_walls(const ObjDev& W, const GeoSetDev& GW, const PairCacheDev& c, cudaStream_t s)
{
    if (W.n > 0) { k_pc_check_walls<<<nblocks(W.n), TPB, 0, s>>>(W, GW, c); note_launch(); }
}
void launch_pair_cache_commit_walls(const ObjDev& W, const PairCacheDev& c, cudaStream_t s)
{
    if (W.n > 0) { k_pc_commit_walls<<<nblocks(W.n), TPB, 0, s>>>(W, c); note_launch(); }
}
void launch_broad_ghost(const ObjDev& P, const GeoSetDev& G, const GhostDev& Gh, PairListDev& L,
                        unsigned int* flags, double probe, cudaStream_t s, double skin, const int* gate,
                        const int* noskin)
{
    cudaMemsetAsync(L.n_pairs, 0, sizeof(int), s);
    if (P.n <= 0) return;
    cudaMemsetAsync(Gh.nsearch, 0, sizeof(int), s);
    k_ghost_searchers<<<nblocks(P.n), TPB, 0, s>>>(P, G, Gh.cells.g, Gh.occ, L, Gh.searchers, Gh.nsearch, skin,
                                                    gate, noskin);
    note_launch();
    const long long groups = std::min<long long>(P.n, 148ll * 8 * (TPB / BROAD_LANES));
    k_broad_cells<true, true, false><<<nblocks(groups * BROAD_LANES), TPB, 0, s>>>(
        P, G, Gh.cells, Gh.pos, Gh.rot, Gh.occ, Gh.searchers, Gh.nsearch, L, NlDev{}, flags, probe, skin, gate,
        noskin);
    note_launch();
}

void launch_narrow(int kind, const ObjDev& P, const GeoSetDev& G, const MatDev& M, const ObjDev& W,
                   const GeoSetDev& GW, const MatDev& MW, const FdGrid& pgrid, const FdGrid& wgrid,
                   const GhostDev* gh, PairListDev& L, const StepArgs& a, int with_force, bool mixed, cudaStream_t s)
{
    cudaMemsetAsync(L.n_slots, 0, 2 * sizeof(int), s);  // slots and contacts
    NarrowArgs n;
    n.P = P; n.G = G; n.M = M; n.W = W; n.GW = GW; n.MW = MW; n.pgrid = pgrid; n.wgrid = wgrid;
    if (gh) n.gh = *gh; else memset(&n.gh, 0, sizeof(n.gh));
    n.L = L; n.a = a; n.with_force = with_force;
    const long long need = ((long long)L.cap_pairs + NARROW_WARPS - 1) / NARROW_WARPS;
    // grid-stride kernels sized in blocks per SM (the pair and slot counts
    // are known only on the device): the defaults fill one resident wave
    const int sel_bps = a.shape[0] > 0 ? a.shape[0] : FD_SELECT_MIN_BLOCKS;
    const int grid = (int)std::max(1ll, std::min(need, 148ll * sel_bps));
    const int pgrid0 = 148 * (a.shape[1] > 0 ? a.shape[1] : FD_PROBE_MIN_BLOCKS);
    const int cgrid = 148 * (a.shape[2] > 0 ? a.shape[2] : 4);
    const int sgrid = 148 * (a.shape[3] > 0 ? a.shape[3] : 4);
#define FD_NARROW_CASE(K)                                                              \
    case K:                                                                            \
        k_select<K><<<grid, NARROW_WARPS * 32, 0, s>>>(n); note_launch();                             \
        if (a.gate) {                                                                  \
            const bool wall = K == FD_PW;                                              \
            k_pc_carry<<<148 * 8, TPB, 0, s>>>(                                        \
                L, P.n, wall ? W.hash : gh ? gh->hash : P.hash, wall ? wgrid : pgrid, a.gate, a.drift, \
                a.disp, a.driftB ? a.driftB : a.drift, a.dispB ? a.dispB : a.disp,      \
                wall ? W.geo : P.geo, wall ? GW.geo : G.geo, (mixed && !wall) ? 1e-4f : 0.f);          \
            note_launch();                                                             \
            if (K == FD_PP) {                                                          \
                cudaMemsetAsync(L.n_test, 0, sizeof(int), s);                          \
                k_slot_filter<<<pgrid0, TPB, 0, s>>>(n);                               \
                note_launch();                                                         \
            }                                                                          \
        }                                                                              \
        if (mixed) {                                                                   \
            k_contact32<K, 0><<<pgrid0, TPB, 0, s>>>(n); note_launch();                               \
            k_contact32<K, 1><<<cgrid, TPB, 0, s>>>(n); note_launch();                                \
        } else {                                                                       \
            k_contact<K, 0><<<pgrid0, TPB, 0, s>>>(n); note_launch();                                 \
            k_contact<K, 1><<<cgrid, TPB, 0, s>>>(n); note_launch();                                  \
        }                                                                              \
        break;
    switch (kind) {
        FD_NARROW_CASE(FD_PP)
        FD_NARROW_CASE(FD_PW)
        FD_NARROW_CASE(FD_GX)
        FD_NARROW_CASE(FD_GY)
        FD_NARROW_CASE(FD_GXY)
    case FD_GR90:
    case FD_GR180:
    case FD_GR270:
        // the sector images differ from the translated ones only in the state
        // the ghost traits read, so they share the ghost kernels
        k_select<FD_GX><<<grid, NARROW_WARPS * 32, 0, s>>>(n); note_launch();
        if (mixed) {
            k_contact32<FD_GX, 0><<<pgrid0, TPB, 0, s>>>(n); note_launch();
            k_contact32<FD_GX, 1><<<cgrid, TPB, 0, s>>>(n); note_launch();
        } else {
            k_contact<FD_GX, 0><<<pgrid0, TPB, 0, s>>>(n); note_launch();
            k_contact<FD_GX, 1><<<cgrid, TPB, 0, s>>>(n); note_launch();
        }
        break;
    }
#undef FD_NARROW_CASE
    if (mixed) {
        k_pair_sum32<<<sgrid, TPB, 0, s>>>(L, with_force);
    } else {
        k_pair_sum<<<sgrid, TPB, 0, s>>>(L, with_force);
    }
    note_launch();
}

void launch_reverse(const ObjDev& P, PairListDev* lists, const int* active, RevDev& R, int* scan_tmp, size_t,
                    cudaStream_t s, const int* gate)
{
    if (P.n <= 0) return;
    RevArgs r;
    for (int k = 0; k < REV_LISTS; ++k) {
        r.L[k] = lists[rev_kind(k)];
        r.active[k] = active[rev_kind(k)];
    }
    r.R = R;
    r.n_obj = P.n;
    r.gate = gate;
    if (gate) {
        k_clear_cells<<<nblocks(P.n), TPB, 0, s>>>(R.cnt, R.fill, P.n, gate); note_launch();
    } else {
        cudaMemsetAsync(R.cnt, 0, sizeof(int) * P.n, s);
        cudaMemsetAsync(R.fill, 0, sizeof(int) * P.n, s);
    }
    const int g = 148 * 8;
    k_rev_count<<<g, TPB, 0, s>>>(r); note_launch();
    scan_exclusive(R.cnt, R.off, P.n, scan_tmp, s, gate);
    k_rev_fill<<<g, TPB, 0, s>>>(r); note_launch();
    k_rev_sort<<<nblocks(P.n), TPB, 0, s>>>(r); note_launch();
}

void launch_bonds(const ObjDev& P, BondDev& B, bool mixed, cudaStream_t s)
{
    if (B.n <= 0) return;
    if (mixed) {
        k_bonds32<<<nblocks(B.n), TPB, 0, s>>>(P, B);
    } else {
        k_bonds<<<nblocks(B.n), TPB, 0, s>>>(P, B);
    }
    note_launch();
}

void launch_contact_view(const PairListDev& L, long long* keys, int* order, unsigned long long* skey,
                         unsigned long long* key_b, int* idx_b, int* bcount, int* bscan, long long n,
                         long long max_key, const ContactViewDev& v, cudaStream_t s)
{
    if (L.cap_contacts <= 0) return;
    k_view_keys<<<148 * 4, TPB, 0, s>>>(L, keys); note_launch();
    radix_sort_keys(keys, L.cap_contacts, max_key, skey, order, key_b, idx_b, bcount, bscan, s);
    if (n > 0) { k_view_gather<<<148 * 4, TPB, 0, s>>>(L, order, n, v); note_launch(); }
}
void launch_bond_view(const BondDev& B, const BondViewDev& v, cudaStream_t s)
{
    if (B.n > 0) { k_bond_view<<<nblocks(B.n), TPB, 0, s>>>(B, v); note_launch(); }
}

void launch_reduce(ObjDev& P, PairListDev* lists, const int* active, const RevDev& R, const BondDev& B, bool mixed,
                   cudaStream_t s)
{
    if (P.n <= 0) return;
    ReduceArgs r;
    r.P = P;
    for (int k = 0; k < FD_NKIND; ++k) { r.L[k] = lists[k]; r.active[k] = active[k]; }
    r.R = R;
    r.B = B;
    if (mixed) {
        k_reduce<float><<<nblocks(P.n), TPB, 0, s>>>(r);
    } else {
        k_reduce<double><<<nblocks(P.n), TPB, 0, s>>>(r);
    }
    note_launch();
}

}  // namespace fd

// ---------------------------------------------------------------------------
// Prefix sum without allocation.
//
// For callers that cannot allocate device memory when they need the scan:
// code that runs inside a device-memory budget owned by another allocator
// (a framework that has reserved the GPU's memory up front, where a
// cudaMalloc can fail), and code for which cudaMalloc's implicit device-wide
// synchronisation is not acceptable.  The scratch (one int per 4096-element
// tile) lives in a fixed device array of this library instead, so the scan
// is limited to FUNDEM_NOALLOC_SCAN_MAX elements.  Every GPU that loads the
// library keeps the 16 KiB array until the process exits.
//
// The array is shared by all calls on a device and keeps the last call's
// contents.  Nothing in it needs to start at zero: every tile sum the scan
// reads is written earlier in the same call.  Calls that overlap on the GPU
// (concurrent streams) race on the array.
// ---------------------------------------------------------------------------
namespace {
constexpr int NOALLOC_TILES = 4096;
static_assert((long long)NOALLOC_TILES * fd::SCAN_TILE == FUNDEM_NOALLOC_SCAN_MAX, "limit and scratch size differ");
static __device__ __align__(256) int g_noalloc_scan_scratch[NOALLOC_TILES];

constexpr int NOALLOC_MAX_DEVICES = 256;
std::mutex g_noalloc_mutex;
int* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

// device address of the scratch on the current device; looked up once per
// device (host code only sees a stand-in for the array's address)
int noalloc_scratch(int** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return FUNDEM_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        int* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_noalloc_scan_scratch) != cudaSuccess || !p) return FUNDEM_ERR_CUDA;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return FUNDEM_OK;
}
}  // namespace

extern "C" int fundem_prefix_sum_noalloc(int* d_prefix, const int* d_count, long long n, void* stream)
{
    if (n < 0 || (n > 0 && (!d_prefix || !d_count))) return FUNDEM_ERR_ARG;
    if (n > FUNDEM_NOALLOC_SCAN_MAX) return FUNDEM_ERR_ARG;
    if (n == 0) return FUNDEM_OK;
    int* scratch = nullptr;
    const int r = noalloc_scratch(&scratch);
    if (r != FUNDEM_OK) return r;
    // n <= NOALLOC_TILES * SCAN_TILE: the tile sums fit the array and their
    // own scan is a single tile, which needs no further scratch
    fd::scan_inclusive(d_count, d_prefix, n, scratch, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? FUNDEM_OK : FUNDEM_ERR_CUDA;
}
