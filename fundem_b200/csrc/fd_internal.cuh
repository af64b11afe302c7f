// fd_internal.cuh -- shared device types and math for the B200 level-set DEM
// timestep (sm_100a).
//
// State layout in HBM (one simulation):
//   particles  pos/vel/angvel/force/torque : double3 AoS (24 B, the layout the
//              reference exposes through LSParticle::position() etc.,
//              kernel/LSParticle.h:768-777), orientation : fd_quat (32 B,
//              scalar first, myQua.h:10-15), material/geometry ids : int.
//   templates  per-geometry table (FdGeo), SDF pool (double and float copies),
//              surface nodes reordered into spatial clusters of <= 32 nodes
//              (one warp-wide batch each) with a per-cluster bounding sphere,
//              and a per-grid-node lower bound on the distance to any cell
//              where the trilinear SDF can be <= 0 (cluster culling).
//   pair lists per kind (particle-particle, particle-wall, three ghost
//              directions): A-major segments, partner ids sorted ascending,
//              per-pair contact segment and per-pair force/torque results.
//   contacts   per kind: node id, partner id, sliding spring (history) and,
//              when records are requested, point/normal/overlap/energies.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// ---------------------------------------------------------------------------
// error flags written by kernels (bitwise OR into a device word)
// ---------------------------------------------------------------------------
enum FdFlag : unsigned int {
    FD_FLAG_PAIR_OVERFLOW = 1u << 0,      // pair list capacity exceeded
    FD_FLAG_CONTACT_OVERFLOW = 1u << 1,   // contact capacity exceeded
    FD_FLAG_NEIGHBOR_OVERFLOW = 1u << 2,  // a particle has more candidates than the per-particle limit
    FD_FLAG_CLUSTER_OVERFLOW = 1u << 3,   // a template has more clusters than the kernel limit
    FD_FLAG_NONFINITE = 1u << 4,          // NaN/Inf in particle state
    FD_FLAG_INDEX = 1u << 5,              // out-of-range index caught by a bounds check
};

// kinds of pair lists
// (GR90, GR180, GR270: the images of sector periodicity, turned about the z
// axis through the domain's min corner)
enum FdKind { FD_PP = 0, FD_PW = 1, FD_GX = 2, FD_GY = 3, FD_GXY = 4, FD_GR90 = 5, FD_GR180 = 6, FD_GR270 = 7,
              FD_NKIND = 8 };

struct __align__(16) fd_quat { double q0, q1, q2, q3; };
struct fd_sym { double xx, yy, zz, xy, xz, yz; };

// per-geometry template table entry
struct FdGeo {
    double3 origin;        // SDF grid origin in the body frame
    double inv_spacing;    // 1 / grid spacing
    double spacing;
    int3 size;             // grid nodes per axis
    long long sdf_off;     // offset into the SDF pools
    long long dist_off;    // offset into the distance-bound pool (one float per grid node)
    long long cellmin_off; // offset into the cell-minimum pool (one float per cell, rounded down)
    int node_off;          // first node (cluster order) in the node pools
    int node_count;
    int clus_off;          // first cluster in the cluster pool
    int clus_count;
    double radius;         // max |node|: the reference's bounding radius (LSParticle.h:101-107)
    double grid_radius;    // max distance from the body origin to a grid-box corner
    double lip;            // Lipschitz bound of the trilinear SDF, per unit length
    double inv_mass;
    fd_sym inertia;
    fd_sym inv_inertia;
};

struct FdCluster {
    double3 centre;  // body frame
    double radius;   // max distance of its nodes from the centre
    int start;       // first node (cluster order) relative to the geometry's node_off
    int count;       // <= 32
};

// uniform cell grid (spatialGrid, myUtility/mySpatialGrid.h:162-256)
struct FdGrid {
    double3 minb, maxb, inv;
    int3 size;
    long long num;
};

// ---------------------------------------------------------------------------
// double3 helpers (plain arithmetic; the compiler may contract mul+add)
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ double3 mk3(double x, double y, double z) { return make_double3(x, y, z); }
__host__ __device__ __forceinline__ double3 operator+(double3 a, double3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ double3 operator-(double3 a, double3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ double3 operator-(double3 a) { return mk3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ double3 operator*(double3 a, double s) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ double3 operator*(double s, double3 a) { return mk3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ double3& operator+=(double3& a, double3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__host__ __device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ double3 cross3(double3 a, double3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ double length3(double3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
__host__ __device__ __forceinline__ double lengthSq3(double3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
__host__ __device__ __forceinline__ bool fd_is_zero(double x) { return fabs(x) <= 1.0e-20; }  // myVec.h:22-25

#ifdef __CUDACC__
// normalize with the device reciprocal square root, as the reference's
// device path does (myVec.h:121-137)
__device__ __forceinline__ double3 fd_normalize(double3 v)
{
    double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (fd_is_zero(l2)) return mk3(0.0, 0.0, 0.0);
    double inv = rsqrt(l2);
    return mk3(v.x * inv, v.y * inv, v.z * inv);
}
__device__ __forceinline__ fd_quat fd_normalize_q(fd_quat q)  // myQua.h:51-62
{
    double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
    if (fd_is_zero(l2)) return q;
    double inv = rsqrt(l2);
    fd_quat r = {q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv};
    return r;
}
// rotateVectorByQuaternion, plain form (myQua.h:104-114)
__device__ __forceinline__ double3 fd_rot(fd_quat q, double3 v)
{
    const double3 qv = mk3(q.q1, q.q2, q.q3);
    const double3 t = cross3(qv, v) * 2.0;
    return v + t * q.q0 + cross3(qv, t);
}
__device__ __forceinline__ double3 fd_rrot(double3 v, fd_quat q)
{
    const double3 qv = mk3(-q.q1, -q.q2, -q.q3);
    const double3 t = cross3(qv, v) * 2.0;
    return v + t * q.q0 + cross3(qv, t);
}

// ---------------------------------------------------------------------------
// The contact-membership arithmetic, written with explicit fused
// multiply-adds so the result does not depend on the compiler's contraction
// choices: node rotation (myQua.h:104-128), squared length (myVec.h:109-112)
// and trilinear value (LSParticleContactDetectionKernel.cuh:4-32).  The
// pattern is the one nvcc's default contraction gives the reference build:
// in a sum of products the leftmost product is fused first and the sum is
// accumulated left to right; differences of products are handled by xm_sub.
// ---------------------------------------------------------------------------
// a*b - c*d with the left (RIGHT = false) or the right product kept exact
template <bool RIGHT> __device__ __forceinline__ double xm_sub(double a, double b, double c, double d)
{
    return RIGHT ? __fma_rn(-c, d, a * b) : __fma_rn(a, b, -(c * d));
}
template <bool RIGHT> __device__ __forceinline__ double3 xm_cross(double3 a, double3 b)
{
    return mk3(xm_sub<RIGHT>(a.y, b.z, a.z, b.y), xm_sub<RIGHT>(a.z, b.x, a.x, b.z), xm_sub<RIGHT>(a.x, b.y, a.y, b.x));
}
__device__ __forceinline__ double xm_len2(double3 v) { return __fma_rn(v.z, v.z, __fma_rn(v.x, v.x, v.y * v.y)); }
template <bool RIGHT> __device__ __forceinline__ double3 xm_rot_qv(double q0, double3 qv, double3 v)
{
    const double3 t = xm_cross<RIGHT>(qv, v) * 2.0;
    const double3 c = xm_cross<RIGHT>(qv, t);
    return mk3(__fma_rn(t.x, q0, v.x) + c.x, __fma_rn(t.y, q0, v.y) + c.y, __fma_rn(t.z, q0, v.z) + c.z);
}
// the reference build keeps the left product exact in the forward rotation and
// the right one in the reverse rotation (negated quaternion components); this
// reproduces its overlaps bit for bit
__device__ __forceinline__ double3 xm_rot(fd_quat q, double3 v) { return xm_rot_qv<false>(q.q0, mk3(q.q1, q.q2, q.q3), v); }
__device__ __forceinline__ double3 xm_rrot(double3 v, fd_quat q) { return xm_rot_qv<true>(q.q0, mk3(-q.q1, -q.q2, -q.q3), v); }
__device__ __forceinline__ double xm_trilinear(double x, double y, double z, const double p[8])
{
    const double wx0 = 1.0 - x, wx1 = x, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
    double s = __fma_rn(p[0] * wx0 * wy0, wz0, p[1] * wx1 * wy0 * wz0);
    s = __fma_rn(p[2] * wx0 * wy1, wz0, s);
    s = __fma_rn(p[3] * wx1 * wy1, wz0, s);
    s = __fma_rn(p[4] * wx0 * wy0, wz1, s);
    s = __fma_rn(p[5] * wx1 * wy0, wz1, s);
    s = __fma_rn(p[6] * wx0 * wy1, wz1, s);
    s = __fma_rn(p[7] * wx1 * wy1, wz1, s);
    return s;
}
// interpolateLevelSetFunctionGradient with its `const int x` parameter
// (LSParticleContactDetectionKernel.cuh:34-77): the x weight uses the
// truncated coordinate.
__device__ __forceinline__ double3 fd_gradient_q(double xd, double y, double z, const double p[8])
{
    const int xi = (int)xd;
    const double wx0 = 1.0 - xi, wx1 = xi, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
    const double gx = (p[1] - p[0]) * wy0 * wz0 + (p[3] - p[2]) * wy1 * wz0 + (p[5] - p[4]) * wy0 * wz1 +
                      (p[7] - p[6]) * wy1 * wz1;
    const double gy = (p[2] - p[0]) * wx0 * wz0 + (p[3] - p[1]) * wx1 * wz0 + (p[6] - p[4]) * wx0 * wz1 +
                      (p[7] - p[5]) * wx1 * wz1;
    const double gz = (p[4] - p[0]) * wx0 * wy0 + (p[5] - p[1]) * wx1 * wy0 + (p[6] - p[2]) * wx0 * wy1 +
                      (p[7] - p[3]) * wx1 * wy1;
    return mk3(gx, gy, gz);
}

// symmetric 3x3 helpers (myMat.h:75-158)
__device__ __forceinline__ double3 fd_smv(fd_sym m, double3 v)
{
    return mk3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
               m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
__device__ __forceinline__ fd_sym fd_rot_tensor(fd_quat q, fd_sym I)
{
    const double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
    const double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
    const double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
    const double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
    const double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
    const double r0x = I.xx * a + I.xy * b + I.xz * c, r0y = I.xy * a + I.yy * b + I.yz * c,
                 r0z = I.xz * a + I.yz * b + I.zz * c;
    const double r1x = I.xx * d + I.xy * e + I.xz * f, r1y = I.xy * d + I.yy * e + I.yz * f,
                 r1z = I.xz * d + I.yz * e + I.zz * f;
    const double r2x = I.xx * g + I.xy * h + I.xz * i, r2y = I.xy * g + I.yy * h + I.yz * i,
                 r2z = I.xz * g + I.yz * h + I.zz * i;
    fd_sym r;
    r.xx = r0x * a + r0y * b + r0z * c;
    r.yy = r1x * d + r1y * e + r1z * f;
    r.zz = r2x * g + r2y * h + r2z * i;
    r.xy = r0x * d + r0y * e + r0z * f;
    r.xz = r0x * g + r0y * h + r0z * i;
    r.yz = r1x * g + r1y * h + r1z * i;
    return r;
}

// calculateGridPosition (mySpatialGrid.h:24-31): truncation toward zero
__device__ __forceinline__ int3 fd_cell_of(double3 p, const FdGrid& g)
{
    return make_int3((int)((p.x - g.minb.x) * g.inv.x), (int)((p.y - g.minb.y) * g.inv.y),
                     (int)((p.z - g.minb.z) * g.inv.z));
}
// linearIndex3D in 64 bits (myVec.h:232-235)
__device__ __forceinline__ long long fd_lin3(int x, int y, int z, int3 s)
{
    return (long long)z * s.y * s.x + (long long)y * s.x + x;
}
// calculateHashKernel (mySpatialGrid.cu:4-26): -1 outside [min, max)
__device__ __forceinline__ long long fd_hash(double3 p, const FdGrid& g)
{
    if (p.x < g.minb.x || p.x >= g.maxb.x) return -1;
    if (p.y < g.minb.y || p.y >= g.maxb.y) return -1;
    if (p.z < g.minb.z || p.z >= g.maxb.z) return -1;
    const int3 c = fd_cell_of(p, g);
    return fd_lin3(c.x, c.y, c.z, g.size);
}
// the clamped 27-cell range a node searches (LSParticleContactDetectionKernel.cu:38-46)
__device__ __forceinline__ void fd_node_range(double3 gp, const FdGrid& g, int3& lo, int3& hi)
{
    int3 c = fd_cell_of(gp, g);
    int3 gs = make_int3(-1, -1, -1), ge = make_int3(1, 1, 1);
    if (c.x <= 0) { c.x = 0; gs.x = 0; }
    if (c.x >= g.size.x - 1) { c.x = g.size.x - 1; ge.x = 0; }
    if (c.y <= 0) { c.y = 0; gs.y = 0; }
    if (c.y >= g.size.y - 1) { c.y = g.size.y - 1; ge.y = 0; }
    if (c.z <= 0) { c.z = 0; gs.z = 0; }
    if (c.z >= g.size.z - 1) { c.z = g.size.z - 1; ge.z = 0; }
    lo = make_int3(c.x + gs.x, c.y + gs.y, c.z + gs.z);
    hi = make_int3(c.x + ge.x, c.y + ge.y, c.z + ge.z);
}
#endif
