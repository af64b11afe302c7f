// fd_api.cu -- host side of libfundem_b200: template preprocessing, device
// memory, step orchestration and the C ABI declared in include/fundem_b200.h.
#include "../../include/fundem_b200.h"
#include "fd_adjoint.cuh"
#include "fd_kernels.cuh"

#include <algorithm>
#include <atomic>
#include <map>
#include <tuple>
#include <cfloat>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using fd::CellTableDev;
using fd::GeoSetDev;
using fd::ObjDev;
using fd::PairListDev;

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
#define FD_CUDA(x)                                                                                   \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// Copies and fills issued on the legacy default stream are not ordered with
// a simulation stream created non-blocking (as PyTorch's streams are), and
// cudaMemset and device-to-device cudaMemcpy may return before they finish.
// The array allocations below, which know no stream, wait for the legacy
// stream after them; everything else goes on the simulation's stream.
inline cudaError_t after_legacy(cudaError_t e) { return e != cudaSuccess ? e : cudaStreamSynchronize(cudaStreamLegacy); }

// A captured step graph holds raw device pointers and is rebuilt when one of
// its simulation's arrays was (re)allocated since the capture.  Allocations
// made inside a call on a simulation (guard() sets t_sim_epoch) bump that
// simulation's counter; any other allocation bumps the global counter, which
// every graph also checks.
std::atomic<unsigned long long> g_alloc_epoch{0};
thread_local unsigned long long* t_sim_epoch = nullptr;
inline void bump_alloc_epoch()
{
    if (t_sim_epoch) ++*t_sim_epoch;
    else g_alloc_epoch.fetch_add(1);
}

template <typename T> struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void alloc(size_t count, bool zero = true)
    {
        release();
        n = count;
        if (count == 0) return;
        bump_alloc_epoch();
        FD_CUDA(cudaMalloc((void**)&p, sizeof(T) * count));
        if (zero) FD_CUDA(after_legacy(cudaMemset(p, 0, sizeof(T) * count)));
    }
    // grow keeping the first `keep` elements
    void grow(size_t count, size_t keep)
    {
        if (count <= n) return;
        bump_alloc_epoch();
        T* q = nullptr;
        FD_CUDA(cudaMalloc((void**)&q, sizeof(T) * count));
        FD_CUDA(after_legacy(cudaMemset(q, 0, sizeof(T) * count)));
        if (p && keep) FD_CUDA(after_legacy(cudaMemcpy(q, p, sizeof(T) * std::min(keep, n), cudaMemcpyDeviceToDevice)));
        if (p) cudaFree(p);
        p = q;
        n = count;
    }
    void upload(const T* h, size_t count, cudaStream_t s)
    {
        if (count) FD_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s)
    {
        if (h.size() > n) alloc(h.size(), false);
        upload(h.data(), h.size(), s);
    }
};

// ---------------------------------------------------------------------------
// host-side template preprocessing
// ---------------------------------------------------------------------------
struct HostGeo {
    double mass = 0.0;
    fd_sym inertia{0, 0, 0, 0, 0, 0};
    double3 origin{0, 0, 0};
    double spacing = 1.0;
    int3 size{2, 2, 2};
    std::vector<double> sdf;
    std::vector<double3> nodes;
};

// Inverse of a symmetric 3x3 matrix by cofactors.  FUNDEM_INERTIA_REFERENCE
// keeps the absolute |det| < 1e-30 -> zero rule of myMat.h:163-194, under
// which mm-scale bodies (det of order 1e-34) never turn.
// FUNDEM_INERTIA_PHYSICAL tests the determinant against the cube of the
// largest diagonal entry instead, so only a matrix singular to 1e-12 relative
// (no mass, a line or point body) gives zero, at any length scale.
fd_sym host_inverse(const fd_sym& A, int mode = FUNDEM_INERTIA_REFERENCE)
{
    const double det = A.xx * (A.yy * A.zz - A.yz * A.yz) + A.xy * (A.yz * A.xz - A.xy * A.zz) +
                       A.xz * (A.xy * A.yz - A.yy * A.xz);
    fd_sym r{0, 0, 0, 0, 0, 0};
    if (mode == FUNDEM_INERTIA_PHYSICAL) {
        const double m = std::max(std::fabs(A.xx), std::max(std::fabs(A.yy), std::fabs(A.zz)));
        if (!(m > 0.0) || !(std::fabs(det) > 1e-12 * m * m * m)) return r;
    } else if (std::fabs(det) < 1e-30) {
        return r;
    }
    const double di = 1.0 / det;
    r.xx = (A.yy * A.zz - A.yz * A.yz) * di;
    r.yy = (A.xx * A.zz - A.xz * A.xz) * di;
    r.zz = (A.xx * A.yy - A.xy * A.xy) * di;
    r.xy = -(A.xy * A.zz - A.xz * A.yz) * di;
    r.xz = (A.xy * A.yz - A.xz * A.yy) * di;
    r.yz = -(A.xx * A.yz - A.xz * A.xy) * di;
    return r;
}

double host_len(double3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// Split node indices into spatially coherent clusters of at most 32 nodes:
// recursive bisection along the widest axis, left part a multiple of 32.
void cluster_nodes(const std::vector<double3>& nodes, std::vector<int>& idx, int lo, int hi,
                   std::vector<std::pair<int, int>>& out)
{
    const int n = hi - lo;
    if (n <= 32) {
        out.push_back({lo, n});
        return;
    }
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int k = lo; k < hi; ++k) {
        const double3 p = nodes[idx[k]];
        const double v[3] = {p.x, p.y, p.z};
        for (int d = 0; d < 3; ++d) { mn[d] = std::min(mn[d], v[d]); mx[d] = std::max(mx[d], v[d]); }
    }
    int axis = 0;
    for (int d = 1; d < 3; ++d)
        if (mx[d] - mn[d] > mx[axis] - mn[axis]) axis = d;
    auto key = [&](int i) { const double3 p = nodes[i]; return axis == 0 ? p.x : (axis == 1 ? p.y : p.z); };
    std::stable_sort(idx.begin() + lo, idx.begin() + hi, [&](int a, int b) { return key(a) < key(b); });
    int left = 32 * (int)std::lround(n / 64.0);
    if (left <= 0) left = 32;
    if (left >= n) left = n - n / 2;
    cluster_nodes(nodes, idx, lo, lo + left, out);
    cluster_nodes(nodes, idx, lo + left, hi, out);
}

// Lower bound, for every grid node, of the distance to the union of cells
// whose corner minimum is <= 0 (the only cells where the trilinear SDF can be
// <= 0).  Exact squared box distance by three separable min-plus passes.
std::vector<float> distance_bound(const HostGeo& g)
{
    const int nx = g.size.x, ny = g.size.y, nz = g.size.z;
    const int cx = nx - 1, cy = ny - 1, cz = nz - 1;
    const double INF = 1e300;
    auto S = [&](int x, int y, int z) { return g.sdf[(size_t)z * ny * nx + (size_t)y * nx + x]; };
    std::vector<double> F((size_t)cx * cy * cz, INF);
    for (int z = 0; z < cz; ++z)
        for (int y = 0; y < cy; ++y)
            for (int x = 0; x < cx; ++x) {
                double m = S(x, y, z);
                for (int dz = 0; dz < 2; ++dz)
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) m = std::min(m, S(x + dx, y + dy, z + dz));
                if (m <= 0.0) F[(size_t)z * cy * cx + (size_t)y * cx + x] = 0.0;
            }
    auto gap2 = [](int c, int a) {
        const int g = std::max(0, std::max(c - a, a - c - 1));
        return (double)g * g;
    };
    // pass x: cells (cz, cy, cx) -> (cz, cy, nx)
    std::vector<double> D1((size_t)cz * cy * nx, INF);
    for (int z = 0; z < cz; ++z)
        for (int y = 0; y < cy; ++y)
            for (int a = 0; a < nx; ++a) {
                double m = INF;
                for (int c = 0; c < cx; ++c) {
                    const double f = F[(size_t)z * cy * cx + (size_t)y * cx + c];
                    if (f < INF) m = std::min(m, f + gap2(c, a));
                }
                D1[(size_t)z * cy * nx + (size_t)y * nx + a] = m;
            }
    std::vector<double> D2((size_t)cz * ny * nx, INF);
    for (int z = 0; z < cz; ++z)
        for (int a = 0; a < ny; ++a)
            for (int x = 0; x < nx; ++x) {
                double m = INF;
                for (int c = 0; c < cy; ++c) {
                    const double f = D1[(size_t)z * cy * nx + (size_t)c * nx + x];
                    if (f < INF) m = std::min(m, f + gap2(c, a));
                }
                D2[(size_t)z * ny * nx + (size_t)a * nx + x] = m;
            }
    std::vector<float> out((size_t)nz * ny * nx);
    for (int a = 0; a < nz; ++a)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                double m = INF;
                for (int c = 0; c < cz; ++c) {
                    const double f = D2[(size_t)c * ny * nx + (size_t)y * nx + x];
                    if (f < INF) m = std::min(m, f + gap2(c, a));
                }
                float r;
                if (m >= INF) r = FLT_MAX;
                else {
                    const double d = std::sqrt(m) * g.spacing * (1.0 - 1e-12);
                    r = (float)d;
                    if ((double)r > d) r = std::nextafter(r, 0.0f);
                }
                out[(size_t)a * ny * nx + (size_t)y * nx + x] = r;
            }
    return out;
}

double lipschitz_bound(const HostGeo& g)
{
    const int nx = g.size.x, ny = g.size.y, nz = g.size.z;
    auto S = [&](int x, int y, int z) { return g.sdf[(size_t)z * ny * nx + (size_t)y * nx + x]; };
    double L[3] = {0, 0, 0};
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                if (x + 1 < nx) L[0] = std::max(L[0], std::fabs(S(x + 1, y, z) - S(x, y, z)));
                if (y + 1 < ny) L[1] = std::max(L[1], std::fabs(S(x, y + 1, z) - S(x, y, z)));
                if (z + 1 < nz) L[2] = std::max(L[2], std::fabs(S(x, y, z + 1) - S(x, y, z)));
            }
    return std::sqrt(L[0] * L[0] + L[1] * L[1] + L[2] * L[2]) / g.spacing * (1.0 + 1e-9);
}

struct GeoSetHost {
    std::vector<HostGeo> geos;
    // device
    DevArray<FdGeo> d_geo;
    DevArray<double> d_sdf;
    DevArray<float> d_sdf32;
    DevArray<float> d_dist;
    DevArray<float> d_cellmin;
    DevArray<double3> d_nodes;
    DevArray<int> d_lid;
    DevArray<FdCluster> d_clusters;
    DevArray<float4> d_nodes32, d_clus_sphere;
    DevArray<int2> d_clus_range;
    std::vector<FdGeo> table;
    // node key (cluster-order index) of every node, by pool offset of the
    // geometry plus the node's original local index
    std::vector<int> key_of;
    double rmax = 0.0, grid_rmax = 0.0;
    bool built = false;

    void build(bool wall, int inertia_mode, cudaStream_t s)
    {
        table.clear();
        key_of.clear();
        std::vector<double> sdf;
        std::vector<float> sdf32, dist, cellmin;
        std::vector<double3> nodes;
        std::vector<int> lid;
        std::vector<FdCluster> clusters;
        rmax = grid_rmax = 0.0;
        for (const HostGeo& g : geos) {
            FdGeo t{};
            t.origin = g.origin;
            t.spacing = g.spacing;
            t.inv_spacing = 1.0 / g.spacing;
            t.size = g.size;
            t.sdf_off = (long long)sdf.size();
            t.dist_off = (long long)dist.size();
            t.cellmin_off = (long long)cellmin.size();
            {
                // per-cell minimum of the eight corner values, rounded down
                const int nx = g.size.x, ny = g.size.y, nz = g.size.z;
                auto S = [&](int x, int y, int z) { return g.sdf[(size_t)z * ny * nx + (size_t)y * nx + x]; };
                for (int z = 0; z < nz - 1; ++z)
                    for (int y = 0; y < ny - 1; ++y)
                        for (int x = 0; x < nx - 1; ++x) {
                            double m = S(x, y, z);
                            for (int d = 1; d < 8; ++d) m = std::min(m, S(x + (d & 1), y + ((d >> 1) & 1), z + (d >> 2)));
                            float f = (float)m;
                            if ((double)f > m) f = std::nextafter(f, -FLT_MAX);
                            cellmin.push_back(f);
                        }
            }
            sdf.insert(sdf.end(), g.sdf.begin(), g.sdf.end());
            for (double v : g.sdf) sdf32.push_back((float)v);
            std::vector<float> D = distance_bound(g);
            dist.insert(dist.end(), D.begin(), D.end());
            double r = 0.0;
            for (const double3& p : g.nodes) r = std::max(r, host_len(p));
            t.radius = r;
            double gr = 0.0;
            for (int c = 0; c < 8; ++c) {
                const double3 corner = make_double3(g.origin.x + ((c & 1) ? (g.size.x - 1) * g.spacing : 0.0),
                                                    g.origin.y + ((c & 2) ? (g.size.y - 1) * g.spacing : 0.0),
                                                    g.origin.z + ((c & 4) ? (g.size.z - 1) * g.spacing : 0.0));
                gr = std::max(gr, host_len(corner));
            }
            t.grid_radius = gr * (1.0 + 1e-9);
            t.lip = lipschitz_bound(g);
            const double mass = wall ? 0.0 : g.mass;
            t.inv_mass = mass > 0.0 ? 1.0 / mass : 0.0;
            t.inertia = mass > 0.0 ? g.inertia : fd_sym{0, 0, 0, 0, 0, 0};
            t.inv_inertia = host_inverse(t.inertia, inertia_mode);
            // clusters
            std::vector<int> idx(g.nodes.size());
            std::iota(idx.begin(), idx.end(), 0);
            std::vector<std::pair<int, int>> parts;
            if (!idx.empty()) cluster_nodes(g.nodes, idx, 0, (int)idx.size(), parts);
            t.node_off = (int)nodes.size();
            t.node_count = (int)g.nodes.size();
            t.clus_off = (int)clusters.size();
            t.clus_count = (int)parts.size();
            for (auto& pr : parts) {
                FdCluster cl{};
                double3 c = make_double3(0, 0, 0);
                for (int k = pr.first; k < pr.first + pr.second; ++k) {
                    const double3 p = g.nodes[idx[k]];
                    c.x += p.x; c.y += p.y; c.z += p.z;
                }
                c.x /= pr.second; c.y /= pr.second; c.z /= pr.second;
                double rr = 0.0;
                for (int k = pr.first; k < pr.first + pr.second; ++k) {
                    const double3 p = g.nodes[idx[k]];
                    rr = std::max(rr, host_len(make_double3(p.x - c.x, p.y - c.y, p.z - c.z)));
                }
                cl.centre = c;
                cl.radius = rr;
                cl.start = pr.first;
                cl.count = pr.second;
                clusters.push_back(cl);
            }
            key_of.resize(t.node_off + idx.size());
            for (size_t j = 0; j < idx.size(); ++j) {
                nodes.push_back(g.nodes[idx[j]]);
                lid.push_back(idx[j]);
                key_of[t.node_off + idx[j]] = (int)j;
            }
            rmax = std::max(rmax, t.radius);
            grid_rmax = std::max(grid_rmax, t.grid_radius);
            table.push_back(t);
        }
        d_geo.alloc(std::max<size_t>(table.size(), 1));
        d_geo.upload(table.data(), table.size(), s);
        d_sdf.alloc(std::max<size_t>(sdf.size(), 1));
        d_sdf.upload(sdf.data(), sdf.size(), s);
        d_sdf32.alloc(std::max<size_t>(sdf32.size(), 1));
        d_sdf32.upload(sdf32.data(), sdf32.size(), s);
        d_dist.alloc(std::max<size_t>(dist.size(), 1));
        d_dist.upload(dist.data(), dist.size(), s);
        d_cellmin.alloc(std::max<size_t>(cellmin.size(), 1));
        d_cellmin.upload(cellmin.data(), cellmin.size(), s);
        d_nodes.alloc(std::max<size_t>(nodes.size(), 1));
        d_nodes.upload(nodes.data(), nodes.size(), s);
        d_lid.alloc(std::max<size_t>(lid.size(), 1));
        d_lid.upload(lid.data(), lid.size(), s);
        d_clusters.alloc(std::max<size_t>(clusters.size(), 1));
        d_clusters.upload(clusters.data(), clusters.size(), s);
        // single-precision copies for the culling stages
        std::vector<float4> n32(nodes.size()), cs32(clusters.size());
        std::vector<int2> cr(clusters.size());
        for (size_t k = 0; k < nodes.size(); ++k)
            n32[k] = make_float4((float)nodes[k].x, (float)nodes[k].y, (float)nodes[k].z, 0.f);
        for (size_t k = 0; k < clusters.size(); ++k) {
            const FdCluster& c = clusters[k];
            cs32[k] = make_float4((float)c.centre.x, (float)c.centre.y, (float)c.centre.z, (float)c.radius);
            cr[k] = make_int2(c.start, c.count);
        }
        d_nodes32.alloc(std::max<size_t>(n32.size(), 1));
        d_nodes32.upload(n32.data(), n32.size(), s);
        d_clus_sphere.alloc(std::max<size_t>(cs32.size(), 1));
        d_clus_sphere.upload(cs32.data(), cs32.size(), s);
        d_clus_range.alloc(std::max<size_t>(cr.size(), 1));
        d_clus_range.upload(cr.data(), cr.size(), s);
        FD_CUDA(cudaStreamSynchronize(s));
        built = true;
    }

    GeoSetDev view() const
    {
        GeoSetDev v;
        v.n = (int)table.size();
        v.geo = d_geo.p;
        v.sdf = d_sdf.p;
        v.sdf32 = d_sdf32.p;
        v.dist = d_dist.p;
        v.cellmin = d_cellmin.p;
        v.nodes = d_nodes.p;
        v.node_lid = d_lid.p;
        v.clusters = d_clusters.p;
        v.nodes32 = d_nodes32.p;
        v.clus_sphere = d_clus_sphere.p;
        v.clus_range = d_clus_range.p;
        v.rmax = rmax;
        v.grid_rmax = grid_rmax;
        return v;
    }
};

struct MatHost {
    std::vector<double> kn, ks, mu, e;
    DevArray<double> d_kn, d_ks, d_mu, d_e;
    void upload(cudaStream_t s)
    {
        d_kn.upload(kn, s);
        d_ks.upload(ks, s);
        d_mu.upload(mu, s);
        d_e.upload(e, s);
    }
    fd::MatDev view() const { return fd::MatDev{d_kn.p, d_ks.p, d_mu.p, d_e.p}; }
};

struct ObjHost {
    std::vector<double3> pos, vel, angvel, force, torque;
    std::vector<fd_quat> q;
    std::vector<int> mat, geo;
    DevArray<double3> d_pos, d_vel, d_angvel, d_force, d_torque;
    DevArray<fd_quat> d_q;
    DevArray<int> d_mat, d_geo, d_node_base;
    DevArray<float4> d_rot;
    DevArray<long long> d_hash;
    int n_dev = 0;
    bool dirty = true;

    int n() const { return (int)pos.size(); }
    void upload(const std::vector<int>& node_base, cudaStream_t s)
    {
        const size_t n = pos.size();
        const size_t m = std::max<size_t>(n, 1);
        d_pos.alloc(m); d_vel.alloc(m); d_angvel.alloc(m); d_force.alloc(m); d_torque.alloc(m);
        d_q.alloc(m); d_mat.alloc(m); d_geo.alloc(m); d_hash.alloc(m); d_node_base.alloc(m); d_rot.alloc(3 * m);
        d_pos.upload(pos.data(), n, s); d_vel.upload(vel.data(), n, s); d_angvel.upload(angvel.data(), n, s);
        d_force.upload(force.data(), n, s); d_torque.upload(torque.data(), n, s); d_q.upload(q.data(), n, s);
        d_mat.upload(mat.data(), n, s); d_geo.upload(geo.data(), n, s);
        d_node_base.upload(node_base.data(), std::min(n, node_base.size()), s);
        n_dev = (int)n;
        dirty = false;
    }
    ObjDev view()
    {
        ObjDev v;
        v.n = n_dev;
        v.pos = d_pos.p; v.vel = d_vel.p; v.angvel = d_angvel.p; v.force = d_force.p; v.torque = d_torque.p;
        v.q = d_q.p; v.mat = d_mat.p; v.geo = d_geo.p; v.hash = d_hash.p; v.node_base = d_node_base.p;
        v.rot = d_rot.p;
        return v;
    }
};

struct PairGen {
    DevArray<int> pairA, pairB, seg_off, seg_cnt, c_off, c_cnt, c_node, c_slave, c_k, counters;
    DevArray<double> pf, c_spring, c_point, c_normal, c_overlap, c_en, c_es;
};

struct PairList {
    PairGen gen[2];
    int cur = 0;
    int cap_pairs = 0, cap_contacts = 0;
    int n_obj = 0;
    // (node, partner) of the list set_contacts uploaded last, in slot order
    std::vector<int> up_node, up_partner;
    // slot and pair scratch of the current step only
    DevArray<int> c_pair, c_hit, p_hist_cnt;
    DevArray<float> c_phi0;  // pair cache: slot bounds of the last rebuild
    DevArray<float> p_bound; // pair cache: per-pair drift bound of a carried step
    DevArray<int> carry_n;   // pair cache: carried steps since the layout was built
    DevArray<int> c_test, n_test;  // pair cache: slots listed for the predicate pass
    DevArray<double> c_force;
    DevArray<int4> p_aux;
    bool allocated = false;

    void alloc(int nobj, int capp, int capc)
    {
        n_obj = nobj;
        cap_pairs = std::max(capp, 16);
        cap_contacts = std::max(capc, 64);
        const size_t m = std::max(nobj, 1);
        for (PairGen& g : gen) {
            g.pairA.alloc(cap_pairs); g.pairB.alloc(cap_pairs); g.seg_off.alloc(m); g.seg_cnt.alloc(m);
            g.c_off.alloc(cap_pairs); g.c_cnt.alloc(cap_pairs); g.pf.alloc((size_t)cap_pairs * 9);
            g.c_node.alloc(cap_contacts); g.c_slave.alloc(cap_contacts); g.c_k.alloc(cap_contacts);
            g.c_spring.alloc((size_t)cap_contacts * 3);
            g.c_point.alloc((size_t)cap_contacts * 3); g.c_normal.alloc((size_t)cap_contacts * 3);
            g.c_overlap.alloc(cap_contacts); g.c_en.alloc(cap_contacts); g.c_es.alloc(cap_contacts);
            g.counters.alloc(3);
        }
        c_pair.alloc(cap_contacts); c_hit.alloc(cap_contacts, false); c_force.alloc((size_t)cap_contacts * 9);
        c_phi0.alloc(cap_contacts, false);
        p_aux.alloc(cap_pairs); p_hist_cnt.alloc(cap_pairs); p_bound.alloc(cap_pairs, false);
        carry_n.alloc(1);
        c_test.alloc(cap_contacts, false);
        n_test.alloc(1);
        allocated = true;
    }
    void grow(int capp, int capc)
    {
        if (capp > cap_pairs) {
            for (PairGen& g : gen) {
                g.pairA.grow(capp, cap_pairs); g.pairB.grow(capp, cap_pairs); g.c_off.grow(capp, cap_pairs);
                g.c_cnt.grow(capp, cap_pairs); g.pf.grow((size_t)capp * 9, (size_t)cap_pairs * 9);
            }
            p_aux.grow(capp, 0);
            p_hist_cnt.grow(capp, 0);
            p_bound.grow(capp, 0);
            cap_pairs = capp;
        }
        if (capc > cap_contacts) {
            for (PairGen& g : gen) {
                g.c_node.grow(capc, cap_contacts); g.c_slave.grow(capc, cap_contacts); g.c_k.grow(capc, cap_contacts);
                g.c_spring.grow((size_t)capc * 3, (size_t)cap_contacts * 3);
                g.c_point.grow((size_t)capc * 3, (size_t)cap_contacts * 3);
                g.c_normal.grow((size_t)capc * 3, (size_t)cap_contacts * 3);
                g.c_overlap.grow(capc, cap_contacts); g.c_en.grow(capc, cap_contacts); g.c_es.grow(capc, cap_contacts);
            }
            c_pair.grow(capc, 0);
            c_hit.grow(capc, 0);
            c_phi0.grow(capc, 0);  // rewritten by the rebuild a grow forces
            c_test.grow(capc, 0);
            c_force.grow((size_t)capc * 9, 0);
            cap_contacts = capc;
        }
    }
    PairListDev view()
    {
        PairGen& c = gen[cur];
        PairGen& o = gen[cur ^ 1];
        PairListDev v;
        v.pairA = c.pairA.p; v.pairB = c.pairB.p; v.seg_off = c.seg_off.p; v.seg_cnt = c.seg_cnt.p;
        v.c_off = c.c_off.p; v.c_cnt = c.c_cnt.p; v.pf = c.pf.p; v.n_pairs = c.counters.p; v.cap_pairs = cap_pairs;
        v.o_pairA = o.pairA.p; v.o_counters = o.counters.p;
        v.o_pairB = o.pairB.p; v.o_seg_off = o.seg_off.p; v.o_seg_cnt = o.seg_cnt.p; v.o_c_off = o.c_off.p;
        v.o_c_cnt = o.c_cnt.p;
        v.c_node = c.c_node.p; v.c_slave = c.c_slave.p; v.c_spring = c.c_spring.p; v.c_point = c.c_point.p;
        v.c_normal = c.c_normal.p; v.c_overlap = c.c_overlap.p; v.c_en = c.c_en.p; v.c_es = c.c_es.p;
        v.n_slots = c.counters.p + 1; v.n_hits = c.counters.p + 2; v.cap_contacts = cap_contacts;
        v.c_pair = c_pair.p; v.c_hit = c_hit.p; v.c_k = c.c_k.p; v.o_c_k = o.c_k.p; v.c_force = c_force.p; v.p_aux = p_aux.p; v.p_hist_cnt = p_hist_cnt.p;
        v.o_c_node = o.c_node.p; v.o_c_spring = o.c_spring.p;
        v.c_phi0 = c_phi0.p;
        v.p_bound = p_bound.p;
        v.carry_n = carry_n.p;
        v.c_test = c_test.p;
        v.n_test = n_test.p;
        return v;
    }
};

// a grid with more cells than this (and than 4 per object) keeps a hash table
// of its occupied cells instead of a dense one
constexpr long long DENSE_CELLS = 1ll << 22;

struct CellTable {
    FdGrid g{};
    bool hashed = false;
    DevArray<int> count, start, fill, sorted, idx_b, bcount, bscan;
    DevArray<unsigned long long> skey, key_b, hkey;
    DevArray<int2> hval;
    unsigned long long hmask = 0;
    int cap = 0;
    void alloc(const FdGrid& grid, int nobj)
    {
        g = grid;
        const size_t m = (size_t)std::max(nobj, 1);
        hashed = g.num > std::max<long long>(4ll * (long long)m, DENSE_CELLS);
        if (hashed) {
            size_t H = 1024;
            while (H < 2 * m) H <<= 1;
            hkey.alloc(H, false);
            hval.alloc(H, false);
            hmask = H - 1;
            count.release();
            start.release();
            fill.release();
        } else {
            count.alloc((size_t)std::max<long long>(g.num, 1));
            start.alloc((size_t)std::max<long long>(g.num, 1), false);
            fill.alloc((size_t)std::max<long long>(g.num, 1), false);
            hkey.release();
            hval.release();
            hmask = 0;
        }
        sorted.alloc(m);
        skey.alloc(m, false);
        key_b.alloc(m, false);
        idx_b.alloc(m, false);
        size_t bc = 0, bs = 0;
        fd::radix_sort_scratch((int)m, bc, bs);
        bcount.alloc(bc, false);
        bscan.alloc(bs, false);
        cap = (int)m;
    }
    CellTableDev view()
    {
        CellTableDev v{};
        v.g = g;
        v.hashed = hashed ? 1 : 0;
        v.count = count.p; v.start = start.p; v.fill = fill.p; v.hkey = hkey.p; v.hval = hval.p; v.hmask = hmask;
        v.sorted = sorted.p; v.skey = skey.p; v.key_b = key_b.p; v.idx_b = idx_b.p;
        v.bcount = bcount.p; v.bscan_tmp = bscan.p; v.nobj_cap = cap;
        return v;
    }
};

struct Ghost {
    DevArray<double3> pos;
    DevArray<long long> hash;
    DevArray<int> occ, searchers, nsearch;
    CellTable cells;
    // sector images only: orientation, velocity, rotation rows
    DevArray<fd_quat> q;
    DevArray<double3> vel;
    DevArray<float4> rot;
    // translated images under the pair cache: which particles have an image
    DevArray<unsigned char> live;
    bool active = false;
    // live: null unless the pair cache covers this image set
    fd::GhostDev view(bool with_live = false)
    {
        return fd::GhostDev{pos.p, hash.p, cells.view(), occ.p, searchers.p, nsearch.p, q.p, vel.p, rot.p,
                            with_live ? live.p : nullptr};
    }
};

struct BondHost {
    std::vector<int> master, slave, active;
    std::vector<double3> point;
    std::vector<double> B, radius, L0, ts, coh, mu, energy;
    std::vector<double3> frames;
    DevArray<int> d_master, d_slave, d_active, d_plist_off, d_plist;
    DevArray<double3> d_point, d_frames;
    DevArray<double> d_B, d_radius, d_L0, d_ts, d_coh, d_mu, d_energy, d_out;
    int n_dev = 0;
    bool dirty = false;
};

}  // namespace

// ---------------------------------------------------------------------------
// the simulation object
// ---------------------------------------------------------------------------
// steps between list-capacity checks inside fundem_step (each check
// synchronises the stream once)
constexpr int CAPACITY_CHECK = 64;
// particle counts from which the particle-particle broad phase keeps a
// neighbour list, and its skin as a fraction of the largest bounding radius
constexpr int NL_MIN_PARTICLES = 8192;
constexpr double NL_SKIN = 0.15;
// pair cache (fundem_set_pair_cache): default skin as a fraction of the
// largest particle bounding radius, and the particle count from which the
// default mode keeps the cache
constexpr double PC_SKIN = 0.01;
constexpr int PC_MIN_PARTICLES = 8192;

// adjoint: per-step records of the contact lists and bonds over one
// checkpoint segment, the host checkpoints, and the reverse-sweep arrays
struct AdjTape {
    int steps = 0;
    int cap[FD_NKIND] = {0, 0, 0, 0, 0};
    DevArray<int> ints[FD_NKIND];        // 9 ints per slot per step
    DevArray<double> dbl[FD_NKIND];      // 16 doubles per slot per step
    DevArray<double> prot;               // turning bodies: ADJ_PREC per particle and step, K + 1 steps
    DevArray<int> nslots;                // per step and kind
    int nbond = 0;
    DevArray<int> bond_active;           // per step and bond
    DevArray<double> bond_rij;           // 3 per step and bond
    DevArray<double> bond_dn;            // 3 per step and bond: n1j - n1i
    fd::AdjRec rec(int k, int t)
    {
        fd::AdjRec r{};
        const long long c = cap[k];
        int* I = ints[k].p + 9ll * c * t;
        double* D = dbl[k].p + 16ll * c * t;
        r.hit = I; r.A = I + c; r.Bp = I + 2 * c; r.B = I + 3 * c; r.geoB = I + 4 * c; r.matB = I + 5 * c;
        r.nid = I + 6 * c; r.hist = I + 7 * c; r.wrap = I + 8 * c;
        r.rel = D; r.vc = D + 3 * c; r.sprev = D + 6 * c; r.qB = D + 9 * c; r.arm = D + 13 * c;
        r.cap = cap[k];
        return r;
    }
    int* ns(int k, int t) { return nslots.p + (long long)t * FD_NKIND + k; }
};

struct AdjCheckpoint {
    std::vector<double> pos, vel, angvel, quat, force, torque;
    std::vector<double> wpos, wvel, wangvel, wquat, wforce, wtorque;
    std::vector<int> node[FD_NKIND], partner[FD_NKIND];
    std::vector<double> spring[FD_NKIND];
    std::vector<int> bond_active;
};

struct AdjState {
    bool on = false;
    int K = 0;
    double3 g{0, 0, 0};
    double dt = 0.0;
    bool dt_set = false;
    int precision = FUNDEM_FP64;       // of the recorded run: its re-runs and Jacobians use it
    long long steps = 0;
    std::vector<AdjCheckpoint> ckpt;   // state at the start of each segment
    std::vector<int> seg_steps;        // steps in each segment
    AdjCheckpoint final_state;
};

struct fundem_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    int precision = FUNDEM_FP64;
    bool mixed() const { return precision == FUNDEM_FP32_MIXED; }
    int records = 1;
    MatHost pmat, wmat;
    GeoSetHost pgeo, wgeo;
    ObjHost P, W;
    BondHost bonds;
    bool perX = false, perY = false;
    bool sector = false;  // quarter-sector periodicity about z through the domain's min corner
    int inertia_mode = FUNDEM_INERTIA_REFERENCE;
    bool geo_dirty = true;
    bool setup_done = false;
    bool detected = false;
    FdGrid pgrid{}, wgrid{};
    CellTable ptab;
    PairList lists[FD_NKIND];
    Ghost ghosts[6];  // X, Y, XY, then the sector images R90, R180, R270
    DevArray<int> scan_tmp;
    DevArray<unsigned int> flags;
    DevArray<unsigned long long> stats;  // narrow-phase work counters (profiling only)
    std::vector<int> node_base;
    long long n_nodes = 0;
    // neighbour list of the particle-particle broad phase (large sets only;
    // small ones search the cell table every step)
    DevArray<double3> nl_ref;
    DevArray<int> nl_vis, nl_cnt, nl_list, nl_ctrl;
    bool use_nl = false;
    int nl_mode = -1;  // -1: from the particle count, 0: off, 1: on (fundem_set_neighbour_list)
    // (re)allocate the neighbour list for the current particle count and
    // request a build at the next detection
    void configure_nl()
    {
        use_nl = nl_mode > 0 || (nl_mode < 0 && P.n() >= NL_MIN_PARTICLES);
        if (!use_nl) return;
        const size_t m = std::max(P.n(), 1);
        nl_ref.alloc(m); nl_vis.alloc(m); nl_cnt.alloc(m); nl_list.alloc(m * fd::NL_MAX, false);
        nl_ctrl.alloc(4);
        const int one = 1;
        FD_CUDA(cudaMemcpyAsync(nl_ctrl.p, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
    }
    fd::NlDev nl_view()
    {
        return fd::NlDev{nl_ref.p, nl_vis.p, nl_cnt.p, nl_list.p, nl_ctrl.p, NL_SKIN * pgeo.rmax, perX, perY, 0.0};
    }
    // contiguous views handed out by fundem_contact_view_get / fundem_bond_view_get
    struct ContactView {
        DevArray<long long> keys;
        DevArray<int> order, idx_b, bcount, bscan, master, slave;
        DevArray<unsigned long long> skey, key_b;
        DevArray<double> point, normal, overlap, en, es, spring;
    };
    ContactView cviews[FD_NKIND];
    DevArray<double> bview_B, bview_energy;
    DevArray<double3> bview_frames;
    // per particle: first wall and wall count it may meet (fundem_set_wall_groups)
    std::vector<int2> wall_groups;
    DevArray<int2> d_wall_groups;
    // pair cache of the particle-particle list (fundem_set_pair_cache): the
    // pairs and contact slots of a rebuild step are kept while no particle
    // drifts more than half the skin; each step still runs the exact
    // predicate on every slot
    DevArray<double3> pc_ref_pos;
    DevArray<fd_quat> pc_ref_q;
    DevArray<int> pc_ref_vis, pc_ctrl;
    DevArray<float> pc_drift;
    DevArray<float4> pc_disp;
    DevArray<double3> pc_wref_pos;
    DevArray<fd_quat> pc_wref_q;
    DevArray<long long> pc_wref_hash;
    DevArray<float> pc_wdrift;
    DevArray<float4> pc_wdisp;
    int pc_mode = -1;          // -1: from the particle count, 0: off, 1: on
    double pc_skin_set = 0.0;  // <= 0: PC_SKIN * the largest bounding radius
    bool pc_on = false;
    bool pc_force = true;      // the next cached step rebuilds
    bool lists_exact = true;   // the lists hold an exact detection (no skin)
    long long pc_steps = 0;    // steps run with the cache
    void configure_pc()
    {
        pc_on = pc_mode > 0 || (pc_mode < 0 && P.n() >= PC_MIN_PARTICLES);
        pc_force = true;
        drop_graph();
        if (!pc_on) return;
        const size_t m = std::max(P.n(), 1);
        pc_ref_pos.alloc(m); pc_ref_q.alloc(m); pc_ref_vis.alloc(m);
        pc_drift.alloc(m, false);
        pc_disp.alloc(m, false);
        const size_t mw = std::max(W.n(), 1);
        pc_wref_pos.alloc(mw); pc_wref_q.alloc(mw); pc_wref_hash.alloc(mw);
        pc_wdrift.alloc(mw, false); pc_wdisp.alloc(mw, false);
        pc_ctrl.alloc(8);
    }
    double pc_skin() const { return pc_skin_set > 0.0 ? pc_skin_set : PC_SKIN * pgeo.rmax; }
    // some particle geometry has a nonzero inverse inertia: its bodies turn,
    // and the adjoint differentiates orientations and angular velocities
    bool adj_turning() const
    {
        for (const FdGeo& g : pgeo.table) {
            const fd_sym& I = g.inv_inertia;
            if (I.xx != 0.0 || I.yy != 0.0 || I.zz != 0.0 || I.xy != 0.0 || I.xz != 0.0 || I.yz != 0.0) return true;
        }
        return false;
    }
    // the adjoint records and re-runs full detections
    bool pc_active() const { return pc_on && !adj.on && recording == nullptr && pc_ctrl.p != nullptr; }
    fd::PairCacheDev pc_view()
    {
        // lever arms of a rotation: a body's nodes (at most r_max from its
        // centre) and a node inside a partner's SDF grid (at most the grid
        // radius from the partner's centre)
        const double reach = std::max(2.0 * pgeo.rmax, pgeo.grid_rmax);
        return fd::PairCacheDev{pc_ref_pos.p, pc_ref_q.p, pc_ref_vis.p, pc_ctrl.p, pc_drift.p, pc_disp.p, pc_skin(),
                                reach, pc_wref_pos.p, pc_wref_q.p, pc_wref_hash.p, pc_wdrift.p, pc_wdisp.p};
    }
    // before steps (outside any stream capture): a pending forced rebuild is
    // written to the device flag
    // before the first cached build after an exact detection (outside any
    // capture): it lists the skin's extra pairs and slots, so each cached
    // list gets room for eight (particle pairs) or 32 (walls and images: few
    // slots per pair without the skin, many more with it) times the exact
    // counts; later builds grow with the capacity checks
    void pc_reserve()
    {
        if (!pc_active() || !pc_force || !lists_exact) return;
        FD_CUDA(cudaStreamSynchronize(stream));
        for (int k : {FD_PP, FD_PW, FD_GX, FD_GY, FD_GXY}) {
            PairList& L = lists[k];
            if (!L.allocated) continue;
            int c[2] = {0, 0};
            FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
            const int f = k == FD_PP ? 8 : 32;
            int needp = f * c[0], needc = f * c[1];
            if (k == FD_PW) {
                // particles reach the walls over the run: room for every
                // particle to meet up to four walls, and for an eighth of
                // the nodes of every pair within the skin of its wall (a flat
                // face parallel to the wall)
                int max_nodes = 1;
                for (const FdGeo& g : pgeo.table) max_nodes = std::max(max_nodes, g.node_count);
                needp = std::max<long long>(needp, (long long)P.n() * std::min(W.n(), 4));
                needc = std::max<long long>(needc, 8ll * P.n() + (long long)c[0] * max_nodes / 8);
            }
            if (needp > L.cap_pairs || needc > L.cap_contacts)
                L.grow(std::max(needp, L.cap_pairs), std::max(needc, L.cap_contacts));
        }
    }
    void pc_prepare()
    {
        if (!pc_active() || !pc_force) return;
        const int one = 1;
        FD_CUDA(cudaMemcpyAsync(pc_ctrl.p, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
        pc_force = false;
        pc_verify = true;
    }
    // after the first steps of a forced rebuild (outside any capture): a
    // cached list that overflowed is grown at once and rebuilt at the next
    // step (its overflow stays reported)
    bool pc_verify = false;
    void pc_check_overflow()
    {
        if (!pc_verify || !pc_active()) return;
        pc_verify = false;
        FD_CUDA(cudaStreamSynchronize(stream));
        bool over = false;
        for (int k : {FD_PP, FD_PW, FD_GX, FD_GY, FD_GXY}) {
            PairList& L = lists[k];
            if (!L.allocated) continue;
            int c[2] = {0, 0};
            FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
            over = over || c[0] > L.cap_pairs || c[1] > L.cap_contacts;
        }
        if (over) {
            ensure_capacity();
            pc_force = true;
        }
    }
    // reverse index over the particle and ghost lists (capacity: their pair
    // capacities together)
    DevArray<int> rev_cnt, rev_off, rev_fill, rev_code;
    // the reverse index holds the pairs of the lists the last step used
    // (a reallocation empties it: the next step builds it whatever the flags)
    bool rev_valid = false;
    fd::RevDev rev_view()
    {
        const int np = std::max(P.n(), 1);
        if (rev_cnt.n < (size_t)np) {
            rev_cnt.alloc(np); rev_off.alloc(np); rev_fill.alloc(np);
            rev_valid = false;
        }
        long long cap = 0;
        for (int k : {FD_PP, FD_GX, FD_GY, FD_GXY, FD_GR90, FD_GR180, FD_GR270})
            if (lists[k].allocated) cap += lists[k].cap_pairs;
        cap = std::max<long long>(cap, 16);
        if (rev_code.n < (size_t)cap) {
            rev_code.alloc((size_t)cap, false);
            rev_valid = false;
        }
        return fd::RevDev{rev_cnt.p, rev_off.p, rev_fill.p, rev_code.p, (int)rev_code.n};
    }
    long long launches = 0;
    long long hook_steps = 0;  // steps of fundem_step and fundem_step_begin, for capacity checks
    // Captured runs of steps (fundem_step_graph).  A capture fixes which of
    // the two list generations each step writes and reads its history from,
    // so there is one graph per generation the run starts on: for an odd
    // number of steps the starting generation alternates between calls.
    struct StepGraph {
        cudaGraphExec_t exec = nullptr;
        int steps = 0;
        double key[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // gravity, dt, precision, records, counters, periodicity
        unsigned long long epoch = 0, gepoch = 0;  // allocation counters at the capture
        long long kernels = 0;                     // kernel launches one replay runs
        long long pc_steps = 0;                    // steps of it that run the pair cache
    };
    StepGraph graphs[2];
    cudaStream_t cap_stream = nullptr;
    bool capturing = false;
    int graph_unchecked = 0;  // steps replayed since the last capacity check
    unsigned long long alloc_epoch = 0;  // device (re)allocations of this simulation
    void drop_graph()
    {
        for (StepGraph& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
    }
    // the particle-wall list (branch 1) and, with translated periodicity,
    // the image lists (branch 0) are detected on streams of their own beside
    // the particle-particle list.  The image branch works on a copy of the
    // positions that the periodic wraps change (the other lists are detected
    // with them unwrapped); the wrapped positions come back at the join.
    cudaStream_t br_stream[2] = {nullptr, nullptr};
    cudaEvent_t br_fork = nullptr, br_join[2] = {nullptr, nullptr};
    DevArray<double3> img_pos;
    ~fundem_sim()
    {
        drop_graph();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        for (int b = 0; b < 2; ++b) {
            if (br_stream[b]) cudaStreamDestroy(br_stream[b]);
            if (br_join[b]) cudaEventDestroy(br_join[b]);
        }
        if (br_fork) cudaEventDestroy(br_fork);
    }
    AdjState adj;
    AdjTape tape;
    AdjTape* recording = nullptr;  // set while a segment is re-run for the reverse sweep
    int record_step = 0;
    std::string last_error;
    // optional CUDA-event timing of kernel groups (fundem_set_profiling)
    bool profiling = false;
    bool counters = false;  // narrow-phase work counters (fundem_set_profiling)
    std::vector<cudaEvent_t> tev[FUNDEM_NTIMERS][2];
    void tbegin(int cat)
    {
        if (!profiling || capturing) return;
        cudaEvent_t e;
        FD_CUDA(cudaEventCreate(&e));
        FD_CUDA(cudaEventRecord(e, stream));
        tev[cat][0].push_back(e);
    }
    void tend(int cat)
    {
        if (!profiling || capturing) return;
        cudaEvent_t e;
        FD_CUDA(cudaEventCreate(&e));
        FD_CUDA(cudaEventRecord(e, stream));
        tev[cat][1].push_back(e);
    }

    void build_node_base()
    {
        node_base.resize(P.pos.size());
        long long acc = 0;
        for (size_t i = 0; i < P.pos.size(); ++i) {
            node_base[i] = (int)acc;
            acc += (long long)pgeo.geos[P.geo[i]].nodes.size();
        }
        n_nodes = acc;
    }

    static FdGrid make_grid(double3 mn, double3 mx, double cell, const FdGrid* prev)
    {
        // spatialGrid::set, mySpatialGrid.h:212-240
        if (mx.x <= mn.x) mx.x = mn.x + cell;
        if (mx.y <= mn.y) mx.y = mn.y + cell;
        if (mx.z <= mn.z) mx.z = mn.z + cell;
        FdGrid g{};
        g.minb = mn;
        g.maxb = mx;
        g.size = prev ? prev->size : make_int3(2, 2, 2);
        g.inv = prev ? prev->inv : make_double3(0, 0, 0);
        if (g.size.x == 0) g.size = make_int3(2, 2, 2);
        if (fd_is_zero(cell)) {
            g.num = 8;
            return g;
        }
        const double dx = mx.x - mn.x, dy = mx.y - mn.y, dz = mx.z - mn.z;
        g.size.x = dx > 2. * cell ? (int)(dx / cell) : 2;
        g.size.y = dy > 2. * cell ? (int)(dy / cell) : 2;
        g.size.z = dz > 2. * cell ? (int)(dz / cell) : 2;
        g.inv.x = dx > 0.0 ? (double)g.size.x / dx : 0.0;
        g.inv.y = dy > 0.0 ? (double)g.size.y / dy : 0.0;
        g.inv.z = dz > 0.0 ? (double)g.size.z / dz : 0.0;
        g.num = (long long)g.size.x * g.size.y * g.size.z;
        return g;
    }

    fd::StepArgs step_args(double dt, double probe = 0.0)
    {
        fd::StepArgs a{};
        a.dt = dt;
        a.probe = probe;
        a.gravity = make_double3(0, 0, 0);
        a.periodic_x = perX;
        a.periodic_y = perY;
        a.sector = sector;
        a.records = records;
        a.flags = flags.p;
        a.stats = counters ? stats.p : nullptr;
        for (int k = 0; k < 4; ++k) a.shape[k] = launch_shape[k];
        return a;
    }
    // narrow-phase launch shape in blocks per SM (0: defaults), set by
    // fundem_set_launch_shape
    int launch_shape[4] = {0, 0, 0, 0};

    fd::BondDev bond_view()
    {
        fd::BondDev b{};
        BondHost& B = bonds;
        b.n = B.n_dev;
        b.master = B.d_master.p; b.slave = B.d_slave.p; b.active = B.d_active.p; b.point = B.d_point.p;
        b.B = B.d_B.p; b.radius = B.d_radius.p; b.L0 = B.d_L0.p; b.ts = B.d_ts.p; b.coh = B.d_coh.p;
        b.mu = B.d_mu.p; b.frames = B.d_frames.p; b.energy = B.d_energy.p; b.out = B.d_out.p;
        b.plist_off = B.d_plist_off.p; b.plist = B.d_plist.p;
        return b;
    }

    void upload_bonds()
    {
        BondHost& B = bonds;
        const size_t n = B.master.size();
        const size_t m = std::max<size_t>(n, 1);
        B.d_master.alloc(m); B.d_slave.alloc(m); B.d_active.alloc(m); B.d_point.alloc(m);
        B.d_B.alloc(4 * m); B.d_radius.alloc(m); B.d_L0.alloc(m); B.d_ts.alloc(m); B.d_coh.alloc(m);
        B.d_mu.alloc(m); B.d_frames.alloc(8 * m); B.d_energy.alloc(6 * m); B.d_out.alloc(9 * m);
        B.d_master.upload(B.master.data(), n, stream); B.d_slave.upload(B.slave.data(), n, stream);
        B.d_active.upload(B.active.data(), n, stream); B.d_point.upload(B.point.data(), n, stream);
        B.d_B.upload(B.B.data(), 4 * n, stream); B.d_radius.upload(B.radius.data(), n, stream);
        B.d_L0.upload(B.L0.data(), n, stream); B.d_ts.upload(B.ts.data(), n, stream);
        B.d_coh.upload(B.coh.data(), n, stream); B.d_mu.upload(B.mu.data(), n, stream);
        B.d_frames.upload(B.frames.data(), 8 * n, stream); B.d_energy.upload(B.energy.data(), 6 * n, stream);
        // per-particle bond lists, bond order within a particle
        const int np = P.n();
        std::vector<int> cnt(np + 1, 0);
        for (size_t k = 0; k < n; ++k) { cnt[B.master[k]]++; cnt[B.slave[k]]++; }
        std::vector<int> off(np + 1, 0);
        for (int i = 0; i < np; ++i) off[i + 1] = off[i] + cnt[i];
        std::vector<int> fillv(np, 0), plist(std::max(off[np], 1));
        for (size_t k = 0; k < n; ++k) {
            plist[off[B.master[k]] + fillv[B.master[k]]++] = (int)(2 * k);
            plist[off[B.slave[k]] + fillv[B.slave[k]]++] = (int)(2 * k + 1);
        }
        B.d_plist_off.alloc(np + 1);
        B.d_plist_off.upload(off.data(), np + 1, stream);
        B.d_plist.alloc(plist.size());
        B.d_plist.upload(plist.data(), plist.size(), stream);
        B.n_dev = (int)n;
        B.dirty = false;
    }

    void setup(double3 mn, double3 mx)
    {
        FD_CUDA(cudaSetDevice(device));
        if (geo_dirty) {
            pgeo.build(false, inertia_mode, stream);
            wgeo.build(true, inertia_mode, stream);
            pmat.upload(stream);
            wmat.upload(stream);
            geo_dirty = false;
        }
        const bool counts_changed = (P.n() != P.n_dev) || !setup_done;
        if (P.dirty || counts_changed) {
            build_node_base();
            P.upload(node_base, stream);
        }
        if (W.dirty || W.n() != W.n_dev) {
            std::vector<int> zeros(W.pos.size(), 0);
            W.upload(zeros, stream);
        }
        if (bonds.dirty || bonds.n_dev != (int)bonds.master.size()) upload_bonds();
        const double pcell = P.n() > 0 ? 2.0 * pgeo.rmax : 0.0;
        const double wcell = W.n() > 0 ? 2.0 * wgeo.rmax : 0.0;
        pgrid = make_grid(mn, mx, pcell, setup_done ? &pgrid : nullptr);
        wgrid = make_grid(mn, mx, wcell, setup_done ? &wgrid : nullptr);
        ptab.alloc(pgrid, P.n());
        configure_nl();
        configure_pc();
        if (!wall_groups.empty()) {
            if ((int)wall_groups.size() != P.n())
                throw std::invalid_argument("wall groups: one entry per particle is needed");
            d_wall_groups.alloc(wall_groups.size(), false);
            d_wall_groups.upload(wall_groups, stream);
        }
        const int np = P.n();
        const int nw = W.n();
        // capacities (grown after the first detection)
        const int kinds_cap[FD_NKIND] = {std::max(64, 8 * np), std::max(64, np * std::min(nw, 4)),
                                         std::max(64, np), std::max(64, np), std::max(64, np),
                                         std::max(64, np), std::max(64, np), std::max(64, np)};
        for (int k = 0; k < FD_NKIND; ++k) {
            if (!lists[k].allocated || counts_changed) lists[k].alloc(np, kinds_cap[k], 2 * kinds_cap[k]);
        }
        const bool act[6] = {perX, perY, perX && perY, sector, sector, sector};
        for (int d = 0; d < 6; ++d) {
            ghosts[d].active = act[d];
            if (act[d]) {
                if (d >= 3) {
                    ghosts[d].q.alloc(std::max(np, 1));
                    ghosts[d].vel.alloc(std::max(np, 1));
                    ghosts[d].rot.alloc(3 * std::max(np, 1));
                }
                ghosts[d].pos.alloc(std::max(np, 1));
                ghosts[d].hash.alloc(std::max(np, 1));
                if (d < 3) ghosts[d].live.alloc(std::max(np, 1));
                ghosts[d].occ.alloc(6);
                ghosts[d].searchers.alloc(std::max(np, 1));
                ghosts[d].nsearch.alloc(1);
                ghosts[d].cells.alloc(pgrid, np);
            }
        }
        if ((perX || perY) && !sector) img_pos.alloc(std::max(np, 1), false);
        for (int b = 0; b < 2; ++b) {
            if (!br_stream[b]) FD_CUDA(cudaStreamCreateWithFlags(&br_stream[b], cudaStreamNonBlocking));
            if (!br_join[b]) FD_CUDA(cudaEventCreateWithFlags(&br_join[b], cudaEventDisableTiming));
        }
        if (!br_fork) FD_CUDA(cudaEventCreateWithFlags(&br_fork, cudaEventDisableTiming));
        size_t st = std::max<size_t>(fd::scan_tmp_size(pgrid.num), fd::scan_tmp_size(np));
        scan_tmp.alloc(st + 16);
        if (!flags.p) flags.alloc(1);
        if (!stats.p) stats.alloc(8);
        FD_CUDA(cudaStreamSynchronize(stream));
        setup_done = true;
    }

    // hash + detection (+ forces) of one step, LSSolver.h:1201-1215
    void detect_all(bool with_force, double dt, double probe = 0.0, bool new_generation = true)
    {
        ObjDev Pv = P.view(), Wv = W.view();
        GeoSetDev G = pgeo.view(), GW = wgeo.view();
        fd::MatDev M = pmat.view(), MW = wmat.view();
        fd::StepArgs a = step_args(dt, probe);
        CellTableDev T = ptab.view();
        // pair cache: steps only (a detection outside a step lists the exact
        // pairs and slots, and the next cached step rebuilds)
        const bool pc = with_force && probe == 0.0 && pc_active();
        fd::PairCacheDev pcv{};
        if (pc) pcv = pc_view();
        tbegin(FUNDEM_T_HASH);
        fd::launch_hash(Pv, pgrid, stream);
        if (pc) {
            fd::launch_pair_cache_check(Pv, pcv, stream);
            pc_steps += 1;
        } else if (pc_on) {
            pc_force = true;
        }
        lists_exact = !pc;
        // with the cache, the particle table serves only rebuild steps
        fd::launch_cell_table(Pv, T, scan_tmp.p, scan_tmp.n, stream, pc ? pcv.ctrl : nullptr);
        // wall hash (visibility and cell for the node test)
        if (W.n_dev > 0) fd::launch_hash(Wv, wgrid, stream);
        if (pc && W.n_dev > 0) fd::launch_pair_cache_check_walls(Wv, GW, pcv, stream);
        tend(FUNDEM_T_HASH);
        int active[FD_NKIND] = {1, 1, 0, 0, 0};
        if (new_generation)
            for (int k = 0; k < FD_NKIND; ++k) lists[k].cur ^= 1;
        PairListDev Lg[6];
        // the translated image sets share the pair cache (not with sector
        // periodicity): their pairs and slots are kept with the particle
        // pairs', and a wrap or an image in a clamped cell rebuilds them
        const bool pcg = pc && !sector;
        int* gctrl = pcg ? pcv.ctrl : nullptr;
        bool img_wrapped = false;
        // PeriodicBoundaryXY2D then PeriodicBoundarySector::updateGhostSpatialGrid
        // (LSSolver.h:780-784), then the detection of every image set, on
        // stream gs with the particle set Pg.  wrap_src non-null: Pg.pos is a
        // separate array, and the first wrap fills it from wrap_src.
        auto image_stage = [&](cudaStream_t gs, ObjDev Pg, const double3* wrap_src) {
            tbegin(FUNDEM_T_GHOST);
            const int kinds[6] = {FD_GX, FD_GY, FD_GXY, FD_GR90, FD_GR180, FD_GR270};
            for (int d = 0; d < 3; ++d) {
                if (!ghosts[d].active) continue;
                if (d < 2) {
                    fd::launch_wrap(Pg, pgrid, d, gs, gctrl, img_wrapped ? nullptr : wrap_src);
                    img_wrapped = true;
                }
                fd::GhostDev gh = ghosts[d].view(pcg);
                fd::launch_ghost_build(Pg, gh, kinds[d], gs, pcg ? pcv.skin : 0.0, gctrl);
            }
            if (pcg) fd::launch_ghost_gate(gctrl, gs);
            for (int d = 0; d < 3; ++d) {
                if (!ghosts[d].active) continue;
                fd::GhostDev gh = ghosts[d].view(pcg);
                ObjDev ghostobj = Pg;
                ghostobj.hash = ghosts[d].hash.p;
                fd::launch_cell_table(ghostobj, gh.cells, scan_tmp.p, scan_tmp.n, gs, pcg ? gctrl + 5 : nullptr);
            }
            if (sector) {
                fd::launch_sector_wrap(Pg, pgrid, gs);
                fd::GhostDev sv[3] = {ghosts[3].view(), ghosts[4].view(), ghosts[5].view()};
                fd::launch_sector_images(Pg, sv, gs);
                for (int d = 3; d < 6; ++d) {
                    ObjDev ghostobj = Pg;
                    ghostobj.hash = ghosts[d].hash.p;
                    fd::launch_cell_table(ghostobj, sv[d - 3].cells, scan_tmp.p, scan_tmp.n, gs);
                }
            }
            for (int d = 0; d < 6; ++d) {
                if (!ghosts[d].active) continue;
                const bool cached = pcg && d < 3;
                fd::GhostDev gh = ghosts[d].view(cached);
                Lg[d] = lists[kinds[d]].view();
                fd::StepArgs ag = a;
                if (cached) {
                    ag.skin = pcv.skin;
                    ag.gate = gctrl + 5;
                    ag.noskin = gctrl + 6;
                    ag.drift = pcv.drift;
                    ag.disp = pcv.disp;
                    fd::launch_broad_ghost(Pg, G, gh, Lg[d], flags.p, probe, gs, pcv.skin, gctrl + 5, gctrl + 6);
                } else {
                    fd::launch_broad_ghost(Pg, G, gh, Lg[d], flags.p, probe, gs);
                }
                ag.rec = recording ? recording->rec(kinds[d], record_step) : fd::AdjRec{};
                fd::launch_narrow(kinds[d], Pg, G, M, Wv, GW, MW, pgrid, wgrid, &gh, Lg[d], ag, with_force, mixed(),
                                  gs);
                if (recording)
                    FD_CUDA(cudaMemcpyAsync(recording->ns(kinds[d], record_step), Lg[d].n_slots, sizeof(int),
                                            cudaMemcpyDeviceToDevice, gs));
                active[kinds[d]] = 1;
            }
            tend(FUNDEM_T_GHOST);
        };
        PairListDev Lpw = lists[FD_PW].view();
        auto wall_stage = [&](cudaStream_t ws) {
            tbegin(FUNDEM_T_BROAD);
            fd::launch_broad_pw(Pv, G, Wv, GW, wgrid, Lpw, flags.p, probe, ws,
                                wall_groups.empty() ? nullptr : d_wall_groups.p, pc ? pcv.skin : 0.0,
                                pc ? pcv.ctrl : nullptr);
            tend(FUNDEM_T_BROAD);
            tbegin(FUNDEM_T_NARROW_PW);
            // the particle-wall list shares the cache (wall drifts and cells
            // in its rebuild flag)
            fd::StepArgs aw = a;
            aw.rec = recording ? recording->rec(FD_PW, record_step) : fd::AdjRec{};
            if (pc) {
                aw.skin = pcv.skin;
                aw.gate = pcv.ctrl;
                aw.drift = pcv.drift;
                aw.disp = pcv.disp;
                aw.driftB = pcv.wdrift;
                aw.dispB = pcv.wdisp;
            }
            fd::launch_narrow(FD_PW, Pv, G, M, Wv, GW, MW, pgrid, wgrid, nullptr, Lpw, aw, with_force, mixed(), ws);
            if (pc && W.n_dev > 0) fd::launch_pair_cache_commit_walls(Wv, pcv, ws);
            if (recording)
                FD_CUDA(cudaMemcpyAsync(recording->ns(FD_PW, record_step), Lpw.n_slots, sizeof(int),
                                        cudaMemcpyDeviceToDevice, ws));
            tend(FUNDEM_T_NARROW_PW);
        };
        // outside per-stage timing the wall list and the images (translated
        // periodicity) run beside the particle-particle list, and the bonds
        // at the end of one of them.  Each branch reads and writes nothing
        // another one writes: its own lists, tables and image arrays; the
        // wall references of the pair cache (branch 1); the wrapped copy of
        // the positions and the pair cache's words 4-7, which the others do
        // not read (branch 0); the bond arrays (the branch that runs the
        // bonds); the flags and counters with atomics.  The pair cache's
        // rebuild flag (word 0) and drifts are written before the fork.
        const bool branches = br_stream[0] && br_stream[1] && (!profiling || capturing);
        const bool img_branch = branches && (perX || perY) && !sector && img_pos.p && img_pos.n >= (size_t)Pv.n;
        // the bonds read only positions (after the wraps) and orientations:
        // they run at the end of a branch, off the particle pairs' path
        fd::BondDev bd = bond_view();
        if (recording && bd.n > 0) {
            bd.rec_active = recording->bond_active.p + (long long)record_step * bd.n;
            bd.rec_rij = recording->bond_rij.p + 3ll * record_step * bd.n;
            bd.rec_dn = recording->bond_dn.p + 3ll * record_step * bd.n;
        }
        bool bonds_done = false;
        if (branches) FD_CUDA(cudaEventRecord(br_fork, stream));
        if (img_branch) {
            FD_CUDA(cudaStreamWaitEvent(br_stream[0], br_fork, 0));
            ObjDev Pg = Pv;
            Pg.pos = img_pos.p;
            image_stage(br_stream[0], Pg, Pv.pos);
            if (with_force && bd.n > 0) {
                fd::launch_bonds(Pg, bd, mixed(), br_stream[0]);
                bonds_done = true;
            }
            FD_CUDA(cudaEventRecord(br_join[0], br_stream[0]));
        }
        if (branches) {
            FD_CUDA(cudaStreamWaitEvent(br_stream[1], br_fork, 0));
            wall_stage(br_stream[1]);
            if (with_force && bd.n > 0 && !bonds_done && !(perX || perY || sector)) {
                fd::launch_bonds(Pv, bd, mixed(), br_stream[1]);
                bonds_done = true;
            }
            FD_CUDA(cudaEventRecord(br_join[1], br_stream[1]));
        }
        PairListDev Lpp = lists[FD_PP].view();
        tbegin(FUNDEM_T_BROAD);
        if (use_nl) {
            fd::NlDev nl = nl_view();
            nl.pair_skin = pc ? pcv.skin : 0.0;
            fd::launch_broad_pp_nl(Pv, G, T, Lpp, nl, flags.p, probe, stream, pc ? pcv.ctrl : nullptr);
        } else {
            fd::launch_broad_pp(Pv, G, T, Lpp, flags.p, probe, stream, pc ? pcv.skin : 0.0, pc ? pcv.ctrl : nullptr);
        }
        tend(FUNDEM_T_BROAD);
        tbegin(FUNDEM_T_NARROW_PP);
        a.rec = recording ? recording->rec(FD_PP, record_step) : fd::AdjRec{};
        {
            fd::StepArgs ap = a;
            if (pc) {
                ap.skin = pcv.skin;
                ap.gate = pcv.ctrl;
                ap.drift = pcv.drift;
                ap.disp = pcv.disp;
            }
            fd::launch_narrow(FD_PP, Pv, G, M, Wv, GW, MW, pgrid, wgrid, nullptr, Lpp, ap, with_force, mixed(), stream);
        }
        if (pc) {
            fd::launch_pair_cache_commit(Pv, pcv, Lpp, stream);
        }
        if (recording)
            FD_CUDA(cudaMemcpyAsync(recording->ns(FD_PP, record_step), Lpp.n_slots, sizeof(int),
                                    cudaMemcpyDeviceToDevice, stream));
        tend(FUNDEM_T_NARROW_PP);
        if (branches) FD_CUDA(cudaStreamWaitEvent(stream, br_join[1], 0));
        else wall_stage(stream);
        if (img_branch) {
            // the image detection ran beside; its wrapped positions replace
            // the ones the particle and wall lists were detected with
            FD_CUDA(cudaStreamWaitEvent(stream, br_join[0], 0));
            if (img_wrapped && Pv.n > 0)
                FD_CUDA(cudaMemcpyAsync(Pv.pos, img_pos.p, sizeof(double3) * Pv.n, cudaMemcpyDeviceToDevice, stream));
        } else if (perX || perY || sector) {
            image_stage(stream, Pv, nullptr);
        }
        auto pc_end = [&] {
            if (!pc) return;
            PairListDev gl[4];
            int ng = 0;
            gl[ng++] = Lpw;
            for (int d = 0; d < 3 && pcg; ++d)
                if (ghosts[d].active) gl[ng++] = Lg[d];
            fd::launch_pair_cache_end(pcv, gl, ng, stream);
        };
        if (!with_force) {
            pc_end();
            FD_CUDA(cudaGetLastError());
            return;
        }
        tbegin(FUNDEM_T_REDUCE);
        PairListDev views[FD_NKIND];
        for (int k = 0; k < FD_NKIND; ++k) views[k] = lists[k].view();
        fd::RevDev rv = rev_view();
        // the reverse index depends only on the lists' pairs: under the pair
        // cache (without sector images, whose lists are detected afresh every
        // step) a step that keeps them keeps the index.  The gate is the
        // rebuild flag of the particle pairs, or of the image lists, which
        // also rebuild with them.
        const bool ghosts_cached = pcg && (ghosts[0].active || ghosts[1].active || ghosts[2].active);
        const int* rev_gate = (pc && !sector && rev_valid) ? (ghosts_cached ? gctrl + 5 : pcv.ctrl) : nullptr;
        fd::launch_reverse(Pv, views, active, rv, scan_tmp.p, scan_tmp.n, stream, rev_gate);
        rev_valid = true;
        if (bd.n > 0 && !bonds_done) fd::launch_bonds(Pv, bd, mixed(), stream);
        fd::launch_reduce(Pv, views, active, rv, bd, mixed(), stream);
        pc_end();

        tend(FUNDEM_T_REDUCE);
        FD_CUDA(cudaGetLastError());
    }

    // copy the device state of a set back into its host mirror
    void pull(ObjHost& O)
    {
        if (!(O.n_dev == O.n() && !O.dirty && O.n() > 0)) return;
        FD_CUDA(cudaStreamSynchronize(stream));
        const size_t n = O.n();
        FD_CUDA(cudaMemcpy(O.pos.data(), O.d_pos.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemcpy(O.vel.data(), O.d_vel.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemcpy(O.angvel.data(), O.d_angvel.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemcpy(O.q.data(), O.d_q.p, sizeof(fd_quat) * n, cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemcpy(O.force.data(), O.d_force.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemcpy(O.torque.data(), O.d_torque.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
    }

    // grow list capacities to three times the last counts when they come
    // within a factor two of the limit (synchronises the stream)
    void ensure_capacity()
    {
        FD_CUDA(cudaStreamSynchronize(stream));
        for (int k = 0; k < FD_NKIND; ++k) {
            PairList& L = lists[k];
            if (!L.allocated) continue;
            int c[2] = {0, 0};
            FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
            const int needp = 2 * c[0] > L.cap_pairs ? 3 * c[0] : 0;
            const int needc = 2 * c[1] > L.cap_contacts ? 3 * c[1] : 0;
            if (needp || needc) {
                L.grow(std::max(needp, L.cap_pairs), std::max(needc, L.cap_contacts));
                // the slot-to-pair map of a cached list is not kept by a growth
                if (k != FD_GR90 && k != FD_GR180 && k != FD_GR270) pc_force = true;
            }
        }
    }

    // detection outside a step: a list that overflowed is grown to the
    // demand its counters recorded and the detection runs again into the same
    // generation (same history source).  Overflow bits raised before the call
    // are kept for fundem_sync.
    // Detection that grows the lists and detects again until nothing
    // overflowed.  The periodic wraps inside a detection move bodies, so a
    // repeated attempt starts again from the state the first one saw.
    void detect_fit(double probe)
    {
        const unsigned int grow_bits = FD_FLAG_PAIR_OVERFLOW | FD_FLAG_CONTACT_OVERFLOW;
        unsigned int f0 = 0;
        FD_CUDA(cudaStreamSynchronize(stream));
        FD_CUDA(cudaMemcpy(&f0, flags.p, sizeof(f0), cudaMemcpyDeviceToHost));
        const size_t np = (size_t)P.n();
        const bool wraps = (perX || perY || sector) && np > 0 && P.n_dev == (int)np;
        DevArray<double3> keep_pos, keep_vel;
        DevArray<fd_quat> keep_q;
        if (wraps) {
            keep_pos.alloc(np);
            keep_vel.alloc(np);
            keep_q.alloc(np);
            FD_CUDA(cudaMemcpyAsync(keep_pos.p, P.d_pos.p, np * sizeof(double3), cudaMemcpyDeviceToDevice, stream));
            FD_CUDA(cudaMemcpyAsync(keep_vel.p, P.d_vel.p, np * sizeof(double3), cudaMemcpyDeviceToDevice, stream));
            FD_CUDA(cudaMemcpyAsync(keep_q.p, P.d_q.p, np * sizeof(fd_quat), cudaMemcpyDeviceToDevice, stream));
        }
        for (int attempt = 0;; ++attempt) {
            if (attempt > 0 && wraps) {
                FD_CUDA(cudaMemcpyAsync(P.d_pos.p, keep_pos.p, np * sizeof(double3), cudaMemcpyDeviceToDevice, stream));
                FD_CUDA(cudaMemcpyAsync(P.d_vel.p, keep_vel.p, np * sizeof(double3), cudaMemcpyDeviceToDevice, stream));
                FD_CUDA(cudaMemcpyAsync(P.d_q.p, keep_q.p, np * sizeof(fd_quat), cudaMemcpyDeviceToDevice, stream));
            }
            if (attempt > 0 || (f0 & grow_bits)) {
                const unsigned int clear = f0 & ~grow_bits;
                FD_CUDA(cudaMemcpyAsync(flags.p, &clear, sizeof(clear), cudaMemcpyHostToDevice, stream));
            }
            detect_all(false, 0.0, probe, attempt == 0);
            ensure_capacity();
            unsigned int f = 0;
            FD_CUDA(cudaMemcpy(&f, flags.p, sizeof(f), cudaMemcpyDeviceToHost));
            if (!(f & grow_bits) || attempt == 3) {
                const unsigned int keep = f | f0;
                FD_CUDA(cudaMemcpyAsync(flags.p, &keep, sizeof(keep), cudaMemcpyHostToDevice, stream));
                break;
            }
        }
    }

    void front(double3 g, double dt)
    {
        ObjDev Pv = P.view(), Wv = W.view();
        tbegin(FUNDEM_T_INTEGRATE);
        fd::launch_kick(Pv, pgeo.view(), g, 0.5 * dt, stream);
        fd::launch_drift(Pv, dt, stream);
        fd::launch_drift(Wv, dt, stream);
        tend(FUNDEM_T_INTEGRATE);
    }
    void back(double3 g, double dt)
    {
        tbegin(FUNDEM_T_INTEGRATE);
        fd::launch_kick(P.view(), pgeo.view(), g, 0.5 * dt, stream);
        tend(FUNDEM_T_INTEGRATE);
    }
    // back() of one step and front() of the next, the particles in one pass
    void back_front(double3 g, double dt)
    {
        ObjDev Pv = P.view(), Wv = W.view();
        tbegin(FUNDEM_T_INTEGRATE);
        fd::launch_kick_drift(Pv, pgeo.view(), g, 0.5 * dt, dt, stream);
        fd::launch_drift(Wv, dt, stream);
        tend(FUNDEM_T_INTEGRATE);
    }
};

namespace {
int guard(fundem_sim* s, const std::function<void()>& f)
{
    // allocations inside the call belong to this simulation
    struct EpochScope {
        unsigned long long* prev;
        explicit EpochScope(unsigned long long* e) : prev(t_sim_epoch) { if (e) t_sim_epoch = e; }
        ~EpochScope() { t_sim_epoch = prev; }
    } scope(s ? &s->alloc_epoch : nullptr);
    // kernels launched inside the call are counted for this simulation
    struct CountScope {
        explicit CountScope(long long* c) { fd::set_launch_counter(c); }
        ~CountScope() { fd::set_launch_counter(nullptr); }
    } counting(s ? &s->launches : nullptr);
    try {
        f();
        return FUNDEM_OK;
    } catch (const CudaError& e) {
        if (s) s->last_error = e.what();
        return FUNDEM_ERR_CUDA;
    } catch (const std::invalid_argument& e) {
        if (s) s->last_error = e.what();
        return FUNDEM_ERR_ARG;
    } catch (const std::logic_error& e) {
        if (s) s->last_error = e.what();
        return FUNDEM_ERR_STATE;
    } catch (const std::exception& e) {
        if (s) s->last_error = e.what();
        return FUNDEM_ERR_CUDA;
    }
}
double3 d3(const double* p) { return make_double3(p[0], p[1], p[2]); }
// host reverse rotation used by bond creation (myQua.h:120-128, host branch)
double3 hrrot(double3 v, const fd_quat& q)
{
    const double3 qv = make_double3(-q.q1, -q.q2, -q.q3);
    const double3 t = cross3(qv, v) * 2.0;
    return v + t * q.q0 + cross3(qv, t);
}
double3 hnormalize(double3 v)
{
    const double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (fd_is_zero(l2)) return make_double3(0, 0, 0);
    const double inv = 1.0 / std::sqrt(l2);
    return make_double3(v.x * inv, v.y * inv, v.z * inv);
}
fd_quat hnormalize_q(fd_quat q)
{
    const double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
    if (fd_is_zero(l2)) return q;
    const double inv = 1.0 / std::sqrt(l2);
    return fd_quat{q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv};
}
}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* fundem_version(void) { return "fundem_b200 0.1 (sm_100a)"; }

const char* fundem_status_string(int s)
{
    switch (s) {
    case FUNDEM_OK: return "ok";
    case FUNDEM_ERR_ARG: return "invalid argument";
    case FUNDEM_ERR_CUDA: return "CUDA error";
    case FUNDEM_ERR_CAPACITY: return "list capacity exceeded";
    case FUNDEM_ERR_STATE: return "call out of order";
    case FUNDEM_ERR_NUMERIC: return "non-finite state";
    }
    return "unknown status";
}

int fundem_create(fundem_sim** out, int device, void* stream)
{
    if (!out) return FUNDEM_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return FUNDEM_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return FUNDEM_ERR_CUDA;
    fundem_sim* s = new fundem_sim();
    s->device = device;
    s->stream = (cudaStream_t)stream;
    *out = s;
    return FUNDEM_OK;
}

int fundem_destroy(fundem_sim* s)
{
    if (!s) return FUNDEM_ERR_ARG;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
    return FUNDEM_OK;
}

int fundem_set_precision(fundem_sim* s, int mode)
{
    if (!s || (mode != FUNDEM_FP64 && mode != FUNDEM_FP32_MIXED)) return FUNDEM_ERR_ARG;
    s->precision = mode;
    return FUNDEM_OK;
}

int fundem_set_neighbour_list(fundem_sim* s, int mode)
{
    if (!s || mode < -1 || mode > 1) return FUNDEM_ERR_ARG;
    s->nl_mode = mode;
    if (!s->setup_done) return FUNDEM_OK;
    return guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        s->configure_nl();
    });
}

int fundem_set_pair_cache(fundem_sim* s, int mode, double skin)
{
    if (!s || mode < -1 || mode > 1 || !(skin >= 0.0)) return FUNDEM_ERR_ARG;
    s->pc_mode = mode;
    s->pc_skin_set = skin;
    if (!s->setup_done) return FUNDEM_OK;
    return guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        s->configure_pc();
    });
}

int fundem_pair_cache_stats(fundem_sim* s, long long* rebuilds, long long* steps, double* skin)
{
    if (!s) return FUNDEM_ERR_ARG;
    return guard(s, [&] {
        int c[2] = {0, 0};
        if (s->pc_ctrl.p) {
            FD_CUDA(cudaStreamSynchronize(s->stream));
            FD_CUDA(cudaMemcpy(c, s->pc_ctrl.p, sizeof(c), cudaMemcpyDeviceToHost));
        }
        if (rebuilds) *rebuilds = c[1];
        if (steps) *steps = s->pc_on ? s->pc_steps : 0;
        if (skin) *skin = s->pc_on ? s->pc_skin() : 0.0;
    });
}

int fundem_set_wall_groups(fundem_sim* s, int n, const int* first, const int* count)
{
    if (!s || n < 0 || (n > 0 && (!first || !count))) return FUNDEM_ERR_ARG;
    if (n > 0 && n != s->P.n()) {
        s->last_error = "wall groups: one entry per particle is needed";
        return FUNDEM_ERR_ARG;
    }
    const int nw = s->W.n();
    for (int i = 0; i < n; ++i)
        if (first[i] < 0 || count[i] < 0 || first[i] + count[i] > nw) {
            s->last_error = "wall groups: a range reaches past the walls";
            return FUNDEM_ERR_ARG;
        }
    return guard(s, [&] {
        s->wall_groups.resize(n);
        for (int i = 0; i < n; ++i) s->wall_groups[i] = make_int2(first[i], count[i]);
        if (s->setup_done && n > 0) {
            s->d_wall_groups.alloc(n, false);
            s->d_wall_groups.upload(s->wall_groups, s->stream);
        }
        s->drop_graph();
    });
}

int fundem_contact_view_get(fundem_sim* s, int kind, fundem_contact_view* out)
{
    if (!s || !out || kind < 0 || kind >= FD_NKIND) return FUNDEM_ERR_ARG;
    *out = fundem_contact_view{};
    PairList& L = s->lists[kind];
    if (!s->setup_done || !L.allocated) return FUNDEM_OK;
    return guard(s, [&] {
        int c[3] = {0, 0, 0};
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        const long long n = c[1] <= L.cap_contacts ? c[2] : 0;
        const size_t cap = (size_t)std::max(L.cap_contacts, 1);
        auto& V = s->cviews[kind];
        if (V.keys.n < cap) {
            V.keys.alloc(cap, false); V.order.alloc(cap, false); V.idx_b.alloc(cap, false);
            V.skey.alloc(cap, false); V.key_b.alloc(cap, false);
            size_t bc = 0, bs = 0;
            fd::radix_sort_scratch((int)cap, bc, bs);
            V.bcount.alloc(bc, false); V.bscan.alloc(bs, false);
            V.master.alloc(cap, false); V.slave.alloc(cap, false); V.overlap.alloc(cap, false);
            V.en.alloc(cap, false); V.es.alloc(cap, false);
            V.point.alloc(3 * cap, false); V.normal.alloc(3 * cap, false); V.spring.alloc(3 * cap, false);
        }
        fd::ContactViewDev v{V.point.p, V.normal.p, V.overlap.p, V.en.p, V.es.p, V.spring.p, V.master.p, V.slave.p};
        const long long max_key = (s->n_nodes + 1) << 32;
        fd::launch_contact_view(L.view(), V.keys.p, V.order.p, V.skey.p, V.key_b.p, V.idx_b.p, V.bcount.p, V.bscan.p,
                                n, max_key, v, s->stream);
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaGetLastError());
        out->point = V.point.p; out->normal = V.normal.p; out->overlap = V.overlap.p;
        out->normal_energy = V.en.p; out->sliding_energy = V.es.p; out->spring = V.spring.p;
        out->master = V.master.p; out->slave = V.slave.p; out->n = n;
    });
}

int fundem_bond_view_get(fundem_sim* s, fundem_bond_view* out)
{
    if (!s || !out) return FUNDEM_ERR_ARG;
    *out = fundem_bond_view{};
    if (!s->setup_done) return FUNDEM_OK;
    return guard(s, [&] {
        fd::BondDev bd = s->bond_view();
        const size_t m = (size_t)std::max(bd.n, 1);
        if (s->bview_B.n < 4 * m) {
            s->bview_B.alloc(4 * m, false);
            s->bview_energy.alloc(6 * m, false);
            s->bview_frames.alloc(8 * m, false);
        }
        fd::BondViewDev v{};
        for (int t = 0; t < 4; ++t) v.B[t] = s->bview_B.p + t * m;
        for (int t = 0; t < 6; ++t) v.energy[t] = s->bview_energy.p + t * m;
        for (int t = 0; t < 8; ++t) v.frames[t] = s->bview_frames.p + t * m;
        fd::launch_bond_view(bd, v, s->stream);
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaGetLastError());
        BondHost& B = s->bonds;
        out->master = B.d_master.p; out->slave = B.d_slave.p; out->activated = B.d_active.p;
        out->center_point = (double*)B.d_point.p; out->radius = B.d_radius.p; out->initial_length = B.d_L0.p;
        out->B1 = v.B[0]; out->B2 = v.B[1]; out->B3 = v.B[2]; out->B4 = v.B[3];
        out->Un = v.energy[0]; out->Us = v.energy[1]; out->Ub = v.energy[2]; out->Ut = v.energy[3];
        out->max_normal_stress = v.energy[4]; out->max_shear_stress = v.energy[5];
        out->tensile_strength = B.d_ts.p; out->cohesion = B.d_coh.p; out->friction = B.d_mu.p;
        for (int t = 0; t < 8; ++t) out->frames[t] = (double*)v.frames[t];
        out->n = bd.n;
    });
}

int fundem_set_records(fundem_sim* s, int full)
{
    if (!s) return FUNDEM_ERR_ARG;
    s->records = full ? 1 : 0;
    return FUNDEM_OK;
}

int fundem_add_material(fundem_sim* s, int wall, double kn, double ks, double mu, double e, int* id_out)
{
    if (!s) return FUNDEM_ERR_ARG;
    MatHost& m = wall ? s->wmat : s->pmat;
    if (wall) { kn = 0.0; ks = 0.0; }
    m.kn.push_back(kn > 0. ? kn : 0.0);
    m.ks.push_back(ks > 0. ? ks : 0.0);
    m.mu.push_back(mu > 0. ? mu : 0.0);
    m.e.push_back((e > 0. && e < 1.0) ? e : 1.0);
    if (id_out) *id_out = (int)m.kn.size() - 1;
    s->geo_dirty = true;
    return FUNDEM_OK;
}

int fundem_add_geometry(fundem_sim* s, int wall, double mass, const double inertia[6], const double origin[3],
                        double spacing, const int size[3], const double* sdf, int n_nodes, const double* nodes,
                        int* id_out)
{
    if (!s || !origin || !size || !sdf || n_nodes < 0 || (n_nodes > 0 && !nodes)) return FUNDEM_ERR_ARG;
    if (size[0] < 2 || size[1] < 2 || size[2] < 2 || !(spacing > 0.0)) return FUNDEM_ERR_ARG;
    HostGeo g;
    g.mass = wall ? 0.0 : mass;
    if (inertia && !wall) g.inertia = fd_sym{inertia[0], inertia[1], inertia[2], inertia[3], inertia[4], inertia[5]};
    g.origin = d3(origin);
    g.spacing = spacing;
    g.size = make_int3(size[0], size[1], size[2]);
    const size_t ns = (size_t)size[0] * size[1] * size[2];
    g.sdf.assign(sdf, sdf + ns);
    for (int k = 0; k < n_nodes; ++k) g.nodes.push_back(d3(nodes + 3 * k));
    GeoSetHost& set = wall ? s->wgeo : s->pgeo;
    set.geos.push_back(std::move(g));
    if (id_out) *id_out = (int)set.geos.size() - 1;
    s->geo_dirty = true;
    return FUNDEM_OK;
}

int fundem_mass_properties(double density, const double origin[3], double h, const int size[3], const double* sdf,
                           double* mass_out, double centroid[3], double inertia[6])
{
    if (!origin || !size || !sdf || size[0] < 2 || size[1] < 2 || size[2] < 2 || !(h > 0.0)) return FUNDEM_ERR_ARG;
    const double PI = 3.14159265358979323846;
    auto H = [&](double phi) {
        const double sp = 1.5;
        if (phi < -sp) return 1.0;
        if (phi > sp) return 0.0;
        const double x = -phi / sp;
        return 0.5 * (1.0 + x + std::sin(PI * x) / PI);
    };
    const double mg = density * h * h * h;
    double mass = 0.0;
    auto idx = [&](int x, int y, int z) { return (size_t)z * size[1] * size[0] + (size_t)y * size[0] + x; };
    for (int x = 0; x < size[0]; x++)
        for (int y = 0; y < size[1]; y++)
            for (int z = 0; z < size[2]; z++) mass += H(sdf[idx(x, y, z)] / h);
    mass *= mg;
    double3 c = make_double3(0, 0, 0);
    fd_sym I{0, 0, 0, 0, 0, 0};
    if (mass > 0.) {
        for (int x = 0; x < size[0]; x++)
            for (int y = 0; y < size[1]; y++)
                for (int z = 0; z < size[2]; z++) {
                    const double w = H(sdf[idx(x, y, z)] / h);
                    c.x += w * (origin[0] + double(x) * h);
                    c.y += w * (origin[1] + double(y) * h);
                    c.z += w * (origin[2] + double(z) * h);
                }
        c = c * (mg / mass);
        for (int x = 0; x < size[0]; x++)
            for (int y = 0; y < size[1]; y++)
                for (int z = 0; z < size[2]; z++) {
                    const double w = H(sdf[idx(x, y, z)] / h);
                    const double3 r = (d3(origin) + h * make_double3(double(x), double(y), double(z))) - c;
                    I.xx += w * (r.y * r.y + r.z * r.z) * mg;
                    I.yy += w * (r.x * r.x + r.z * r.z) * mg;
                    I.zz += w * (r.y * r.y + r.x * r.x) * mg;
                    I.xy -= w * r.x * r.y * mg;
                    I.xz -= w * r.x * r.z * mg;
                    I.yz -= w * r.y * r.z * mg;
                }
    }
    if (mass_out) *mass_out = mass;
    if (centroid) { centroid[0] = c.x; centroid[1] = c.y; centroid[2] = c.z; }
    if (inertia) {
        inertia[0] = I.xx; inertia[1] = I.yy; inertia[2] = I.zz;
        inertia[3] = I.xy; inertia[4] = I.xz; inertia[5] = I.yz;
    }
    return FUNDEM_OK;
}

int fundem_add_objects(fundem_sim* s, int wall, int n, const double* pos, const double* vel, const double* angvel,
                       const double* quat, const int* mat, const int* geo)
{
    if (!s || n < 0 || (n > 0 && (!pos || !quat || !mat || !geo))) return FUNDEM_ERR_ARG;
    ObjHost& O = wall ? s->W : s->P;
    const MatHost& M = wall ? s->wmat : s->pmat;
    const GeoSetHost& G = wall ? s->wgeo : s->pgeo;
    {
        int r = guard(s, [&] { s->pull(O); });
        if (r) return r;
    }
    for (int i = 0; i < n; ++i) {
        // LSParticle::addParticle rejects unknown ids, LSParticle.h:276-286
        if (mat[i] < 0 || mat[i] >= (int)M.kn.size()) return FUNDEM_ERR_ARG;
        if (geo[i] < 0 || geo[i] >= (int)G.geos.size()) return FUNDEM_ERR_ARG;
    }
    for (int i = 0; i < n; ++i) {
        O.pos.push_back(d3(pos + 3 * i));
        O.vel.push_back(vel ? d3(vel + 3 * i) : make_double3(0, 0, 0));
        O.angvel.push_back(angvel ? d3(angvel + 3 * i) : make_double3(0, 0, 0));
        O.force.push_back(make_double3(0, 0, 0));
        O.torque.push_back(make_double3(0, 0, 0));
        O.q.push_back(hnormalize_q(fd_quat{quat[4 * i], quat[4 * i + 1], quat[4 * i + 2], quat[4 * i + 3]}));
        O.mat.push_back(mat[i]);
        O.geo.push_back(geo[i]);
    }
    O.dirty = true;
    return FUNDEM_OK;
}

int fundem_set_wall_motion(fundem_sim* s, int index, const double vel[3], const double angvel[3])
{
    if (!s || index < 0 || index >= s->W.n()) return FUNDEM_ERR_ARG;
    return guard(s, [&] {
        s->pull(s->W);
        if (vel) s->W.vel[index] = d3(vel);
        if (angvel) s->W.angvel[index] = d3(angvel);
        s->W.dirty = true;
    });
}

int fundem_move(fundem_sim* s, int wall, int index, const double offset[3])
{
    if (!s || !offset) return FUNDEM_ERR_ARG;
    ObjHost& O = wall ? s->W : s->P;
    if (index < 0 || index >= O.n()) return FUNDEM_ERR_ARG;
    return guard(s, [&] {
        s->pull(O);
        O.pos[index] = O.pos[index] + d3(offset);
        O.dirty = true;
    });
}

int fundem_add_bonds(fundem_sim* s, int n, const int* master, const int* slave, const double* point,
                     const double* normal, const double* radius, const double* length, const double* young,
                     const double* poisson, const double* tensile, const double* cohesion, const double* friction)
{
    if (!s || n < 0) return FUNDEM_ERR_ARG;
    if (n > 0 && (!master || !slave || !point || !normal || !radius || !length || !young || !poisson))
        return FUNDEM_ERR_ARG;
    // bonds are built from the current host-side state (the reference reads
    // positionHostRef/orientationHostRef, LSSolver.h:300-316)
    {
        int r = guard(s, [&] { s->pull(s->P); });
        if (r) return r;
    }
    const double PI = 3.14159265358979323846;
    BondHost& B = s->bonds;
    int added = 0;
    for (int k = 0; k < n; ++k) {
        const int mi = master[k], sj = slave[k];
        if (mi < 0 || sj < 0 || mi >= s->P.n() || sj >= s->P.n()) continue;  // LSSolver.h:300
        const double3 gn = d3(normal + 3 * k);
        const double Rb = radius[k], Lb = length[k], Eb = young[k], nu = poisson[k];
        if (fd_is_zero(lengthSq3(gn)) || Rb <= 0. || Lb <= 0. || Eb <= 0. || nu <= -1.0 || nu >= 0.5) continue;
        const double Gb = Eb / (2. * (1. + nu));
        const double Ab = PI * Rb * Rb;
        const double Ib = Ab * Rb * Rb / 4.;
        const double Jb = 2. * Ib;
        const double Kn = Eb * Ab / Lb, Kt = Gb * Jb / Lb, Ks = 12. * Eb * Ib / (Lb * Lb * Lb), Kb = Eb * Ib / Lb;
        const double B1 = Kn, B2 = Lb * Lb * Ks, B4 = Kt, B3 = Kb - B2 / 4. - B4 / 2.;
        const double3 nn = gn * (1.0 / std::sqrt(gn.x * gn.x + gn.y * gn.y + gn.z * gn.z));
        const double3 c = d3(point + 3 * k);
        const double3 gpi = c + (0.5 * Lb) * nn, gpj = c - (0.5 * Lb) * nn;
        const fd_quat qi = s->P.q[mi], qj = s->P.q[sj];
        const double3 lpi = hrrot(gpi - s->P.pos[mi], qi);
        const double3 lpj = hrrot(gpj - s->P.pos[sj], qj);
        const double3 n1i = -nn;
        const double3 ref = (std::fabs(n1i.x) < 0.9) ? make_double3(1., 0., 0.) : make_double3(0., 1., 0.);
        const double3 n2i = hnormalize(cross3(ref, n1i));
        const double3 n3i = hnormalize(cross3(n1i, n2i));
        const double3 n1j = -n1i, n2j = n2i, n3j = n3i;
        B.master.push_back(mi);
        B.slave.push_back(sj);
        B.active.push_back(1);
        B.point.push_back(c);
        B.B.insert(B.B.end(), {B1, B2, B3, B4});
        B.radius.push_back(Rb);
        B.L0.push_back(Lb);
        B.ts.push_back(tensile ? tensile[k] : 0.0);
        B.coh.push_back(cohesion ? cohesion[k] : 0.0);
        B.mu.push_back(friction ? friction[k] : 0.0);
        B.energy.insert(B.energy.end(), {0., 0., 0., 0., 0., 0.});
        B.frames.push_back(hnormalize(hrrot(n1i, qi)));
        B.frames.push_back(hnormalize(hrrot(n2i, qi)));
        B.frames.push_back(hnormalize(hrrot(n3i, qi)));
        B.frames.push_back(lpi);
        B.frames.push_back(hnormalize(hrrot(n1j, qj)));
        B.frames.push_back(hnormalize(hrrot(n2j, qj)));
        B.frames.push_back(hnormalize(hrrot(n3j, qj)));
        B.frames.push_back(lpj);
        ++added;
    }
    B.dirty = true;
    return added == n ? FUNDEM_OK : FUNDEM_ERR_ARG;
}

int fundem_set_periodic(fundem_sim* s, int x, int y)
{
    if (!s) return FUNDEM_ERR_ARG;
    s->perX = x != 0;
    s->perY = y != 0;
    return FUNDEM_OK;
}

int fundem_set_periodic_sector(fundem_sim* s, int on)
{
    if (!s) return FUNDEM_ERR_ARG;
    s->sector = on != 0;
    return FUNDEM_OK;
}

int fundem_set_inertia_mode(fundem_sim* s, int mode)
{
    if (!s || (mode != FUNDEM_INERTIA_REFERENCE && mode != FUNDEM_INERTIA_PHYSICAL)) return FUNDEM_ERR_ARG;
    if (mode != s->inertia_mode) {
        s->inertia_mode = mode;
        s->geo_dirty = true;
    }
    return FUNDEM_OK;
}

int fundem_setup(fundem_sim* s, const double mn[3], const double mx[3])
{
    if (!s || !mn || !mx) return FUNDEM_ERR_ARG;
    if (!(mx[0] - mn[0] > 0.0) || !(mx[1] - mn[1] > 0.0) || !(mx[2] - mn[2] > 0.0)) return FUNDEM_ERR_ARG;
    return guard(s, [&] { s->setup(d3(mn), d3(mx)); });
}

int fundem_detect(fundem_sim* s)
{
    if (!s) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        s->detect_fit(0.0);
        s->detected = true;
    });
}

int fundem_detect_proximity(fundem_sim* s, double gap)
{
    if (!s || !(gap >= 0.0)) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        s->detect_fit(gap);
    });
}

int fundem_step_begin(fundem_sim* s, const double g[3], double dt)
{
    if (!s || !g) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        if (++s->hook_steps % CAPACITY_CHECK == 0) s->ensure_capacity();
        s->pc_check_overflow();
        s->pc_reserve();
        s->pc_prepare();
        s->front(d3(g), dt);
        s->detect_all(true, dt);
    });
}

int fundem_step_end(fundem_sim* s, const double g[3], double dt)
{
    if (!s || !g) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] { s->back(d3(g), dt); });
}

int fundem_step(fundem_sim* s, int nsteps, const double g[3], double dt)
{
    if (!s || !g || nsteps < 0) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        for (int k = 0; k < nsteps; ++k) {
            // list capacities follow the counts every CAPACITY_CHECK steps,
            // counted across calls
            if (++s->hook_steps % CAPACITY_CHECK == 0) s->ensure_capacity();
            s->pc_check_overflow();
            s->pc_reserve();
            s->pc_prepare();
            // the host checks above touch no particle state: a step's first
            // half kick and drift run with the previous step's second half
            // kick (back_front), ahead of them
            if (k == 0) s->front(d3(g), dt);
            s->detect_all(true, dt);
            if (k + 1 < nsteps) s->back_front(d3(g), dt);
            else s->back(d3(g), dt);
        }
        FD_CUDA(cudaGetLastError());
    });
}

int fundem_step_graph(fundem_sim* s, int nsteps, const double g[3], double dt)
{
    if (!s || !g || nsteps < 1) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        s->pc_check_overflow();  // before the graph is looked up: these may grow the lists
        s->pc_reserve();
        const double key[8] = {g[0], g[1], g[2], dt, (double)s->precision, (double)s->records,
                               (double)s->counters,
                               (double)(s->pc_active() * 8 + s->sector * 4 + s->perX * 2 + s->perY)};
        auto reusable = [&](const fundem_sim::StepGraph& G) {
            bool same = G.exec && G.steps == nsteps && G.epoch == s->alloc_epoch && G.gepoch == g_alloc_epoch.load();
            for (int k = 0; k < 8 && same; ++k) same = G.key[k] == key[k];
            return same;
        };
        // grow the lists ahead of their counts every CAPACITY_CHECK steps, as
        // fundem_step does, and always before a capture (which also makes
        // every lazy allocation of a step first)
        if (!reusable(s->graphs[s->lists[FD_PP].cur]) || s->graph_unchecked >= CAPACITY_CHECK) {
            s->ensure_capacity();
            s->rev_view();
            s->graph_unchecked = 0;
        }
        s->graph_unchecked += nsteps;
        // the generation the run starts on (all lists flip together)
        fundem_sim::StepGraph& G = s->graphs[s->lists[FD_PP].cur];
        if (!reusable(G)) {
            if (G.exec) cudaGraphExecDestroy(G.exec);
            G.exec = nullptr;
            if (!s->cap_stream) FD_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
            const cudaStream_t own = s->stream;
            const unsigned long long epoch = s->alloc_epoch, gepoch = g_alloc_epoch.load();
            s->stream = s->cap_stream;
            s->capturing = true;
            const long long launches0 = s->launches, pc_steps0 = s->pc_steps;
            cudaGraph_t graph = nullptr;
            cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
            try {
                if (e != cudaSuccess) throw CudaError(cudaGetErrorString(e));
                for (int k = 0; k < nsteps; ++k) {
                    if (k == 0) s->front(d3(g), dt);
                    s->detect_all(true, dt);
                    if (k + 1 < nsteps) s->back_front(d3(g), dt);
                    else s->back(d3(g), dt);
                }
            } catch (...) {
                cudaStreamEndCapture(s->stream, &graph);
                if (graph) cudaGraphDestroy(graph);
                s->stream = own;
                s->capturing = false;
                throw;
            }
            e = cudaStreamEndCapture(s->stream, &graph);
            s->stream = own;
            s->capturing = false;
            FD_CUDA(e);
            if (s->alloc_epoch != epoch || g_alloc_epoch.load() != gepoch) {
                cudaGraphDestroy(graph);
                throw std::logic_error("a device allocation happened while the steps were captured");
            }
            e = cudaGraphInstantiate(&G.exec, graph, 0);
            cudaGraphDestroy(graph);
            FD_CUDA(e);
            // the capture noted the kernels without running them: they count
            // when a replay runs them
            G.kernels = s->launches - launches0;
            s->launches = launches0;
            G.pc_steps = s->pc_steps - pc_steps0;
            s->pc_steps = pc_steps0;
            G.steps = nsteps;
            std::copy(key, key + 8, G.key);
            G.epoch = epoch;
            G.gepoch = gepoch;
            // capturing flipped the host's generation index nsteps times
            // without running a step; put it back so the launch below
            // starts from the generation it was captured for
            if (nsteps & 1)
                for (int k = 0; k < FD_NKIND; ++k) s->lists[k].cur ^= 1;
        }
        s->pc_prepare();
        FD_CUDA(cudaGraphLaunch(G.exec, s->stream));
        s->launches += G.kernels;
        s->pc_steps += G.pc_steps;
        // the launch leaves the newest lists in the generation nsteps flips on
        if (nsteps & 1)
            for (int k = 0; k < FD_NKIND; ++k) s->lists[k].cur ^= 1;
    });
}

int fundem_sync(fundem_sim* s)
{
    if (!s) return FUNDEM_ERR_ARG;
    unsigned int f = 0;
    int r = guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        if (s->setup_done) s->ensure_capacity();
        FD_CUDA(cudaGetLastError());
        if (s->flags.p) FD_CUDA(cudaMemcpy(&f, s->flags.p, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    });
    if (r) return r;
    if (f & (FD_FLAG_PAIR_OVERFLOW | FD_FLAG_CONTACT_OVERFLOW | FD_FLAG_NEIGHBOR_OVERFLOW | FD_FLAG_CLUSTER_OVERFLOW))
        return FUNDEM_ERR_CAPACITY;
    if (f & FD_FLAG_NONFINITE) return FUNDEM_ERR_NUMERIC;
    return FUNDEM_OK;
}

int fundem_status_word(fundem_sim* s, unsigned int* out)
{
    if (!s || !out) return FUNDEM_ERR_ARG;
    *out = 0;
    if (!s->flags.p) return FUNDEM_OK;
    return guard(s, [&] {
        FD_CUDA(cudaMemcpyAsync(out, s->flags.p, sizeof(unsigned int), cudaMemcpyDeviceToHost, s->stream));
    });
}

int fundem_num_objects(fundem_sim* s, int wall, int* n)
{
    if (!s || !n) return FUNDEM_ERR_ARG;
    *n = wall ? s->W.n() : s->P.n();
    return FUNDEM_OK;
}

int fundem_get_objects(fundem_sim* s, int wall, double* pos, double* vel, double* angvel, double* quat, double* force,
                       double* torque)
{
    if (!s) return FUNDEM_ERR_ARG;
    ObjHost& O = wall ? s->W : s->P;
    return guard(s, [&] {
        const size_t n = O.n();
        const bool dev = (O.n_dev == (int)n) && !O.dirty && n > 0;
        auto get = [&](double* dst, const void* dsrc, const void* hsrc, size_t bytes) {
            if (!dst || bytes == 0) return;
            if (dev) FD_CUDA(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToHost, s->stream));
            else std::memcpy(dst, hsrc, bytes);
        };
        get(pos, O.d_pos.p, O.pos.data(), sizeof(double3) * n);
        get(vel, O.d_vel.p, O.vel.data(), sizeof(double3) * n);
        get(angvel, O.d_angvel.p, O.angvel.data(), sizeof(double3) * n);
        get(quat, O.d_q.p, O.q.data(), sizeof(fd_quat) * n);
        get(force, O.d_force.p, O.force.data(), sizeof(double3) * n);
        get(torque, O.d_torque.p, O.torque.data(), sizeof(double3) * n);
        FD_CUDA(cudaStreamSynchronize(s->stream));
    });
}

int fundem_set_objects(fundem_sim* s, int wall, const double* pos, const double* vel, const double* angvel,
                       const double* quat, const double* force, const double* torque)
{
    if (!s) return FUNDEM_ERR_ARG;
    ObjHost& O = wall ? s->W : s->P;
    return guard(s, [&] {
        s->pc_force = true;  // the pair cache rebuilds at the next step
        const size_t n = O.n();
        const bool dev = (O.n_dev == (int)n) && !O.dirty && n > 0;
        // with the state on the device, the device copy is the one kept (the
        // host copy is refreshed from it wherever it is read, pull())
        auto put = [&](void* ddst, void* hdst, const double* src, size_t bytes) {
            if (!src || bytes == 0) return;
            if (dev) FD_CUDA(cudaMemcpyAsync(ddst, src, bytes, cudaMemcpyHostToDevice, s->stream));
            else std::memcpy(hdst, src, bytes);
        };
        put(O.d_pos.p, O.pos.data(), pos, sizeof(double3) * n);
        put(O.d_vel.p, O.vel.data(), vel, sizeof(double3) * n);
        put(O.d_angvel.p, O.angvel.data(), angvel, sizeof(double3) * n);
        put(O.d_q.p, O.q.data(), quat, sizeof(fd_quat) * n);
        put(O.d_force.p, O.force.data(), force, sizeof(double3) * n);
        put(O.d_torque.p, O.torque.data(), torque, sizeof(double3) * n);
        FD_CUDA(cudaStreamSynchronize(s->stream));
    });
}

int fundem_device_view_get(fundem_sim* s, int wall, fundem_device_view* out)
{
    if (!s || !out) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    ObjHost& O = wall ? s->W : s->P;
    out->pos = (double*)O.d_pos.p;
    out->vel = (double*)O.d_vel.p;
    out->angvel = (double*)O.d_angvel.p;
    out->force = (double*)O.d_force.p;
    out->torque = (double*)O.d_torque.p;
    out->quat = (double*)O.d_q.p;
    out->mat = O.d_mat.p;
    out->geo = O.d_geo.p;
    out->n = O.n_dev;
    return FUNDEM_OK;
}

int fundem_num_pairs(fundem_sim* s, int kind, long long* n)
{
    if (!s || !n || kind < 0 || kind >= FD_NKIND) return FUNDEM_ERR_ARG;
    *n = 0;
    PairList& L = s->lists[kind];
    if (!L.allocated) return FUNDEM_OK;
    return guard(s, [&] {
        int c[2] = {0, 0};
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        *n = std::min(c[0], L.cap_pairs);
    });
}

int fundem_num_contacts(fundem_sim* s, int kind, long long* n)
{
    if (!s || !n || kind < 0 || kind >= FD_NKIND) return FUNDEM_ERR_ARG;
    *n = 0;
    PairList& L = s->lists[kind];
    if (!L.allocated) return FUNDEM_OK;
    return guard(s, [&] {
        int c[3] = {0, 0, 0};
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(c, L.gen[L.cur].counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        *n = c[1] <= L.cap_contacts ? c[2] : 0;
    });
}

int fundem_get_contacts(fundem_sim* s, int kind, int* node, int* partner, double* point, double* normal,
                        double* overlap, double* spring, double* en, double* es)
{
    if (!s || kind < 0 || kind >= FD_NKIND) return FUNDEM_ERR_ARG;
    PairList& L = s->lists[kind];
    if (!L.allocated) return FUNDEM_OK;
    return guard(s, [&] {
        int c[3] = {0, 0, 0};
        FD_CUDA(cudaStreamSynchronize(s->stream));
        PairGen& g = L.gen[L.cur];
        FD_CUDA(cudaMemcpy(c, g.counters.p, sizeof(c), cudaMemcpyDeviceToHost));
        // an overflowed list holds no valid contacts (fundem_num_contacts gives 0)
        const size_t n = (size_t)(c[1] <= L.cap_contacts ? c[1] : 0);
        std::vector<int> hn(n), hs(n);
        std::vector<double> hsp(3 * n), hpt(3 * n), hnm(3 * n), hov(n), hen(n), hes(n);
        if (n) {
            FD_CUDA(cudaMemcpy(hn.data(), g.c_node.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hs.data(), g.c_slave.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hsp.data(), g.c_spring.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hpt.data(), g.c_point.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hnm.data(), g.c_normal.p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hov.data(), g.c_overlap.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hen.data(), g.c_en.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
            FD_CUDA(cudaMemcpy(hes.data(), g.c_es.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
        }
        // slots that hold no contact carry node id -1
        std::vector<size_t> order;
        order.reserve(n);
        for (size_t k = 0; k < n; ++k)
            if (hn[k] >= 0) order.push_back(k);
        // the caller sized its arrays with fundem_num_contacts
        if (order.size() != (size_t)c[2])
            throw std::runtime_error("contact list inconsistent: " + std::to_string(order.size()) + " contacts in " +
                                     std::to_string(n) + " slots, counter " + std::to_string(c[2]));
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            return hn[a] != hn[b] ? hn[a] < hn[b] : hs[a] < hs[b];
        });
        for (size_t k = 0; k < order.size(); ++k) {
            const size_t j = order[k];
            if (node) node[k] = hn[j];
            if (partner) partner[k] = hs[j];
            for (int d = 0; d < 3; ++d) {
                if (spring) spring[3 * k + d] = hsp[3 * j + d];
                if (point) point[3 * k + d] = hpt[3 * j + d];
                if (normal) normal[3 * k + d] = hnm[3 * j + d];
            }
            if (overlap) overlap[k] = hov[j];
            if (en) en[k] = hen[j];
            if (es) es[k] = hes[j];
        }
    });
}

int fundem_set_contacts(fundem_sim* s, int kind, long long n, const int* node, const int* partner, const double* spring)
{
    if (!s || kind < 0 || kind >= FD_NKIND || n < 0 || (n > 0 && (!node || !partner || !spring))) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    PairList& L = s->lists[kind];
    return guard(s, [&] {
        s->pc_force = true;  // the pair cache rebuilds at the next step
        // group by (particle of node, partner); the list becomes the current
        // generation so the next detection reads it as history
        const int np = s->P.n();
        std::vector<size_t> order((size_t)n);
        std::iota(order.begin(), order.end(), 0);
        auto owner = [&](int nid) {
            return (int)(std::upper_bound(s->node_base.begin(), s->node_base.end(), nid) - s->node_base.begin()) - 1;
        };
        for (long long k = 0; k < n; ++k)
            if (node[k] < 0 || node[k] >= s->n_nodes) throw std::invalid_argument("node id out of range");
        // within a pair, slots ascend in node key (the order the detection
        // writes them in, which the history search relies on)
        auto key = [&](int nid) {
            const int o = owner(nid);
            return s->pgeo.key_of[s->pgeo.table[s->P.geo[o]].node_off + (nid - s->node_base[o])];
        };
        std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            const int oa = owner(node[a]), ob = owner(node[b]);
            if (oa != ob) return oa < ob;
            if (partner[a] != partner[b]) return partner[a] < partner[b];
            return key(node[a]) < key(node[b]);
        });
        std::vector<int> pairA, pairB, c_off, c_cnt, seg_off(np, 0), seg_cnt(np, 0), cn, cs, ck;
        std::vector<double> csp;
        for (size_t t = 0; t < order.size(); ++t) {
            const size_t k = order[t];
            const int A = owner(node[k]), B = partner[k];
            if (pairA.empty() || pairA.back() != A || pairB.back() != B) {
                if (seg_cnt[A] == 0) seg_off[A] = (int)pairA.size();
                seg_cnt[A]++;
                pairA.push_back(A);
                pairB.push_back(B);
                c_off.push_back((int)cn.size());
                c_cnt.push_back(0);
            }
            c_cnt.back()++;
            cn.push_back(node[k]);
            cs.push_back(B);
            ck.push_back(key(node[k]));
            csp.insert(csp.end(), {spring[3 * k], spring[3 * k + 1], spring[3 * k + 2]});
        }
        L.grow(std::max<int>(L.cap_pairs, (int)pairA.size() * 2), std::max<int>(L.cap_contacts, (int)cn.size() * 2));
        PairGen& g = L.gen[L.cur];
        g.pairA.upload(pairA.data(), pairA.size(), s->stream);
        g.pairB.upload(pairB.data(), pairB.size(), s->stream);
        g.seg_off.upload(seg_off.data(), np, s->stream);
        g.seg_cnt.upload(seg_cnt.data(), np, s->stream);
        g.c_off.upload(c_off.data(), c_off.size(), s->stream);
        g.c_cnt.upload(c_cnt.data(), c_cnt.size(), s->stream);
        g.c_node.upload(cn.data(), cn.size(), s->stream);
        g.c_slave.upload(cs.data(), cs.size(), s->stream);
        g.c_k.upload(ck.data(), ck.size(), s->stream);
        L.up_node = cn;
        L.up_partner = cs;
        g.c_spring.upload(csp.data(), csp.size(), s->stream);
        const int counters[3] = {(int)pairA.size(), (int)cn.size(), (int)cn.size()};
        g.counters.upload(counters, 3, s->stream);
        FD_CUDA(cudaStreamSynchronize(s->stream));
    });
}

int fundem_num_bonds(fundem_sim* s, int* n)
{
    if (!s || !n) return FUNDEM_ERR_ARG;
    *n = (int)s->bonds.master.size();
    return FUNDEM_OK;
}

int fundem_get_bonds(fundem_sim* s, int* activated, double* point, double* energy6)
{
    if (!s) return FUNDEM_ERR_ARG;
    BondHost& B = s->bonds;
    return guard(s, [&] {
        const size_t n = B.master.size();
        const bool dev = B.n_dev == (int)n && !B.dirty && n > 0;
        FD_CUDA(cudaStreamSynchronize(s->stream));
        if (activated) {
            if (dev) FD_CUDA(cudaMemcpy(activated, B.d_active.p, sizeof(int) * n, cudaMemcpyDeviceToHost));
            else std::memcpy(activated, B.active.data(), sizeof(int) * n);
        }
        if (point) {
            if (dev) FD_CUDA(cudaMemcpy(point, B.d_point.p, sizeof(double3) * n, cudaMemcpyDeviceToHost));
            else std::memcpy(point, B.point.data(), sizeof(double3) * n);
        }
        if (energy6) {
            if (dev) FD_CUDA(cudaMemcpy(energy6, B.d_energy.p, sizeof(double) * 6 * n, cudaMemcpyDeviceToHost));
            else std::memcpy(energy6, B.energy.data(), sizeof(double) * 6 * n);
        }
    });
}

int fundem_set_bond_activation(fundem_sim* s, const int* activated)
{
    if (!s || !activated) return FUNDEM_ERR_ARG;
    BondHost& B = s->bonds;
    return guard(s, [&] {
        const size_t n = B.master.size();
        std::memcpy(B.active.data(), activated, sizeof(int) * n);
        if (B.n_dev == (int)n && !B.dirty && n > 0)
            FD_CUDA(cudaMemcpyAsync(B.d_active.p, activated, sizeof(int) * n, cudaMemcpyHostToDevice, s->stream));
    });
}

int fundem_get_geometry(fundem_sim* s, int wall, int geo, double* radius, double* inv_mass, double inertia[6],
                        double inv_inertia[6])
{
    if (!s) return FUNDEM_ERR_ARG;
    GeoSetHost& G = wall ? s->wgeo : s->pgeo;
    if (geo < 0 || geo >= (int)G.geos.size()) return FUNDEM_ERR_ARG;
    const HostGeo& g = G.geos[geo];
    double r = 0.0;
    for (const double3& p : g.nodes) r = std::max(r, host_len(p));
    const double mass = wall ? 0.0 : g.mass;
    const fd_sym I = mass > 0.0 ? g.inertia : fd_sym{0, 0, 0, 0, 0, 0};
    const fd_sym Ii = host_inverse(I, s->inertia_mode);
    if (radius) *radius = r;
    if (inv_mass) *inv_mass = mass > 0.0 ? 1.0 / mass : 0.0;
    if (inertia) { inertia[0] = I.xx; inertia[1] = I.yy; inertia[2] = I.zz; inertia[3] = I.xy; inertia[4] = I.xz; inertia[5] = I.yz; }
    if (inv_inertia) { inv_inertia[0] = Ii.xx; inv_inertia[1] = Ii.yy; inv_inertia[2] = Ii.zz; inv_inertia[3] = Ii.xy; inv_inertia[4] = Ii.xz; inv_inertia[5] = Ii.yz; }
    return FUNDEM_OK;
}

int fundem_get_grid(fundem_sim* s, int wall, double minb[3], double maxb[3], double inv_cell[3], int size[3])
{
    if (!s) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    const FdGrid& g = wall ? s->wgrid : s->pgrid;
    if (minb) { minb[0] = g.minb.x; minb[1] = g.minb.y; minb[2] = g.minb.z; }
    if (maxb) { maxb[0] = g.maxb.x; maxb[1] = g.maxb.y; maxb[2] = g.maxb.z; }
    if (inv_cell) { inv_cell[0] = g.inv.x; inv_cell[1] = g.inv.y; inv_cell[2] = g.inv.z; }
    if (size) { size[0] = g.size.x; size[1] = g.size.y; size[2] = g.size.z; }
    return FUNDEM_OK;
}

int fundem_set_profiling(fundem_sim* s, int on)
{
    if (!s) return FUNDEM_ERR_ARG;
    if (on & ~(FUNDEM_PROF_TIMERS | FUNDEM_PROF_COUNTERS)) return FUNDEM_ERR_ARG;
    s->profiling = (on & FUNDEM_PROF_TIMERS) != 0;
    s->counters = (on & FUNDEM_PROF_COUNTERS) != 0;
    return FUNDEM_OK;
}

int fundem_kernel_time(fundem_sim* s, int group, double* ms_total, long long* count)
{
    if (!s || group < 0 || group >= FUNDEM_NTIMERS || !ms_total || !count) return FUNDEM_ERR_ARG;
    return guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        auto& a = s->tev[group][0];
        auto& b = s->tev[group][1];
        double t = 0.0;
        const size_t n = std::min(a.size(), b.size());
        for (size_t k = 0; k < n; ++k) {
            float ms = 0.f;
            FD_CUDA(cudaEventElapsedTime(&ms, a[k], b[k]));
            t += ms;
        }
        for (cudaEvent_t e : a) cudaEventDestroy(e);
        for (cudaEvent_t e : b) cudaEventDestroy(e);
        a.clear();
        b.clear();
        *ms_total = t;
        *count = (long long)n;
    });
}

int fundem_prefix_sum(int* d_prefix, const int* d_count, long long n, void* stream)
{
    if (n < 0 || n > 0x7fffffffLL || (n > 0 && (!d_prefix || !d_count))) return FUNDEM_ERR_ARG;
    if (n == 0) return FUNDEM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t ntmp = fd::scan_tmp_size(n);
    int* tmp = nullptr;
    if (cudaMallocAsync((void**)&tmp, ntmp * sizeof(int), s) != cudaSuccess) return FUNDEM_ERR_CUDA;
    fd::scan_inclusive(d_count, d_prefix, n, tmp, s);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(tmp, s);
    return e == cudaSuccess ? FUNDEM_OK : FUNDEM_ERR_CUDA;
}

int fundem_hash_sort(const long long* d_hash, int n, long long num_cells, int* d_sorted, long long* d_sorted_hash,
                     void* stream)
{
    if (n < 0 || num_cells < 0 || (n > 0 && (!d_hash || !d_sorted))) return FUNDEM_ERR_ARG;
    if (n == 0) return FUNDEM_OK;
    cudaStream_t s = (cudaStream_t)stream;
    size_t bc = 0, bs = 0;
    fd::radix_sort_scratch(n, bc, bs);
    // one block of scratch: sorted keys, second key buffer, second index
    // buffer, block counts and their scan temporary
    const size_t bytes = sizeof(unsigned long long) * 2 * (size_t)n + sizeof(int) * ((size_t)n + bc + bs) + 256;
    char* tmp = nullptr;
    if (cudaMallocAsync((void**)&tmp, bytes, s) != cudaSuccess) return FUNDEM_ERR_CUDA;
    unsigned long long* okey = reinterpret_cast<unsigned long long*>(tmp);
    unsigned long long* key_b = okey + n;
    int* idx_b = reinterpret_cast<int*>(key_b + n);
    int* bcount = idx_b + n;
    int* bscan = bcount + bc;
    fd::radix_sort_keys(d_hash, n, num_cells, okey, d_sorted, key_b, idx_b, bcount, bscan, s);
    if (d_sorted_hash)
        cudaMemcpyAsync(d_sorted_hash, okey, sizeof(long long) * (size_t)n, cudaMemcpyDeviceToDevice, s);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(tmp, s);
    return e == cudaSuccess ? FUNDEM_OK : FUNDEM_ERR_CUDA;
}

int fundem_work_counters(fundem_sim* s, unsigned long long out[5])
{
    if (!s || !out) return FUNDEM_ERR_ARG;
    if (!s->stats.p) { for (int k = 0; k < 5; ++k) out[k] = 0; return FUNDEM_OK; }
    return guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(out, s->stats.p, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        FD_CUDA(cudaMemsetAsync(s->stats.p, 0, 8 * sizeof(unsigned long long), s->stream));
    });
}

int fundem_set_launch_shape(fundem_sim* s, const int blocks_per_sm[4])
{
    if (!s || !blocks_per_sm) return FUNDEM_ERR_ARG;
    for (int k = 0; k < 4; ++k)
        if (blocks_per_sm[k] < 0 || blocks_per_sm[k] > 64) {
            s->last_error = "blocks per SM must lie in 0 (the default) .. 64";
            return FUNDEM_ERR_ARG;
        }
    return guard(s, [&] {
        for (int k = 0; k < 4; ++k) s->launch_shape[k] = blocks_per_sm[k];
        s->drop_graph();  // recorded graphs hold the old grids
    });
}

int fundem_get_launch_shape(fundem_sim* s, int blocks_per_sm[4])
{
    if (!s || !blocks_per_sm) return FUNDEM_ERR_ARG;
    const int def[4] = {FD_SELECT_MIN_BLOCKS, FD_PROBE_MIN_BLOCKS, 4, 4};
    for (int k = 0; k < 4; ++k) blocks_per_sm[k] = s->launch_shape[k] > 0 ? s->launch_shape[k] : def[k];
    return FUNDEM_OK;
}

int fundem_slot_counters(fundem_sim* s, unsigned long long out[2])
{
    if (!s || !out) return FUNDEM_ERR_ARG;
    if (!s->stats.p) { out[0] = out[1] = 0; return FUNDEM_OK; }
    return guard(s, [&] {
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(out, s->stats.p + 5, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    });
}

const char* fundem_last_error(fundem_sim* s)
{
    return s ? s->last_error.c_str() : "";
}

int fundem_launch_count(fundem_sim* s, long long* n)
{
    if (!s || !n) return FUNDEM_ERR_ARG;
    *n = s->launches;
    return FUNDEM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// adjoint: checkpoints, segment re-runs with recording, reverse sweep
// ---------------------------------------------------------------------------
namespace {

void adj_check(int r)
{
    if (r != FUNDEM_OK) throw std::runtime_error(std::string("adjoint: ") + fundem_status_string(r));
}

void adj_snapshot(fundem_sim* s, AdjCheckpoint& c)
{
    int np = 0, nw = 0;
    adj_check(fundem_num_objects(s, 0, &np));
    adj_check(fundem_num_objects(s, 1, &nw));
    auto grab = [&](int wall, int n, std::vector<double>& x, std::vector<double>& v, std::vector<double>& w,
                    std::vector<double>& q, std::vector<double>& f, std::vector<double>& t) {
        x.assign(3 * n, 0.0); v.assign(3 * n, 0.0); w.assign(3 * n, 0.0); q.assign(4 * n, 0.0);
        f.assign(3 * n, 0.0); t.assign(3 * n, 0.0);
        if (n > 0) adj_check(fundem_get_objects(s, wall, x.data(), v.data(), w.data(), q.data(), f.data(), t.data()));
    };
    grab(0, np, c.pos, c.vel, c.angvel, c.quat, c.force, c.torque);
    grab(1, nw, c.wpos, c.wvel, c.wangvel, c.wquat, c.wforce, c.wtorque);
    for (int k = 0; k < FD_NKIND; ++k) {
        long long n = 0;
        adj_check(fundem_num_contacts(s, k, &n));
        c.node[k].assign(n, 0); c.partner[k].assign(n, 0); c.spring[k].assign(3 * n, 0.0);
        if (n > 0)
            adj_check(fundem_get_contacts(s, k, c.node[k].data(), c.partner[k].data(), nullptr, nullptr, nullptr,
                                          c.spring[k].data(), nullptr, nullptr));
    }
    int nb = 0;
    adj_check(fundem_num_bonds(s, &nb));
    c.bond_active.assign(nb, 0);
    if (nb > 0) adj_check(fundem_get_bonds(s, c.bond_active.data(), nullptr, nullptr));
}

void adj_restore(fundem_sim* s, AdjCheckpoint& c)
{
    if (!c.quat.empty())
        adj_check(fundem_set_objects(s, 0, c.pos.data(), c.vel.data(), c.angvel.data(), c.quat.data(), c.force.data(),
                                     c.torque.data()));
    if (!c.wquat.empty())
        adj_check(fundem_set_objects(s, 1, c.wpos.data(), c.wvel.data(), c.wangvel.data(), c.wquat.data(),
                                     c.wforce.data(), c.wtorque.data()));
    for (int k = 0; k < FD_NKIND; ++k) {
        if (!s->lists[k].allocated) continue;
        adj_check(fundem_set_contacts(s, k, (long long)c.node[k].size(), c.node[k].data(), c.partner[k].data(),
                                      c.spring[k].data()));
    }
    if (!c.bond_active.empty()) adj_check(fundem_set_bond_activation(s, c.bond_active.data()));
}

}  // namespace

extern "C" {

int fundem_adjoint_begin(fundem_sim* s, int checkpoint_interval)
{
    if (!s || checkpoint_interval < 1) return FUNDEM_ERR_ARG;
    if (!s->setup_done || !s->detected) return FUNDEM_ERR_STATE;
    if (s->sector) {
        s->last_error = "the adjoint does not differentiate through the turned images of sector periodicity";
        return FUNDEM_ERR_STATE;
    }
    if (s->adj_turning() && !s->bonds.master.empty()) {
        s->last_error = "the adjoint differentiates bonds between bodies that do not turn only: a particle "
                        "geometry can rotate and the run has bonds";
        return FUNDEM_ERR_STATE;
    }
    return guard(s, [&] {
        AdjState& A = s->adj;
        A = AdjState{};
        A.on = true;
        s->pc_force = true;  // the adjoint runs full detections; the cache rebuilds afterwards
        A.precision = s->precision;
        A.K = checkpoint_interval;
        A.ckpt.emplace_back();
        adj_snapshot(s, A.ckpt.back());
        A.seg_steps.push_back(0);
    });
}

int fundem_adjoint_forward(fundem_sim* s, int nsteps, const double g[3], double dt)
{
    if (!s || !g || nsteps < 0 || !(dt > 0.0)) return FUNDEM_ERR_ARG;
    AdjState& A = s->adj;
    if (!A.on) return FUNDEM_ERR_STATE;
    const double3 gg = make_double3(g[0], g[1], g[2]);
    if (A.dt_set && (A.dt != dt || A.g.x != gg.x || A.g.y != gg.y || A.g.z != gg.z)) {
        s->last_error = "the adjoint needs one time step and one gravity over the recording";
        return FUNDEM_ERR_ARG;
    }
    if (s->precision != A.precision) {
        s->last_error = "the precision changed since fundem_adjoint_begin";
        return FUNDEM_ERR_STATE;
    }
    A.g = gg;
    A.dt = dt;
    A.dt_set = true;
    const int r = guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        for (int k = 0; k < nsteps; ++k) {
            if (A.seg_steps.back() == A.K) {
                A.ckpt.emplace_back();
                adj_snapshot(s, A.ckpt.back());
                A.seg_steps.push_back(0);
            }
            if (A.steps % CAPACITY_CHECK == 0) s->ensure_capacity();
            s->front(gg, dt);
            s->detect_all(true, dt);
            s->back(gg, dt);
            A.seg_steps.back() += 1;
            A.steps += 1;
        }
        FD_CUDA(cudaGetLastError());
    });
    if (r != FUNDEM_OK) return r;
    return fundem_sync(s);
}

int fundem_adjoint_backward(fundem_sim* s, const double* dl_dpos, const double* dl_dvel, double* dl_dvel0,
                            double* dl_dparams)
{
    return fundem_adjoint_backward_rot(s, dl_dpos, dl_dvel, nullptr, nullptr, dl_dvel0, nullptr, dl_dparams);
}

int fundem_adjoint_backward_rot(fundem_sim* s, const double* dl_dpos, const double* dl_dvel, const double* dl_dquat,
                                const double* dl_dangvel, double* dl_dvel0, double* dl_dangvel0, double* dl_dparams)
{
    if (!s || !dl_dpos || !dl_dvel || !dl_dvel0 || !dl_dparams) return FUNDEM_ERR_ARG;
    AdjState& A = s->adj;
    if (!A.on || A.steps == 0) return FUNDEM_ERR_STATE;
    if (s->precision != A.precision) {
        s->last_error = "the precision changed since fundem_adjoint_begin";
        return FUNDEM_ERR_STATE;
    }
    return guard(s, [&] {
        FD_CUDA(cudaSetDevice(s->device));
        adj_snapshot(s, A.final_state);
        s->ensure_capacity();
        const int np = s->P.n();
        const int nmat = (int)s->pmat.kn.size();
        const int K = A.K;
        // tape for one segment
        AdjTape& T = s->tape;
        T.steps = K;
        // lists the step fills: particle pairs, walls, and the ghost
        // directions in use (the adjoint refuses sector periodicity); the
        // others keep no tape and are skipped by the sweep
        bool used[FD_NKIND] = {};
        used[FD_PP] = used[FD_PW] = true;
        used[FD_GX] = s->ghosts[0].active;
        used[FD_GY] = s->ghosts[1].active;
        used[FD_GXY] = s->ghosts[2].active;
        for (int k = 0; k < FD_NKIND; ++k) {
            T.cap[k] = (used[k] && s->lists[k].allocated) ? s->lists[k].cap_contacts : 0;
            const size_t c = (size_t)std::max(T.cap[k], 1);
            T.ints[k].alloc(9 * c * K, false);
            T.dbl[k].alloc(16 * c * K, false);
        }
        T.nslots.alloc((size_t)K * FD_NKIND);
        fd::BondDev bd = s->bond_view();
        T.nbond = bd.n;
        T.bond_active.alloc((size_t)std::max(bd.n, 1) * K);
        T.bond_rij.alloc((size_t)std::max(bd.n, 1) * 3 * K);
        T.bond_dn.alloc((size_t)std::max(bd.n, 1) * 3 * K);
        DevArray<double> xb, vb, vhb, Fb, Feb, pgrad, Sb[2][FD_NKIND];
        xb.alloc(3 * (size_t)np); vb.alloc(3 * (size_t)np); vhb.alloc(3 * (size_t)np);
        Fb.alloc(3 * (size_t)np); Feb.alloc(3 * (size_t)np); pgrad.alloc(4 * (size_t)std::max(nmat, 1));
        // turning bodies: orientation and angular-velocity adjoints and the
        // per-step record of orientations, angular velocities and torques
        const bool rot = s->adj_turning();
        DevArray<double> qb, wb, whb, Tb, Teb;
        if (rot) {
            qb.alloc(4 * (size_t)np); wb.alloc(3 * (size_t)np); whb.alloc(3 * (size_t)np);
            Tb.alloc(3 * (size_t)np); Teb.alloc(3 * (size_t)np);
            T.prot.alloc((size_t)fd::ADJ_PREC * np * (K + 1), false);
            if (dl_dquat) qb.upload(dl_dquat, 4 * (size_t)np, s->stream);
            if (dl_dangvel) wb.upload(dl_dangvel, 3 * (size_t)np, s->stream);
        }
        for (int k = 0; k < FD_NKIND; ++k) {
            Sb[0][k].alloc(3 * (size_t)std::max(T.cap[k], 1));
            Sb[1][k].alloc(3 * (size_t)std::max(T.cap[k], 1));
        }
        xb.upload(dl_dpos, 3 * (size_t)np, s->stream);
        vb.upload(dl_dvel, 3 * (size_t)np, s->stream);
        const ObjDev Pv = s->P.view();
        fd::AdjParticles ap{np, Pv.geo, Pv.mat, Pv.angvel, s->pgeo.view(), xb.p, vb.p, vhb.p, Fb.p, Feb.p, pgrad.p,
                            rot ? 1 : 0, nullptr, nullptr, qb.p, wb.p, whb.p, Tb.p, Teb.p};
        const size_t prs = (size_t)fd::ADJ_PREC * np;  // record doubles per step
        std::map<std::tuple<int, int, int>, double3> carry;
        int cur = 0;
        for (int seg = (int)A.ckpt.size() - 1; seg >= 0; --seg) {
            const int ns = A.seg_steps[seg];
            if (ns == 0) continue;
            adj_restore(s, A.ckpt[seg]);
            // re-run the segment, recording every step
            s->recording = &T;
            if (rot) fd::adj_record_rot(s->P.view(), T.prot.p, fd::ADJ_REC_QW | fd::ADJ_REC_T, s->stream);
            for (int t = 0; t < ns; ++t) {
                s->record_step = t;
                s->front(A.g, A.dt);
                if (rot) fd::adj_record_rot(s->P.view(), T.prot.p + prs * (t + 1), fd::ADJ_REC_QW, s->stream);
                s->detect_all(true, A.dt);
                s->back(A.g, A.dt);
                if (rot) fd::adj_record_rot(s->P.view(), T.prot.p + prs * (t + 1), fd::ADJ_REC_T, s->stream);
            }
            s->recording = nullptr;
            FD_CUDA(cudaStreamSynchronize(s->stream));
            unsigned int f = 0;
            FD_CUDA(cudaMemcpy(&f, s->flags.p, sizeof(f), cudaMemcpyDeviceToHost));
            if (f & (FD_FLAG_PAIR_OVERFLOW | FD_FLAG_CONTACT_OVERFLOW | FD_FLAG_NEIGHBOR_OVERFLOW))
                throw std::runtime_error("adjoint: a contact list overflowed while a segment was re-run");
            // spring adjoints of the segment's last step, from the later segment
            for (int k = 0; k < FD_NKIND; ++k)
                FD_CUDA(cudaMemsetAsync(Sb[cur][k].p, 0, Sb[cur][k].n * sizeof(double), s->stream));
            if (!carry.empty()) {
                const int t = ns - 1;
                for (int k = 0; k < FD_NKIND; ++k) {
                    if (T.cap[k] == 0) continue;
                    int nsl = 0;
                    FD_CUDA(cudaMemcpy(&nsl, T.ns(k, t), sizeof(int), cudaMemcpyDeviceToHost));
                    nsl = std::min(nsl, T.cap[k]);
                    if (nsl <= 0) continue;
                    const fd::AdjRec R = T.rec(k, t);
                    std::vector<int> hit(nsl), nid(nsl), B(nsl);
                    FD_CUDA(cudaMemcpy(hit.data(), R.hit, sizeof(int) * nsl, cudaMemcpyDeviceToHost));
                    FD_CUDA(cudaMemcpy(nid.data(), R.nid, sizeof(int) * nsl, cudaMemcpyDeviceToHost));
                    FD_CUDA(cudaMemcpy(B.data(), R.B, sizeof(int) * nsl, cudaMemcpyDeviceToHost));
                    std::vector<double> sb(3 * (size_t)nsl, 0.0);
                    bool any = false;
                    for (int i = 0; i < nsl; ++i) {
                        if (!hit[i]) continue;
                        auto it = carry.find(std::make_tuple(k, nid[i], B[i]));
                        if (it == carry.end()) continue;
                        sb[3 * i] = it->second.x; sb[3 * i + 1] = it->second.y; sb[3 * i + 2] = it->second.z;
                        any = true;
                    }
                    if (any)
                        FD_CUDA(cudaMemcpyAsync(Sb[cur][k].p, sb.data(), sizeof(double) * sb.size(),
                                                cudaMemcpyHostToDevice, s->stream));
                }
            }
            // reverse sweep over the segment
            for (int t = ns - 1; t >= 0; --t) {
                if (rot) {
                    ap.pr_prev = T.prot.p + prs * t;
                    ap.pr_cur = T.prot.p + prs * (t + 1);
                }
                fd::adj_force(ap, A.dt, s->stream);
                const int prv = cur ^ 1;
                for (int k = 0; k < FD_NKIND; ++k)
                    FD_CUDA(cudaMemsetAsync(Sb[prv][k].p, 0, Sb[prv][k].n * sizeof(double), s->stream));
                for (int k = 0; k < FD_NKIND; ++k) {
                    if (T.cap[k] == 0) continue;
                    fd::AdjContactArgs c{};
                    c.rec = T.rec(k, t);
                    c.period = make_double3(s->pgrid.maxb.x - s->pgrid.minb.x, s->pgrid.maxb.y - s->pgrid.minb.y, 0.0);
                    c.nslots = T.ns(k, t);
                    c.M = s->pmat.view();
                    c.MW = s->wmat.view();
                    c.GW = s->wgeo.view();
                    c.wall_angvel = s->W.view().angvel;
                    c.Sb_cur = Sb[cur][k].p;
                    c.Sb_prev = Sb[prv][k].p;
                    c.sb_prev_cap = T.cap[k];
                    c.dt = A.dt;
                    fd::adj_contacts(ap, c, s->stream);
                }
                if (bd.n > 0) {
                    fd::AdjBondArgs b{bd.n, bd.master, bd.slave, T.bond_active.p + (long long)t * bd.n,
                                      T.bond_rij.p + 3ll * t * bd.n, bd.B, bd.L0, T.bond_dn.p + 3ll * t * bd.n};
                    fd::adj_bonds(ap, b, s->stream);
                }
                fd::adj_particles(ap, A.dt, s->stream);
                cur = prv;
            }
            FD_CUDA(cudaGetLastError());
            // spring adjoints of the restored lists (the state before the
            // segment), keyed for the earlier segment
            carry.clear();
            FD_CUDA(cudaStreamSynchronize(s->stream));
            for (int k = 0; k < FD_NKIND; ++k) {
                const PairList& L = s->lists[k];
                const size_t n = L.up_node.size();
                if (T.cap[k] == 0 || n == 0) continue;
                std::vector<double> sb(3 * n);
                FD_CUDA(cudaMemcpy(sb.data(), Sb[cur][k].p, sizeof(double) * 3 * std::min<size_t>(n, T.cap[k]),
                                   cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < std::min<size_t>(n, T.cap[k]); ++i)
                    if (sb[3 * i] != 0.0 || sb[3 * i + 1] != 0.0 || sb[3 * i + 2] != 0.0)
                        carry[std::make_tuple(k, L.up_node[i], L.up_partner[i])] =
                            make_double3(sb[3 * i], sb[3 * i + 1], sb[3 * i + 2]);
            }
        }
        FD_CUDA(cudaStreamSynchronize(s->stream));
        FD_CUDA(cudaMemcpy(dl_dvel0, vb.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost));
        if (dl_dangvel0) {
            if (rot) FD_CUDA(cudaMemcpy(dl_dangvel0, wb.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost));
            else std::fill(dl_dangvel0, dl_dangvel0 + 3 * (size_t)np, 0.0);
        }
        FD_CUDA(cudaMemcpy(dl_dparams, pgrad.p, sizeof(double) * 4 * nmat, cudaMemcpyDeviceToHost));
        adj_restore(s, A.final_state);
        FD_CUDA(cudaStreamSynchronize(s->stream));
    });
}

// ---------------------------------------------------------------------------
// checkpoint files: the state a restart needs, FP64 little-endian
//   "FDCK" u32 version=2, i32 np, i32 nw, i32 nb,
//   particles: pos, vel, angvel (3 np each), quat (4 np), force, torque (3 np each)
//   walls: the same with nw
//   version 2: i32 number of kinds K (version 1 files hold the first 5)
//   per kind (K): i64 n, node (n i32), partner (n i32), spring (3n f64)
//   bonds: activation (nb i32)
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {
constexpr uint32_t CKPT_MAGIC = 0x4b434446u;  // "FDCK"

template <typename T> void put(std::FILE* f, const T* p, size_t n)
{
    if (n && std::fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("checkpoint: write failed");
}
template <typename T> void get(std::FILE* f, T* p, size_t n)
{
    if (n && std::fread(p, sizeof(T), n, f) != n) throw std::runtime_error("checkpoint: file truncated");
}
}  // namespace

extern "C" {

int fundem_checkpoint_write(fundem_sim* s, const char* path)
{
    if (!s || !path) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        AdjCheckpoint c;
        adj_snapshot(s, c);
        std::FILE* f = std::fopen(path, "wb");
        if (!f) throw std::invalid_argument(std::string("cannot open ") + path);
        try {
            const uint32_t head[2] = {CKPT_MAGIC, 2u};
            const int32_t counts[3] = {(int32_t)(c.pos.size() / 3), (int32_t)(c.wpos.size() / 3),
                                       (int32_t)c.bond_active.size()};
            const int32_t nkind = FD_NKIND;
            put(f, head, 2);
            put(f, counts, 3);
            for (auto* v : {&c.pos, &c.vel, &c.angvel, &c.quat, &c.force, &c.torque, &c.wpos, &c.wvel, &c.wangvel,
                            &c.wquat, &c.wforce, &c.wtorque})
                put(f, v->data(), v->size());
            put(f, &nkind, 1);
            for (int k = 0; k < FD_NKIND; ++k) {
                const int64_t n = (int64_t)c.node[k].size();
                put(f, &n, 1);
                put(f, c.node[k].data(), c.node[k].size());
                put(f, c.partner[k].data(), c.partner[k].size());
                put(f, c.spring[k].data(), c.spring[k].size());
            }
            put(f, c.bond_active.data(), c.bond_active.size());
        } catch (...) {
            std::fclose(f);
            throw;
        }
        if (std::fclose(f) != 0) throw std::runtime_error("checkpoint: write failed");
    });
}

int fundem_checkpoint_read(fundem_sim* s, const char* path)
{
    if (!s || !path) return FUNDEM_ERR_ARG;
    if (!s->setup_done) return FUNDEM_ERR_STATE;
    return guard(s, [&] {
        s->pc_force = true;  // the pair cache rebuilds at the next step
        std::FILE* f = std::fopen(path, "rb");
        if (!f) throw std::invalid_argument(std::string("cannot open ") + path);
        AdjCheckpoint c;
        try {
            uint32_t head[2];
            int32_t counts[3];
            get(f, head, 2);
            if (head[0] != CKPT_MAGIC || (head[1] != 1u && head[1] != 2u))
                throw std::invalid_argument("not a checkpoint file");
            get(f, counts, 3);
            int np = 0, nw = 0, nb = 0;
            adj_check(fundem_num_objects(s, 0, &np));
            adj_check(fundem_num_objects(s, 1, &nw));
            adj_check(fundem_num_bonds(s, &nb));
            if (counts[0] != np || counts[1] != nw || counts[2] != nb)
                throw std::invalid_argument("checkpoint: object or bond counts differ from the simulation");
            auto rd = [&](std::vector<double>& v, size_t n) { v.resize(n); get(f, v.data(), n); };
            rd(c.pos, 3 * np); rd(c.vel, 3 * np); rd(c.angvel, 3 * np); rd(c.quat, 4 * np);
            rd(c.force, 3 * np); rd(c.torque, 3 * np);
            rd(c.wpos, 3 * nw); rd(c.wvel, 3 * nw); rd(c.wangvel, 3 * nw); rd(c.wquat, 4 * nw);
            rd(c.wforce, 3 * nw); rd(c.wtorque, 3 * nw);
            int32_t nkind = 5;
            if (head[1] == 2u) get(f, &nkind, 1);
            if (nkind < 0 || nkind > FD_NKIND) throw std::invalid_argument("checkpoint: bad number of kinds");
            for (int k = 0; k < nkind; ++k) {
                int64_t n = 0;
                get(f, &n, 1);
                if (n < 0 || n > (int64_t)1 << 31) throw std::invalid_argument("checkpoint: bad contact count");
                c.node[k].resize(n); c.partner[k].resize(n); c.spring[k].resize(3 * n);
                get(f, c.node[k].data(), n);
                get(f, c.partner[k].data(), n);
                get(f, c.spring[k].data(), 3 * n);
            }
            c.bond_active.resize(nb);
            get(f, c.bond_active.data(), nb);
        } catch (...) {
            std::fclose(f);
            throw;
        }
        std::fclose(f);
        adj_restore(s, c);
        s->detected = true;
        FD_CUDA(cudaStreamSynchronize(s->stream));
    });
}

int fundem_adjoint_end(fundem_sim* s)
{
    if (!s) return FUNDEM_ERR_ARG;
    s->adj = AdjState{};
    s->pc_force = true;
    return FUNDEM_OK;
}

}  // extern "C"

