// fd_levelset.cu -- level-set templates on the GPU: the signed-distance grid of
// an analytic shape or of a closed triangle mesh, one thread per grid node.
//
// The reference builds these grids on the host, one virtual call per node
// (kernel/helper/LevelSetObjectGenerator.h:122-224, Base::buildGrid).  Each
// node stores f / |grad f| when |grad f| > 1e-12, else +-h/2 by the sign of f.
// The implicit functions follow the reference classes:
//   Superellipsoid  LevelSetObjectGenerator.h:1264-1354
//   Sphere          :1628-1661
//   BoxWall         :1781-1867
//   CylinderWall    :2050-2131 (its end-cap gradient is the unnormalised axis
//                   vector, so grid values there are divided by the axis length)
//   triangle mesh   :888-953 (closest point over all triangles, sign by the
//                   winding number |sum of solid angles / 4 pi| > 0.5)
// This file is compiled with -fmad=false: every add and multiply rounds on its
// own as in the reference's host code, so the grids differ from a host build
// only where CUDA's pow and atan2 round differently from the host library.
#include <cfloat>
#include <cmath>

#include "fundem_b200.h"

namespace {

struct Vec { double x, y, z; };

__device__ __forceinline__ Vec mk(double x, double y, double z) { return Vec{x, y, z}; }
__device__ __forceinline__ Vec operator+(Vec a, Vec b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ Vec operator-(Vec a, Vec b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ Vec operator-(Vec a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ Vec operator*(double s, Vec a) { return mk(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ Vec operator*(Vec a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
// vector / scalar multiplies by the reciprocal, as the reference's double3 does (myVec.h:55-59)
__device__ __forceinline__ Vec operator/(Vec a, double s)
{
    const double inv = 1.0 / s;
    return mk(a.x * inv, a.y * inv, a.z * inv);
}
__device__ __forceinline__ double dot(Vec a, Vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Vec cross(Vec a, Vec b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double len(Vec a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
// host-side normalisation of the reference (myVec.h:121-137): v * (1 / sqrt(|v|^2)), zero below 1e-20
__device__ __forceinline__ Vec unit(Vec v)
{
    const double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (fabs(l2) <= 1.0e-20) return mk(0.0, 0.0, 0.0);
    const double inv = 1.0 / sqrt(l2);
    return mk(v.x * inv, v.y * inv, v.z * inv);
}
__device__ __forceinline__ double sign_no_zero(double v) { return v >= 0.0 ? 1.0 : -1.0; }

struct Shape {
    int kind;
    int flip;  // positive inside: value and gradient negated
    double p[8];
};

// Superellipsoid |x/rx|^(2/ee) + |y/ry|^(2/ee))^(ee/en) + |z/rz|^(2/en) - 1 and its gradient
__device__ void eval_superellipsoid(const double* p, Vec x, double& f, Vec& g)
{
    const double rx = p[0], ry = p[1], rz = p[2], ee = p[3], en = p[4];
    const double ix = 1.0 / rx, iy = 1.0 / ry, iz = 1.0 / rz;
    const double ax = fabs(x.x * ix), ay = fabs(x.y * iy), az = fabs(x.z * iz);
    const double exy = 2.0 / ee, ez = 2.0 / en, eo = ee / en;
    const double sxy = pow(fabs(ax), exy) + pow(fabs(ay), exy);
    f = pow(fabs(sxy), eo) + pow(fabs(az), ez) - 1.0;
    const double tiny = 1e-30;
    const double outer = pow(fabs(fmax(sxy, tiny)), eo - 1.0);
    const double dsx = exy * pow(fabs(fmax(ax, tiny)), exy - 1.0) * sign_no_zero(x.x) * ix;
    const double dsy = exy * pow(fabs(fmax(ay, tiny)), exy - 1.0) * sign_no_zero(x.y) * iy;
    const double dz = ez * pow(fabs(fmax(az, tiny)), ez - 1.0) * sign_no_zero(x.z) * iz;
    g = mk(eo * outer * dsx, eo * outer * dsy, dz);
}

__device__ void eval_sphere(const double* p, Vec x, double& f, Vec& g)
{
    const double d = len(x);
    f = d - p[0];
    if (d > 1e-30) g = x / d;  // at the centre the gradient stays zero
}

__device__ void eval_box(const double* p, Vec x, double& f, Vec& g)
{
    const Vec hb = mk(0.5 * p[0], 0.5 * p[1], 0.5 * p[2]);
    const Vec q = mk(fabs(x.x) - hb.x, fabs(x.y) - hb.y, fabs(x.z) - hb.z);
    const Vec qo = mk(fmax(q.x, 0.0), fmax(q.y, 0.0), fmax(q.z, 0.0));
    const double out = len(qo);
    const double in = fmin(fmax(q.x, fmax(q.y, q.z)), 0.0);
    f = out + in;
    if (out > 1e-30) {
        g = qo / out;
        if (x.x < 0.0 && q.x > 0.0) g.x = -g.x;
        if (x.y < 0.0 && q.y > 0.0) g.y = -g.y;
        if (x.z < 0.0 && q.z > 0.0) g.z = -g.z;
    } else {
        // inside: the normal of the nearest face
        const double fx = hb.x - fabs(x.x), fy = hb.y - fabs(x.y), fz = hb.z - fabs(x.z);
        if (fx <= fy && fx <= fz) g = mk(x.x >= 0.0 ? 1.0 : -1.0, 0.0, 0.0);
        else if (fy <= fx && fy <= fz) g = mk(0.0, x.y >= 0.0 ? 1.0 : -1.0, 0.0);
        else g = mk(0.0, 0.0, x.z >= 0.0 ? 1.0 : -1.0);
    }
}

// capped cylinder between points A (p[0..2]) and B (p[3..5]) of radius p[6]
__device__ void eval_cylinder(const double* p, Vec x, double& f, Vec& g)
{
    const Vec A = mk(p[0], p[1], p[2]), B = mk(p[3], p[4], p[5]);
    const double r = p[6];
    const Vec axis = B - A;
    const double L = len(axis);
    const Vec dir = axis / L;
    const Vec rel = x - A;
    const double s = dot(rel, dir);
    const double sc = fmax(0.0, fmin(s, L));
    const Vec on_axis = A + sc * dir;
    const bool in_radius = len(cross(rel, dir)) <= r;
    const bool in_length = s >= 0.0 && s <= L;
    const bool near_a = s < 0.5 * L;
    if (in_radius && in_length) {
        const Vec radial = x - on_axis;
        const double rs = len(radial) - r;
        const double as = near_a ? -s : s - L;
        if (fabs(rs) <= fabs(as)) {
            f = rs;
            g = unit(radial);
        } else {
            f = as;
            g = near_a ? -axis : axis;
        }
    } else if (!in_radius && in_length) {
        const Vec radial = x - on_axis;
        f = len(radial) - r;
        g = unit(radial);
    } else if (!in_radius && !in_length) {
        const Vec rim = on_axis + unit(rel - s * dir) * r;
        f = len(x - rim);
        g = unit(x - rim);
    } else {
        f = s < 0.0 ? -s : s - L;
        g = s < 0.0 ? -axis : axis;
    }
}

__device__ __forceinline__ double grid_value(double f, Vec g, double h)
{
    const double gn = len(g);
    if (gn > 1e-12) return f / gn;
    return (f <= 0.0 ? -1.0 : 1.0) * 0.5 * h;
}

__device__ __forceinline__ Vec node_point(double3 o, double h, long long id, int3 n)
{
    const int i = (int)(id % n.x);
    const int j = (int)((id / n.x) % n.y);
    const int k = (int)(id / ((long long)n.x * n.y));
    return mk(o.x + double(i) * h, o.y + double(j) * h, o.z + double(k) * h);
}

__global__ void k_levelset_analytic(Shape s, double3 o, double h, int3 n, long long total, double* __restrict__ out)
{
    for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < total;
         id += (long long)gridDim.x * blockDim.x) {
        const Vec x = node_point(o, h, id, n);
        double f = 0.0;
        Vec g = mk(0.0, 0.0, 0.0);
        switch (s.kind) {
        case FUNDEM_SHAPE_SUPERELLIPSOID: eval_superellipsoid(s.p, x, f, g); break;
        case FUNDEM_SHAPE_SPHERE: eval_sphere(s.p, x, f, g); break;
        case FUNDEM_SHAPE_BOX: eval_box(s.p, x, f, g); break;
        default: eval_cylinder(s.p, x, f, g); break;
        }
        if (s.flip) { f = -f; g = -g; }
        out[id] = grid_value(f, g, h);
    }
}

// closest point of triangle abc to p: the Voronoi-region walk of Ericson,
// "Real-Time Collision Detection" (2005), section 5.1.5
__device__ __forceinline__ Vec closest_on_triangle(Vec p, Vec a, Vec b, Vec c)
{
    const Vec ab = b - a, ac = c - a, ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return a;
    const Vec bp = p - b;
    const double d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0 && d4 <= d3) return b;
    const double vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return a + (d1 / (d1 - d3)) * ab;
    const Vec cp = p - c;
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return c;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return a + (d2 / (d2 - d6)) * ac;
    const double va = d3 * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0)
        return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b);
    const double inv = 1.0 / (va + vb + vc);
    return a + ab * (vb * inv) + ac * (vc * inv);
}

// signed solid angle of triangle abc seen from p (Van Oosterom and Strackee, 1983)
__device__ __forceinline__ double solid_angle(Vec p, Vec a, Vec b, Vec c)
{
    const Vec r0 = a - p, r1 = b - p, r2 = c - p;
    const double l0 = len(r0), l1 = len(r1), l2 = len(r2);
    if (l0 < 1e-30 || l1 < 1e-30 || l2 < 1e-30) return 0.0;
    const double num = dot(r0, cross(r1, r2));
    const double den = l0 * l1 * l2 + dot(r0, r1) * l2 + dot(r1, r2) * l0 + dot(r2, r0) * l1;
    return 2.0 * atan2(num, den);
}

constexpr int MESH_BLOCK = 128;

// one thread per grid node; the triangles stream through shared memory in
// tiles of MESH_BLOCK, every thread of the block reading the same triangle
// (a broadcast).  The solid angles are summed in triangle order.
__global__ void __launch_bounds__(MESH_BLOCK) k_levelset_mesh(const double* __restrict__ tri, int ntri, int flip,
                                                              double3 o, double h, int3 n, long long total,
                                                              double* __restrict__ out)
{
    __shared__ double s_tri[MESH_BLOCK * 9];
    const long long id = blockIdx.x * (long long)MESH_BLOCK + threadIdx.x;
    const bool live = id < total;
    const Vec x = live ? node_point(o, h, id, n) : mk(0.0, 0.0, 0.0);
    double best = DBL_MAX;
    Vec near = x;
    double wsum = 0.0;
    for (int t0 = 0; t0 < ntri; t0 += MESH_BLOCK) {
        const int nt = min(MESH_BLOCK, ntri - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < nt * 9; k += MESH_BLOCK) s_tri[k] = tri[(long long)t0 * 9 + k];
        __syncthreads();
        if (!live) continue;
        for (int t = 0; t < nt; ++t) {
            const double* T = s_tri + t * 9;
            const Vec a = mk(T[0], T[1], T[2]), b = mk(T[3], T[4], T[5]), c = mk(T[6], T[7], T[8]);
            const Vec q = closest_on_triangle(x, a, b, c);
            const Vec dq = x - q;
            const double d2 = dot(dq, dq);
            if (d2 < best) {
                best = d2;
                near = q;
            }
            wsum += solid_angle(x, a, b, c);
        }
    }
    if (!live) return;
    const double d = len(x - near);
    const bool inside = fabs(wsum / (4.0 * 3.14159265358979323846)) > 0.5;
    double f = inside ? -d : d;
    Vec g = mk(0.0, 0.0, 0.0);
    if (d > 1e-30) {
        const Vec u = (x - near) / d;
        g = inside ? -u : u;
    }
    if (flip) { f = -f; g = -g; }
    out[id] = grid_value(f, g, h);
}

}  // namespace

extern "C" int fundem_levelset_grid(int device, void* stream, const fundem_shape* shape, const double origin[3],
                                    double spacing, const int size[3], double* sdf)
{
    if (!shape || !origin || !size || !sdf || !(spacing > 0.0)) return FUNDEM_ERR_ARG;
    if (size[0] <= 0 || size[1] <= 0 || size[2] <= 0) return FUNDEM_ERR_ARG;
    const long long total = (long long)size[0] * size[1] * size[2];
    if (total > (1LL << 31)) return FUNDEM_ERR_ARG;
    const int kind = shape->kind;
    if (kind < FUNDEM_SHAPE_SUPERELLIPSOID || kind > FUNDEM_SHAPE_MESH) return FUNDEM_ERR_ARG;
    const double* p = shape->param;
    switch (kind) {
    case FUNDEM_SHAPE_SUPERELLIPSOID:
        if (!(p[0] > 0.0 && p[1] > 0.0 && p[2] > 0.0 && p[3] > 0.0 && p[4] > 0.0)) return FUNDEM_ERR_ARG;
        break;
    case FUNDEM_SHAPE_SPHERE:
        if (!(p[0] > 0.0)) return FUNDEM_ERR_ARG;
        break;
    case FUNDEM_SHAPE_BOX:
        if (!(p[0] > 0.0 && p[1] > 0.0 && p[2] > 0.0)) return FUNDEM_ERR_ARG;
        break;
    case FUNDEM_SHAPE_CYLINDER: {
        const double dx = p[3] - p[0], dy = p[4] - p[1], dz = p[5] - p[2];
        if (!(p[6] > 0.0) || !(std::sqrt(dx * dx + dy * dy + dz * dz) > 1e-30)) return FUNDEM_ERR_ARG;
        break;
    }
    default: {
        const int nv = shape->n_vertices, nt = shape->n_triangles;
        if (nv <= 0 || nt <= 0 || !shape->vertices || !shape->triangles) return FUNDEM_ERR_ARG;
        for (int t = 0; t < nt; ++t) {
            const int* T = shape->triangles + 3 * t;
            for (int k = 0; k < 3; ++k)
                if (T[k] < 0 || T[k] >= nv) return FUNDEM_ERR_ARG;
            if (T[0] == T[1] || T[1] == T[2] || T[2] == T[0]) return FUNDEM_ERR_ARG;
        }
    }
    }

    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return FUNDEM_ERR_CUDA;
    if (device >= 0 && device != prev && cudaSetDevice(device) != cudaSuccess) return FUNDEM_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    const double3 o = make_double3(origin[0], origin[1], origin[2]);
    const int3 n = make_int3(size[0], size[1], size[2]);
    double* d_out = nullptr;
    double* d_tri = nullptr;
    int status = FUNDEM_OK;
    cudaError_t e = cudaMallocAsync((void**)&d_out, total * sizeof(double), s);
    if (e == cudaSuccess && kind == FUNDEM_SHAPE_MESH) {
        // triangle corners gathered on the host: 9 doubles per triangle
        const int nt = shape->n_triangles;
        double* h_tri = new double[(size_t)nt * 9];
        for (int t = 0; t < nt; ++t)
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) h_tri[t * 9 + k * 3 + c] = shape->vertices[3 * shape->triangles[3 * t + k] + c];
        e = cudaMallocAsync((void**)&d_tri, (size_t)nt * 9 * sizeof(double), s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_tri, h_tri, (size_t)nt * 9 * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        delete[] h_tri;
    }
    if (e == cudaSuccess) {
        if (kind == FUNDEM_SHAPE_MESH) {
            const long long blocks = (total + MESH_BLOCK - 1) / MESH_BLOCK;
            k_levelset_mesh<<<(unsigned)blocks, MESH_BLOCK, 0, s>>>(d_tri, shape->n_triangles, shape->positive_inside != 0,
                                                                    o, spacing, n, total, d_out);
        } else {
            Shape sh;
            sh.kind = kind;
            sh.flip = shape->positive_inside != 0;
            for (int k = 0; k < 8; ++k) sh.p[k] = p[k];
            int sms = 148;
            int dev = 0;
            if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            const long long want = (total + 255) / 256;
            const long long cap = (long long)sms * 16;
            k_levelset_analytic<<<(unsigned)(want < cap ? want : cap), 256, 0, s>>>(sh, o, spacing, n, total, d_out);
        }
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(sdf, d_out, total * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (d_out) cudaFreeAsync(d_out, s);
    if (d_tri) cudaFreeAsync(d_tri, s);
    const cudaError_t e2 = cudaStreamSynchronize(s);
    if (e != cudaSuccess || e2 != cudaSuccess) status = FUNDEM_ERR_CUDA;
    if (device >= 0 && device != prev) cudaSetDevice(prev);
    return status;
}
