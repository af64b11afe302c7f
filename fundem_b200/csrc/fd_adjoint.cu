// fd_adjoint.cu -- reverse sweep of the timestep for translating bodies.
//
// The forward step (LSSolver.h:1033-1107 with the contact law of
// contactKernel.cuh:4-77 and the bond law of contactKernel.cuh:138-199) is
//   v_h     = v_n + (F_n / m + g) dt / 2
//   x_{n+1} = x_n + v_h dt
//   (F_{n+1}, S_{n+1}) = Phi(x_{n+1}, v_h, S_n; kn, ks, damping ratio, mu)
//   v_{n+1} = v_h + (F_{n+1} / m + g) dt / 2
// with S the tangential springs.  Its reverse, given the adjoints of x_{n+1},
// v_{n+1}, F_{n+1} (from the next step's first half-kick) and S_{n+1}:
//   Fbar_{n+1} += vbar_{n+1} dt / (2 m)
//   [Phi^T]  xbar_{n+1}, vbar_h, Sbar_n, parameter adjoints
//   vbar_h  += vbar_{n+1} + xbar_{n+1} dt
//   xbar_n   = xbar_{n+1};  vbar_n = vbar_h;  Fbar_n = vbar_h dt / (2 m)
// Contact topology is frozen at each step (replayed from the forward
// record), including the stick/slip branch of each contact and bond
// breakage.  Orientations do not change (zero inverse inertia), so only
// translations are differentiated.
//
// Phi^T is applied contact by contact: the local Jacobian of (force, new
// spring) with respect to (node position relative to the partner, relative
// velocity, previous spring, kn, ks, damping ratio, mu) comes from
// forward-mode dual numbers evaluated along the recorded state; the
// transposed products are added to the particles with atomics.
#include <cuda_runtime.h>

#include "fd_adjoint.cuh"

namespace fd {
namespace {

constexpr int ADJ_TPB = 128;

// ---------------------------------------------------------------------------
// forward-mode dual numbers with N derivative directions over the scalar type
// T (double for the FP64 step, float for the mixed-precision one); scalar
// operands are doubles converted to T
// ---------------------------------------------------------------------------
template <int N, typename T = double>
struct Dual {
    T v;
    T d[N];
    __device__ Dual() {}
    __device__ Dual(double x) : v((T)x)
    {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = T(0);
    }
    __device__ static Dual var(double x, int i)
    {
        Dual r(x);
        r.d[i] = T(1);
        return r;
    }
};
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator+(const Dual<N, T>& a, const Dual<N, T>& b)
{
    Dual<N, T> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator-(const Dual<N, T>& a, const Dual<N, T>& b)
{
    Dual<N, T> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator-(const Dual<N, T>& a)
{
    Dual<N, T> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator*(const Dual<N, T>& a, const Dual<N, T>& b)
{
    Dual<N, T> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator*(const Dual<N, T>& a, double sd)
{
    const T s = (T)sd;
    Dual<N, T> r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator*(double s, const Dual<N, T>& a)
{
    return a * s;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator/(const Dual<N, T>& a, const Dual<N, T>& b)
{
    Dual<N, T> r;
    const T ib = T(1) / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator/(double a, const Dual<N, T>& b)
{
    return Dual<N, T>(a) / b;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator+(const Dual<N, T>& a, double s)
{
    Dual<N, T> r = a;
    r.v += (T)s;
    return r;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> operator-(double s, const Dual<N, T>& a)
{
    return (-a) + s;
}
template <int N, typename T> __device__ __forceinline__ Dual<N, T> dsqrt(const Dual<N, T>& a)
{
    Dual<N, T> r;
    r.v = sqrt(a.v);
    const T g = r.v > T(0) ? T(0.5) / r.v : T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * g;
    return r;
}

template <typename T> struct V3 {
    T x, y, z;
};
template <typename T> __device__ __forceinline__ V3<T> operator+(const V3<T>& a, const V3<T>& b)
{
    return V3<T>{a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename T> __device__ __forceinline__ V3<T> operator-(const V3<T>& a, const V3<T>& b)
{
    return V3<T>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename T> __device__ __forceinline__ V3<T> operator-(const V3<T>& a) { return V3<T>{-a.x, -a.y, -a.z}; }
template <typename T> __device__ __forceinline__ V3<T> scale(const T& s, const V3<T>& a)
{
    return V3<T>{s * a.x, s * a.y, s * a.z};
}
template <typename T> __device__ __forceinline__ T vdot(const V3<T>& a, const V3<T>& b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

// ---------------------------------------------------------------------------
// one contact: (force on A, new spring) from (node relative to the partner,
// relative velocity, previous spring, kn, ks, damping ratio, mu).  The same
// expressions as the forward step; the cell of the SDF lookup is the one the
// recorded state falls in.
// ---------------------------------------------------------------------------
constexpr int NDIR = 13;  // rel 3, vc 3, sprev 3, kn, ks, diss, mu

// T is the scalar type of the duals (the launches use double).  The cell and
// the position inside it come from the recorded double-precision node
// offset, as in the forward kernels.
template <typename T>
__device__ bool contact_dual(const V3<Dual<NDIR, T>>& rel, const double3 reld, V3<Dual<NDIR, T>> vc,
                             const V3<Dual<NDIR, T>>& sprev, const Dual<NDIR, T>& kn, const Dual<NDIR, T>& ks,
                             const Dual<NDIR, T>& diss, const Dual<NDIR, T>& mu, double m, double dt,
                             const FdGeo& GB, const T* sdf, const double qB[4], const double3 wA, const double3 wB,
                             V3<Dual<NDIR, T>>& F, V3<Dual<NDIR, T>>& snew)
{
    using D13 = Dual<NDIR, T>;
    // rotation matrix of the partner (rows: world <- body)
    const double q0 = qB[0], q1 = qB[1], q2 = qB[2], q3 = qB[3];
    const double R[9] = {1.0 - 2.0 * (q2 * q2 + q3 * q3), 2.0 * (q1 * q2 - q0 * q3), 2.0 * (q1 * q3 + q0 * q2),
                         2.0 * (q1 * q2 + q0 * q3), 1.0 - 2.0 * (q1 * q1 + q3 * q3), 2.0 * (q2 * q3 - q0 * q1),
                         2.0 * (q1 * q3 - q0 * q2), 2.0 * (q2 * q3 + q0 * q1), 1.0 - 2.0 * (q1 * q1 + q2 * q2)};
    // node in the partner's body frame, then grid coordinates
    const D13 lx = rel.x * R[0] + rel.y * R[3] + rel.z * R[6];
    const D13 ly = rel.x * R[1] + rel.y * R[4] + rel.z * R[7];
    const D13 lz = rel.x * R[2] + rel.y * R[5] + rel.z * R[8];
    const D13 gx = (lx + (-GB.origin.x)) * GB.inv_spacing;
    const D13 gy = (ly + (-GB.origin.y)) * GB.inv_spacing;
    const D13 gz = (lz + (-GB.origin.z)) * GB.inv_spacing;
    const double gxd = (reld.x * R[0] + reld.y * R[3] + reld.z * R[6] + (-GB.origin.x)) * GB.inv_spacing;
    const double gyd = (reld.x * R[1] + reld.y * R[4] + reld.z * R[7] + (-GB.origin.y)) * GB.inv_spacing;
    const double gzd = (reld.x * R[2] + reld.y * R[5] + reld.z * R[8] + (-GB.origin.z)) * GB.inv_spacing;
    const int i0 = (int)floor(gxd), j0 = (int)floor(gyd), k0 = (int)floor(gzd);
    if (i0 < 0 || j0 < 0 || k0 < 0 || i0 >= GB.size.x - 1 || j0 >= GB.size.y - 1 || k0 >= GB.size.z - 1)
        return false;
    D13 fx = gx, fy = gy, fz = gz;
    fx.v = (T)(gxd - (double)i0);
    fy.v = (T)(gyd - (double)j0);
    fz.v = (T)(gzd - (double)k0);
    const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
    const T* S = sdf + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
    const double p[8] = {S[0], S[1], S[sx], S[sx + 1], S[sxy], S[sxy + 1], S[sxy + sx], S[sxy + sx + 1]};
    const D13 ux = 1.0 - fx, uy = 1.0 - fy, uz = 1.0 - fz;
    const D13 phi = ((p[0] * ux + p[1] * fx) * uy + (p[2] * ux + p[3] * fx) * fy) * uz +
                    ((p[4] * ux + p[5] * fx) * uy + (p[6] * ux + p[7] * fx) * fy) * fz;
    const D13 ov = -phi;
    // gradient with the truncated x weight (LSParticleContactDetectionKernel.cuh:34)
    const D13 ggx = (p[1] - p[0]) * (uy * uz) + (p[3] - p[2]) * (fy * uz) + (p[5] - p[4]) * (uy * fz) +
                    (p[7] - p[6]) * (fy * fz);
    const D13 ggy = (p[2] - p[0]) * uz + (p[6] - p[4]) * fz;
    const D13 ggz = (p[4] - p[0]) * uy + (p[6] - p[2]) * fy;
    const V3<D13> nw{ggx * R[0] + ggy * R[1] + ggz * R[2], ggx * R[3] + ggy * R[4] + ggz * R[5],
                     ggx * R[6] + ggy * R[7] + ggz * R[8]};
    const D13 nl = dsqrt(vdot(nw, nw));
    if (!(nl.v > 0.0)) return false;
    const V3<D13> n = V3<D13>{nw.x / nl, nw.y / nl, nw.z / nl};
    // The contact point is the node moved by n overlap / 2
    // (LSParticleContactDetectionKernel.cu:268-281), so with turning bodies
    // the velocity wA x (c - rA) - wB x (c - rB) moves with the point:
    // its derivative adds wA x dh - wB x (drel + dh), h = n overlap / 2.
    if (wA.x != 0.0 || wA.y != 0.0 || wA.z != 0.0 || wB.x != 0.0 || wB.y != 0.0 || wB.z != 0.0) {
        const D13 half = ov * 0.5;
        V3<D13> dh = scale(half, n), dr = rel;
        dh.x.v = dh.y.v = dh.z.v = 0.0;  // derivative parts only
        dr.x.v = dr.y.v = dr.z.v = 0.0;
        const V3<D13> drh = dr + dh;
        vc.x = vc.x + (dh.z * wA.y - dh.y * wA.z) - (drh.z * wB.y - drh.y * wB.z);
        vc.y = vc.y + (dh.x * wA.z - dh.z * wA.x) - (drh.x * wB.z - drh.z * wB.x);
        vc.z = vc.z + (dh.y * wA.x - dh.x * wA.y) - (drh.y * wB.x - drh.x * wB.y);
    }
    F = V3<D13>{D13(0.0), D13(0.0), D13(0.0)};
    snew = F;
    if (!(ov.v > 0.0)) return true;
    const D13 cn = 2.0 * diss * dsqrt(m * kn);
    const D13 vcn = vdot(vc, n);
    const V3<D13> vn = scale(vcn, n);
    const V3<D13> fn = scale(kn * ov, n) - scale(cn, vn);
    const D13 cs = 2.0 * diss * dsqrt(m * ks);
    const V3<D13> vs = vc - vn;
    V3<D13> sp{D13(0.0), D13(0.0), D13(0.0)};
    if (mu.v > 0.0 && ks.v > 0.0) {
        V3<D13> p1 = sprev - scale(vdot(sprev, n), n);
        const D13 ap1 = dsqrt(vdot(p1, p1));
        if (ap1.v > 1.0e-20) p1 = scale(dsqrt(vdot(sprev, sprev)) / ap1, p1);
        sp = p1 + scale(D13(dt), vs);
        V3<D13> sf = scale(-ks, sp) - scale(cs, vs);
        const D13 asf = dsqrt(vdot(sf, sf));
        const D13 afn = dsqrt(vdot(fn, fn));
        if (asf.v > 1.0e-20 && asf.v > mu.v * afn.v) {
            sf = scale(mu * afn / asf, sf);
            const V3<D13> t = sf + scale(cs, vs);
            const D13 iks = D13(-1.0) / ks;
            sp = scale(iks, t);
        }
    }
    snew = sp;
    F = fn + (scale(-ks, sp) - scale(cs, vs));
    return true;
}

__device__ __forceinline__ void atomic_add3(double* a, double x, double y, double z)
{
    atomicAdd(a, x);
    atomicAdd(a + 1, y);
    atomicAdd(a + 2, z);
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// Fbar = Fext + vbar dt / (2 m); vhbar = vbar
__global__ void k_adj_force(AdjParticles a, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double im = a.G.geo[a.geo[i]].inv_mass;
    for (int c = 0; c < 3; ++c) {
        a.Fb[3 * i + c] = a.Feb[3 * i + c] + 0.5 * dt * im * a.vb[3 * i + c];
        a.vhb[3 * i + c] = a.vb[3 * i + c];
    }
}

// the contacts of one list at one step
template <typename T>
__global__ void __launch_bounds__(ADJ_TPB) k_adj_contact(AdjParticles a, AdjContactArgs c)
{
    using D13 = Dual<NDIR, T>;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int nslots = min(*c.nslots, c.rec.cap);
    if (s >= nslots || !c.rec.hit[s]) return;
    const AdjRec& R = c.rec;
    const int A = R.A[s], Bp = R.Bp[s];
    const int mi = a.mat[A], mj = R.matB[s];
    const bool wall = Bp < 0;
    // effective parameters, as the forward contact law forms them
    const double kni = c.M.kn[mi], ksi = c.M.ks[mi], mui = c.M.mu[mi], ei = c.M.e[mi];
    const double knj = wall ? kni : c.M.kn[mj], ksj = wall ? ksi : c.M.ks[mj];
    const double muj = wall ? c.MW.mu[mj] : c.M.mu[mj], ej = wall ? c.MW.e[mj] : c.M.e[mj];
    double kn, ks, dk_i, dk_j, ds_i, ds_j;
    if (wall) {
        kn = kni; ks = ksi; dk_i = 1.0; dk_j = 0.0; ds_i = 1.0; ds_j = 0.0;
    } else {
        kn = (kni > 0. && knj > 0.) ? kni * knj / (kni + knj) : 0.;
        ks = (ksi > 0. && ksj > 0.) ? ksi * ksj / (ksi + ksj) : 0.;
        dk_i = (kni > 0. && knj > 0.) ? knj * knj / ((kni + knj) * (kni + knj)) : 0.;
        dk_j = (kni > 0. && knj > 0.) ? kni * kni / ((kni + knj) * (kni + knj)) : 0.;
        ds_i = (ksi > 0. && ksj > 0.) ? ksj * ksj / ((ksi + ksj) * (ksi + ksj)) : 0.;
        ds_j = (ksi > 0. && ksj > 0.) ? ksi * ksi / ((ksi + ksj) * (ksi + ksj)) : 0.;
    }
    const double mu = fmin(mui, muj);
    double res = fmin(ei, ej);
    const double lr = log(res);
    const double diss = -lr / sqrt(lr * lr + 3.14159265358979323846 * 3.14159265358979323846);
    const double invMi = a.G.geo[a.geo[A]].inv_mass;
    const double invMj = wall ? 0.0 : a.G.geo[a.geo[Bp]].inv_mass;
    double m = 0.0;
    if (invMi > 0. || invMj > 0.) m = 1.0 / (invMi + invMj);
    // duals
    V3<D13> rel{D13::var(R.rel[3 * s], 0), D13::var(R.rel[3 * s + 1], 1), D13::var(R.rel[3 * s + 2], 2)};
    V3<D13> vc{D13::var(R.vc[3 * s], 3), D13::var(R.vc[3 * s + 1], 4), D13::var(R.vc[3 * s + 2], 5)};
    V3<D13> sprev{D13::var(R.sprev[3 * s], 6), D13::var(R.sprev[3 * s + 1], 7), D13::var(R.sprev[3 * s + 2], 8)};
    const D13 dkn = D13::var(kn, 9), dks = D13::var(ks, 10), ddiss = D13::var(diss, 11), dmu = D13::var(mu, 12);
    const FdGeo& GB = wall ? c.GW.geo[R.geoB[s]] : a.G.geo[R.geoB[s]];
    const T* sdf;
    if constexpr (sizeof(T) == sizeof(double)) sdf = wall ? c.GW.sdf : a.G.sdf;
    else sdf = wall ? c.GW.sdf32 : a.G.sdf32;
    const double qB[4] = {R.qB[4 * s], R.qB[4 * s + 1], R.qB[4 * s + 2], R.qB[4 * s + 3]};
    const double3 wA = a.angvel[A], wB = wall ? c.wall_angvel[R.B[s]] : a.angvel[Bp];
    V3<D13> F, snew;
    const double3 reld = make_double3(R.rel[3 * s], R.rel[3 * s + 1], R.rel[3 * s + 2]);
    if (!contact_dual<T>(rel, reld, vc, sprev, dkn, dks, ddiss, dmu, m, c.dt, GB, sdf, qB, wA, wB, F, snew))
        return;
    // A contact with a particle's own periodic image has no reaction
    // (contactKernel.cu:207-291), and its node offset and relative velocity
    // do not move with the particle.
    const bool react = !wall && Bp != A;
    // output adjoints: force on A (and its reaction), new spring
    double fb[3] = {a.Fb[3 * A], a.Fb[3 * A + 1], a.Fb[3 * A + 2]};
    if (react) {
        fb[0] -= a.Fb[3 * Bp];
        fb[1] -= a.Fb[3 * Bp + 1];
        fb[2] -= a.Fb[3 * Bp + 2];
    }
    const double sb[3] = {c.Sb_cur[3 * s], c.Sb_cur[3 * s + 1], c.Sb_cur[3 * s + 2]};
    double g[NDIR];
#pragma unroll
    for (int k = 0; k < NDIR; ++k)
        g[k] = fb[0] * (double)F.x.d[k] + fb[1] * (double)F.y.d[k] + fb[2] * (double)F.z.d[k] +
               sb[0] * (double)snew.x.d[k] + sb[1] * (double)snew.y.d[k] + sb[2] * (double)snew.z.d[k];
    // positions (the node offset is fixed: d rel / d x_A = I, d rel / d x_B = -I)
    if (wall || react) {
        atomic_add3(a.xb + 3 * A, g[0], g[1], g[2]);
        atomic_add3(a.vhb + 3 * A, g[3], g[4], g[5]);
    }
    if (react) {
        atomic_add3(a.xb + 3 * Bp, -g[0], -g[1], -g[2]);
        atomic_add3(a.vhb + 3 * Bp, -g[3], -g[4], -g[5]);
    }
    const int h = R.hist[s];
    if (h >= 0 && h < c.sb_prev_cap) atomic_add3(c.Sb_prev + 3 * h, g[6], g[7], g[8]);
    // parameters, per material: kn, ks, damping ratio, mu
    atomicAdd(&a.pgrad[4 * mi + 0], g[9] * dk_i);
    atomicAdd(&a.pgrad[4 * mi + 1], g[10] * ds_i);
    if (!wall) {
        atomicAdd(&a.pgrad[4 * mj + 0], g[9] * dk_j);
        atomicAdd(&a.pgrad[4 * mj + 1], g[10] * ds_j);
    }
    if (ei <= ej) atomicAdd(&a.pgrad[4 * mi + 2], g[11]);
    else if (!wall) atomicAdd(&a.pgrad[4 * mj + 2], g[11]);
    if (mui <= muj) atomicAdd(&a.pgrad[4 * mi + 3], g[12]);
    else if (!wall) atomicAdd(&a.pgrad[4 * mj + 3], g[12]);
}

// the bonds at one step: force F(r) on the master, -F on the slave, with the
// body frames fixed (no rotation)
template <typename T>
__global__ void k_adj_bond(AdjParticles a, AdjBondArgs b)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= b.n || !b.active[k]) return;
    using D3 = Dual<3, T>;
    const int i = b.master[k], j = b.slave[k];
    const V3<D3> r{D3::var(b.rij[3 * k], 0), D3::var(b.rij[3 * k + 1], 1), D3::var(b.rij[3 * k + 2], 2)};
    const D3 D = dsqrt(vdot(r, r));
    if (!(D.v > 1.0e-20)) return;
    const double B1 = b.B[4 * k], B2 = b.B[4 * k + 1], D0 = b.L0[k];
    const V3<D3> e{-(r.x / D), -(r.y / D), -(r.z / D)};
    const V3<D3> dnv{D3(b.dn[3 * k]), D3(b.dn[3 * k + 1]), D3(b.dn[3 * k + 2])};
    const D3 dne = vdot(dnv, e);
    const D3 c1 = B1 * (D + (-D0));
    const D3 c2 = B2 / (2.0 * D);
    const V3<D3> F = scale(c1, e) + scale(c2, dnv - scale(dne, e));
    const double fb[3] = {a.Fb[3 * i] - a.Fb[3 * j], a.Fb[3 * i + 1] - a.Fb[3 * j + 1], a.Fb[3 * i + 2] - a.Fb[3 * j + 2]};
    double g[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) g[t] = fb[0] * (double)F.x.d[t] + fb[1] * (double)F.y.d[t] + fb[2] * (double)F.z.d[t];
    atomic_add3(a.xb + 3 * i, g[0], g[1], g[2]);
    atomic_add3(a.xb + 3 * j, -g[0], -g[1], -g[2]);
}

// vhbar += xbar dt; vbar = vhbar; Fext = vhbar dt / (2 m)
__global__ void k_adj_particle(AdjParticles a, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double im = a.G.geo[a.geo[i]].inv_mass;
    for (int c = 0; c < 3; ++c) {
        const double vh = a.vhb[3 * i + c] + dt * a.xb[3 * i + c];
        a.vb[3 * i + c] = vh;
        a.Feb[3 * i + c] = 0.5 * dt * im * vh;
    }
}

}  // namespace

void adj_force(const AdjParticles& a, double dt, cudaStream_t s)
{
    if (a.n > 0) { k_adj_force<<<(a.n + 255) / 256, 256, 0, s>>>(a, dt); count_launch(); }
}
// Both precisions of the step are swept with double-precision Jacobians: the
// single-precision evaluation of a contact's Jacobian gave non-finite
// gradients on a 4,096-particle pour, where contacts separate from the walls.
void adj_contacts(const AdjParticles& a, const AdjContactArgs& c, cudaStream_t s)
{
    if (c.rec.cap > 0) { k_adj_contact<double><<<(c.rec.cap + ADJ_TPB - 1) / ADJ_TPB, ADJ_TPB, 0, s>>>(a, c); count_launch(); }
}
void adj_bonds(const AdjParticles& a, const AdjBondArgs& b, cudaStream_t s)
{
    if (b.n > 0) { k_adj_bond<double><<<(b.n + 255) / 256, 256, 0, s>>>(a, b); count_launch(); }
}
void adj_particles(const AdjParticles& a, double dt, cudaStream_t s)
{
    if (a.n > 0) { k_adj_particle<<<(a.n + 255) / 256, 256, 0, s>>>(a, dt); count_launch(); }
}

}  // namespace fd
