// fd_adjoint.cu -- reverse sweep of the timestep.
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
// Turning bodies add (particleIntegrationKernel.cu:3-48, myQua.h:77-93)
//   w_h     = w_n + W(q_n, w_n, T_n) dt / 2,  W = I_w^-1 (T - w x I_w w),
//             I_w = R(q) I R(q)^T
//   q_{n+1} = normalise(q_n + (0, w_h dt / 2) (x) q_n)
//   (F, T_{n+1}, S_{n+1}) = Phi(x, q_{n+1}, v_h, w_h, S_n; ...)
//   w_{n+1} = w_h + W(q_{n+1}, w_h, T_{n+1}) dt / 2
// reversed with forward-mode duals over (q, w) per particle, and the torques'
// lever arms and the partner's orientation in Phi's Jacobian.
// Contact topology is frozen at each step (replayed from the forward
// record), including the stick/slip branch of each contact and bond
// breakage.
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

// ---------------------------------------------------------------------------
// turning bodies.  The forward step's rotational parts, written over dual
// numbers with the forward kernels' expressions:
//   rot(q, v)   = v + t q0 + qv x t, t = 2 qv x v          (myQua.h:104-114)
//   rrot(v, q)  = rot with qv negated                       (myQua.h:120-128)
//   W(q, w, T)  = Iw^-1 (T - w x (Iw w)), Iw = R I R^T      (particleIntegrationKernel.cu:3-32)
//   qint(q, w)  = normalize(q + (0, w dt / 2) (x) q)        (myQua.h:77-93)
// ---------------------------------------------------------------------------
template <typename D> __device__ __forceinline__ V3<D> vcross(const V3<D>& a, const V3<D>& b)
{
    return V3<D>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename D> __device__ __forceinline__ V3<D> qrot(const D q[4], const V3<D>& v, bool inverse)
{
    const V3<D> qv = inverse ? V3<D>{-q[1], -q[2], -q[3]} : V3<D>{q[1], q[2], q[3]};
    const V3<D> c = vcross(qv, v);
    const V3<D> t{c.x * 2.0, c.y * 2.0, c.z * 2.0};
    const V3<D> u = vcross(qv, t);
    return V3<D>{v.x + t.x * q[0] + u.x, v.y + t.y * q[0] + u.y, v.z + t.z * q[0] + u.z};
}
// symmetric tensor R(q) I R(q)^T as fd_rot_tensor forms it: xx yy zz xy xz yz
template <typename D> __device__ __forceinline__ void rot_tensor_d(const D q[4], const fd_sym& I, D r[6])
{
    const D q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
    const D q11 = 2.0 * q1 * q1, q22 = 2.0 * q2 * q2, q33 = 2.0 * q3 * q3;
    const D a = 1.0 - q22 - q33, b = 2.0 * (q1 * q2 - q0 * q3), c = 2.0 * (q1 * q3 + q0 * q2);
    const D d = 2.0 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2.0 * (q2 * q3 - q0 * q1);
    const D g = 2.0 * (q1 * q3 - q0 * q2), h = 2.0 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
    const D r0x = a * I.xx + b * I.xy + c * I.xz, r0y = a * I.xy + b * I.yy + c * I.yz, r0z = a * I.xz + b * I.yz + c * I.zz;
    const D r1x = d * I.xx + e * I.xy + f * I.xz, r1y = d * I.xy + e * I.yy + f * I.yz, r1z = d * I.xz + e * I.yz + f * I.zz;
    const D r2x = g * I.xx + h * I.xy + i * I.xz, r2y = g * I.xy + h * I.yy + i * I.yz, r2z = g * I.xz + h * I.yz + i * I.zz;
    r[0] = r0x * a + r0y * b + r0z * c;
    r[1] = r1x * d + r1y * e + r1z * f;
    r[2] = r2x * g + r2y * h + r2z * i;
    r[3] = r0x * d + r0y * e + r0z * f;
    r[4] = r0x * g + r0y * h + r0z * i;
    r[5] = r1x * g + r1y * h + r1z * i;
}
template <typename D> __device__ __forceinline__ V3<D> smv_d(const D m[6], const V3<D>& v)
{
    return V3<D>{m[0] * v.x + m[3] * v.y + m[4] * v.z, m[3] * v.x + m[1] * v.y + m[5] * v.z,
                 m[4] * v.x + m[5] * v.y + m[2] * v.z};
}
// the angular acceleration of the half kick
template <typename D>
__device__ __forceinline__ V3<D> w_accel(const D q[4], const V3<D>& w, const double3 T, const FdGeo& g)
{
    D Iw[6], Ii[6];
    rot_tensor_d(q, g.inertia, Iw);
    rot_tensor_d(q, g.inv_inertia, Ii);
    const V3<D> L = smv_d(Iw, w);
    const V3<D> c = vcross(w, L);
    const V3<D> r{D(T.x) - c.x, D(T.y) - c.y, D(T.z) - c.z};
    return smv_d(Ii, r);
}
template <typename D> __device__ __forceinline__ void qint_d(const D q[4], const V3<D>& w, double dt, D out[4])
{
    const V3<D> v{w.x * (0.5 * dt), w.y * (0.5 * dt), w.z * (0.5 * dt)};
    D s[4];
    s[0] = q[0] + (-(q[1] * v.x) - q[2] * v.y - q[3] * v.z);
    s[1] = q[1] + (q[0] * v.x + q[3] * v.y - q[2] * v.z);
    s[2] = q[2] + (-(q[3] * v.x) + q[0] * v.y + q[1] * v.z);
    s[3] = q[3] + (q[2] * v.x - q[1] * v.y + q[0] * v.z);
    const D l2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + s[3] * s[3];
    if (!(l2.v > 1.0e-20)) {
        for (int k = 0; k < 4; ++k) out[k] = s[k];
        return;
    }
    const D inv = 1.0 / dsqrt(l2);
    for (int k = 0; k < 4; ++k) out[k] = s[k] * inv;
}

// One contact between turning bodies: (force on A, torques on A and on the
// partner, new spring) from the node relative to the partner's centre
// (rel), the node relative to A's centre (arm), the partner's orientation,
// the velocity difference vA - vB, both angular velocities, the previous
// spring and the four parameters.  shiftA, shiftB: the periodic shifts of the
// force-side centres (the lever arms are measured from the wrapped centres).
template <int N>
__device__ bool contact_dual_rot(const V3<Dual<N>>& rel, const V3<Dual<N>>& arm, const Dual<N> qB[4],
                                 const V3<Dual<N>>& dv, const V3<Dual<N>>& wA, const V3<Dual<N>>& wB,
                                 const V3<Dual<N>>& sprev, const Dual<N>& kn, const Dual<N>& ks,
                                 const Dual<N>& diss, const Dual<N>& mu, const double3 reld, const double qBd[4],
                                 const double3 shiftA, const double3 shiftB, double m, double dt, const FdGeo& GB,
                                 const double* sdf, V3<Dual<N>>& F, V3<Dual<N>>& TA, V3<Dual<N>>& TB,
                                 V3<Dual<N>>& snew)
{
    using DN = Dual<N>;
    // the cell from the recorded double-precision state (frozen topology)
    const double q0 = qBd[0], q1 = qBd[1], q2 = qBd[2], q3 = qBd[3];
    const double R[9] = {1.0 - 2.0 * (q2 * q2 + q3 * q3), 2.0 * (q1 * q2 - q0 * q3), 2.0 * (q1 * q3 + q0 * q2),
                         2.0 * (q1 * q2 + q0 * q3), 1.0 - 2.0 * (q1 * q1 + q3 * q3), 2.0 * (q2 * q3 - q0 * q1),
                         2.0 * (q1 * q3 - q0 * q2), 2.0 * (q2 * q3 + q0 * q1), 1.0 - 2.0 * (q1 * q1 + q2 * q2)};
    const double gxd = (reld.x * R[0] + reld.y * R[3] + reld.z * R[6] + (-GB.origin.x)) * GB.inv_spacing;
    const double gyd = (reld.x * R[1] + reld.y * R[4] + reld.z * R[7] + (-GB.origin.y)) * GB.inv_spacing;
    const double gzd = (reld.x * R[2] + reld.y * R[5] + reld.z * R[8] + (-GB.origin.z)) * GB.inv_spacing;
    const int i0 = (int)floor(gxd), j0 = (int)floor(gyd), k0 = (int)floor(gzd);
    if (i0 < 0 || j0 < 0 || k0 < 0 || i0 >= GB.size.x - 1 || j0 >= GB.size.y - 1 || k0 >= GB.size.z - 1)
        return false;
    // the node in the partner's body frame, grid coordinates, fractions
    const V3<DN> lp = qrot(qB, rel, true);
    DN fx = (lp.x + (-GB.origin.x)) * GB.inv_spacing, fy = (lp.y + (-GB.origin.y)) * GB.inv_spacing,
       fz = (lp.z + (-GB.origin.z)) * GB.inv_spacing;
    fx.v = gxd - (double)i0;
    fy.v = gyd - (double)j0;
    fz.v = gzd - (double)k0;
    const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
    const double* S = sdf + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
    const double p[8] = {S[0], S[1], S[sx], S[sx + 1], S[sxy], S[sxy + 1], S[sxy + sx], S[sxy + sx + 1]};
    const DN ux = 1.0 - fx, uy = 1.0 - fy, uz = 1.0 - fz;
    const DN phi = ((p[0] * ux + p[1] * fx) * uy + (p[2] * ux + p[3] * fx) * fy) * uz +
                   ((p[4] * ux + p[5] * fx) * uy + (p[6] * ux + p[7] * fx) * fy) * fz;
    const DN ov = -phi;
    // gradient with the truncated x weight, turned to the world frame
    const V3<DN> gb{(p[1] - p[0]) * (uy * uz) + (p[3] - p[2]) * (fy * uz) + (p[5] - p[4]) * (uy * fz) +
                        (p[7] - p[6]) * (fy * fz),
                    (p[2] - p[0]) * uz + (p[6] - p[4]) * fz, (p[4] - p[0]) * uy + (p[6] - p[2]) * fy};
    const V3<DN> nw = qrot(qB, gb, false);
    const DN l2 = vdot(nw, nw);
    if (!(l2.v > 1.0e-20)) return false;
    const DN inv = 1.0 / dsqrt(l2);
    const V3<DN> n{nw.x * inv, nw.y * inv, nw.z * inv};
    // contact point: the node moved by n overlap / 2; lever arms from the
    // force-side centres
    const DN half = ov * 0.5;
    const V3<DN> h = scale(half, n);
    const V3<DN> rA{arm.x + h.x + (-shiftA.x), arm.y + h.y + (-shiftA.y), arm.z + h.z + (-shiftA.z)};
    const V3<DN> rB{rel.x + h.x + (-shiftB.x), rel.y + h.y + (-shiftB.y), rel.z + h.z + (-shiftB.z)};
    const V3<DN> vc = dv + vcross(wA, rA) - vcross(wB, rB);
    F = V3<DN>{DN(0.0), DN(0.0), DN(0.0)};
    snew = F;
    TA = F;
    TB = F;
    if (!(ov.v > 0.0)) return true;
    const DN cn = 2.0 * diss * dsqrt(m * kn);
    const DN vcn = vdot(vc, n);
    const V3<DN> vn = scale(vcn, n);
    const V3<DN> fn = scale(kn * ov, n) - scale(cn, vn);
    const DN cs = 2.0 * diss * dsqrt(m * ks);
    const V3<DN> vs = vc - vn;
    V3<DN> sp{DN(0.0), DN(0.0), DN(0.0)};
    if (mu.v > 0.0 && ks.v > 0.0) {
        V3<DN> p1 = sprev - scale(vdot(sprev, n), n);
        const DN ap1 = dsqrt(vdot(p1, p1));
        if (ap1.v > 1.0e-20) p1 = scale(dsqrt(vdot(sprev, sprev)) / ap1, p1);
        sp = p1 + scale(DN(dt), vs);
        V3<DN> sf = scale(-ks, sp) - scale(cs, vs);
        const DN asf = dsqrt(vdot(sf, sf));
        const DN afn = dsqrt(vdot(fn, fn));
        if (asf.v > 1.0e-20 && asf.v > mu.v * afn.v) {
            sf = scale(mu * afn / asf, sf);
            const V3<DN> t = sf + scale(cs, vs);
            const DN iks = DN(-1.0) / ks;
            sp = scale(iks, t);
        }
    }
    snew = sp;
    F = fn + (scale(-ks, sp) - scale(cs, vs));
    TA = vcross(rA, F);
    TB = vcross(rB, -F);
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
    const FdGeo& geo = a.G.geo[a.geo[i]];
    const double im = geo.inv_mass;
    for (int c = 0; c < 3; ++c) {
        a.Fb[3 * i + c] = a.Feb[3 * i + c] + 0.5 * dt * im * a.vb[3 * i + c];
        a.vhb[3 * i + c] = a.vb[3 * i + c];
    }
    if (!a.rot) return;
    // second half kick w' = wh + W(q', wh, T') dt / 2 (skipped for fixed bodies)
    const double h = 0.5 * dt;
    const double wb[3] = {a.wb[3 * i], a.wb[3 * i + 1], a.wb[3 * i + 2]};
    double Tb[3] = {a.Teb[3 * i], a.Teb[3 * i + 1], a.Teb[3 * i + 2]};
    double whb[3] = {wb[0], wb[1], wb[2]};
    if (im != 0.0) {
        using D7 = Dual<7>;
        const double* pc = a.pr_cur + (long long)ADJ_PREC * i;
        D7 q[4];
        for (int k = 0; k < 4; ++k) q[k] = D7::var(pc[k], k);
        const V3<D7> w{D7::var(pc[4], 4), D7::var(pc[5], 5), D7::var(pc[6], 6)};
        const double3 T = make_double3(pc[7], pc[8], pc[9]);
        const V3<D7> acc = w_accel(q, w, T, geo);
        for (int k = 0; k < 7; ++k) {
            const double g = h * (wb[0] * acc.x.d[k] + wb[1] * acc.y.d[k] + wb[2] * acc.z.d[k]);
            if (k < 4) a.qb[4 * i + k] += g;
            else whb[k - 4] += g;
        }
        // the torque enters linearly through the inverse inertia in the world frame
        double Ii[6];
        {
            const double qd[4] = {pc[0], pc[1], pc[2], pc[3]};
            rot_tensor_d(qd, geo.inv_inertia, Ii);
        }
        Tb[0] += h * (Ii[0] * wb[0] + Ii[3] * wb[1] + Ii[4] * wb[2]);
        Tb[1] += h * (Ii[3] * wb[0] + Ii[1] * wb[1] + Ii[5] * wb[2]);
        Tb[2] += h * (Ii[4] * wb[0] + Ii[5] * wb[1] + Ii[2] * wb[2]);
    }
    for (int c = 0; c < 3; ++c) {
        a.Tb[3 * i + c] = Tb[c];
        a.whb[3 * i + c] = whb[c];
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
    const FdGeo& geo = a.G.geo[a.geo[i]];
    const double im = geo.inv_mass;
    for (int c = 0; c < 3; ++c) {
        const double vh = a.vhb[3 * i + c] + dt * a.xb[3 * i + c];
        a.vb[3 * i + c] = vh;
        a.Feb[3 * i + c] = 0.5 * dt * im * vh;
    }
    if (!a.rot) return;
    using D7 = Dual<7>;
    const double* pp = a.pr_prev + (long long)ADJ_PREC * i;
    const double* pc = a.pr_cur + (long long)ADJ_PREC * i;
    // drift q' = qint(q_n, wh): q and the angular velocity at force time
    double qbn[4] = {0.0, 0.0, 0.0, 0.0};
    double whb[3] = {a.whb[3 * i], a.whb[3 * i + 1], a.whb[3 * i + 2]};
    {
        D7 q[4], qo[4];
        for (int k = 0; k < 4; ++k) q[k] = D7::var(pp[k], k);
        const V3<D7> w{D7::var(pc[4], 4), D7::var(pc[5], 5), D7::var(pc[6], 6)};
        qint_d(q, w, dt, qo);
        const double qb1[4] = {a.qb[4 * i], a.qb[4 * i + 1], a.qb[4 * i + 2], a.qb[4 * i + 3]};
        for (int k = 0; k < 7; ++k) {
            const double g = qb1[0] * qo[0].d[k] + qb1[1] * qo[1].d[k] + qb1[2] * qo[2].d[k] + qb1[3] * qo[3].d[k];
            if (k < 4) qbn[k] += g;
            else whb[k - 4] += g;
        }
    }
    // first half kick wh = w_n + W(q_n, w_n, T_n) dt / 2 (skipped for fixed
    // bodies), w_n the angular velocity the previous step ended with
    double wbn[3] = {whb[0], whb[1], whb[2]};
    double Teb[3] = {0.0, 0.0, 0.0};
    if (im != 0.0) {
        const double h = 0.5 * dt;
        D7 q[4];
        for (int k = 0; k < 4; ++k) q[k] = D7::var(pp[k], k);
        const V3<D7> w{D7::var(pp[10], 4), D7::var(pp[11], 5), D7::var(pp[12], 6)};
        const V3<D7> acc = w_accel(q, w, make_double3(pp[7], pp[8], pp[9]), geo);
        for (int k = 0; k < 7; ++k) {
            const double g = h * (whb[0] * acc.x.d[k] + whb[1] * acc.y.d[k] + whb[2] * acc.z.d[k]);
            if (k < 4) qbn[k] += g;
            else wbn[k - 4] += g;
        }
        double Ii[6];
        const double qd[4] = {pp[0], pp[1], pp[2], pp[3]};
        rot_tensor_d(qd, geo.inv_inertia, Ii);
        Teb[0] = h * (Ii[0] * whb[0] + Ii[3] * whb[1] + Ii[4] * whb[2]);
        Teb[1] = h * (Ii[3] * whb[0] + Ii[1] * whb[1] + Ii[5] * whb[2]);
        Teb[2] = h * (Ii[4] * whb[0] + Ii[5] * whb[1] + Ii[2] * whb[2]);
    }
    for (int k = 0; k < 4; ++k) a.qb[4 * i + k] = qbn[k];
    for (int c = 0; c < 3; ++c) {
        a.wb[3 * i + c] = wbn[c];
        a.Teb[3 * i + c] = Teb[c];
    }
}

// the record of turning bodies at a step: orientation and angular velocity
// after the drift and first half kick, torque after the forces
__global__ void k_adj_record(ObjDev P, double* dst, int what)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    double* d = dst + (long long)ADJ_PREC * i;
    if (what & ADJ_REC_QW) {
        const fd_quat q = P.q[i];
        const double3 w = P.angvel[i];
        d[0] = q.q0; d[1] = q.q1; d[2] = q.q2; d[3] = q.q3;
        d[4] = w.x; d[5] = w.y; d[6] = w.z;
    }
    if (what & ADJ_REC_T) {
        const double3 t = P.torque[i];
        const double3 w = P.angvel[i];
        d[7] = t.x; d[8] = t.y; d[9] = t.z;
        d[10] = w.x; d[11] = w.y; d[12] = w.z;
    }
}

// the contacts of one list at one step, turning bodies: two dual passes of 13
// directions each (relative node position, velocity difference, previous
// spring and the four parameters; then A's lever arm, the partner's
// orientation and both angular velocities), with force, both torques and
// new spring as outputs
__global__ void __launch_bounds__(ADJ_TPB) k_adj_contact_rot(AdjParticles a, AdjContactArgs c)
{
    using D13 = Dual<NDIR>;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int nslots = min(*c.nslots, c.rec.cap);
    if (s >= nslots || !c.rec.hit[s]) return;
    const AdjRec& R = c.rec;
    const int A = R.A[s], Bp = R.Bp[s];
    const int mi = a.mat[A], mj = R.matB[s];
    const bool wall = Bp < 0;
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
    const double lr = log(fmin(ei, ej));
    const double diss = -lr / sqrt(lr * lr + 3.14159265358979323846 * 3.14159265358979323846);
    const double invMi = a.G.geo[a.geo[A]].inv_mass;
    const double invMj = wall ? 0.0 : a.G.geo[a.geo[Bp]].inv_mass;
    double m = 0.0;
    if (invMi > 0. || invMj > 0.) m = 1.0 / (invMi + invMj);
    const FdGeo& GB = wall ? c.GW.geo[R.geoB[s]] : a.G.geo[R.geoB[s]];
    const double* sdf = wall ? c.GW.sdf : a.G.sdf;
    const double reld[3] = {R.rel[3 * s], R.rel[3 * s + 1], R.rel[3 * s + 2]};
    const double armd[3] = {R.arm[3 * s], R.arm[3 * s + 1], R.arm[3 * s + 2]};
    const double qBd[4] = {R.qB[4 * s], R.qB[4 * s + 1], R.qB[4 * s + 2], R.qB[4 * s + 3]};
    const double* pA = a.pr_cur + (long long)ADJ_PREC * A;
    const double wAd[3] = {pA[4], pA[5], pA[6]};
    double wBd[3];
    if (wall) {
        const double3 ww = c.wall_angvel[R.B[s]];
        wBd[0] = ww.x; wBd[1] = ww.y; wBd[2] = ww.z;
    } else {
        const double* pB = a.pr_cur + (long long)ADJ_PREC * Bp;
        wBd[0] = pB[4]; wBd[1] = pB[5]; wBd[2] = pB[6];
    }
    const int code = R.wrap[s];
    const double3 shiftA = make_double3((code % 3 - 1) * c.period.x, ((code / 3) % 3 - 1) * c.period.y, 0.0);
    const double3 shiftB = make_double3(((code / 9) % 3 - 1) * c.period.x, ((code / 27) % 3 - 1) * c.period.y, 0.0);
    const double3 rel3 = make_double3(reld[0], reld[1], reld[2]);
    // the velocity difference behind the recorded relative velocity: the
    // lever arms at the recorded state, from the same cell as the dual passes
    double dvd[3];
    {
        const double q0 = qBd[0], q1 = qBd[1], q2 = qBd[2], q3 = qBd[3];
        const double Rm[9] = {1.0 - 2.0 * (q2 * q2 + q3 * q3), 2.0 * (q1 * q2 - q0 * q3), 2.0 * (q1 * q3 + q0 * q2),
                              2.0 * (q1 * q2 + q0 * q3), 1.0 - 2.0 * (q1 * q1 + q3 * q3), 2.0 * (q2 * q3 - q0 * q1),
                              2.0 * (q1 * q3 - q0 * q2), 2.0 * (q2 * q3 + q0 * q1), 1.0 - 2.0 * (q1 * q1 + q2 * q2)};
        const double gx = (reld[0] * Rm[0] + reld[1] * Rm[3] + reld[2] * Rm[6] + (-GB.origin.x)) * GB.inv_spacing;
        const double gy = (reld[0] * Rm[1] + reld[1] * Rm[4] + reld[2] * Rm[7] + (-GB.origin.y)) * GB.inv_spacing;
        const double gz = (reld[0] * Rm[2] + reld[1] * Rm[5] + reld[2] * Rm[8] + (-GB.origin.z)) * GB.inv_spacing;
        const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
        if (i0 < 0 || j0 < 0 || k0 < 0 || i0 >= GB.size.x - 1 || j0 >= GB.size.y - 1 || k0 >= GB.size.z - 1) return;
        const double fx = gx - i0, fy = gy - j0, fz = gz - k0;
        const long long sx = GB.size.x, sxy = (long long)GB.size.x * GB.size.y;
        const double* S = sdf + GB.sdf_off + (long long)k0 * sxy + (long long)j0 * sx + i0;
        const double p[8] = {S[0], S[1], S[sx], S[sx + 1], S[sxy], S[sxy + 1], S[sxy + sx], S[sxy + sx + 1]};
        const double ux = 1 - fx, uy = 1 - fy, uz = 1 - fz;
        const double ov = -(((p[0] * ux + p[1] * fx) * uy + (p[2] * ux + p[3] * fx) * fy) * uz +
                            ((p[4] * ux + p[5] * fx) * uy + (p[6] * ux + p[7] * fx) * fy) * fz);
        using D1 = Dual<1>;
        const D1 qB[4] = {D1(qBd[0]), D1(qBd[1]), D1(qBd[2]), D1(qBd[3])};
        const V3<D1> gb{D1((p[1] - p[0]) * uy * uz + (p[3] - p[2]) * fy * uz + (p[5] - p[4]) * uy * fz +
                           (p[7] - p[6]) * fy * fz),
                        D1((p[2] - p[0]) * uz + (p[6] - p[4]) * fz), D1((p[4] - p[0]) * uy + (p[6] - p[2]) * fy)};
        const V3<D1> nw = qrot(qB, gb, false);
        const double nl = sqrt(nw.x.v * nw.x.v + nw.y.v * nw.y.v + nw.z.v * nw.z.v);
        if (!(nl > 0.0)) return;
        const double hx = 0.5 * ov * nw.x.v / nl, hy = 0.5 * ov * nw.y.v / nl, hz = 0.5 * ov * nw.z.v / nl;
        const double rA[3] = {armd[0] + hx - shiftA.x, armd[1] + hy - shiftA.y, armd[2] + hz - shiftA.z};
        const double rB[3] = {reld[0] + hx - shiftB.x, reld[1] + hy - shiftB.y, reld[2] + hz - shiftB.z};
        // vc = dv + wA x rA - wB x rB
        const double vc[3] = {R.vc[3 * s], R.vc[3 * s + 1], R.vc[3 * s + 2]};
        dvd[0] = vc[0] - (wAd[1] * rA[2] - wAd[2] * rA[1]) + (wBd[1] * rB[2] - wBd[2] * rB[1]);
        dvd[1] = vc[1] - (wAd[2] * rA[0] - wAd[0] * rA[2]) + (wBd[2] * rB[0] - wBd[0] * rB[2]);
        dvd[2] = vc[2] - (wAd[0] * rA[1] - wAd[1] * rA[0]) + (wBd[0] * rB[1] - wBd[1] * rB[0]);
    }
    // a contact with a particle's own periodic image has no reaction
    const bool react = !wall && Bp != A;
    double fb[3] = {a.Fb[3 * A], a.Fb[3 * A + 1], a.Fb[3 * A + 2]};
    if (react) {
        fb[0] -= a.Fb[3 * Bp];
        fb[1] -= a.Fb[3 * Bp + 1];
        fb[2] -= a.Fb[3 * Bp + 2];
    }
    const double tA[3] = {a.Tb[3 * A], a.Tb[3 * A + 1], a.Tb[3 * A + 2]};
    const double tB[3] = {react ? a.Tb[3 * Bp] : 0.0, react ? a.Tb[3 * Bp + 1] : 0.0, react ? a.Tb[3 * Bp + 2] : 0.0};
    const double sb[3] = {c.Sb_cur[3 * s], c.Sb_cur[3 * s + 1], c.Sb_cur[3 * s + 2]};
    auto project = [&](const V3<D13>& F, const V3<D13>& TA, const V3<D13>& TB, const V3<D13>& sn, double* g) {
        for (int k = 0; k < NDIR; ++k)
            g[k] = fb[0] * F.x.d[k] + fb[1] * F.y.d[k] + fb[2] * F.z.d[k] + tA[0] * TA.x.d[k] +
                   tA[1] * TA.y.d[k] + tA[2] * TA.z.d[k] + tB[0] * TB.x.d[k] + tB[1] * TB.y.d[k] +
                   tB[2] * TB.z.d[k] + sb[0] * sn.x.d[k] + sb[1] * sn.y.d[k] + sb[2] * sn.z.d[k];
    };
    double g1[NDIR], g2[NDIR];
    {
        // pass 1: rel, dv, sprev, kn, ks, diss, mu
        const V3<D13> rel{D13::var(reld[0], 0), D13::var(reld[1], 1), D13::var(reld[2], 2)};
        const V3<D13> dv{D13::var(dvd[0], 3), D13::var(dvd[1], 4), D13::var(dvd[2], 5)};
        const V3<D13> sprev{D13::var(R.sprev[3 * s], 6), D13::var(R.sprev[3 * s + 1], 7),
                            D13::var(R.sprev[3 * s + 2], 8)};
        const V3<D13> arm{D13(armd[0]), D13(armd[1]), D13(armd[2])};
        const D13 qB[4] = {D13(qBd[0]), D13(qBd[1]), D13(qBd[2]), D13(qBd[3])};
        const V3<D13> wA{D13(wAd[0]), D13(wAd[1]), D13(wAd[2])}, wB{D13(wBd[0]), D13(wBd[1]), D13(wBd[2])};
        V3<D13> F, TA, TB, sn;
        if (!contact_dual_rot<NDIR>(rel, arm, qB, dv, wA, wB, sprev, D13::var(kn, 9), D13::var(ks, 10),
                                    D13::var(diss, 11), D13::var(mu, 12), rel3, qBd, shiftA, shiftB, m, c.dt, GB,
                                    sdf, F, TA, TB, sn))
            return;
        project(F, TA, TB, sn, g1);
    }
    {
        // pass 2: arm, qB, wA, wB
        const V3<D13> rel{D13(reld[0]), D13(reld[1]), D13(reld[2])};
        const V3<D13> dv{D13(dvd[0]), D13(dvd[1]), D13(dvd[2])};
        const V3<D13> sprev{D13(R.sprev[3 * s]), D13(R.sprev[3 * s + 1]), D13(R.sprev[3 * s + 2])};
        const V3<D13> arm{D13::var(armd[0], 0), D13::var(armd[1], 1), D13::var(armd[2], 2)};
        const D13 qB[4] = {D13::var(qBd[0], 3), D13::var(qBd[1], 4), D13::var(qBd[2], 5), D13::var(qBd[3], 6)};
        const V3<D13> wA{D13::var(wAd[0], 7), D13::var(wAd[1], 8), D13::var(wAd[2], 9)};
        const V3<D13> wB{D13::var(wBd[0], 10), D13::var(wBd[1], 11), D13::var(wBd[2], 12)};
        V3<D13> F, TA, TB, sn;
        if (!contact_dual_rot<NDIR>(rel, arm, qB, dv, wA, wB, sprev, D13(kn), D13(ks), D13(diss), D13(mu), rel3, qBd,
                                    shiftA, shiftB, m, c.dt, GB, sdf, F, TA, TB, sn))
            return;
        project(F, TA, TB, sn, g2);
    }
    // positions and velocities (the node offset moves with A's centre and
    // orientation: rel = xA + arm - xB)
    if (wall || react) {
        atomic_add3(a.xb + 3 * A, g1[0], g1[1], g1[2]);
        atomic_add3(a.vhb + 3 * A, g1[3], g1[4], g1[5]);
    }
    if (react) {
        atomic_add3(a.xb + 3 * Bp, -g1[0], -g1[1], -g1[2]);
        atomic_add3(a.vhb + 3 * Bp, -g1[3], -g1[4], -g1[5]);
    }
    // A's orientation, through arm (which rel contains): arm = rot(qA, n),
    // n the node in A's body frame
    {
        using D4 = Dual<4>;
        const double* qAp = pA;  // orientation after the drift
        const D4 qA[4] = {D4::var(qAp[0], 0), D4::var(qAp[1], 1), D4::var(qAp[2], 2), D4::var(qAp[3], 3)};
        const D4 qAc[4] = {D4(qAp[0]), D4(qAp[1]), D4(qAp[2]), D4(qAp[3])};
        const V3<D4> nb = qrot(qAc, V3<D4>{D4(armd[0]), D4(armd[1]), D4(armd[2])}, true);
        const V3<D4> arm4 = qrot(qA, V3<D4>{D4(nb.x.v), D4(nb.y.v), D4(nb.z.v)}, false);
        const double ga[3] = {g1[0] + g2[0], g1[1] + g2[1], g1[2] + g2[2]};
        for (int k = 0; k < 4; ++k)
            atomicAdd(&a.qb[4 * A + k], ga[0] * arm4.x.d[k] + ga[1] * arm4.y.d[k] + ga[2] * arm4.z.d[k]);
    }
    if (!wall) {
        for (int k = 0; k < 4; ++k) atomicAdd(&a.qb[4 * Bp + k], g2[3 + k]);
        atomic_add3(a.whb + 3 * Bp, g2[10], g2[11], g2[12]);
    }
    atomic_add3(a.whb + 3 * A, g2[7], g2[8], g2[9]);
    const int hs = R.hist[s];
    if (hs >= 0 && hs < c.sb_prev_cap) atomic_add3(c.Sb_prev + 3 * hs, g1[6], g1[7], g1[8]);
    atomicAdd(&a.pgrad[4 * mi + 0], g1[9] * dk_i);
    atomicAdd(&a.pgrad[4 * mi + 1], g1[10] * ds_i);
    if (!wall) {
        atomicAdd(&a.pgrad[4 * mj + 0], g1[9] * dk_j);
        atomicAdd(&a.pgrad[4 * mj + 1], g1[10] * ds_j);
    }
    if (ei <= ej) atomicAdd(&a.pgrad[4 * mi + 2], g1[11]);
    else if (!wall) atomicAdd(&a.pgrad[4 * mj + 2], g1[11]);
    if (mui <= muj) atomicAdd(&a.pgrad[4 * mi + 3], g1[12]);
    else if (!wall) atomicAdd(&a.pgrad[4 * mj + 3], g1[12]);
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
    if (c.rec.cap <= 0) return;
    if (a.rot) k_adj_contact_rot<<<(c.rec.cap + ADJ_TPB - 1) / ADJ_TPB, ADJ_TPB, 0, s>>>(a, c);
    else k_adj_contact<double><<<(c.rec.cap + ADJ_TPB - 1) / ADJ_TPB, ADJ_TPB, 0, s>>>(a, c);
    count_launch();
}
void adj_record_rot(const ObjDev& P, double* dst, int what, cudaStream_t s)
{
    if (P.n > 0) { k_adj_record<<<(P.n + 255) / 256, 256, 0, s>>>(P, dst, what); count_launch(); }
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
