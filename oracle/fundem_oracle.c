/*
 * fundem_oracle.c -- CPU restatement of FunDEM's level-set DEM timestep.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Every function
 * cites the reference file:line it restates; paths are relative to the
 * reference's kernel/ directory unless stated otherwise.
 *
 * Floating point: the contact-membership arithmetic (node rotation, relative
 * position, radius test, body-frame grid coordinate and trilinear value) is
 * written with explicit fma() calls in the pattern nvcc's default contraction
 * gives the reference build (sums of products accumulated left to right; in
 * a difference of products the left product is fused, except in the reverse
 * rotation, whose negated quaternion components make the right one fused),
 * so that pair lists and overlaps compare bit for bit with the reference run
 * on a GPU.  Everything else is plain IEEE double with
 * contraction disabled (-ffp-contract=off).  Device-only intrinsics of the
 * reference (rsqrt in normalize) are replaced by 1/sqrt, as the reference's own
 * host path does (myVec.h:128-134); this moves normals by about one ulp.
 */
#include "fundem_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double x, y, z; } d3;
typedef struct { double q0, q1, q2, q3; } qt;
typedef struct { double xx, yy, zz, xy, xz, yz; } sm;

static int g_fma = 1;
/* which product each contracted a*b - c*d keeps exact: bit0 forward rotation
   t = q x v, bit1 forward q x t, bit2 reverse rotation t, bit3 reverse q x t,
   bit4 first sum of the trilinear value; set bit = right-hand product fused.
   12 (the reverse rotation, whose quaternion components are negated, fuses
   the right-hand product; everything else the left) reproduces every overlap
   of the reference build bit for bit (tests/test_oracle_cpu.py). */
static int g_pattern = 12;
void orc_set_fma_mode(int mode) { g_fma = mode ? 1 : 0; }
int orc_get_fma_mode(void) { return g_fma; }
void orc_set_fma_pattern(int p) { g_pattern = p; }
void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* small vector helpers (myVec.h:34-137, myQua.h:10-128)                      */
/* ------------------------------------------------------------------------- */
static inline d3 v3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 add(d3 a, d3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 sub(d3 a, d3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 mul(d3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline d3 neg(d3 a) { return v3(-a.x, -a.y, -a.z); }
static inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 cross(d3 a, d3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double len2(d3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
static inline double len(d3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline int is_zero(double x) { return fabs(x) <= 1.0e-20; } /* myVec.h:22-25 */
static inline d3 normalize3(d3 v) /* myVec.h:121-137, host branch */
{
    double l2 = v.x * v.x + v.y * v.y + v.z * v.z;
    if (is_zero(l2)) return v3(0, 0, 0);
    double inv = 1.0 / sqrt(l2);
    return v3(v.x * inv, v.y * inv, v.z * inv);
}
static inline qt normalizeq(qt q) /* myQua.h:51-62, host branch */
{
    double l2 = q.q0 * q.q0 + q.q1 * q.q1 + q.q2 * q.q2 + q.q3 * q.q3;
    if (is_zero(l2)) return q;
    double inv = 1.0 / sqrt(l2);
    qt r = {q.q0 * inv, q.q1 * inv, q.q2 * inv, q.q3 * inv};
    return r;
}
static const double PI = 3.14159265358979323846; /* myVec.h:13-16 */

/* --- contraction-aware pieces used by the membership predicate ----------- */
/* a*b - c*d as nvcc contracts it: fma(a, b, -(c*d)) */
static inline double msub(double a, double b, double c, double d)
{
    return g_fma ? fma(a, b, -(c * d)) : a * b - c * d;
}
static inline double msub_p(double a, double b, double c, double d, int right)
{
    if (!g_fma) return a * b - c * d;
    return right ? fma(-c, d, a * b) : fma(a, b, -(c * d));
}
static inline d3 cross_p(d3 a, d3 b, int right)
{
    return v3(msub_p(a.y, b.z, a.z, b.y, right), msub_p(a.z, b.x, a.x, b.z, right), msub_p(a.x, b.y, a.y, b.x, right));
}
/* x*x + y*y + z*z contracted: fma(z, z, fma(x, x, y*y)) */
static inline double len2_c(d3 v)
{
    return g_fma ? fma(v.z, v.z, fma(v.x, v.x, v.y * v.y)) : len2(v);
}
static inline d3 cross_c(d3 a, d3 b)
{
    return v3(msub(a.y, b.z, a.z, b.y), msub(a.z, b.x, a.x, b.z), msub(a.x, b.y, a.y, b.x));
}
/* v + t*s + w  (per component) -> fma(t, s, v) + w */
static inline double ats(double v, double t, double s, double w)
{
    return g_fma ? fma(t, s, v) + w : (v + t * s) + w;
}
/* rotateVectorByQuaternion, myQua.h:104-114 */
static inline d3 rotq_c(qt q, d3 v)
{
    d3 qv = v3(q.q1, q.q2, q.q3);
    d3 t = mul(cross_p(qv, v, g_pattern & 1), 2.0);
    d3 c = cross_p(qv, t, (g_pattern >> 1) & 1);
    return v3(ats(v.x, t.x, q.q0, c.x), ats(v.y, t.y, q.q0, c.y), ats(v.z, t.z, q.q0, c.z));
}
/* reverseRotateVectorByQuaternion, myQua.h:120-128 */
static inline d3 rrotq_c(d3 v, qt q)
{
    d3 qv = v3(-q.q1, -q.q2, -q.q3);
    d3 t = mul(cross_p(qv, v, (g_pattern >> 2) & 1), 2.0);
    d3 c = cross_p(qv, t, (g_pattern >> 3) & 1);
    return v3(ats(v.x, t.x, q.q0, c.x), ats(v.y, t.y, q.q0, c.y), ats(v.z, t.z, q.q0, c.z));
}
/* plain versions for everything outside the membership predicate */
static inline d3 rotq(qt q, d3 v)
{
    d3 qv = v3(q.q1, q.q2, q.q3);
    d3 t = mul(cross(qv, v), 2.0);
    return add(add(v, mul(t, q.q0)), cross(qv, t));
}
static inline d3 rrotq(d3 v, qt q)
{
    d3 qv = v3(-q.q1, -q.q2, -q.q3);
    d3 t = mul(cross(qv, v), 2.0);
    return add(add(v, mul(t, q.q0)), cross(qv, t));
}
/* interpolateLevelSetFunctionValue, LSParticleContactDetectionKernel.cuh:4-32 */
static inline double trilinear_c(double x, double y, double z, const double p[8])
{
    const double wx0 = 1.0 - x, wx1 = x, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
    if (!g_fma)
        return p[0] * wx0 * wy0 * wz0 + p[1] * wx1 * wy0 * wz0 + p[2] * wx0 * wy1 * wz0 +
               p[3] * wx1 * wy1 * wz0 + p[4] * wx0 * wy0 * wz1 + p[5] * wx1 * wy0 * wz1 +
               p[6] * wx0 * wy1 * wz1 + p[7] * wx1 * wy1 * wz1;
    double s = (g_pattern & 16) ? fma(p[1] * wx1 * wy0, wz0, p[0] * wx0 * wy0 * wz0)
                                : fma(p[0] * wx0 * wy0, wz0, p[1] * wx1 * wy0 * wz0);
    s = fma(p[2] * wx0 * wy1, wz0, s);
    s = fma(p[3] * wx1 * wy1, wz0, s);
    s = fma(p[4] * wx0 * wy0, wz1, s);
    s = fma(p[5] * wx1 * wy0, wz1, s);
    s = fma(p[6] * wx0 * wy1, wz1, s);
    s = fma(p[7] * wx1 * wy1, wz1, s);
    return s;
}
/* interpolateLevelSetFunctionGradient, LSParticleContactDetectionKernel.cuh:34-77.
   The x argument is declared `const int` in the reference: the fractional
   coordinate is truncated to 0 before the weights are formed. */
static inline d3 gradient_q(double xd, double y, double z, const double p[8])
{
    const int xi = (int)xd;
    const double wx0 = 1.0 - xi, wx1 = xi, wy0 = 1.0 - y, wy1 = y, wz0 = 1.0 - z, wz1 = z;
    double gx = (p[1] - p[0]) * wy0 * wz0 + (p[3] - p[2]) * wy1 * wz0 + (p[5] - p[4]) * wy0 * wz1 +
                (p[7] - p[6]) * wy1 * wz1;
    double gy = (p[2] - p[0]) * wx0 * wz0 + (p[3] - p[1]) * wx1 * wz0 + (p[6] - p[4]) * wx0 * wz1 +
                (p[7] - p[5]) * wx1 * wz1;
    double gz = (p[4] - p[0]) * wx0 * wy0 + (p[5] - p[1]) * wx1 * wy0 + (p[6] - p[2]) * wx0 * wy1 +
                (p[7] - p[3]) * wx1 * wy1;
    return v3(gx, gy, gz);
}

/* ------------------------------------------------------------------------- */
/* symmetric matrices (myMat.h:15-194)                                        */
/* ------------------------------------------------------------------------- */
static inline d3 smv(sm m, d3 v)
{
    return v3(m.xx * v.x + m.xy * v.y + m.xz * v.z, m.xy * v.x + m.yy * v.y + m.yz * v.z,
              m.xz * v.x + m.yz * v.y + m.zz * v.z);
}
/* rotateTensorByQuaternion, myMat.h:107-158 */
static sm rot_tensor(qt q, sm I)
{
    double q0 = q.q0, q1 = q.q1, q2 = q.q2, q3 = q.q3;
    double q11 = 2 * q1 * q1, q22 = 2 * q2 * q2, q33 = 2 * q3 * q3;
    double a = 1.0 - q22 - q33, b = 2 * (q1 * q2 - q0 * q3), c = 2 * (q1 * q3 + q0 * q2);
    double d = 2 * (q1 * q2 + q0 * q3), e = 1.0 - q11 - q33, f = 2 * (q2 * q3 - q0 * q1);
    double g = 2 * (q1 * q3 - q0 * q2), h = 2 * (q2 * q3 + q0 * q1), i = 1.0 - q11 - q22;
    double r0x = I.xx * a + I.xy * b + I.xz * c, r0y = I.xy * a + I.yy * b + I.yz * c,
           r0z = I.xz * a + I.yz * b + I.zz * c;
    double r1x = I.xx * d + I.xy * e + I.xz * f, r1y = I.xy * d + I.yy * e + I.yz * f,
           r1z = I.xz * d + I.yz * e + I.zz * f;
    double r2x = I.xx * g + I.xy * h + I.xz * i, r2y = I.xy * g + I.yy * h + I.yz * i,
           r2z = I.xz * g + I.yz * h + I.zz * i;
    sm r;
    r.xx = r0x * a + r0y * b + r0z * c;
    r.yy = r1x * d + r1y * e + r1z * f;
    r.zz = r2x * g + r2y * h + r2z * i;
    r.xy = r0x * d + r0y * e + r0z * f;
    r.xz = r0x * g + r0y * h + r0z * i;
    r.yz = r1x * g + r1y * h + r1z * i;
    return r;
}
/* inverse with the |det| < 1e-30 -> zero quirk, myMat.h:163-194; with
   physical != 0 the determinant is tested against the cube of the largest
   diagonal entry (1e-12 relative) instead, the project's scale-aware rule */
static sm inverse_sm_mode(sm A, int physical)
{
    const double det = A.xx * (A.yy * A.zz - A.yz * A.yz) + A.xy * (A.yz * A.xz - A.xy * A.zz) +
                       A.xz * (A.xy * A.yz - A.yy * A.xz);
    sm r = {0, 0, 0, 0, 0, 0};
    if (physical) {
        double m = fabs(A.xx);
        if (fabs(A.yy) > m) m = fabs(A.yy);
        if (fabs(A.zz) > m) m = fabs(A.zz);
        if (!(m > 0.0) || !(fabs(det) > 1e-12 * m * m * m)) return r;
    } else if (fabs(det) < 1e-30) {
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
static sm inverse_sm(sm A) { return inverse_sm_mode(A, 0); }
void orc_inverse_sym(const double in[6], double out[6])
{
    sm a = {in[0], in[1], in[2], in[3], in[4], in[5]};
    sm r = inverse_sm(a);
    out[0] = r.xx; out[1] = r.yy; out[2] = r.zz; out[3] = r.xy; out[4] = r.xz; out[5] = r.yz;
}

/* ------------------------------------------------------------------------- */
/* data model                                                                 */
/* ------------------------------------------------------------------------- */
#define GROW(ptr, n, cap)                                                          \
    do {                                                                           \
        if ((n) >= (cap)) {                                                        \
            (cap) = (cap) ? 2 * (cap) : 16;                                        \
            (ptr) = realloc((ptr), sizeof(*(ptr)) * (size_t)(cap));                \
        }                                                                          \
    } while (0)

typedef struct {
    int n, cap;
    double *kn, *ks, *mu, *e;
} mat_set;

typedef struct {
    int n, cap;
    double *radius, *inv_mass, *inv_spacing;
    sm *inertia, *inv_inertia;
    d3* origin;
    int* size; /* 3 per geometry */
    long long* sdf_start; /* exclusive start of each geometry's SDF */
    int* node_start;      /* exclusive start of each geometry's nodes */
    int* node_count;
    double* sdf;
    long long sdf_len, sdf_cap;
    d3* nodes;
    int node_len, node_cap;
} geo_set;

typedef struct {
    d3 minb, maxb, inv;
    int size[3];
    long long num;
    int *start, *end;
} grid_t;

typedef struct {
    int n, cap;
    d3 *pos, *vel, *angvel, *force, *torque;
    qt* q;
    int *mat, *geo;
    int *hash_value, *hash_index;
    long long n_nodes, node_cap;
    int *node_pid, *node_lid;
    mat_set mats;
    geo_set geos;
    grid_t g;
} obj_set;

typedef struct {
    long long n_master;
    int *count, *prefix, *prefix_old;
    long long n, cap; /* current list */
    int *master, *slave;
    d3 *point, *normal, *spring;
    double *overlap, *en, *es;
    long long n_old;
    int* slave_old;
    d3* spring_old;
    int initialized;
} contacts;

typedef struct {
    int active;
    int n;
    d3 *pos, *vel;
    qt* q;
    int *hash_value, *hash_index;
    grid_t g;
    contacts c;
} ghost_t;

typedef struct {
    int n, cap;
    int *master, *slave, *active;
    d3* point;
    double *radius, *L0, *B1, *B2, *B3, *B4, *ts, *coh, *mu;
    double *un, *us, *ub, *ut, *sn, *ss;
    d3 *mn1, *mn2, *mn3, *mp, *sn1, *sn2, *sn3, *sp;
} bonds_t;

struct orc_world {
    obj_set P, W;
    contacts PP, PW;
    ghost_t GX, GY, GXY;
    ghost_t R90, R180, R270; /* sector images, PeriodicBoundary.h:319-425 */
    int perX, perY, sector;
    int physical_inertia; /* 0: the reference's inverse() rule */
    bonds_t B;
};

orc_world* orc_create(void) { return (orc_world*)calloc(1, sizeof(orc_world)); }

static void free_contacts(contacts* c)
{
    free(c->count); free(c->prefix); free(c->prefix_old);
    free(c->master); free(c->slave); free(c->point); free(c->normal); free(c->spring);
    free(c->overlap); free(c->en); free(c->es); free(c->slave_old); free(c->spring_old);
}
static void free_obj(obj_set* o)
{
    free(o->pos); free(o->vel); free(o->angvel); free(o->force); free(o->torque); free(o->q);
    free(o->mat); free(o->geo); free(o->hash_value); free(o->hash_index); free(o->node_pid);
    free(o->node_lid);
    free(o->mats.kn); free(o->mats.ks); free(o->mats.mu); free(o->mats.e);
    geo_set* g = &o->geos;
    free(g->radius); free(g->inv_mass); free(g->inv_spacing); free(g->inertia);
    free(g->inv_inertia); free(g->origin); free(g->size); free(g->sdf_start);
    free(g->node_start); free(g->node_count); free(g->sdf); free(g->nodes);
    free(o->g.start); free(o->g.end);
}
static void free_ghost(ghost_t* g)
{
    free(g->pos); free(g->vel); free(g->q); free(g->hash_value); free(g->hash_index);
    free(g->g.start); free(g->g.end);
    free_contacts(&g->c);
}
void orc_destroy(orc_world* w)
{
    if (!w) return;
    free_obj(&w->P); free_obj(&w->W);
    free_contacts(&w->PP); free_contacts(&w->PW);
    free_ghost(&w->GX); free_ghost(&w->GY); free_ghost(&w->GXY);
    free_ghost(&w->R90); free_ghost(&w->R180); free_ghost(&w->R270);
    bonds_t* b = &w->B;
    free(b->master); free(b->slave); free(b->active); free(b->point); free(b->radius);
    free(b->L0); free(b->B1); free(b->B2); free(b->B3); free(b->B4); free(b->ts); free(b->coh);
    free(b->mu); free(b->un); free(b->us); free(b->ub); free(b->ut); free(b->sn); free(b->ss);
    free(b->mn1); free(b->mn2); free(b->mn3); free(b->mp); free(b->sn1); free(b->sn2);
    free(b->sn3); free(b->sp);
    free(w);
}

/* ------------------------------------------------------------------------- */
/* host setup                                                                 */
/* ------------------------------------------------------------------------- */
/* LSParticle::addMaterial clamps, LSParticle.h:221-231; walls pass kn=ks=0
   (LSSolver.h:175-183) */
int orc_add_material(orc_world* w, int wall, double kn, double ks, double mu, double e)
{
    mat_set* m = wall ? &w->W.mats : &w->P.mats;
    if (m->n >= m->cap) {
        m->cap = m->cap ? 2 * m->cap : 8;
        m->kn = realloc(m->kn, sizeof(double) * m->cap);
        m->ks = realloc(m->ks, sizeof(double) * m->cap);
        m->mu = realloc(m->mu, sizeof(double) * m->cap);
        m->e = realloc(m->e, sizeof(double) * m->cap);
    }
    if (wall) { kn = 0.0; ks = 0.0; }
    m->kn[m->n] = kn > 0. ? kn : 0.0;
    m->ks[m->n] = ks > 0. ? ks : 0.0;
    m->mu[m->n] = mu > 0. ? mu : 0.0;
    m->e[m->n] = (e > 0. && e < 1.0) ? e : 1.0;
    return m->n++;
}

/* LSParticle::addGeometry + geometryInfo::pushHost, LSParticle.h:233-267, 74-117;
   walls: LSSolver.h:196-213 (mass 0, zero inertia) */
int orc_add_geometry(orc_world* w, int wall, double mass, const double inertia[6],
                     const double origin[3], double spacing, const int size[3],
                     const double* sdf, int n_nodes, const double* nodes)
{
    if (size[0] < 2 || size[1] < 2 || size[2] < 2) return -1;
    if (spacing <= 0.0) return -1;
    geo_set* g = wall ? &w->W.geos : &w->P.geos;
    if (wall) mass = 0.0;
    if (g->n >= g->cap) {
        g->cap = g->cap ? 2 * g->cap : 8;
        g->radius = realloc(g->radius, sizeof(double) * g->cap);
        g->inv_mass = realloc(g->inv_mass, sizeof(double) * g->cap);
        g->inv_spacing = realloc(g->inv_spacing, sizeof(double) * g->cap);
        g->inertia = realloc(g->inertia, sizeof(sm) * g->cap);
        g->inv_inertia = realloc(g->inv_inertia, sizeof(sm) * g->cap);
        g->origin = realloc(g->origin, sizeof(d3) * g->cap);
        g->size = realloc(g->size, sizeof(int) * 3 * g->cap);
        g->sdf_start = realloc(g->sdf_start, sizeof(long long) * g->cap);
        g->node_start = realloc(g->node_start, sizeof(int) * g->cap);
        g->node_count = realloc(g->node_count, sizeof(int) * g->cap);
    }
    const int k = g->n;
    sm I = {0, 0, 0, 0, 0, 0};
    if (mass > 0.0 && inertia) {
        I.xx = inertia[0]; I.yy = inertia[1]; I.zz = inertia[2];
        I.xy = inertia[3]; I.xz = inertia[4]; I.yz = inertia[5];
    }
    g->inv_mass[k] = mass > 0.0 ? 1.0 / mass : 0.0;
    g->inertia[k] = I;
    g->inv_inertia[k] = inverse_sm_mode(I, wall ? 0 : w->physical_inertia);
    g->origin[k] = v3(origin[0], origin[1], origin[2]);
    g->inv_spacing[k] = 1.0 / spacing;
    g->size[3 * k] = size[0]; g->size[3 * k + 1] = size[1]; g->size[3 * k + 2] = size[2];
    long long nsdf = (long long)size[0] * size[1] * size[2];
    g->sdf_start[k] = g->sdf_len;
    if (g->sdf_len + nsdf > g->sdf_cap) {
        while (g->sdf_len + nsdf > g->sdf_cap) g->sdf_cap = g->sdf_cap ? 2 * g->sdf_cap : 4096;
        g->sdf = realloc(g->sdf, sizeof(double) * g->sdf_cap);
    }
    memcpy(g->sdf + g->sdf_len, sdf, sizeof(double) * nsdf);
    g->sdf_len += nsdf;
    g->node_start[k] = g->node_len;
    g->node_count[k] = n_nodes;
    if (g->node_len + n_nodes > g->node_cap) {
        while (g->node_len + n_nodes > g->node_cap) g->node_cap = g->node_cap ? 2 * g->node_cap : 1024;
        g->nodes = realloc(g->nodes, sizeof(d3) * g->node_cap);
    }
    double r = 0.0;
    for (int i = 0; i < n_nodes; ++i) {
        d3 p = v3(nodes[3 * i], nodes[3 * i + 1], nodes[3 * i + 2]);
        g->nodes[g->node_len + i] = p;
        double l = len(p);
        if (l > r) r = l;
    }
    g->node_len += n_nodes;
    g->radius[k] = r;
    return g->n++;
}

/* mass, centroid, inertia from a smoothed Heaviside of the SDF,
   LSSolver.h:503-565 (smooth parameter 1.5 at :512) */
static double smooth_heaviside(double phi, double s)
{
    if (s <= 0.0) return (phi > 0.0) ? 0.0 : 1.0;
    if (phi < -s) return 1.0;
    if (phi > s) return 0.0;
    const double x = -phi / s;
    return 0.5 * (1.0 + x + sin(PI * x) / PI);
}
int orc_mass_properties(double density, const double origin[3], double h, const int size[3],
                        const double* sdf, double* mass_out, double centroid_out[3],
                        double inertia_out[6])
{
    if (size[0] < 2 || size[1] < 2 || size[2] < 2 || h <= 0.0) return -1;
    double mass = 0.0;
    const double mg = density * h * h * h;
    for (int x = 0; x < size[0]; x++)
        for (int y = 0; y < size[1]; y++)
            for (int z = 0; z < size[2]; z++) {
                const long long idx = (long long)z * size[1] * size[0] + (long long)y * size[0] + x;
                mass += smooth_heaviside(sdf[idx] / h, 1.5);
            }
    mass *= mg;
    d3 c = v3(0, 0, 0);
    sm I = {0, 0, 0, 0, 0, 0};
    if (mass > 0.) {
        for (int x = 0; x < size[0]; x++)
            for (int y = 0; y < size[1]; y++)
                for (int z = 0; z < size[2]; z++) {
                    const long long idx = (long long)z * size[1] * size[0] + (long long)y * size[0] + x;
                    const double H = smooth_heaviside(sdf[idx] / h, 1.5);
                    c.x += H * (origin[0] + (double)x * h);
                    c.y += H * (origin[1] + (double)y * h);
                    c.z += H * (origin[2] + (double)z * h);
                }
        c = mul(c, mg / mass);
        for (int x = 0; x < size[0]; x++)
            for (int y = 0; y < size[1]; y++)
                for (int z = 0; z < size[2]; z++) {
                    const long long idx = (long long)z * size[1] * size[0] + (long long)y * size[0] + x;
                    const double H = smooth_heaviside(sdf[idx] / h, 1.5);
                    d3 r = sub(add(v3(origin[0], origin[1], origin[2]),
                                   mul(v3((double)x, (double)y, (double)z), h)),
                               c);
                    I.xx += H * (r.y * r.y + r.z * r.z) * mg;
                    I.yy += H * (r.x * r.x + r.z * r.z) * mg;
                    I.zz += H * (r.y * r.y + r.x * r.x) * mg;
                    I.xy -= H * r.x * r.y * mg;
                    I.xz -= H * r.x * r.z * mg;
                    I.yz -= H * r.y * r.z * mg;
                }
    }
    *mass_out = mass;
    centroid_out[0] = c.x; centroid_out[1] = c.y; centroid_out[2] = c.z;
    inertia_out[0] = I.xx; inertia_out[1] = I.yy; inertia_out[2] = I.zz;
    inertia_out[3] = I.xy; inertia_out[4] = I.xz; inertia_out[5] = I.yz;
    return 0;
}

/* LSParticle::addParticle, LSParticle.h:269-328 */
int orc_add_object(orc_world* w, int wall, const double pos[3], const double vel[3],
                   const double angvel[3], const double q[4], int mat, int geo)
{
    obj_set* o = wall ? &w->W : &w->P;
    if (mat < 0 || mat >= o->mats.n) return -1;
    if (geo < 0 || geo >= o->geos.n) return -1;
    if (o->n >= o->cap) {
        o->cap = o->cap ? 2 * o->cap : 64;
        o->pos = realloc(o->pos, sizeof(d3) * o->cap);
        o->vel = realloc(o->vel, sizeof(d3) * o->cap);
        o->angvel = realloc(o->angvel, sizeof(d3) * o->cap);
        o->force = realloc(o->force, sizeof(d3) * o->cap);
        o->torque = realloc(o->torque, sizeof(d3) * o->cap);
        o->q = realloc(o->q, sizeof(qt) * o->cap);
        o->mat = realloc(o->mat, sizeof(int) * o->cap);
        o->geo = realloc(o->geo, sizeof(int) * o->cap);
        o->hash_value = realloc(o->hash_value, sizeof(int) * o->cap);
        o->hash_index = realloc(o->hash_index, sizeof(int) * o->cap);
    }
    const int i = o->n;
    const int nn = o->geos.node_count[geo];
    if (o->n_nodes + nn > o->node_cap) {
        while (o->n_nodes + nn > o->node_cap) o->node_cap = o->node_cap ? 2 * o->node_cap : 4096;
        o->node_pid = realloc(o->node_pid, sizeof(int) * o->node_cap);
        o->node_lid = realloc(o->node_lid, sizeof(int) * o->node_cap);
    }
    for (int k = 0; k < nn; ++k) {
        o->node_pid[o->n_nodes + k] = i;
        o->node_lid[o->n_nodes + k] = o->geos.node_start[geo] + k;
    }
    o->n_nodes += nn;
    o->pos[i] = v3(pos[0], pos[1], pos[2]);
    o->vel[i] = v3(vel[0], vel[1], vel[2]);
    o->angvel[i] = v3(angvel[0], angvel[1], angvel[2]);
    o->force[i] = v3(0, 0, 0);
    o->torque[i] = v3(0, 0, 0);
    qt qq = {q[0], q[1], q[2], q[3]};
    o->q[i] = normalizeq(qq);
    o->mat[i] = mat;
    o->geo[i] = geo;
    o->hash_value[i] = -1;
    o->hash_index[i] = -1;
    return o->n++;
}

/* VBondedInteraction::add, VBondedInteraction.h:10-22, 74-195 */
static d3 frame_n2(d3 n1)
{
    const d3 ref = (fabs(n1.x) < 0.9) ? v3(1., 0., 0.) : v3(0., 1., 0.);
    return normalize3(cross(ref, n1));
}
int orc_add_bond(orc_world* w, int master, int slave, const double point[3],
                 const double normal[3], double Rb, double Lb, double Eb, double nu,
                 double tensile, double cohesion, double mu)
{
    /* LSSolver::addBondedInteraction range check, LSSolver.h:300 */
    if (master >= w->P.n || slave >= w->P.n || master < 0 || slave < 0) return -1;
    d3 gn = v3(normal[0], normal[1], normal[2]);
    if (is_zero(len2(gn))) return -1;
    if (Rb <= 0. || Lb <= 0. || Eb <= 0. || nu <= -1.0 || nu >= 0.5) return -1;
    bonds_t* b = &w->B;
    if (b->n >= b->cap) {
        b->cap = b->cap ? 2 * b->cap : 64;
#define RE(p) b->p = realloc(b->p, sizeof(*b->p) * b->cap)
        RE(master); RE(slave); RE(active); RE(point); RE(radius); RE(L0); RE(B1); RE(B2);
        RE(B3); RE(B4); RE(ts); RE(coh); RE(mu); RE(un); RE(us); RE(ub); RE(ut); RE(sn);
        RE(ss); RE(mn1); RE(mn2); RE(mn3); RE(mp); RE(sn1); RE(sn2); RE(sn3); RE(sp);
#undef RE
    }
    const double Gb = Eb / (2. * (1. + nu));
    const double Ab = PI * Rb * Rb;
    const double Ib = Ab * Rb * Rb / 4.;
    const double Jb = 2. * Ib;
    const double Kn = Eb * Ab / Lb;
    const double Kt = Gb * Jb / Lb;
    const double Ks = 12. * Eb * Ib / (Lb * Lb * Lb);
    const double Kb = Eb * Ib / Lb;
    const double B1 = Kn, B2 = Lb * Lb * Ks, B4 = Kt, B3 = Kb - B2 / 4. - B4 / 2.;
    const d3 n = mul(gn, 1.0 / len(gn));
    const d3 c = v3(point[0], point[1], point[2]);
    const d3 gpi = add(c, mul(n, 0.5 * Lb));
    const d3 gpj = sub(c, mul(n, 0.5 * Lb));
    const qt qi = w->P.q[master], qj = w->P.q[slave];
    const d3 lpi = rrotq(sub(gpi, w->P.pos[master]), qi);
    const d3 lpj = rrotq(sub(gpj, w->P.pos[slave]), qj);
    const d3 n1i = neg(n);
    const d3 n2i = frame_n2(n1i);
    const d3 n3i = normalize3(cross(n1i, n2i));
    const d3 n1j = neg(n1i), n2j = n2i, n3j = n3i;
    const int k = b->n;
    b->master[k] = master; b->slave[k] = slave; b->active[k] = 1; b->point[k] = c;
    b->radius[k] = Rb; b->L0[k] = Lb; b->B1[k] = B1; b->B2[k] = B2; b->B3[k] = B3; b->B4[k] = B4;
    b->un[k] = b->us[k] = b->ub[k] = b->ut[k] = b->sn[k] = b->ss[k] = 0.;
    b->ts[k] = tensile; b->coh[k] = cohesion; b->mu[k] = mu;
    /* VBondPoint::pushHost normalises the local vectors, VBondedInteraction.h:31-37 */
    b->mn1[k] = normalize3(rrotq(n1i, qi));
    b->mn2[k] = normalize3(rrotq(n2i, qi));
    b->mn3[k] = normalize3(rrotq(n3i, qi));
    b->mp[k] = lpi;
    b->sn1[k] = normalize3(rrotq(n1j, qj));
    b->sn2[k] = normalize3(rrotq(n2j, qj));
    b->sn3[k] = normalize3(rrotq(n3j, qj));
    b->sp[k] = lpj;
    return b->n++;
}

void orc_set_periodic(orc_world* w, int x, int y) { w->perX = x ? 1 : 0; w->perY = y ? 1 : 0; }
void orc_set_sector(orc_world* w, int on) { w->sector = on ? 1 : 0; }

/* inverse-inertia rule: 0 the reference's, 1 scale-aware; recomputes the
   particle geometries already added */
void orc_set_inertia_mode(orc_world* w, int physical)
{
    w->physical_inertia = physical ? 1 : 0;
    for (int k = 0; k < w->P.geos.n; ++k) w->P.geos.inv_inertia[k] = inverse_sm_mode(w->P.geos.inertia[k], w->physical_inertia);
}

/* spatialGrid::set, mySpatialGrid.h:212-240 */
static void grid_set(grid_t* g, d3 minb, d3 maxb, double cell)
{
    if (maxb.x <= minb.x) maxb.x = minb.x + cell;
    if (maxb.y <= minb.y) maxb.y = minb.y + cell;
    if (maxb.z <= minb.z) maxb.z = minb.z + cell;
    g->minb = minb;
    g->maxb = maxb;
    if (g->size[0] == 0) { g->size[0] = g->size[1] = g->size[2] = 2; g->num = 8; }
    if (is_zero(cell)) {
        g->num = 8;
    } else {
        const d3 ds = sub(maxb, minb);
        g->size[0] = ds.x > 2. * cell ? (int)(ds.x / cell) : 2;
        g->size[1] = ds.y > 2. * cell ? (int)(ds.y / cell) : 2;
        g->size[2] = ds.z > 2. * cell ? (int)(ds.z / cell) : 2;
        g->inv.x = ds.x > 0.0 ? (double)g->size[0] / ds.x : 0.0;
        g->inv.y = ds.y > 0.0 ? (double)g->size[1] / ds.y : 0.0;
        g->inv.z = ds.z > 0.0 ? (double)g->size[2] / ds.z : 0.0;
        g->num = (long long)g->size[0] * g->size[1] * g->size[2];
    }
    g->start = realloc(g->start, sizeof(int) * g->num);
    g->end = realloc(g->end, sizeof(int) * g->num);
    for (long long i = 0; i < g->num; ++i) g->start[i] = g->end[i] = -1;
}

static void contacts_init(contacts* c, long long n_master)
{
    /* SolidInteraction::initialize, SolidInteraction.h:23-49: keeps history
       when the master count is unchanged */
    if (n_master <= c->n_master && c->initialized) return;
    long long n0 = c->initialized ? c->n_master : 0;
    c->count = realloc(c->count, sizeof(int) * (n_master ? n_master : 1));
    c->prefix = realloc(c->prefix, sizeof(int) * (n_master ? n_master : 1));
    c->prefix_old = realloc(c->prefix_old, sizeof(int) * (n_master ? n_master : 1));
    int last = (n0 > 0) ? c->prefix[n0 - 1] : 0;
    for (long long i = n0; i < n_master; ++i) { c->prefix[i] = last; c->count[i] = 0; c->prefix_old[i] = 0; }
    if (!c->initialized) {
        for (long long i = 0; i < n_master; ++i) { c->prefix[i] = 0; c->prefix_old[i] = 0; c->count[i] = 0; }
    }
    c->n_master = n_master;
    c->initialized = 1;
}

static void ghost_init(ghost_t* gh, const obj_set* P)
{
    /* Ghost::initialize, PeriodicBoundary.h:23-39 (zero-filled device arrays) */
    gh->active = 1;
    if (gh->n != P->n) {
        gh->n = P->n;
        gh->pos = realloc(gh->pos, sizeof(d3) * (P->n ? P->n : 1));
        gh->vel = realloc(gh->vel, sizeof(d3) * (P->n ? P->n : 1));
        gh->q = realloc(gh->q, sizeof(qt) * (P->n ? P->n : 1));
        gh->hash_value = realloc(gh->hash_value, sizeof(int) * (P->n ? P->n : 1));
        gh->hash_index = realloc(gh->hash_index, sizeof(int) * (P->n ? P->n : 1));
        memset(gh->pos, 0, sizeof(d3) * P->n);
        memset(gh->vel, 0, sizeof(d3) * P->n);
        memset(gh->q, 0, sizeof(qt) * P->n);
    }
    gh->g.minb = P->g.minb; gh->g.maxb = P->g.maxb; gh->g.inv = P->g.inv;
    gh->g.size[0] = P->g.size[0]; gh->g.size[1] = P->g.size[1]; gh->g.size[2] = P->g.size[2];
    gh->g.num = P->g.num;
    gh->g.start = realloc(gh->g.start, sizeof(int) * gh->g.num);
    gh->g.end = realloc(gh->g.end, sizeof(int) * gh->g.num);
    contacts_init(&gh->c, P->n_nodes);
}

/* LSSolver::upload, LSSolver.h:692-703; LSParticle::initialize LSParticle.h:371-386 */
int orc_setup(orc_world* w, const double minb[3], const double maxb[3])
{
    const d3 mn = v3(minb[0], minb[1], minb[2]), mx = v3(maxb[0], maxb[1], maxb[2]);
    const d3 ds = sub(mx, mn);
    if (ds.x <= 0.0 || ds.y <= 0.0 || ds.z <= 0.0) return -1; /* LSSolver.h:646-663 */
    obj_set* sets[2] = {&w->P, &w->W};
    for (int s = 0; s < 2; ++s) {
        obj_set* o = sets[s];
        double cell = 0.0;
        if (o->n > 0) {
            for (int k = 0; k < o->geos.n; ++k)
                if (o->geos.radius[k] > cell) cell = o->geos.radius[k];
            cell *= 2.0;
        }
        grid_set(&o->g, mn, mx, cell);
    }
    contacts_init(&w->PP, w->P.n_nodes);
    contacts_init(&w->PW, w->P.n_nodes);
    if (w->perX) ghost_init(&w->GX, &w->P);
    else w->GX.active = 0;
    if (w->perY) ghost_init(&w->GY, &w->P);
    else w->GY.active = 0;
    if (w->perX && w->perY) ghost_init(&w->GXY, &w->P);
    else w->GXY.active = 0;
    ghost_t* sec[3] = {&w->R90, &w->R180, &w->R270};
    for (int d = 0; d < 3; ++d) {
        if (w->sector) ghost_init(sec[d], &w->P);
        else sec[d]->active = 0;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* hashing and cell tables                                                    */
/* ------------------------------------------------------------------------- */
static inline int lin3(int x, int y, int z, const int* s) /* myVec.h:232-235 */
{
    return z * s[1] * s[0] + y * s[0] + x;
}
/* calculateGridPosition, mySpatialGrid.h:24-31 (truncation toward zero) */
static inline void cellpos(d3 p, d3 mn, d3 inv, int out[3])
{
    out[0] = (int)((p.x - mn.x) * inv.x);
    out[1] = (int)((p.y - mn.y) * inv.y);
    out[2] = (int)((p.z - mn.z) * inv.z);
}
/* calculateHashKernel, mySpatialGrid.cu:4-26 */
static int hash_of(d3 p, const grid_t* g)
{
    if (p.x < g->minb.x || p.x >= g->maxb.x) return -1;
    if (p.y < g->minb.y || p.y >= g->maxb.y) return -1;
    if (p.z < g->minb.z || p.z >= g->maxb.z) return -1;
    int c[3];
    cellpos(p, g->minb, g->inv, c);
    return lin3(c[0], c[1], c[2], g->size);
}
typedef struct { int h, i; } hpair;
static int cmp_hpair(const void* a, const void* b)
{
    const hpair* x = (const hpair*)a; const hpair* y = (const hpair*)b;
    if (x->h != y->h) return x->h < y->h ? -1 : 1;
    return x->i < y->i ? -1 : (x->i > y->i);
}
/* buildHashStartEnd, buildHashStartEnd.cu:47-137: stable sort of (hash, index),
   start/end per cell, values outside [0, numGrid) ignored.  hash_value is left
   sorted, as thrust::sort_by_key leaves it. */
static void build_start_end(int n, int* hv, int* hi, grid_t* g)
{
    for (long long c = 0; c < g->num; ++c) g->start[c] = g->end[c] = -1;
    if (n <= 0) return;
    hpair* tmp = (hpair*)malloc(sizeof(hpair) * n);
    for (int i = 0; i < n; ++i) { tmp[i].h = hv[i]; tmp[i].i = i; }
    qsort(tmp, n, sizeof(hpair), cmp_hpair);
    for (int i = 0; i < n; ++i) { hv[i] = tmp[i].h; hi[i] = tmp[i].i; }
    free(tmp);
    for (int i = 0; i < n; ++i) {
        const int h = hv[i];
        if (h < 0 || h >= g->num) continue;
        if (i == 0 || hv[i - 1] != h) g->start[h] = i;
        if (i == n - 1 || hv[i + 1] != h) g->end[h] = i + 1;
    }
}
static void update_grid(obj_set* o)
{
    for (int i = 0; i < o->n; ++i) o->hash_value[i] = hash_of(o->pos[i], &o->g);
    build_start_end(o->n, o->hash_value, o->hash_index, &o->g);
}

/* ------------------------------------------------------------------------- */
/* node-vs-SDF detection, LSParticleContactDetectionKernel.cu:4-607           */
/* ------------------------------------------------------------------------- */
typedef struct {
    /* master side (always real particles) */
    const obj_set* M;
    /* slave side */
    const d3* s_pos;
    const qt* s_q;
    const int* s_geo;
    const int* s_hash_index;
    const grid_t* s_grid;
    const geo_set* s_geos;
    int pp; /* 1: particle-particle rules (A<B and radius test) */
} detect_ctx;

/* Evaluate one (node, slave) candidate exactly as the reference does.
   Returns 1 if overlap >= 0; fills overlap and (if want) point/normal. */
static inline int node_candidate(const detect_ctx* cx, int idxA, d3 gp, int idxB, double* ov,
                                 d3* point, d3* normal, int want)
{
    if (cx->pp && idxA >= idxB) return 0;
    const int geoB = cx->s_geo[idxB];
    const geo_set* G = cx->s_geos;
    const d3 rel = v3(gp.x - cx->s_pos[idxB].x, gp.y - cx->s_pos[idxB].y, gp.z - cx->s_pos[idxB].z);
    if (cx->pp) {
        const double rB = G->radius[geoB];
        if (len2_c(rel) > rB * rB) return 0;
    }
    const qt qB = cx->s_q[idxB];
    const d3 lp = rrotq_c(rel, qB);
    const d3 o = G->origin[geoB];
    const double is = G->inv_spacing[geoB];
    const int* sz = G->size + 3 * geoB;
    const double gx = (lp.x - o.x) * is, gy = (lp.y - o.y) * is, gz = (lp.z - o.z) * is;
    const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
    if (i0 < 0 || j0 < 0 || k0 < 0) return 0;
    if (i0 >= sz[0] - 1 || j0 >= sz[1] - 1 || k0 >= sz[2] - 1) return 0;
    const int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
    const double x = gx - (double)i0, y = gy - (double)j0, z = gz - (double)k0;
    const double* S = G->sdf + G->sdf_start[geoB];
    double p[8];
    p[0] = S[lin3(i0, j0, k0, sz)];
    p[1] = S[lin3(i1, j0, k0, sz)];
    p[2] = S[lin3(i0, j1, k0, sz)];
    p[3] = S[lin3(i1, j1, k0, sz)];
    p[4] = S[lin3(i0, j0, k1, sz)];
    p[5] = S[lin3(i1, j0, k1, sz)];
    p[6] = S[lin3(i0, j1, k1, sz)];
    p[7] = S[lin3(i1, j1, k1, sz)];
    const double overlap = -trilinear_c(x, y, z, p);
    if (!(overlap >= 0.)) return 0;
    *ov = overlap;
    if (want) {
        d3 n = gradient_q(x, y, z, p);
        n = rotq(qB, n);
        n = normalize3(n);
        *normal = n;
        *point = add(gp, mul(n, 0.5 * overlap));
    }
    return 1;
}

/* the 27-cell loop shared by count and write passes (LSParticleContactDetectionKernel.cu:37-58) */
static long long detect_node(const detect_ctx* cx, long long idx, int write, contacts* c,
                             long long base_w, long long base_old, long long end_old)
{
    const obj_set* M = cx->M;
    const int idxA = M->node_pid[idx];
    const int lid = M->node_lid[idx];
    const d3 node = M->geos.nodes[lid];
    const d3 r = rotq_c(M->q[idxA], node);
    const d3 gp = v3(r.x + M->pos[idxA].x, r.y + M->pos[idxA].y, r.z + M->pos[idxA].z);
    const grid_t* g = cx->s_grid;
    int cp[3];
    cellpos(gp, g->minb, g->inv, cp);
    int st[3] = {-1, -1, -1}, en[3] = {1, 1, 1};
    for (int d = 0; d < 3; ++d) {
        if (cp[d] <= 0) { cp[d] = 0; st[d] = 0; }
        if (cp[d] >= g->size[d] - 1) { cp[d] = g->size[d] - 1; en[d] = 0; }
    }
    long long count = 0;
    for (int zz = st[2]; zz <= en[2]; zz++)
        for (int yy = st[1]; yy <= en[1]; yy++)
            for (int xx = st[0]; xx <= en[0]; xx++) {
                const int h = lin3(cp[0] + xx, cp[1] + yy, cp[2] + zz, g->size);
                const int s = g->start[h];
                if (s == -1) continue;
                const int e = g->end[h];
                for (int i = s; i < e; i++) {
                    const int idxB = cx->s_hash_index[i];
                    double ov;
                    d3 pt, nm;
                    if (!node_candidate(cx, idxA, gp, idxB, &ov, &pt, &nm, write)) continue;
                    if (write) {
                        const long long k = base_w + count;
                        c->point[k] = pt;
                        c->normal[k] = nm;
                        c->overlap[k] = ov;
                        c->master[k] = (int)idx;
                        c->slave[k] = idxB;
                        d3 ss = v3(0., 0., 0.);
                        for (long long j = base_old; j < end_old; j++)
                            if (idxB == c->slave_old[j]) { ss = c->spring_old[j]; break; }
                        c->spring[k] = ss;
                        c->en[k] = 0.;
                        c->es[k] = 0.;
                    }
                    count++;
                }
            }
    return count;
}

static void ensure_cap(contacts* c, long long n)
{
    if (n <= c->cap) return;
    long long cap = c->cap ? c->cap : 1024;
    while (cap < n) cap *= 2;
    c->master = realloc(c->master, sizeof(int) * cap);
    c->slave = realloc(c->slave, sizeof(int) * cap);
    c->point = realloc(c->point, sizeof(d3) * cap);
    c->normal = realloc(c->normal, sizeof(d3) * cap);
    c->spring = realloc(c->spring, sizeof(d3) * cap);
    c->overlap = realloc(c->overlap, sizeof(double) * cap);
    c->en = realloc(c->en, sizeof(double) * cap);
    c->es = realloc(c->es, sizeof(double) * cap);
    c->slave_old = realloc(c->slave_old, sizeof(int) * cap);
    c->spring_old = realloc(c->spring_old, sizeof(d3) * cap);
    c->cap = cap;
}

/* count -> prefix -> numPair -> savePreviousStep -> write
   (LSSolver.h:786-912, SolidInteraction.h:92-151) */
static void detect(const detect_ctx* cx, contacts* c)
{
    const long long nm = c->n_master;
    if (nm <= 0) { c->n = 0; return; }
#pragma omp parallel for schedule(dynamic, 256)
    for (long long idx = 0; idx < nm; ++idx) c->count[idx] = (int)detect_node(cx, idx, 0, c, 0, 0, 0);
    memcpy(c->prefix_old, c->prefix, sizeof(int) * nm);
    long long acc = 0;
    for (long long idx = 0; idx < nm; ++idx) { acc += c->count[idx]; c->prefix[idx] = (int)acc; }
    const long long nold = c->n;
    ensure_cap(c, acc > nold ? acc : nold);
    memcpy(c->slave_old, c->slave, sizeof(int) * nold);
    memcpy(c->spring_old, c->spring, sizeof(d3) * nold);
    c->n_old = nold;
    c->n = acc;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long idx = 0; idx < nm; ++idx) {
        const long long base_w = idx > 0 ? c->prefix[idx - 1] : 0;
        const long long end_w = c->prefix[idx];
        if (end_w - base_w == 0) continue;
        const long long base_old = idx > 0 ? c->prefix_old[idx - 1] : 0;
        const long long end_old = c->prefix_old[idx];
        detect_node(cx, idx, 1, c, base_w, base_old, end_old);
    }
}

/* ------------------------------------------------------------------------- */
/* contact law, contactKernel.cuh:4-77                                        */
/* ------------------------------------------------------------------------- */
static d3 sliding_spring(d3 prev, d3 sv, d3 n, d3 fn, double mu, double k, double c, double dt)
{
    d3 spring = v3(0., 0., 0.);
    if (mu > 0. && k > 0.) {
        d3 p1 = sub(prev, mul(n, dot(prev, n)));
        const double ap1 = len(p1);
        if (!is_zero(ap1)) p1 = mul(p1, len(prev) / ap1);
        spring = add(p1, mul(sv, dt));
        d3 sf = sub(mul(spring, -k), mul(sv, c));
        const double asf = len(sf);
        const double afn = len(fn);
        if (!is_zero(asf) && asf > mu * afn) {
            const double ratio = mu * afn / asf;
            sf = mul(sf, ratio);
            spring = mul(add(sf, mul(sv, c)), -1.0 / k);
            /* reference: -(springForce + c*v) / stiffness, operator/ multiplies
               by the reciprocal (myVec.h:55-59) */
        }
    }
    return spring;
}
/* 0: the reference's single-precision square roots in the damping terms
   (contactKernel.cuh:51, 53, 58); 1: double precision, a smooth variant for
   finite-difference checks of derivatives (test use only) */
static int g_sqrt64 = 0;
void orc_set_damping_sqrt64(int on) { g_sqrt64 = on ? 1 : 0; }
static inline double damp_sqrt(double x) { return g_sqrt64 ? sqrt(x) : (double)sqrtf((float)x); }

static void linear_contact(d3* F, d3* spring, d3 vc, d3 n, double delta, double dt, double kn,
                           double ks, double mu, double res, double m)
{
    if (delta > 0.) {
        const double lr = log(res);
        const double diss = -lr / damp_sqrt(lr * lr + PI * PI);
        const double cn = 2. * diss * damp_sqrt(m * kn);
        const d3 vn = mul(n, dot(vc, n));
        const d3 fn = sub(mul(n, kn * delta), mul(vn, cn));
        const double cs = 2. * diss * damp_sqrt(m * ks);
        const d3 vs = sub(vc, vn);
        *spring = sliding_spring(*spring, vs, n, fn, mu, ks, cs, dt);
        const d3 fs = sub(mul(*spring, -ks), mul(vs, cs));
        *F = add(fn, fs);
    } else {
        *spring = v3(0., 0., 0.);
    }
}

/* per-contact force for the three list kinds (contactKernel.cu:46-291).  Writes
   spring/energies in place; returns force on the master particle and the slave
   index (or -1 when no slave reaction applies). */
static void contact_forces(orc_world* w, contacts* c, int kind, const ghost_t* gh, double dt,
                           d3* Fout, int* jout)
{
    const obj_set* P = &w->P;
    const obj_set* W = &w->W;
    const long long n = c->n;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < n; ++k) {
        const int i = P->node_pid[c->master[k]];
        const d3 ri = P->pos[i], vi = P->vel[i], wi = P->angvel[i];
        const double invMi = P->geos.inv_mass[P->geo[i]];
        const int mi = P->mat[i];
        const double kni = P->mats.kn[mi], ksi = P->mats.ks[mi], mui = P->mats.mu[mi], ei = P->mats.e[mi];
        const int j = c->slave[k];
        d3 rj, vj, wj;
        double kn = 0., ks = 0., effM = 0., mu, res;
        if (kind == ORC_PW) {
            rj = W->pos[j]; vj = W->vel[j]; wj = W->angvel[j];
            const int mj = W->mat[j];
            mu = fmin(mui, W->mats.mu[mj]);
            res = fmin(ei, W->mats.e[mj]);
            if (invMi > 0.) effM = 1. / invMi;
            kn = kni; ks = ksi;
        } else {
            if (kind == ORC_PP) { rj = P->pos[j]; vj = P->vel[j]; }
            else { rj = gh->pos[j]; vj = gh->vel[j]; }
            wj = P->angvel[j];
            const double invMj = P->geos.inv_mass[P->geo[j]];
            const int mj = P->mat[j];
            const double knj = P->mats.kn[mj], ksj = P->mats.ks[mj];
            if (kni > 0. && knj > 0.) kn = kni * knj / (kni + knj);
            if (ksi > 0. && ksj > 0.) ks = ksi * ksj / (ksi + ksj);
            if (invMi > 0. || invMj > 0.) effM = 1. / (invMi + invMj);
            res = fmin(ei, P->mats.e[mj]);
            mu = fmin(mui, P->mats.mu[mj]);
        }
        const d3 rc = c->point[k], nij = c->normal[k];
        const double delta = c->overlap[k];
        const d3 vc = sub(add(vi, cross(wi, sub(rc, ri))), add(vj, cross(wj, sub(rc, rj))));
        d3 F = v3(0., 0., 0.);
        d3 es = c->spring[k];
        linear_contact(&F, &es, vc, nij, delta, dt, kn, ks, mu, res, effM);
        c->spring[k] = es;
        c->en[k] = 0.5 * delta * delta * kn;
        c->es[k] = 0.5 * len2(es) * ks;
        Fout[k] = F;
        jout[k] = (kind == ORC_PW) ? -1 : ((kind != ORC_PP && i == j) ? -1 : j);
    }
    /* deterministic accumulation in list order (the reference uses FP64
       atomics, contactKernel.cu:120-123, whose order is unspecified) */
    for (long long k = 0; k < n; ++k) {
        const int i = P->node_pid[c->master[k]];
        const d3 F = Fout[k];
        const d3 rc = c->point[k];
        P->force[i] = add(P->force[i], F);
        P->torque[i] = add(P->torque[i], cross(sub(rc, P->pos[i]), F));
        const int j = jout[k];
        if (j >= 0) {
            const d3 rj = (kind == ORC_PP) ? P->pos[j] : gh->pos[j];
            P->force[j] = add(P->force[j], neg(F));
            P->torque[j] = add(P->torque[j], cross(sub(rc, rj), neg(F)));
        }
    }
}

static void run_contact_forces(orc_world* w, contacts* c, int kind, const ghost_t* gh, double dt)
{
    if (c->n <= 0) return;
    d3* F = (d3*)malloc(sizeof(d3) * c->n);
    int* j = (int*)malloc(sizeof(int) * c->n);
    contact_forces(w, c, kind, gh, dt, F, j);
    free(F);
    free(j);
}

/* ------------------------------------------------------------------------- */
/* bonds, contactKernel.cuh:138-199 and contactKernel.cu:293-371               */
/* ------------------------------------------------------------------------- */
static int vbond(d3* Fij, d3* Mij, d3* Mji, double* Un, double* Us, double* Ub, double* Ut,
                 double* sn, double* ss, d3 rbi, d3 rbj, d3 n1i, d3 n2i, d3 n3i, d3 n1j, d3 n2j,
                 d3 n3j, double B1, double B2, double B3, double B4, double R, double L0,
                 double ts, double coh, double mu)
{
    const d3 rij = sub(rbi, rbj);
    const double D = len(rij);
    if (is_zero(D)) return 1;
    const d3 nij = normalize3(rij);
    const d3 e = neg(nij);
    const double D0 = L0;
    *Un = 0.5 * B1 * (D - D0) * (D - D0);
    *Us = B2 * (0.5 * dot(sub(n1j, n1i), e) - 0.25 * dot(n1i, n1j) + 0.75);
    *Ub = (0.25 * B2 + B3 + 0.5 * B4) * (dot(n1i, n1j) + 1.);
    *Ut = -0.5 * B4 * (dot(n1i, n1j) + dot(n2i, n2j) + dot(n3i, n3j) - 1);
    const d3 dn = sub(n1j, n1i);
    *Fij = add(mul(e, B1 * (D - D0)), mul(sub(dn, mul(e, dot(dn, e))), B2 / (2 * D)));
    const d3 MTB = sub(mul(cross(n1j, n1i), B3), mul(add(cross(n2j, n2i), cross(n3j, n3i)), 0.5 * B4));
    *Mij = add(mul(cross(e, n1i), -0.5 * B2), MTB);
    *Mji = sub(mul(cross(e, n1j), 0.5 * B2), MTB);
    const double bnf = dot(*Fij, nij);
    const d3 bsf = sub(*Fij, mul(nij, bnf));
    const double btt = dot(MTB, nij);
    const d3 bbt = sub(MTB, mul(nij, btt));
    const double A = R * R * PI;
    const double I = A * R * R / 4.;
    const double J = 2 * I;
    *sn = -bnf / A + len(bbt) / I * R;
    *ss = len(bsf) / A + fabs(btt) / J * R;
    if (ts > 0. && *sn > ts) return 0;
    else if (coh > 0. && *ss > coh - mu * *sn) return 0;
    return 1;
}
static void bond_forces(orc_world* w)
{
    bonds_t* b = &w->B;
    obj_set* P = &w->P;
    for (int k = 0; k < b->n; ++k) {
        if (b->active[k] == 0) {
            b->un[k] = b->us[k] = b->ub[k] = b->ut[k] = b->sn[k] = b->ss[k] = 0.;
            continue;
        }
        const int i = b->master[k], j = b->slave[k];
        const qt qi = P->q[i], qj = P->q[j];
        const d3 n1i = rotq(qi, b->mn1[k]), n2i = rotq(qi, b->mn2[k]), n3i = rotq(qi, b->mn3[k]);
        const d3 n1j = rotq(qj, b->sn1[k]), n2j = rotq(qj, b->sn2[k]), n3j = rotq(qj, b->sn3[k]);
        const d3 ri = P->pos[i], rj = P->pos[j];
        const d3 rbi = add(rotq(qi, b->mp[k]), ri);
        const d3 rbj = add(rotq(qj, b->sp[k]), rj);
        b->point[k] = mul(add(rbi, rbj), 0.5);
        d3 F = v3(0, 0, 0), Mij = v3(0, 0, 0), Mji = v3(0, 0, 0);
        b->active[k] = vbond(&F, &Mij, &Mji, &b->un[k], &b->us[k], &b->ub[k], &b->ut[k], &b->sn[k],
                             &b->ss[k], rbi, rbj, n1i, n2i, n3i, n1j, n2j, n3j, b->B1[k], b->B2[k],
                             b->B3[k], b->B4[k], b->radius[k], b->L0[k], b->ts[k], b->coh[k], b->mu[k]);
        P->force[i] = add(P->force[i], F);
        P->torque[i] = add(P->torque[i], add(Mij, cross(sub(rbi, ri), F)));
        P->force[j] = add(P->force[j], neg(F));
        P->torque[j] = add(P->torque[j], add(Mji, cross(sub(rbj, rj), neg(F))));
    }
}

/* ------------------------------------------------------------------------- */
/* integration, particleIntegrationKernel.cu:3-48, myQua.h:77-93               */
/* ------------------------------------------------------------------------- */
static void kick(obj_set* P, d3 g, double h)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P->n; ++i) {
        const int geo = P->geo[i];
        const double invM = P->geos.inv_mass[geo];
        if (is_zero(invM)) continue;
        P->vel[i] = add(P->vel[i], mul(add(mul(P->force[i], invM), g), h));
        const d3 wv = P->angvel[i];
        const qt q = P->q[i];
        const d3 Iw = smv(rot_tensor(q, P->geos.inertia[geo]), wv);
        P->angvel[i] = add(wv, mul(smv(rot_tensor(q, P->geos.inv_inertia[geo]), sub(P->torque[i], cross(wv, Iw))), h));
    }
}
static qt quat_integrate(qt q, d3 w, double dt)
{
    const d3 v = mul(w, 0.5 * dt);
    qt d;
    d.q0 = -q.q1 * v.x - q.q2 * v.y - q.q3 * v.z;
    d.q1 = q.q0 * v.x + q.q3 * v.y - q.q2 * v.z;
    d.q2 = -q.q3 * v.x + q.q0 * v.y + q.q1 * v.z;
    d.q3 = q.q2 * v.x - q.q1 * v.y + q.q0 * v.z;
    qt s = {q.q0 + d.q0, q.q1 + d.q1, q.q2 + d.q2, q.q3 + d.q3};
    return normalizeq(s);
}
static void drift(obj_set* P, double dt)
{
#pragma omp parallel for schedule(static)
    for (int i = 0; i < P->n; ++i) {
        P->pos[i] = add(P->pos[i], mul(P->vel[i], dt));
        P->q[i] = quat_integrate(P->q[i], P->angvel[i], dt);
    }
}

/* ------------------------------------------------------------------------- */
/* periodic ghosts, PeriodicBoundary.h:221-317, mySpatialGrid.cu:28-152,214-240 */
/* ------------------------------------------------------------------------- */
static void wrap(obj_set* P, int dim)
{
    const grid_t* g = &P->g;
    for (int i = 0; i < P->n; ++i) {
        d3 p = P->pos[i];
        if (dim == 0) {
            const double L = g->maxb.x - g->minb.x;
            if (p.x < g->minb.x) p.x += L;
            else if (p.x >= g->maxb.x) p.x -= L;
        } else {
            const double L = g->maxb.y - g->minb.y;
            if (p.y < g->minb.y) p.y += L;
            else if (p.y >= g->maxb.y) p.y -= L;
        }
        P->pos[i] = p;
    }
}
static void ghost_positions(ghost_t* gh, const obj_set* P, int kind)
{
    const grid_t* g = &P->g;
    const d3 ox = v3(g->maxb.x - g->minb.x, 0., 0.), oy = v3(0., g->maxb.y - g->minb.y, 0.);
    for (int i = 0; i < P->n; ++i) {
        const d3 p = P->pos[i];
        int c[3];
        cellpos(p, g->minb, g->inv, c);
        d3 r = p;
        if (kind == ORC_GX && c[0] == 0) r = add(r, ox);
        if (kind == ORC_GY && c[1] == 0) r = add(r, oy);
        if (kind == ORC_GXY && c[0] == 0 && c[1] == 0) r = add(r, add(ox, oy));
        gh->pos[i] = r;
    }
}
/* calculateGhostHashKernel (note the z test against maxBound.y, :236) */
static void ghost_grid(ghost_t* gh)
{
    const grid_t* g = &gh->g;
    for (int i = 0; i < gh->n; ++i) {
        const d3 p = gh->pos[i];
        int c[3];
        cellpos(p, g->minb, g->inv, c);
        int out = 0;
        if (p.x < g->minb.x) { c[0] = 0; out = 1; }
        else if (p.x >= g->maxb.x) { c[0] = g->size[0] - 1; out = 1; }
        if (p.y < g->minb.y) { c[1] = 0; out = 1; }
        else if (p.y >= g->maxb.y) { c[1] = g->size[1] - 1; out = 1; }
        if (p.z < g->minb.z) { c[2] = 0; out = 1; }
        else if (p.z >= g->maxb.y) { c[2] = g->size[2] - 1; out = 1; }
        gh->hash_value[i] = out ? lin3(c[0], c[1], c[2], g->size) : -1;
    }
    build_start_end(gh->n, gh->hash_value, gh->hash_index, &gh->g);
}
/* rotateVector, myVec.h:143-182 (host branch): v rotated by the angle |om|
   about om, exp([om]x) v = v + (sin t / t) om x v + ((1 - cos t) / t^2) om x (om x v) */
static d3 rot_by_omega(d3 v, d3 om)
{
    const double th2 = dot(om, om);
    if (is_zero(th2)) {
        const d3 oxv = cross(om, v), oo = cross(om, oxv);
        return add(add(v, oxv), mul(oo, 0.5));
    }
    const double inv = 1.0 / sqrt(th2);
    const double th = th2 * inv;
    const double sn = sin(th), cs = cos(th);
    const double A = sn * inv, B = (1.0 - cs) * (inv * inv);
    const d3 oxv = cross(om, v), oo = cross(om, oxv);
    return add(add(v, mul(oxv, A)), mul(oo, B));
}
/* rotateQuaternion, myQua.h:131-180: r(om) * q (Hamilton product), normalised */
static qt rot_quat_by_omega(qt q, d3 om)
{
    const double th2 = om.x * om.x + om.y * om.y + om.z * om.z;
    if (is_zero(th2)) return q;
    const double th = sqrt(th2);
    const double inv = 1.0 / th;
    const double ux = om.x * inv, uy = om.y * inv, uz = om.z * inv;
    const double half = 0.5 * th;
    const double c = cos(half), sn = sin(half);
    const double r0 = c, r1 = sn * ux, r2 = sn * uy, r3 = sn * uz;
    qt o;
    o.q0 = r0 * q.q0 - r1 * q.q1 - r2 * q.q2 - r3 * q.q3;
    o.q1 = r0 * q.q1 + r1 * q.q0 + r2 * q.q3 - r3 * q.q2;
    o.q2 = r0 * q.q2 - r1 * q.q3 + r2 * q.q0 + r3 * q.q1;
    o.q3 = r0 * q.q3 + r1 * q.q2 - r2 * q.q1 + r3 * q.q0;
    return normalizeq(o);
}
/* velocity, position about the domain's min corner, and orientation of a body
   turned by the angle a about z */
static void sector_turn(d3* v, d3* p, qt* q, d3 mn, double a)
{
    const d3 om = v3(0., 0., a);
    *v = rot_by_omega(*v, om);
    *p = add(mn, rot_by_omega(sub(*p, mn), om));
    *q = rot_quat_by_omega(*q, om);
}
/* updateVelocityPositionOrientationOutOfSectorKernel, mySpatialGrid.cu:58-85:
   a body that left the quarter sector x >= min.x, y >= min.y through one face
   comes back through the other */
static void sector_wrap(obj_set* P)
{
    const d3 mn = P->g.minb;
    for (int i = 0; i < P->n; ++i) {
        d3 v = P->vel[i], p = P->pos[i];
        qt q = P->q[i];
        if (p.x < mn.x && p.y >= mn.y) sector_turn(&v, &p, &q, mn, -0.5 * PI);
        if (p.y < mn.y && p.x >= mn.x) sector_turn(&v, &p, &q, mn, 0.5 * PI);
        P->vel[i] = v;
        P->pos[i] = p;
        P->q[i] = q;
    }
}
/* calculateSectorGhostVelocityPositionOrientationKernel, mySpatialGrid.cu:154-213:
   images turned by +90 degrees (bodies in the first cell row in y), -90
   degrees (first cell column in x) and 180 degrees (the corner cell); every
   other image is a copy of the body */
static void sector_images(orc_world* w)
{
    const obj_set* P = &w->P;
    const grid_t* g = &P->g;
    for (int i = 0; i < P->n; ++i) {
        const d3 p = P->pos[i], v = P->vel[i];
        const qt q = P->q[i];
        ghost_t* im[3] = {&w->R90, &w->R180, &w->R270};
        for (int d = 0; d < 3; ++d) { im[d]->pos[i] = p; im[d]->vel[i] = v; im[d]->q[i] = q; }
        int c[3];
        cellpos(p, g->minb, g->inv, c);
        if (c[1] == 0) {
            sector_turn(&w->R90.vel[i], &w->R90.pos[i], &w->R90.q[i], g->minb, 0.5 * PI);
            if (c[0] == 0) {
                sector_turn(&w->R270.vel[i], &w->R270.pos[i], &w->R270.q[i], g->minb, -0.5 * PI);
                sector_turn(&w->R180.vel[i], &w->R180.pos[i], &w->R180.q[i], g->minb, PI);
            }
        } else if (c[0] == 0) {
            sector_turn(&w->R270.vel[i], &w->R270.pos[i], &w->R270.q[i], g->minb, -0.5 * PI);
        }
    }
}
static void update_ghost_grids(orc_world* w)
{
    obj_set* P = &w->P;
    ghost_t* list[3] = {&w->GX, &w->GY, &w->GXY};
    const int kinds[3] = {ORC_GX, ORC_GY, ORC_GXY};
    for (int d = 0; d < 3; ++d) {
        ghost_t* gh = list[d];
        if (!gh->active) continue;
        if (d == 0) wrap(P, 0);
        if (d == 1) wrap(P, 1);
        ghost_positions(gh, P, kinds[d]);
        ghost_grid(gh);
        memcpy(gh->q, P->q, sizeof(qt) * P->n);
        memcpy(gh->vel, P->vel, sizeof(d3) * P->n);
    }
    /* PeriodicBoundarySector::updateGhostSpatialGrid, PeriodicBoundary.h:351-383 */
    if (w->sector) {
        sector_wrap(P);
        sector_images(w);
        ghost_grid(&w->R90);
        ghost_grid(&w->R180);
        ghost_grid(&w->R270);
    }
}

static void detect_pp(orc_world* w)
{
    detect_ctx cx = {&w->P, w->P.pos, w->P.q, w->P.geo, w->P.hash_index, &w->P.g, &w->P.geos, 1};
    detect(&cx, &w->PP);
}
static void detect_pw(orc_world* w)
{
    detect_ctx cx = {&w->P, w->W.pos, w->W.q, w->W.geo, w->W.hash_index, &w->W.g, &w->W.geos, 0};
    detect(&cx, &w->PW);
}
static void detect_ghosts(orc_world* w)
{
    ghost_t* list[6] = {&w->GX, &w->GY, &w->GXY, &w->R90, &w->R180, &w->R270};
    for (int d = 0; d < 6; ++d) {
        ghost_t* gh = list[d];
        if (!gh->active) continue;
        detect_ctx cx = {&w->P, gh->pos, gh->q, w->P.geo, gh->hash_index, &gh->g, &w->P.geos, 0};
        detect(&cx, &gh->c);
    }
}

/* ------------------------------------------------------------------------- */
/* orchestration, LSSolver.h:1091-1229                                        */
/* ------------------------------------------------------------------------- */
int orc_initial_detect(orc_world* w)
{
    update_grid(&w->P);
    update_grid(&w->W);
    detect_pp(w);
    detect_pw(w);
    if (w->perX || w->perY || w->sector) {
        update_ghost_grids(w);
        detect_ghosts(w);
    }
    return 0;
}
int orc_half_kick(orc_world* w, const double g[3], double dt)
{
    kick(&w->P, v3(g[0], g[1], g[2]), 0.5 * dt);
    return 0;
}
int orc_front(orc_world* w, const double g[3], double dt)
{
    kick(&w->P, v3(g[0], g[1], g[2]), 0.5 * dt);
    drift(&w->P, dt);
    drift(&w->W, dt);
    return 0;
}
int orc_detect_and_force(orc_world* w, double dt)
{
    update_grid(&w->P);
    update_grid(&w->W);
    detect_pp(w);
    detect_pw(w);
    if (w->perX || w->perY || w->sector) {
        update_ghost_grids(w);
        detect_ghosts(w);
    }
    for (int i = 0; i < w->P.n; ++i) { w->P.force[i] = v3(0, 0, 0); w->P.torque[i] = v3(0, 0, 0); }
    run_contact_forces(w, &w->PP, ORC_PP, NULL, dt);
    run_contact_forces(w, &w->PW, ORC_PW, NULL, dt);
    if (w->GX.active) run_contact_forces(w, &w->GX.c, ORC_GX, &w->GX, dt);
    if (w->GY.active) run_contact_forces(w, &w->GY.c, ORC_GY, &w->GY, dt);
    if (w->GXY.active) run_contact_forces(w, &w->GXY.c, ORC_GXY, &w->GXY, dt);
    if (w->R90.active) run_contact_forces(w, &w->R90.c, ORC_GR90, &w->R90, dt);
    if (w->R180.active) run_contact_forces(w, &w->R180.c, ORC_GR180, &w->R180, dt);
    if (w->R270.active) run_contact_forces(w, &w->R270.c, ORC_GR270, &w->R270, dt);
    bond_forces(w);
    return 0;
}
int orc_step(orc_world* w, const double g[3], double dt)
{
    orc_front(w, g, dt);
    orc_detect_and_force(w, dt);
    orc_half_kick(w, g, dt);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* accessors                                                                  */
/* ------------------------------------------------------------------------- */
int orc_num_objects(orc_world* w, int wall) { return wall ? w->W.n : w->P.n; }
long long orc_num_nodes(orc_world* w) { return w->P.n_nodes; }

void orc_get_state(orc_world* w, int wall, double* pos, double* vel, double* angvel, double* q,
                   double* force, double* torque)
{
    obj_set* o = wall ? &w->W : &w->P;
    for (int i = 0; i < o->n; ++i) {
        if (pos) { pos[3 * i] = o->pos[i].x; pos[3 * i + 1] = o->pos[i].y; pos[3 * i + 2] = o->pos[i].z; }
        if (vel) { vel[3 * i] = o->vel[i].x; vel[3 * i + 1] = o->vel[i].y; vel[3 * i + 2] = o->vel[i].z; }
        if (angvel) { angvel[3 * i] = o->angvel[i].x; angvel[3 * i + 1] = o->angvel[i].y; angvel[3 * i + 2] = o->angvel[i].z; }
        if (q) { q[4 * i] = o->q[i].q0; q[4 * i + 1] = o->q[i].q1; q[4 * i + 2] = o->q[i].q2; q[4 * i + 3] = o->q[i].q3; }
        if (force) { force[3 * i] = o->force[i].x; force[3 * i + 1] = o->force[i].y; force[3 * i + 2] = o->force[i].z; }
        if (torque) { torque[3 * i] = o->torque[i].x; torque[3 * i + 1] = o->torque[i].y; torque[3 * i + 2] = o->torque[i].z; }
    }
}
void orc_set_state(orc_world* w, int wall, const double* pos, const double* vel,
                   const double* angvel, const double* q, const double* force, const double* torque)
{
    obj_set* o = wall ? &w->W : &w->P;
    for (int i = 0; i < o->n; ++i) {
        if (pos) o->pos[i] = v3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        if (vel) o->vel[i] = v3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        if (angvel) o->angvel[i] = v3(angvel[3 * i], angvel[3 * i + 1], angvel[3 * i + 2]);
        if (q) { qt t = {q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]}; o->q[i] = t; }
        if (force) o->force[i] = v3(force[3 * i], force[3 * i + 1], force[3 * i + 2]);
        if (torque) o->torque[i] = v3(torque[3 * i], torque[3 * i + 1], torque[3 * i + 2]);
    }
}
void orc_get_geometry(orc_world* w, int wall, int geo, double* radius, double* inv_mass,
                      double inertia[6], double inv_inertia[6])
{
    geo_set* g = wall ? &w->W.geos : &w->P.geos;
    if (geo < 0 || geo >= g->n) return;
    if (radius) *radius = g->radius[geo];
    if (inv_mass) *inv_mass = g->inv_mass[geo];
    if (inertia) {
        sm I = g->inertia[geo];
        inertia[0] = I.xx; inertia[1] = I.yy; inertia[2] = I.zz; inertia[3] = I.xy; inertia[4] = I.xz; inertia[5] = I.yz;
    }
    if (inv_inertia) {
        sm I = g->inv_inertia[geo];
        inv_inertia[0] = I.xx; inv_inertia[1] = I.yy; inv_inertia[2] = I.zz; inv_inertia[3] = I.xy; inv_inertia[4] = I.xz; inv_inertia[5] = I.yz;
    }
}
void orc_get_grid(orc_world* w, int wall, double minb[3], double maxb[3], double inv_cell[3], int size[3])
{
    grid_t* g = wall ? &w->W.g : &w->P.g;
    minb[0] = g->minb.x; minb[1] = g->minb.y; minb[2] = g->minb.z;
    maxb[0] = g->maxb.x; maxb[1] = g->maxb.y; maxb[2] = g->maxb.z;
    inv_cell[0] = g->inv.x; inv_cell[1] = g->inv.y; inv_cell[2] = g->inv.z;
    size[0] = g->size[0]; size[1] = g->size[1]; size[2] = g->size[2];
}
static contacts* kind_list(orc_world* w, int kind)
{
    switch (kind) {
    case ORC_PP: return &w->PP;
    case ORC_PW: return &w->PW;
    case ORC_GX: return &w->GX.c;
    case ORC_GY: return &w->GY.c;
    case ORC_GXY: return &w->GXY.c;
    case ORC_GR90: return &w->R90.c;
    case ORC_GR180: return &w->R180.c;
    case ORC_GR270: return &w->R270.c;
    }
    return NULL;
}
long long orc_num_contacts(orc_world* w, int kind)
{
    contacts* c = kind_list(w, kind);
    return c ? c->n : -1;
}
void orc_get_contacts(orc_world* w, int kind, int* master, int* slave, double* point,
                      double* normal, double* overlap, double* spring, double* en, double* es)
{
    contacts* c = kind_list(w, kind);
    if (!c) return;
    for (long long k = 0; k < c->n; ++k) {
        if (master) master[k] = c->master[k];
        if (slave) slave[k] = c->slave[k];
        if (point) { point[3 * k] = c->point[k].x; point[3 * k + 1] = c->point[k].y; point[3 * k + 2] = c->point[k].z; }
        if (normal) { normal[3 * k] = c->normal[k].x; normal[3 * k + 1] = c->normal[k].y; normal[3 * k + 2] = c->normal[k].z; }
        if (overlap) overlap[k] = c->overlap[k];
        if (spring) { spring[3 * k] = c->spring[k].x; spring[3 * k + 1] = c->spring[k].y; spring[3 * k + 2] = c->spring[k].z; }
        if (en) en[k] = c->en[k];
        if (es) es[k] = c->es[k];
    }
}
int orc_set_contacts(orc_world* w, int kind, long long n, const int* master, const int* slave,
                     const double* spring)
{
    contacts* c = kind_list(w, kind);
    if (!c || !c->initialized) return -1;
    ensure_cap(c, n);
    for (long long i = 0; i < c->n_master; ++i) c->count[i] = 0;
    for (long long k = 0; k < n; ++k) {
        if (master[k] < 0 || master[k] >= c->n_master) return -1;
        if (k > 0 && master[k] < master[k - 1]) return -1;
        c->master[k] = master[k];
        c->slave[k] = slave[k];
        c->spring[k] = v3(spring[3 * k], spring[3 * k + 1], spring[3 * k + 2]);
        c->count[master[k]]++;
    }
    long long acc = 0;
    for (long long i = 0; i < c->n_master; ++i) { acc += c->count[i]; c->prefix[i] = (int)acc; }
    c->n = n;
    return 0;
}
int orc_num_bonds(orc_world* w) { return w->B.n; }
void orc_get_bonds(orc_world* w, int* activated, double* point, double* un, double* us,
                   double* ub, double* ut, double* sn, double* ss)
{
    bonds_t* b = &w->B;
    for (int k = 0; k < b->n; ++k) {
        if (activated) activated[k] = b->active[k];
        if (point) { point[3 * k] = b->point[k].x; point[3 * k + 1] = b->point[k].y; point[3 * k + 2] = b->point[k].z; }
        if (un) un[k] = b->un[k];
        if (us) us[k] = b->us[k];
        if (ub) ub[k] = b->ub[k];
        if (ut) ut[k] = b->ut[k];
        if (sn) sn[k] = b->sn[k];
        if (ss) ss[k] = b->ss[k];
    }
}
void orc_set_bond_activation(orc_world* w, const int* activated)
{
    for (int k = 0; k < w->B.n; ++k) w->B.active[k] = activated[k];
}
void orc_get_bond_params(orc_world* w, double* b1234, double* f)
{
    bonds_t* b = &w->B;
    for (int k = 0; k < b->n; ++k) {
        if (b1234) { b1234[4 * k] = b->B1[k]; b1234[4 * k + 1] = b->B2[k]; b1234[4 * k + 2] = b->B3[k]; b1234[4 * k + 3] = b->B4[k]; }
        if (f) {
            d3 v[8] = {b->mn1[k], b->mn2[k], b->mn3[k], b->mp[k], b->sn1[k], b->sn2[k], b->sn3[k], b->sp[k]};
            for (int t = 0; t < 8; ++t) { f[24 * k + 3 * t] = v[t].x; f[24 * k + 3 * t + 1] = v[t].y; f[24 * k + 3 * t + 2] = v[t].z; }
        }
    }
}
