/*
 * CPU oracle for the rigid-body contact-solve hot path.  TEST INFRASTRUCTURE ONLY:
 * this file is the checker that the CUDA product is compared against.  Nothing in
 * the product links, loads or calls it; only the tests, the smoke check and the
 * bench's CPU-baseline leg do.
 *
 * It restates, expression for expression and in the same order, the float32
 * arithmetic of the reference's Warp kernels:
 *   src/motion_engine/contact_engine_gpu.py            (relaxed Jacobi, int64 fixed point)
 *   src/motion_engine/contact_engine_gpu_colored.py    (feature sort, manifold, pairs, JP colouring)
 *   src/motion_engine/contact_engine_gpu_fixed_frame.py / _applied_warm.py /
 *   _deferred_force.py / _color_cache.py               (the ColorCache chain)
 *
 * The reference kernels were JIT-compiled by Warp 1.13.0 through nvrtc with
 * floating-point contraction ON (fuse_fp=True, the default), so the golden arrays
 * carry the compiler's fused-multiply-add choices.  Every multiply-add site below
 * is therefore written with an explicit fmaf() or explicit separate rounding, and
 * the choice per builtin is a variant switch (g_fv[]).  The pinned defaults are the
 * ones that reproduce the reference's golden arrays bit for bit
 * (reports/cross_hardware_l4.npz, jacobi stack8 / lattice1000).
 *
 * Build: gcc -O2 -ffp-contract=off -fno-fast-math (the Makefile beside this file).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* variant switches for the contraction pattern of each builtin / site */
/* ------------------------------------------------------------------ */
enum {
    FV_DOT = 0,     /* wp.dot(vec3, vec3)                                  */
    FV_CROSS,       /* wp.cross                                            */
    FV_MATVEC,      /* mat33 * vec3                                        */
    FV_MATMUL,      /* mat33 * mat33                                       */
    FV_QROT,        /* wp.quat_rotate                                      */
    FV_QMUL,        /* quat * quat                                         */
    FV_QNORM,       /* wp.normalize(quat)                                  */
    FV_VNORM,       /* wp.normalize(vec3)                                  */
    FV_SITE_GRAV,   /* v + g*dt                          CEG:44           */
    FV_SITE_VT,     /* vrel - vn*nrm                     CEG:99           */
    FV_SITE_T1,     /* aa - dot(aa,n)*n                  CEG:105          */
    FV_SITE_MAG,    /* a1*a1 + a2*a2                     CEG:124          */
    FV_SITE_JT,     /* (a1-o1)*t1 + 0.5*(a2-o2)*t2       CEG:128          */
    FV_SITE_APPLY,  /* v + relax*dv                      CEG:142          */
    FV_SITE_INTX,   /* xc + (v+pv)*dt                    CEG:178          */
    FV_SITE_INTQ,   /* q + 0.5*wq*q*dt                   CEG:179          */
    FV_SITE_IMP,    /* jn*n + jt1*t1 + jt2*t2            applied_warm:38  */
    FV_COUNT
};
/* pinned: builtins in their first-product-fused form (variant 0), every user-level
 * multiply-add site contracted (1) -- reproduces the golden arrays bit for bit */
static int g_fv[32] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 1, 1, 1};

OR_API void or_set_variant(int idx, int val) { if (idx >= 0 && idx < 32) g_fv[idx] = val; }
OR_API int or_get_variant(int idx) { return (idx >= 0 && idx < 32) ? g_fv[idx] : -1; }

typedef struct { float x, y, z; } v3;
typedef struct { float m[3][3]; } m33;            /* row-major, m[row][col] */
typedef struct { float x, y, z, w; } qt;          /* Warp order (x, y, z, w) */

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vscale(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }

/* a*b + c, contracted or not */
static inline float mad(int fused, float a, float b, float c) { return fused ? fmaf(a, b, c) : a * b + c; }
/* c - a*b, contracted or not */
static inline float msub(int fused, float c, float a, float b) { return fused ? fmaf(-a, b, c) : c - a * b; }

static inline float dot3(v3 a, v3 b)
{
    switch (g_fv[FV_DOT]) {
    case 0: return fmaf(a.z, b.z, fmaf(a.x, b.x, a.y * b.y));          /* a0b0+a1b1+a2b2, first product fused */
    case 1: return fmaf(a.z, b.z, fmaf(a.y, b.y, fmaf(a.x, b.x, 0.0f))); /* loop from zero */
    case 2: return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));          /* second product fused */
    default: return (a.x * b.x + a.y * b.y) + a.z * b.z;
    }
}
static inline v3 cross3(v3 a, v3 b)
{
    switch (g_fv[FV_CROSS]) {
    case 0: return V(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
    case 1: return V(fmaf(-a.z, b.y, a.y * b.z), fmaf(-a.x, b.z, a.z * b.x), fmaf(-a.y, b.x, a.x * b.y));
    default: return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    }
}
static inline float len3(v3 a) { return sqrtf(dot3(a, a)); }

static inline float row_dot(const float *r, v3 b)
{
    switch (g_fv[FV_MATVEC]) {
    case 0: return fmaf(r[2], b.z, fmaf(r[0], b.x, r[1] * b.y));
    case 1: return fmaf(r[2], b.z, fmaf(r[1], b.y, r[0] * b.x));
    case 2: return fmaf(r[2], b.z, fmaf(r[1], b.y, fmaf(r[0], b.x, 0.0f)));
    default: return (r[0] * b.x + r[1] * b.y) + r[2] * b.z;
    }
}
static inline v3 matvec(const m33 *M, v3 b) { return V(row_dot(M->m[0], b), row_dot(M->m[1], b), row_dot(M->m[2], b)); }

static inline float mm_el(float a0, float a1, float a2, float b0, float b1, float b2)
{
    switch (g_fv[FV_MATMUL]) {
    case 0: return fmaf(a2, b2, fmaf(a1, b1, fmaf(a0, b0, 0.0f)));
    case 1: return fmaf(a2, b2, fmaf(a0, b0, a1 * b1));
    case 2: return fmaf(a2, b2, fmaf(a1, b1, a0 * b0));
    default: return (a0 * b0 + a1 * b1) + a2 * b2;
    }
}
static m33 matmul(const m33 *A, const m33 *B)
{
    m33 R;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            R.m[i][j] = mm_el(A->m[i][0], A->m[i][1], A->m[i][2], B->m[0][j], B->m[1][j], B->m[2][j]);
    return R;
}
static m33 transpose(const m33 *A)
{
    m33 R;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R.m[i][j] = A->m[j][i];
    return R;
}

/* wp.quat_rotate(q, x) = x*(2w^2-1) + q.xyz*2*dot(q.xyz,x) + cross(q.xyz,x)*w*2 */
static v3 quat_rotate(qt q, v3 x)
{
    if (g_fv[FV_QROT] == 0) {
        float c = fmaf(2.0f * q.w, q.w, -1.0f);
        float d = 2.0f * fmaf(q.z, x.z, fmaf(q.x, x.x, q.y * x.y));
        float cx = fmaf(q.y, x.z, -(q.z * x.y)), cy = fmaf(q.z, x.x, -(q.x * x.z)), cz = fmaf(q.x, x.y, -(q.y * x.x));
        return V(fmaf(cx * q.w, 2.0f, fmaf(x.x, c, q.x * d)),
                 fmaf(cy * q.w, 2.0f, fmaf(x.y, c, q.y * d)),
                 fmaf(cz * q.w, 2.0f, fmaf(x.z, c, q.z * d)));
    } else {
        float c = 2.0f * q.w * q.w - 1.0f;
        float d = 2.0f * ((q.x * x.x + q.y * x.y) + q.z * x.z);
        float cx = q.y * x.z - q.z * x.y, cy = q.z * x.x - q.x * x.z, cz = q.x * x.y - q.y * x.x;
        return V((x.x * c + q.x * d) + cx * q.w * 2.0f, (x.y * c + q.y * d) + cy * q.w * 2.0f,
                 (x.z * c + q.z * d) + cz * q.w * 2.0f);
    }
}
/* wp.quat_to_matrix: columns are the rotated unit axes */
static m33 quat_to_matrix(qt q)
{
    v3 c1 = quat_rotate(q, V(1.0f, 0.0f, 0.0f));
    v3 c2 = quat_rotate(q, V(0.0f, 1.0f, 0.0f));
    v3 c3 = quat_rotate(q, V(0.0f, 0.0f, 1.0f));
    m33 R = {{{c1.x, c2.x, c3.x}, {c1.y, c2.y, c3.y}, {c1.z, c2.z, c3.z}}};
    return R;
}
static qt qmul(qt a, qt b)
{
    qt r;
    if (g_fv[FV_QMUL] == 0) {
        r.x = fmaf(-b.y, a.z, fmaf(a.y, b.z, fmaf(a.w, b.x, b.w * a.x)));
        r.y = fmaf(-b.z, a.x, fmaf(a.z, b.x, fmaf(a.w, b.y, b.w * a.y)));
        r.z = fmaf(-b.x, a.y, fmaf(a.x, b.y, fmaf(a.w, b.z, b.w * a.z)));
        r.w = fmaf(-a.z, b.z, fmaf(-a.y, b.y, fmaf(a.w, b.w, -(a.x * b.x))));
    } else {
        r.x = ((a.w * b.x + b.w * a.x) + a.y * b.z) - b.y * a.z;
        r.y = ((a.w * b.y + b.w * a.y) + a.z * b.x) - b.z * a.x;
        r.z = ((a.w * b.z + b.w * a.z) + a.x * b.y) - b.x * a.y;
        r.w = ((a.w * b.w - a.x * b.x) - a.y * b.y) - a.z * b.z;
    }
    return r;
}
static float qdot(qt a, qt b)
{
    switch (g_fv[FV_DOT]) {
    case 0: return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.x, b.x, a.y * b.y)));
    case 1: return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, fmaf(a.x, b.x, 0.0f))));
    case 2: return fmaf(a.w, b.w, fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)));
    default: return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w;
    }
}
static qt qnormalize(qt q)
{
    float l = sqrtf(qdot(q, q));
    qt r;
    if (l > 0.0f) {
        if (g_fv[FV_QNORM] == 0) {
            float il = 1.0f / l;
            r.x = q.x * il; r.y = q.y * il; r.z = q.z * il; r.w = q.w * il;
        } else {
            r.x = q.x / l; r.y = q.y / l; r.z = q.z / l; r.w = q.w / l;
        }
    } else {
        r.x = 0.0f; r.y = 0.0f; r.z = 0.0f; r.w = 1.0f;
    }
    return r;
}
static v3 vnormalize(v3 a)
{
    float l = len3(a);
    if (l > 0.0f) {
        if (g_fv[FV_VNORM] == 0) return vdivs(a, l);
        float il = 1.0f / l;
        return vscale(a, il);
    }
    return V(0.0f, 0.0f, 0.0f);
}

/* ------------------------------------------------------------------ */
/* constants of the reference (contact_engine_gpu.py:25-26)            */
/* ------------------------------------------------------------------ */
#define K_G 9.81f
#define K_R 0.05f
#define K_2R 0.1f
#define K_BETA 0.2f
#define K_SLOP 1e-4f
#define K_SCALE 1.0e10f

static inline v3 ld3(const float *a, int i) { return V(a[3 * i], a[3 * i + 1], a[3 * i + 2]); }
static inline void st3(float *a, int i, v3 v) { a[3 * i] = v.x; a[3 * i + 1] = v.y; a[3 * i + 2] = v.z; }
static inline qt ldq(const float *a, int i) { qt q = {a[4 * i], a[4 * i + 1], a[4 * i + 2], a[4 * i + 3]}; return q; }
static inline void stq(float *a, int i, qt q) { a[4 * i] = q.x; a[4 * i + 1] = q.y; a[4 * i + 2] = q.z; a[4 * i + 3] = q.w; }
static inline m33 ldm(const float *a, int i) { m33 M; memcpy(&M, a + 9 * i, sizeof M); return M; }

/* ------------------------------------------------------------------ */
/* per-body kernels (CEG:40-59, CEG:171-180)                           */
/* ------------------------------------------------------------------ */
/* k_grav, CEG:40-44 */
static void body_gravity(int N, float *v, const float *invM, float dt)
{
    int f = g_fv[FV_SITE_GRAV];
    for (int i = 0; i < N; ++i)
        if (invM[i] > 0.0f) {
            v3 a = ld3(v, i);
            a = V(mad(f, 0.0f, dt, a.x), mad(f, 0.0f, dt, a.y), mad(f, -K_G, dt, a.z));
            st3(v, i, a);
        }
}
/* k_invIw, CEG:46-53: R * IbInv * R^T, zero for kinematic bodies */
static void body_inv_inertia(int N, const float *q, const float *IbInv, const int *kin, float *invIw)
{
    for (int i = 0; i < N; ++i) {
        m33 out;
        if (kin[i] == 1) {
            memset(&out, 0, sizeof out);
        } else {
            m33 Rm = quat_to_matrix(ldq(q, i));
            m33 Ib = ldm(IbInv, i);
            m33 t = matmul(&Rm, &Ib);
            m33 Rt = transpose(&Rm);
            out = matmul(&t, &Rt);
        }
        memcpy(invIw + 9 * i, &out, sizeof out);
    }
}
/* k_worldp, CEG:55-59.  Beads of body b are rest[off[b] .. off[b+1]) (uniform P in the reference). */
static void bead_world(int nbead, const float *xc, const float *q, const float *rest, const int *owner, float *allp)
{
    for (int g = 0; g < nbead; ++g) {
        int b = owner[g];
        st3(allp, g, vadd(ld3(xc, b), quat_rotate(ldq(q, b), ld3(rest, g))));
    }
}
/* k_integ, CEG:171-180 */
static void body_integrate(int N, float *xc, float *q, const float *v, const float *w, const float *pv,
                           const float *po, const float *invM, float dt)
{
    int fx = g_fv[FV_SITE_INTX], fq = g_fv[FV_SITE_INTQ];
    for (int i = 0; i < N; ++i) {
        if (invM[i] <= 0.0f) continue;
        v3 x = ld3(xc, i), s = vadd(ld3(v, i), ld3(pv, i));
        st3(xc, i, V(mad(fx, s.x, dt, x.x), mad(fx, s.y, dt, x.y), mad(fx, s.z, dt, x.z)));
        v3 ww = vadd(ld3(w, i), ld3(po, i));
        qt wq = {0.5f * ww.x, 0.5f * ww.y, 0.5f * ww.z, 0.5f * 0.0f};
        qt qi = ldq(q, i);
        qt p = qmul(wq, qi);
        qt qn = {mad(fq, p.x, dt, qi.x), mad(fq, p.y, dt, qi.y), mad(fq, p.z, dt, qi.z), mad(fq, p.w, dt, qi.w)};
        stq(q, i, qnormalize(qn));
    }
}

/* ------------------------------------------------------------------ */
/* broadphase + bead contact generation (CEG:61-79, COL:102-122)       */
/* A uniform grid of cell 2R is used here; the contact SET it produces */
/* is the set of the reference's hash-grid query (every pair closer   */
/* than 2R), so only the order differs, and the order never reaches   */
/* the result: Jacobi sums in int64, the coloured path sorts by        */
/* feature key first.                                                  */
/* ------------------------------------------------------------------ */
typedef struct {
    int C, cap, overflow;
    int *bi, *bj, *fa, *fb;
    float *pA, *pB, *n, *pen;
} contacts_t;

static void push_contact(contacts_t *c, int bi, int bj, v3 pA, v3 pB, v3 n, float pen, int fa, int fb)
{
    if (c->C >= c->cap) { c->overflow++; return; }
    int k = c->C++;
    c->bi[k] = bi; c->bj[k] = bj; st3(c->pA, k, pA); st3(c->pB, k, pB); st3(c->n, k, n);
    c->pen[k] = pen; c->fa[k] = fa; c->fb[k] = fb;
}

typedef struct { int64_t key; int idx; } cellent_t;
static int cmp_cell(const void *a, const void *b)
{
    const cellent_t *x = a, *y = b;
    if (x->key < y->key) return -1;
    if (x->key > y->key) return 1;
    return x->idx - y->idx;
}
static inline int64_t cell_key(int ix, int iy, int iz)
{
    return ((int64_t)(ix + (1 << 20)) << 42) | ((int64_t)(iy + (1 << 20)) << 21) | (int64_t)(iz + (1 << 20));
}

static void gen_contacts(int nbead, const float *allp, const int *owner, contacts_t *out)
{
    cellent_t *cells = malloc(sizeof(cellent_t) * (size_t)(nbead > 0 ? nbead : 1));
    for (int g = 0; g < nbead; ++g) {
        v3 p = ld3(allp, g);
        cells[g].key = cell_key((int)floorf(p.x / K_2R), (int)floorf(p.y / K_2R), (int)floorf(p.z / K_2R));
        cells[g].idx = g;
    }
    qsort(cells, nbead, sizeof(cellent_t), cmp_cell);
    out->C = 0; out->overflow = 0;
    for (int g = 0; g < nbead; ++g) {
        v3 xi = ld3(allp, g);
        int bi = owner[g];
        float s = xi.z - K_R;
        if (s < 0.0f) push_contact(out, bi, -1, xi, V(0, 0, 0), V(0, 0, 1), -s, g, -1);
        int cx = (int)floorf(xi.x / K_2R), cy = (int)floorf(xi.y / K_2R), cz = (int)floorf(xi.z / K_2R);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    int64_t k = cell_key(cx + dx, cy + dy, cz + dz);
                    int lo = 0, hi = nbead;
                    while (lo < hi) {
                        int mid = (lo + hi) >> 1;
                        if (cells[mid].key < k) lo = mid + 1; else hi = mid;
                    }
                    for (int t = lo; t < nbead && cells[t].key == k; ++t) {
                        int j = cells[t].idx;
                        if (j > g && owner[j] != bi) {
                            v3 xj = ld3(allp, j);
                            v3 dvec = vsub(xi, xj);
                            float dist = len3(dvec);
                            if (dist < K_2R && dist > 1e-9f)
                                push_contact(out, bi, owner[j], xi, xj, vdivs(dvec, dist), K_2R - dist, g, j);
                        }
                    }
                }
    }
    free(cells);
}

/* ------------------------------------------------------------------ */
/* relaxed Jacobi with int64 fixed-point accumulation (CEG:31-169)    */
/* ------------------------------------------------------------------ */
/* _acc, CEG:31-38 */
static inline void acc3(int64_t *ax, int64_t *ay, int64_t *az, int b, v3 d, float sign, float scale)
{
    double sc = (double)(sign * scale);
    ax[b] += (int64_t)round((double)d.x * sc);
    ay[b] += (int64_t)round((double)d.y * sc);
    az[b] += (int64_t)round((double)d.z * sc);
}

typedef struct {
    int64_t *a[6];
} accum_t;

/* k_jac_vel, CEG:81-131 */
static void jacobi_velocity(const contacts_t *c, float *jn, float *jt1, float *jt2, const float *xc, const float *v,
                            const float *w, const float *invIw, const float *invM, float mu, float scale, accum_t *A)
{
    int fvt = g_fv[FV_SITE_VT], ft1 = g_fv[FV_SITE_T1], fmag = g_fv[FV_SITE_MAG], fjt = g_fv[FV_SITE_JT];
    for (int k = 0; k < c->C; ++k) {
        int bi = c->bi[k], bj = c->bj[k];
        v3 nrm = ld3(c->n, k);
        v3 rA = vsub(ld3(c->pA, k), ld3(xc, bi));
        float iMA = invM[bi];
        m33 IA = ldm(invIw, bi), IB;
        v3 va = vadd(ld3(v, bi), cross3(ld3(w, bi), rA));
        v3 vb = V(0, 0, 0), rB = V(0, 0, 0);
        float iMB = 0.0f;
        if (bj >= 0) {
            rB = vsub(ld3(c->pB, k), ld3(xc, bj));
            vb = vadd(ld3(v, bj), cross3(ld3(w, bj), rB));
            iMB = invM[bj];
            IB = ldm(invIw, bj);
        }
        v3 vrel = vsub(va, vb);
        float vn = dot3(vrel, nrm);
        v3 vt = V(msub(fvt, vrel.x, vn, nrm.x), msub(fvt, vrel.y, vn, nrm.y), msub(fvt, vrel.z, vn, nrm.z));
        float mt = len3(vt);
        v3 t1 = vdivs(vt, mt);
        if (mt <= 5e-3f) {
            v3 aa = V(1.0f, 0.0f, 0.0f);
            if (fabsf(nrm.x) >= 0.9f) aa = V(0.0f, 1.0f, 0.0f);
            float dd = dot3(aa, nrm);
            t1 = vnormalize(V(msub(ft1, aa.x, dd, nrm.x), msub(ft1, aa.y, dd, nrm.y), msub(ft1, aa.z, dd, nrm.z)));
        }
        v3 t2 = cross3(nrm, t1);
        v3 rnA = cross3(rA, nrm);
        float meff = iMA + dot3(rnA, matvec(&IA, rnA));
        v3 rnB;
        if (bj >= 0) {
            rnB = cross3(rB, nrm);
            meff = (meff + iMB) + dot3(rnB, matvec(&IB, rnB));
        }
        if (meff < 1e-12f) continue;
        float dj = -vn / meff;
        float nw = fmaxf(0.0f, jn[k] + dj);
        dj = nw - jn[k];
        jn[k] = nw;
        v3 Jn = vscale(nrm, dj);
        acc3(A->a[0], A->a[1], A->a[2], bi, vscale(Jn, iMA), 1.0f, scale);
        acc3(A->a[3], A->a[4], A->a[5], bi, matvec(&IA, cross3(rA, Jn)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A->a[0], A->a[1], A->a[2], bj, vscale(Jn, iMB), -1.0f, scale);
            acc3(A->a[3], A->a[4], A->a[5], bj, matvec(&IB, cross3(rB, Jn)), -1.0f, scale);
        }
        v3 rtA1 = cross3(rA, t1);
        float meft1 = iMA + dot3(rtA1, matvec(&IA, rtA1));
        v3 rtA2 = cross3(rA, t2);
        float meft2 = iMA + dot3(rtA2, matvec(&IA, rtA2));
        if (bj >= 0) {
            v3 rtB1 = cross3(rB, t1);
            meft1 = (meft1 + iMB) + dot3(rtB1, matvec(&IB, rtB1));
            v3 rtB2 = cross3(rB, t2);
            meft2 = (meft2 + iMB) + dot3(rtB2, matvec(&IB, rtB2));
        }
        float o1 = jt1[k], o2 = jt2[k];
        float a1 = o1 - dot3(vrel, t1) / meft1;
        float a2 = o2 - dot3(vrel, t2) / meft2;
        float mag = sqrtf(fmag ? fmaf(a1, a1, a2 * a2) : a1 * a1 + a2 * a2);
        float lim = mu * jn[k];
        if (mag > lim && mag > 1e-12f) {
            a1 = a1 * lim / mag;
            a2 = a2 * lim / mag;
        }
        jt1[k] = a1;
        jt2[k] = a2;
        float e1 = a1 - o1, e2 = 0.5f * (a2 - o2);
        v3 Jt;
        if (fjt) Jt = V(fmaf(e1, t1.x, e2 * t2.x), fmaf(e1, t1.y, e2 * t2.y), fmaf(e1, t1.z, e2 * t2.z));
        else Jt = vadd(vscale(t1, e1), vscale(t2, e2));
        acc3(A->a[0], A->a[1], A->a[2], bi, vscale(Jt, iMA), 1.0f, scale);
        acc3(A->a[3], A->a[4], A->a[5], bi, matvec(&IA, cross3(rA, Jt)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A->a[0], A->a[1], A->a[2], bj, vscale(Jt, iMB), -1.0f, scale);
            acc3(A->a[3], A->a[4], A->a[5], bj, matvec(&IB, cross3(rB, Jt)), -1.0f, scale);
        }
    }
}

/* k_apply, CEG:133-143 */
static void jacobi_apply(int N, float *v, float *w, float relax, float scale, accum_t *A)
{
    int f = g_fv[FV_SITE_APPLY];
    float inv = 1.0f / scale;
    for (int i = 0; i < N; ++i) {
        float d[6];
        for (int k = 0; k < 6; ++k) d[k] = (float)((double)A->a[k][i] * (double)inv);
        v3 a = ld3(v, i), b = ld3(w, i);
        st3(v, i, V(mad(f, relax, d[0], a.x), mad(f, relax, d[1], a.y), mad(f, relax, d[2], a.z)));
        st3(w, i, V(mad(f, relax, d[3], b.x), mad(f, relax, d[4], b.y), mad(f, relax, d[5], b.z)));
        for (int k = 0; k < 6; ++k) A->a[k][i] = 0;
    }
}

/* k_jac_pos, CEG:145-169 */
static void jacobi_position(const contacts_t *c, float *jp, const float *xc, const float *pv, const float *po,
                            const float *invIw, const float *invM, float dt, float scale, accum_t *A)
{
    for (int k = 0; k < c->C; ++k) {
        int bi = c->bi[k], bj = c->bj[k];
        v3 nrm = ld3(c->n, k);
        v3 rA = vsub(ld3(c->pA, k), ld3(xc, bi));
        float iMA = invM[bi];
        m33 IA = ldm(invIw, bi), IB;
        v3 rel = vadd(ld3(pv, bi), cross3(ld3(po, bi), rA));
        v3 rB = V(0, 0, 0);
        float iMB = 0.0f;
        if (bj >= 0) {
            rB = vsub(ld3(c->pB, k), ld3(xc, bj));
            rel = vsub(rel, vadd(ld3(pv, bj), cross3(ld3(po, bj), rB)));
            iMB = invM[bj];
            IB = ldm(invIw, bj);
        }
        v3 rnA = cross3(rA, nrm);
        float meff = iMA + dot3(rnA, matvec(&IA, rnA));
        if (bj >= 0) {
            v3 rnB = cross3(rB, nrm);
            meff = (meff + iMB) + dot3(rnB, matvec(&IB, rnB));
        }
        if (meff < 1e-12f) continue;
        float bias = K_BETA * fmaxf(c->pen[k] - K_SLOP, 0.0f) / dt;
        float dj = (bias - dot3(rel, nrm)) / meff;
        float nw = fmaxf(0.0f, jp[k] + dj);
        dj = nw - jp[k];
        jp[k] = nw;
        v3 Jn = vscale(nrm, dj);
        acc3(A->a[0], A->a[1], A->a[2], bi, vscale(Jn, iMA), 1.0f, scale);
        acc3(A->a[3], A->a[4], A->a[5], bi, matvec(&IA, cross3(rA, Jn)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A->a[0], A->a[1], A->a[2], bj, vscale(Jn, iMB), -1.0f, scale);
            acc3(A->a[3], A->a[4], A->a[5], bj, matvec(&IB, cross3(rB, Jn)), -1.0f, scale);
        }
    }
}

/* ------------------------------------------------------------------ */
/* one Jacobi step: RelaxedJacobiContactEngine.step, CEG:252-280       */
/* ------------------------------------------------------------------ */
OR_API int or_jacobi_step(int N, int nbead, const float *rest, const int *owner, float *xc, float *q, float *v,
                          float *w, float *pv, float *po, const float *invM, const float *IbInv, const int *kin,
                          const double *M,
                          double dt, int substeps, int vit, int pit, float relax, float mu, int maxc,
                          double *force, int *ncontacts)
{
    float *invIw = malloc(sizeof(float) * 9 * (size_t)N);
    float *allp = malloc(sizeof(float) * 3 * (size_t)nbead);
    /* pv/po persist across calls: the reference zeroes them only in a substep that has contacts */
    float *vgrav = malloc(sizeof(float) * 3 * (size_t)N);
    contacts_t c;
    c.cap = maxc;
    c.bi = malloc(sizeof(int) * maxc); c.bj = malloc(sizeof(int) * maxc);
    c.fa = malloc(sizeof(int) * maxc); c.fb = malloc(sizeof(int) * maxc);
    c.pA = malloc(sizeof(float) * 3 * maxc); c.pB = malloc(sizeof(float) * 3 * maxc);
    c.n = malloc(sizeof(float) * 3 * maxc); c.pen = malloc(sizeof(float) * maxc);
    float *jn = malloc(sizeof(float) * maxc), *jt1 = malloc(sizeof(float) * maxc);
    float *jt2 = malloc(sizeof(float) * maxc), *jp = malloc(sizeof(float) * maxc);
    accum_t A;
    for (int k = 0; k < 6; ++k) A.a[k] = calloc((size_t)N, sizeof(int64_t));
    for (int s = 0; s < substeps; ++s) {
        double sdt_d = dt / substeps;
        float sdt = (float)sdt_d;
        body_gravity(N, v, invM, sdt);
        body_inv_inertia(N, q, IbInv, kin, invIw);
        bead_world(nbead, xc, q, rest, owner, allp);
        gen_contacts(nbead, allp, owner, &c);
        int C = c.C;
        if (ncontacts) ncontacts[s] = C + c.overflow;
        memcpy(vgrav, v, sizeof(float) * 3 * N);
        if (C > 0) {
            memset(jn, 0, sizeof(float) * C); memset(jt1, 0, sizeof(float) * C);
            memset(jt2, 0, sizeof(float) * C); memset(jp, 0, sizeof(float) * C);
            memset(pv, 0, sizeof(float) * 3 * N); memset(po, 0, sizeof(float) * 3 * N);
            for (int k = 0; k < 6; ++k) memset(A.a[k], 0, sizeof(int64_t) * N);
            for (int it = 0; it < vit; ++it) {
                jacobi_velocity(&c, jn, jt1, jt2, xc, v, w, invIw, invM, mu, K_SCALE, &A);
                jacobi_apply(N, v, w, relax, K_SCALE, &A);
            }
            for (int it = 0; it < pit; ++it) {
                jacobi_position(&c, jp, xc, pv, po, invIw, invM, sdt, K_SCALE, &A);
                jacobi_apply(N, pv, po, relax, K_SCALE, &A);
            }
        }
        body_integrate(N, xc, q, v, w, pv, po, invM, sdt);
        /* contact force on the host in float64: M * (v_post - v_grav) / sdt, kinematic rows 0 */
        for (int i = 0; i < N; ++i)
            for (int k = 0; k < 3; ++k) {
                float dvf = v[3 * i + k] - vgrav[3 * i + k];
                force[3 * i + k] = kin[i] ? 0.0 : (M[i] * (double)dvf) / sdt_d;
            }
    }
    free(invIw); free(allp); free(vgrav);
    free(c.bi); free(c.bj); free(c.fa); free(c.fb); free(c.pA); free(c.pB); free(c.n); free(c.pen);
    free(jn); free(jt1); free(jt2); free(jp);
    for (int k = 0; k < 6; ++k) free(A.a[k]);
    return c.overflow ? 2 : 0;
}
