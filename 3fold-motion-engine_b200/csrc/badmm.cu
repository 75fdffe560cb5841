// Batched proximal ADMM for many small contact problems, with its adjoint: the reference's
// BatchProxADMMGPU (src/motion_engine/ncp/ncp_batch_gpu.py:918-1313, "NB").
//
// The reference runs every step as a separate kernel over the whole batch (133 launches per
// ADMM iteration, ~35 000 graph nodes per step and gradient).  Here ONE warp owns one problem
// for the whole solve: its J (3 nc x nv), M^-1 (nv x nv), M^-1 J^T, the dense Delassus G and
// every vector live in the warp's shared memory, the set-up, the ADMM iterations, the refreshes,
// the active set and both gradient directions run in one launch, and the only synchronisation
// is __syncwarp.  The arithmetic is the reference's, float64:
//  * set-up (NB:974-1000): b = J v_free, the scale bound kappa, M^-1 J^T (k_mj), G (k_gdense),
//    G's spectrum by cyclic Jacobi in the fixed pair order (k_jacobi; the rotations' row and
//    column updates spread over the lanes), the diagonal blocks and their largest eigenvalue
//    (k_gd3, f_eigmax), eta and the per-contact step (k_eta), the bilateral regime test by a
//    Cholesky solve (k_bilat), rho (k_rho), the block-Jacobi preconditioner (k_pjac);
//  * the matrix-free product G x + (eta + rho) x (NB:326-388): y = J^T x per contact, then
//    M^-1 y per contact rounded at a power-of-two scale 2^floor(log2(2^52 / (kappa |x|inf)))
//    and summed in int64 (exact: the sum does not depend on the order), w = acc / scale, then J w;
//  * ADMM (NB:466-543, 1075-1099): x-step by block-Jacobi preconditioned CG warm-started from
//    the last x, z = proj_K(x + gamma / rho), gamma += rho (x - z), and every `refresh_every`
//    iterations u = G z + b, the slip speeds, the natural residual and the convergence mask (a
//    converged problem freezes x, z and gamma);
//  * the gradient (NB:556-808, 1145-1206): the active set (open / stick / slip with its
//    projector Z and diagonal D), the Schur preconditioner, and grad_affine -- the de Saxce
//    sigma map is affine, so it is solved by 1 + n_calls - 2 + 1 applications of the
//    CG-solved fixed-branch system and one (I - B) sigma = a elimination -- for the direction
//    db = dt J M^-1 e_j (and v+'s response) and for mu at each problem's first slip contact.
#include <math_constants.h>

#include "b2c_common.cuh"

namespace b2c {
namespace badmm {

constexpr double kTiny = 1.0e-300;
constexpr double kScaleBound = 4.503599627370496e15;  // 2^52

// one problem's working set in the warp's shared memory
struct Env {
    double *J, *Mi, *MJ, *G, *A, *yt, *wv, *vf;
    double *bb, *x, *zv, *gam, *r, *zz, *pv, *Ap, *rhs, *tmp, *tmp2, *u, *pinh, *dbv, *ZtHp, *yv, *dlam, *Dv, *what,
        *bw, *ev;
    double *mu, *s, *eta, *rhoc, *slipf, *sig, *sigo, *siga, *res, *gnorm;
    double *Gd, *Pj, *Zm, *Ps;  // 9 per contact, row-major
    double *Bm, *Aw, *rw;
    int *sidx;
    int C, NV, M;
    double kap, rho;
    int mask, nslip;
};

__host__ __device__ inline size_t env_doubles(int C, int NV)
{
    const size_t M = 3 * (size_t)C;
    return M * NV * 2 + (size_t)NV * NV + M * M * 2 + (size_t)C * NV + 2 * (size_t)NV + 24 * M + 10 * (size_t)C +
           36 * (size_t)C + 2 * (size_t)C * C + C;
}
__host__ __device__ inline size_t env_bytes(int C, int NV)
{
    return env_doubles(C, NV) * 8 + (size_t)C * 4 + 16;
}

__device__ inline Env carve(double *base, int C, int NV)
{
    Env E;
    E.C = C;
    E.NV = NV;
    E.M = 3 * C;
    const int M = E.M;
    double *p = base;
    auto take = [&](size_t n) {
        double *q = p;
        p += n;
        return q;
    };
    E.J = take((size_t)M * NV);
    E.MJ = take((size_t)M * NV);
    E.Mi = take((size_t)NV * NV);
    E.G = take((size_t)M * M);
    E.A = take((size_t)M * M);
    E.yt = take((size_t)C * NV);
    E.wv = take(NV);
    E.vf = take(NV);
    double **vecs[] = {&E.bb, &E.x, &E.zv, &E.gam, &E.r, &E.zz, &E.pv, &E.Ap, &E.rhs, &E.tmp, &E.tmp2, &E.u,
                       &E.pinh, &E.dbv, &E.ZtHp, &E.yv, &E.dlam, &E.Dv, &E.what, &E.bw, &E.ev};
    for (double **v : vecs) *v = take(M);
    take(3 * (size_t)M);  // (24 vectors of M reserved)
    double **cvec[] = {&E.mu, &E.s, &E.eta, &E.rhoc, &E.slipf, &E.sig, &E.sigo, &E.siga, &E.res, &E.gnorm};
    for (double **v : cvec) *v = take(C);
    E.Gd = take(9 * (size_t)C);
    E.Pj = take(9 * (size_t)C);
    E.Zm = take(9 * (size_t)C);
    E.Ps = take(9 * (size_t)C);
    E.Bm = take((size_t)C * C);
    E.Aw = take((size_t)C * C);
    E.rw = take(C);
    E.sidx = reinterpret_cast<int *>(p);
    E.kap = 0.0;
    E.rho = 0.0;
    E.mask = 1;
    E.nslip = 0;
    return E;
}

__device__ __forceinline__ int lane_id() { return (int)(threadIdx.x & 31); }
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// f_proj (NB:113-126)
__device__ __forceinline__ void proj3(const double z[3], double mu, double out[3])
{
    const double zn = z[0], zt = sqrt(z[1] * z[1] + z[2] * z[2]);
    if (zt <= mu * zn) {
        out[0] = z[0];
        out[1] = z[1];
        out[2] = z[2];
    } else if (mu * zt <= -zn) {
        out[0] = out[1] = out[2] = 0.0;
    } else {
        const double s = (zn + mu * zt) / (1.0 + mu * mu);
        const double f = mu * s / zt;
        out[0] = s;
        out[1] = f * z[1];
        out[2] = f * z[2];
    }
}

// 3x3 inverse (adjugate over determinant; zero when singular)
__device__ inline void inv3(const double a[9], double o[9])
{
    const double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[2] * a[7] - a[1] * a[8], c02 = a[1] * a[5] - a[2] * a[4];
    const double c10 = a[5] * a[6] - a[3] * a[8], c11 = a[0] * a[8] - a[2] * a[6], c12 = a[2] * a[3] - a[0] * a[5];
    const double c20 = a[3] * a[7] - a[4] * a[6], c21 = a[1] * a[6] - a[0] * a[7], c22 = a[0] * a[4] - a[1] * a[3];
    const double det = a[0] * c00 + a[1] * c10 + a[2] * c20;
    const double adj[9] = {c00, c01, c02, c10, c11, c12, c20, c21, c22};
    for (int i = 0; i < 9; ++i) o[i] = det != 0.0 ? adj[i] / det : 0.0;
}

// f_eigmax (NB:130-146): largest eigenvalue of a symmetric 3x3 block, closed form
__device__ inline double eigmax3(const double A[9])
{
    const double p1 = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    const double q = (A[0] + A[4] + A[8]) / 3.0;
    double out = fmax(A[0], fmax(A[4], A[8]));
    if (p1 > 0.0) {
        const double p2 = (A[0] - q) * (A[0] - q) + (A[4] - q) * (A[4] - q) + (A[8] - q) * (A[8] - q) + 2.0 * p1;
        const double p = sqrt(p2 / 6.0);
        if (p > 1.0e-300) {
            double Bm[9];
            for (int i = 0; i < 9; ++i) Bm[i] = (A[i] - ((i % 4) == 0 ? q : 0.0)) / p;
            const double det = Bm[0] * (Bm[4] * Bm[8] - Bm[5] * Bm[7]) - Bm[1] * (Bm[3] * Bm[8] - Bm[5] * Bm[6]) +
                               Bm[2] * (Bm[3] * Bm[7] - Bm[4] * Bm[6]);
            const double r = fmin(1.0, fmax(-1.0, det / 2.0));
            out = q + 2.0 * p * cos(acos(r) / 3.0);
        }
    }
    return out;
}

// the matrix-free product (k_scale, k_jt, k_mscat, k_acc2w, k_gath): xout = G xin + (eta + rho') xin.
// Lane k (< nv) owns row k of M^-1: it forms every contact's M^-1 (J^T x)_c entry k with the
// contacts' sums interleaved (independent chains), rounds each at the scale and adds them in its
// own int64 register -- exact, so no atomics and no order dependence.  The scale is a power of
// two, so acc / scale is the exact product acc * 2^-e.
template <int kC>
__device__ void matvec(Env &E, const double *xin, double *xout, bool use_rho)
{
    const int ln = lane_id(), C = E.C, NV = E.NV, M = E.M;
    double m = ln < M ? fabs(xin[ln]) : 0.0;
    m = warp_max(m);
    const double t = E.kap * m;
    double scal = 1.0, inv = 1.0;
    if (t > 0.0) {
        int e = ilogb(kScaleBound / t);  // floor(log2(2^52 / t)), exactly
        e = e < -1000 ? -1000 : (e > 1000 ? 1000 : e);
        scal = ldexp(1.0, e);
        inv = ldexp(1.0, -e);
    }
    if (ln < NV) {
#pragma unroll
        for (int c = 0; c < kC; ++c) {
            const double *jr = E.J + (size_t)(3 * c) * NV + ln;
            E.yt[c * NV + ln] = jr[0] * xin[3 * c] + jr[NV] * xin[3 * c + 1] + jr[2 * NV] * xin[3 * c + 2];
        }
    }
    __syncwarp();
    if (ln < NV) {
        double sc[kC];
#pragma unroll
        for (int c = 0; c < kC; ++c) sc[c] = 0.0;
        const double *mrow = E.Mi + (size_t)ln * NV;
        for (int l = 0; l < NV; ++l) {
            const double ml = mrow[l];
#pragma unroll
            for (int c = 0; c < kC; ++c) sc[c] = sc[c] + ml * E.yt[c * NV + l];
        }
        long long acc = 0;
#pragma unroll
        for (int c = 0; c < kC; ++c) acc += llround(sc[c] * scal);
        E.wv[ln] = (double)acc * inv;
    }
    __syncwarp();
    const double rr = use_rho ? E.rho : 0.0;
    if (ln < M) {
        double u = 0.0;
        const double *jrow = E.J + (size_t)ln * NV;
        for (int k = 0; k < NV; ++k) u = u + jrow[k] * E.wv[k];
        xout[ln] = u + (E.eta[ln / 3] + rr) * xin[ln];
    }
    __syncwarp();
}

// k_dot (NB:408-416): the products lane by lane, summed by a butterfly; IEEE addition is
// commutative, so every lane ends with the same bits
__device__ __forceinline__ double dot(const Env &E, const double *a, const double *b)
{
    const int ln = lane_id();
    double s = ln < E.M ? a[ln] * b[ln] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = s + __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// k_papply: z = P r per contact
__device__ __forceinline__ void papply(const Env &E, const double *P, const double *r, double *z)
{
    for (int i = lane_id(); i < E.M; i += 32) {
        const int c = i / 3, row = i - 3 * c;
        const double *p = P + 9 * c + 3 * row;
        z[i] = p[0] * r[3 * c] + p[1] * r[3 * c + 1] + p[2] * r[3 * c + 2];
    }
    __syncwarp();
}

// the Schur operator of the fixed-branch system (NB:1040-1043): yout = Z^T G Z y + D y
template <int kC>
__device__ void sopv(Env &E, const double *y, double *yout)
{
    const int ln = lane_id();
    for (int i = ln; i < E.M; i += 32) {
        const int c = i / 3, row = i - 3 * c;
        const double *z = E.Zm + 9 * c + 3 * row;
        E.tmp[i] = z[0] * y[3 * c] + z[1] * y[3 * c + 1] + z[2] * y[3 * c + 2];
    }
    __syncwarp();
    matvec<kC>(E, E.tmp, E.tmp2, false);
    for (int i = ln; i < E.M; i += 32) {
        const int c = i / 3, col = i - 3 * c;
        const double *z = E.Zm + 9 * c;
        const double t = z[col] * E.tmp2[3 * c] + z[3 + col] * E.tmp2[3 * c + 1] + z[6 + col] * E.tmp2[3 * c + 2];
        yout[i] = t + E.Dv[i] * y[i];
    }
    __syncwarp();
}

enum Op { kOpAdmm = 0, kOpSchur = 1 };

// _pcg (NB:1048-1073); the x update skips a frozen problem when use_mask
template <int kC>
__device__ void pcg(Env &E, const double *rhs, double *x, int n_it, Op op, const double *P, bool warm_zero,
                    bool use_mask)
{
    const int ln = lane_id(), M = E.M;
    auto apply = [&](const double *v, double *o) {
        if (op == kOpAdmm) matvec<kC>(E, v, o, true);
        else sopv<kC>(E, v, o);
    };
    if (warm_zero) {
        for (int i = ln; i < M; i += 32) {
            x[i] = 0.0;
            E.r[i] = rhs[i];
        }
        __syncwarp();
    } else {
        apply(x, E.Ap);
        for (int i = ln; i < M; i += 32) E.r[i] = rhs[i] - E.Ap[i];
        __syncwarp();
    }
    papply(E, P, E.r, E.zz);
    for (int i = ln; i < M; i += 32) E.pv[i] = E.zz[i];
    __syncwarp();
    double s0 = dot(E, E.r, E.zz);
    const bool upd = !use_mask || E.mask != 0;
    for (int it = 0; it < n_it; ++it) {
        apply(E.pv, E.Ap);
        const double s1 = dot(E, E.pv, E.Ap);
        const double s2 = (s1 > 0.0 || s1 < 0.0) ? s0 / s1 : 0.0;
        for (int i = ln; i < M; i += 32) {
            if (upd) x[i] = x[i] + 1.0 * s2 * E.pv[i];
            E.r[i] = E.r[i] + -1.0 * s2 * E.Ap[i];
        }
        __syncwarp();
        papply(E, P, E.r, E.zz);
        const double s3 = dot(E, E.r, E.zz);
        const double s4 = (s0 > 0.0 || s0 < 0.0) ? s3 / s0 : 0.0;
        for (int i = ln; i < M; i += 32) E.pv[i] = E.zz[i] + s4 * E.pv[i];
        __syncwarp();
        s0 = s3;
    }
}

// one ADMM iteration (NB:1075-1082)
template <int kC>
__device__ void admm_iter(Env &E, int cg_iters)
{
    const int ln = lane_id(), M = E.M;
    for (int i = ln; i < M; i += 32) {
        const int c = i / 3;
        const double g = E.bb[i] + ((i - 3 * c) == 0 ? E.mu[c] * E.s[c] : 0.0);
        E.rhs[i] = -((g + E.gam[i]) - E.rho * E.zv[i]);
    }
    __syncwarp();
    pcg<kC>(E, E.rhs, E.x, cg_iters, kOpAdmm, E.Pj, false, true);
    if (E.mask != 0) {
        for (int c = ln; c < E.C; c += 32) {
            double v[3], z[3];
            for (int k = 0; k < 3; ++k) v[k] = E.x[3 * c + k] + E.gam[3 * c + k] / E.rho;
            proj3(v, E.mu[c], z);
            for (int k = 0; k < 3; ++k) E.zv[3 * c + k] = z[k];
        }
        __syncwarp();
        for (int i = ln; i < M; i += 32) E.gam[i] = E.gam[i] + E.rho * (E.x[i] - E.zv[i]);
        __syncwarp();
    }
}

// the Cadoux refresh, the natural residual and the mask (NB:1084-1092, 498-543)
template <int kC>
__device__ double refresh(Env &E, double tol, bool desax)
{
    const int ln = lane_id();
    matvec<kC>(E, E.zv, E.tmp2, false);
    for (int i = ln; i < E.M; i += 32) E.u[i] = E.tmp2[i] + E.bb[i];
    __syncwarp();
    for (int c = ln; c < E.C; c += 32) {
        const double *uu = E.u + 3 * c;
        const double ut = sqrt(uu[1] * uu[1] + uu[2] * uu[2]);
        E.s[c] = ut;
        double w[3] = {uu[0], uu[1], uu[2]};
        if (desax) w[0] = uu[0] + E.mu[c] * ut;
        double q[3], pr[3];
        for (int k = 0; k < 3; ++k) q[k] = E.zv[3 * c + k] - E.rhoc[c] * w[k];
        proj3(q, E.mu[c], pr);
        const double d0 = fabs(E.zv[3 * c] - pr[0]), d1 = fabs(E.zv[3 * c + 1] - pr[1]),
                     d2 = fabs(E.zv[3 * c + 2] - pr[2]);
        E.res[c] = fmax(d0, fmax(d1, d2));
    }
    __syncwarp();
    double m = 0.0;
    for (int c = 0; c < E.C; ++c) {  // NaN-propagating maximum (k_resmax)
        const double v = E.res[c];
        if (v != v) m = v;
        else if (v > m) m = v;
    }
    if (E.mask == 1 && m < tol) E.mask = 0;
    return m;
}

// set-up of one problem (NB:974-1000, 1013-1022, k_pjac)
__device__ void setup(Env &E, const b2c_admm &P, const b2c_admm_params &prm, int e)
{
    const int ln = lane_id(), C = E.C, NV = E.NV, M = E.M;
    const double *Jg = P.J + (size_t)e * M * NV, *Mg = P.Minv + (size_t)e * NV * NV, *vg = P.v_free + (size_t)e * NV;
    for (int i = ln; i < M * NV; i += 32) E.J[i] = Jg[i];
    for (int i = ln; i < NV * NV; i += 32) E.Mi[i] = Mg[i];
    for (int i = ln; i < NV; i += 32) E.vf[i] = vg[i];
    for (int c = ln; c < C; c += 32) E.mu[c] = P.mu[(size_t)e * C + c];
    __syncwarp();
    for (int i = ln; i < M; i += 32) {
        double s = 0.0;
        for (int k = 0; k < NV; ++k) s = s + E.J[i * NV + k] * E.vf[k];
        E.bb[i] = P.b_in ? P.b_in[(size_t)e * M + i] : s;
    }
    // kappa = C max_i sum_l |M^-1_il| max_(c,k) sum_r |J_(3c+r)k| + 1e-300
    double m1 = 0.0, m2 = 0.0;
    for (int i = ln; i < NV; i += 32) {
        double s = 0.0;
        for (int l = 0; l < NV; ++l) s = s + fabs(E.Mi[i * NV + l]);
        m1 = fmax(m1, s);
    }
    for (int q = ln; q < C * NV; q += 32) {
        const int c = q / NV, k = q - c * NV;
        m2 = fmax(m2, fabs(E.J[(3 * c) * NV + k]) + fabs(E.J[(3 * c + 1) * NV + k]) + fabs(E.J[(3 * c + 2) * NV + k]));
    }
    m1 = warp_max(m1);
    m2 = warp_max(m2);
    E.kap = (double)C * m1 * m2 + 1e-300;
    // M^-1 J^T (k_mj) and G = J M^-1 J^T (k_gdense)
    for (int q = ln; q < M * NV; q += 32) {
        const int i = q / NV, k = q - i * NV;
        double s = 0.0;
        for (int l = 0; l < NV; ++l) s = s + E.Mi[k * NV + l] * E.J[i * NV + l];
        E.MJ[q] = s;
    }
    __syncwarp();
    for (int q = ln; q < M * M; q += 32) {
        const int i = q / M, j = q - i * M;
        double s = 0.0;
        for (int k = 0; k < NV; ++k) s = s + E.J[i * NV + k] * E.MJ[j * NV + k];
        E.G[q] = s;
        E.A[q] = s;
    }
    __syncwarp();
    // spectrum: cyclic Jacobi in the fixed pair order (k_jacobi); lane k updates row / column k
    for (int sw = 0; sw < prm.jacobi_sweeps; ++sw)
        for (int p = 0; p < M - 1; ++p)
            for (int q = p + 1; q < M; ++q) {
                const double apq = E.A[p * M + q];
                if (apq > kTiny || apq < -kTiny) {
                    const double app = E.A[p * M + p], aqq = E.A[q * M + q];
                    const double th = (aqq - app) / (2.0 * apq);
                    double t = 1.0 / (fabs(th) + sqrt(th * th + 1.0));
                    if (th < 0.0) t = -t;
                    const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
                    __syncwarp();
                    for (int k = ln; k < M; k += 32) {
                        const double akp = E.A[k * M + p], akq = E.A[k * M + q];
                        E.A[k * M + p] = c * akp - sn * akq;
                        E.A[k * M + q] = sn * akp + c * akq;
                    }
                    __syncwarp();
                    for (int k = ln; k < M; k += 32) {
                        const double apk = E.A[p * M + k], aqk = E.A[q * M + k];
                        E.A[p * M + k] = c * apk - sn * aqk;
                        E.A[q * M + k] = sn * apk + c * aqk;
                    }
                    __syncwarp();
                }
            }
    for (int i = ln; i < M; i += 32) E.ev[i] = E.A[i * M + i];
    // diagonal blocks, their largest eigenvalue, eta, the per-contact step (k_gd3, k_eta)
    for (int c = ln; c < C; c += 32) {
        double W[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) W[3 * i + j] = E.G[(3 * c + i) * M + 3 * c + j];
        for (int i = 0; i < 9; ++i) E.Gd[9 * c + i] = W[i];
        const double gn = eigmax3(W);
        E.gnorm[c] = gn;
        E.eta[c] = prm.alpha_eta * gn;
        const double s = gn + E.eta[c];
        E.rhoc[c] = s > 0.0 ? 1.0 / s : 1.0;
    }
    __syncwarp();
    // the regime (k_bilat): Cholesky of G with floored pivots, then -G^-1 b against the cones;
    // run by lane 0 (a 3 nc x 3 nc factorisation)
    int bind = 0;
    if (prm.rho_mode == B2C_ADMM_RHO_REGIME) {
        if (ln == 0) {
            for (int i = 0; i < M * M; ++i) E.A[i] = E.G[i];
            for (int k = 0; k < M; ++k) {
                double d = E.A[k * M + k];
                for (int j = 0; j < k; ++j) d = d - E.A[k * M + j] * E.A[k * M + j];
                if (d < kTiny) d = kTiny;
                d = sqrt(d);
                E.A[k * M + k] = d;
                for (int i = k + 1; i < M; ++i) {
                    double s = E.A[i * M + k];
                    for (int j = 0; j < k; ++j) s = s - E.A[i * M + j] * E.A[k * M + j];
                    E.A[i * M + k] = s / d;
                }
            }
            for (int i = 0; i < M; ++i) {
                double s = -E.bb[i];
                for (int j = 0; j < i; ++j) s = s - E.A[i * M + j] * E.bw[j];
                E.bw[i] = s / E.A[i * M + i];
            }
            for (int ii = 0; ii < M; ++ii) {
                const int i = M - 1 - ii;
                double s = E.bw[i];
                for (int j = i + 1; j < M; ++j) s = s - E.A[j * M + i] * E.bw[j];
                E.bw[i] = s / E.A[i * M + i];
            }
            for (int c = 0; c < C; ++c) {
                const double lnrm = E.bw[3 * c], lt = sqrt(E.bw[3 * c + 1] * E.bw[3 * c + 1] + E.bw[3 * c + 2] * E.bw[3 * c + 2]);
                if (lnrm <= 0.0 || lt > E.mu[c] * lnrm) bind = 1;
            }
        }
        bind = __shfl_sync(0xffffffffu, bind, 0);
    }
    // rho (k_rho): sqrt(lmin+ lmax) | lmin+ | lmax | the regime's choice
    double mx = -1.0e300;
    for (int i = 0; i < M; ++i) mx = fmax(mx, E.ev[i]);
    const double thr = 1e-12 * mx;
    double mn = mx;
    for (int i = 0; i < M; ++i) {
        const double v = E.ev[i];
        if (v > thr && v < mn) mn = v;
    }
    double rho = sqrt(mn * mx);
    if (prm.rho_mode == B2C_ADMM_RHO_LMIN) rho = mn;
    if (prm.rho_mode == B2C_ADMM_RHO_LMAX) rho = mx;
    if (prm.rho_mode == B2C_ADMM_RHO_REGIME) rho = bind ? mx : mn;
    if (prm.rho_mode == B2C_ADMM_RHO_GIVEN) rho = P.rho[e];
    E.rho = rho;
    // block-Jacobi preconditioner (k_pjac) and the reset (NB:1100-1110)
    for (int c = ln; c < C; c += 32) {
        double W[9];
        const double sh = E.eta[c] + rho;
        for (int i = 0; i < 9; ++i) W[i] = E.Gd[9 * c + i] + ((i % 4) == 0 ? sh : 0.0);
        inv3(W, E.Pj + 9 * c);
    }
    for (int i = ln; i < M; i += 32) {
        E.gam[i] = 0.0;
        E.zv[i] = 0.0;
        E.x[i] = 0.0;
        E.u[i] = 0.0;
    }
    for (int c = ln; c < C; c += 32) E.s[c] = 0.0;
    E.mask = 1;
    __syncwarp();
}

// the active set (k_lamscale, k_active, k_slipidx, k_sjac: NB:546-627), from lam = zv and u
__device__ void build_active(Env &E, double tol_lam, double tol_rel)
{
    const int ln = lane_id(), C = E.C;
    double lsc = 1.0e-30;
    for (int i = 0; i < E.M; ++i) lsc = fmax(lsc, fabs(E.zv[i]));
    for (int c = ln; c < C; c += 32) {
        const double *L = E.zv + 3 * c;
        const double lnrm = L[0], lt = sqrt(L[1] * L[1] + L[2] * L[2]);
        double Z[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double D[3] = {0, 0, 0}, wh[3] = {0, 0, 0}, sf = 0.0;
        const double mu = E.mu[c];
        if (lnrm <= tol_lam + tol_rel * lsc) {  // open
            D[0] = D[1] = D[2] = 1.0;
        } else if (lt >= mu * lnrm * (1.0 - tol_rel) - tol_lam) {  // slip
            const double w1 = E.u[3 * c + 1], w2 = E.u[3 * c + 2];
            double nw = sqrt(w1 * w1 + w2 * w2);
            if (nw < 1.0e-300) nw = 1.0e-300;
            const double h1 = w1 / nw, h2 = w2 / nw;
            Z[0] = 1.0;
            Z[3] = -mu * h1;
            Z[6] = -mu * h2;
            Z[4] = -h2;
            Z[7] = h1;
            D[1] = nw / fmax(mu * lnrm, 1.0e-300);
            D[2] = 1.0;
            sf = 1.0;
            wh[1] = h1;
            wh[2] = h2;
        } else {  // stick
            Z[0] = Z[4] = Z[8] = 1.0;
        }
        for (int i = 0; i < 9; ++i) E.Zm[9 * c + i] = Z[i];
        for (int k = 0; k < 3; ++k) {
            E.Dv[3 * c + k] = D[k];
            E.what[3 * c + k] = wh[k];
        }
        E.slipf[c] = sf;
        // Schur preconditioner: (Z^T (Gd + eta I) Z + diag D)^-1
        double Q[9], T[9], S[9];
        for (int i = 0; i < 9; ++i) Q[i] = E.Gd[9 * c + i] + ((i % 4) == 0 ? E.eta[c] : 0.0);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s = s + Z[3 * k + i] * Q[3 * k + j];
                T[3 * i + j] = s;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s = s + T[3 * i + k] * Z[3 * k + j];
                S[3 * i + j] = s;
            }
        S[0] += D[0];
        S[4] += D[1];
        S[8] += D[2];
        inv3(S, E.Ps + 9 * c);
    }
    __syncwarp();
    int n = 0;
    for (int c = 0; c < C; ++c)
        if (E.slipf[c] > 0.5) {
            if (ln == 0) E.sidx[n] = c;
            ++n;
        }
    for (int c = n + ln; c < C; c += 32) E.sidx[c] = -1;
    E.nslip = n;
    __syncwarp();
}

// one application of the affine sigma map (NB:1162-1170)
template <int kC>
__device__ void grad_once(Env &E, int cg)
{
    const int ln = lane_id(), M = E.M;
    for (int i = ln; i < M; i += 32) {
        const int c = i / 3;
        double v = -E.ZtHp[i];
        if (E.slipf[c] > 0.5 && i == 3 * c) v = v - E.mu[c] * E.sig[c];
        E.rhs[i] = v;
    }
    __syncwarp();
    pcg<kC>(E, E.rhs, E.yv, cg, kOpSchur, E.Ps, true, false);
    for (int i = ln; i < M; i += 32) {
        const int c = i / 3, row = i - 3 * c;
        const double *z = E.Zm + 9 * c + 3 * row;
        E.dlam[i] = (z[0] * E.yv[3 * c] + z[1] * E.yv[3 * c + 1] + z[2] * E.yv[3 * c + 2]) + E.pinh[i];
    }
    __syncwarp();
    matvec<kC>(E, E.dlam, E.tmp2, false);
    for (int c = ln; c < E.C; c += 32)
        E.sigo[c] = E.slipf[c] > 0.5 ? E.what[3 * c + 1] * (E.tmp2[3 * c + 1] + E.dbv[3 * c + 1]) +
                                            E.what[3 * c + 2] * (E.tmp2[3 * c + 2] + E.dbv[3 * c + 2])
                                      : 0.0;
    __syncwarp();
}

// grad_affine (NB:1172-1186): dlam for the current (pinh, dbv)
template <int kC>
__device__ void grad_affine(Env &E, int n_calls, int cg)
{
    const int ln = lane_id(), C = E.C, M = E.M;
    const int K = n_calls - 2;
    matvec<kC>(E, E.pinh, E.tmp, false);
    for (int i = ln; i < M; i += 32) E.tmp2[i] = E.tmp[i] + E.dbv[i];
    __syncwarp();
    for (int i = ln; i < M; i += 32) {
        const int c = i / 3, col = i - 3 * c;
        const double *z = E.Zm + 9 * c;
        E.ZtHp[i] = z[col] * E.tmp2[3 * c] + z[3 + col] * E.tmp2[3 * c + 1] + z[6 + col] * E.tmp2[3 * c + 2];
    }
    for (int c = ln; c < C; c += 32) E.sig[c] = 0.0;
    __syncwarp();
    grad_once<kC>(E, cg);
    for (int c = ln; c < C; c += 32) E.siga[c] = E.sigo[c];
    __syncwarp();
    for (int j = 0; j < K; ++j) {
        for (int c = ln; c < C; c += 32) E.sig[c] = 0.0;
        __syncwarp();
        if (ln == 0 && j >= 0 && j < E.nslip) E.sig[E.sidx[j]] = 1.0;
        __syncwarp();
        grad_once<kC>(E, cg);
        if (j < E.nslip)
            for (int i = ln; i < E.nslip; i += 32) {
                const int c = E.sidx[i];
                E.Bm[i * C + j] = E.sigo[c] - E.siga[c];
            }
        __syncwarp();
    }
    // (I - B) sigma = a over the slip contacts: Gauss with partial pivoting, lane 0 (k_solvesig)
    if (ln == 0) {
        for (int c = 0; c < C; ++c) E.sig[c] = 0.0;
        const int n = E.nslip;
        if (n > 0) {
            for (int i = 0; i < n; ++i) {
                for (int j = 0; j < n; ++j) E.Aw[i * C + j] = (i == j ? 1.0 : 0.0) - E.Bm[i * C + j];
                E.rw[i] = E.siga[E.sidx[i]];
            }
            for (int k = 0; k < n; ++k) {
                int piv = k;
                double big = fabs(E.Aw[k * C + k]);
                for (int i = k + 1; i < n; ++i) {
                    const double v = fabs(E.Aw[i * C + k]);
                    if (v > big) {
                        big = v;
                        piv = i;
                    }
                }
                if (piv != k) {
                    for (int j = 0; j < n; ++j) {
                        const double t = E.Aw[k * C + j];
                        E.Aw[k * C + j] = E.Aw[piv * C + j];
                        E.Aw[piv * C + j] = t;
                    }
                    const double t = E.rw[k];
                    E.rw[k] = E.rw[piv];
                    E.rw[piv] = t;
                }
                const double d = E.Aw[k * C + k];
                if (d > kTiny || d < -kTiny)
                    for (int i = k + 1; i < n; ++i) {
                        const double f = E.Aw[i * C + k] / d;
                        for (int j = k; j < n; ++j) E.Aw[i * C + j] = E.Aw[i * C + j] - f * E.Aw[k * C + j];
                        E.rw[i] = E.rw[i] - f * E.rw[k];
                    }
            }
            for (int ii = 0; ii < n; ++ii) {
                const int i = n - 1 - ii;
                double s = E.rw[i];
                for (int j = i + 1; j < n; ++j) s = s - E.Aw[i * C + j] * E.sig[E.sidx[j]];
                const double d = E.Aw[i * C + i];
                if (d > kTiny || d < -kTiny) E.sig[E.sidx[i]] = s / d;
            }
        }
    }
    __syncwarp();
    grad_once<kC>(E, cg);
}

template <int kC>
__global__ void __launch_bounds__(32, 16) k_admm(b2c_admm P, b2c_admm_params prm)
{
    extern __shared__ double s_env[];
    const int e = blockIdx.x;
    if (e >= P.n_env) return;
    const int ln = lane_id(), C = P.nc, NV = P.nv, M = 3 * C;
    Env E = carve(s_env, C, NV);
    setup(E, P, prm, e);
    double resm = CUDART_NAN;
    if (prm.flags & B2C_ADMM_FORWARD) {
        for (int i = 0; i < prm.n_iter; ++i) {
            admm_iter<kC>(E, prm.cg_iters);
            const int k = prm.chunk > 0 ? i % prm.chunk : i;
            if (prm.refresh_every > 0 && (k + 1) % prm.refresh_every == 0) resm = refresh<kC>(E, prm.tol, prm.desax != 0);
        }
    } else {
        // the impulses and velocities are given (the gradient of an outside solve)
        for (int i = ln; i < M; i += 32) {
            E.zv[i] = P.lam[(size_t)e * M + i];
            E.u[i] = P.u[(size_t)e * M + i];
        }
        __syncwarp();
    }
    // v+ = v_free + M^-1 J^T lam (NB:1057-1062)
    matvec<kC>(E, E.zv, E.tmp, false);
    if (prm.flags & B2C_ADMM_FORWARD) {
        for (int i = ln; i < M; i += 32) {
            P.lam[(size_t)e * M + i] = E.zv[i];
            P.u[(size_t)e * M + i] = E.u[i];
        }
        for (int k = ln; k < NV; k += 32) P.v_plus[(size_t)e * NV + k] = E.vf[k] + E.wv[k];
        if (ln == 0) {
            if (P.res) P.res[e] = resm;
            if (P.mask) P.mask[e] = E.mask;
            if (P.rho) P.rho[e] = E.rho;
        }
    }
    if (prm.flags & (B2C_ADMM_GRADIENT | B2C_ADMM_GRAD_GIVEN)) {
        build_active(E, 1e-10, 1e-6);
        const int n_calls = prm.n_calls > 0 ? prm.n_calls : C + 2;
        const int j = prm.jdir;
        for (int i = ln; i < M; i += 32) {
            E.pinh[i] = 0.0;
            E.dbv[i] = (prm.flags & B2C_ADMM_GRAD_GIVEN) ? P.dbv_in[(size_t)e * M + i] : prm.dt * E.MJ[i * NV + j];
        }
        __syncwarp();
        grad_affine<kC>(E, n_calls, prm.grad_cg);
        for (int i = ln; i < M; i += 32) P.dlam_tau[(size_t)e * M + i] = E.dlam[i];
        if (!(prm.flags & B2C_ADMM_GRAD_GIVEN)) {
            matvec<kC>(E, E.dlam, E.tmp, false);
            for (int k = ln; k < NV; k += 32) P.dv_tau[(size_t)e * NV + k] = prm.dt * E.Mi[k * NV + j] + E.wv[k];
            // mu at the first slip contact (k_pmu): pinh = -lam_n w_hat there, db = 0
            for (int i = ln; i < M; i += 32) {
                E.pinh[i] = 0.0;
                E.dbv[i] = 0.0;
            }
            __syncwarp();
            if (ln == 0 && E.nslip > 0) {
                const int cc = E.sidx[0];
                E.pinh[3 * cc + 1] = -E.zv[3 * cc] * E.what[3 * cc + 1];
                E.pinh[3 * cc + 2] = -E.zv[3 * cc] * E.what[3 * cc + 2];
            }
            __syncwarp();
            if (prm.do_mu) grad_affine<kC>(E, n_calls, prm.grad_cg);
            for (int i = ln; i < M; i += 32) P.dlam_mu[(size_t)e * M + i] = prm.do_mu ? E.dlam[i] : 0.0;
        }
        for (int c = ln; c < C; c += 32)
            P.labels[(size_t)e * C + c] = E.slipf[c] > 0.5 ? 2 : (E.Zm[9 * c] == 0.0 ? 0 : 1);
        if (ln == 0) P.nslip[e] = E.nslip;
    }
}

}  // namespace badmm
}  // namespace b2c

extern "C" int64_t b2c_admm_smem_bytes(int32_t nc, int32_t nv)
{
    if (nc < 1 || nc > B2C_ADMM_MAX_CONTACTS || nv < 1 || nv > B2C_ADMM_MAX_DOFS) return -1;
    return (int64_t)b2c::badmm::env_bytes(nc, nv);
}

extern "C" int32_t b2c_admm_solve(const b2c_admm *a, const b2c_admm_params *p, b2c_stream st)
{
    using namespace b2c;
    if (!a || !p) {
        set_error("b2c_admm_solve: null argument");
        return B2C_EARG;
    }
    if (a->n_env < 0 || a->nc < 1 || a->nc > B2C_ADMM_MAX_CONTACTS || a->nv < 1 || a->nv > B2C_ADMM_MAX_DOFS) {
        set_error("b2c_admm_solve: n_env %d, nc %d (1..%d), nv %d (1..%d) out of range", a->n_env, a->nc,
                  B2C_ADMM_MAX_CONTACTS, a->nv, B2C_ADMM_MAX_DOFS);
        return B2C_EARG;
    }
    const bool fwd = (p->flags & B2C_ADMM_FORWARD) != 0, grad = (p->flags & B2C_ADMM_GRADIENT) != 0,
               given = (p->flags & B2C_ADMM_GRAD_GIVEN) != 0;
    if (fwd == given || (grad && given) || p->jdir < 0 || p->jdir >= a->nv || p->n_iter < 0 || p->cg_iters < 0 ||
        p->grad_cg < 0 || p->n_calls > a->nc + 2 || p->rho_mode < 0 || p->rho_mode > B2C_ADMM_RHO_GIVEN) {
        set_error("b2c_admm_solve: bad parameters (flags %d: exactly one of FORWARD and GRAD_GIVEN; jdir %d)", p->flags,
                  p->jdir);
        return B2C_EARG;
    }
    if (!a->J || !a->Minv || !a->v_free || !a->mu || !a->lam || !a->u ||
        (fwd && !a->v_plus) || ((grad || given) && (!a->dlam_tau || !a->labels || !a->nslip)) ||
        (grad && (!a->dv_tau || !a->dlam_mu)) || (given && !a->dbv_in) ||
        (p->rho_mode == B2C_ADMM_RHO_GIVEN && !a->rho)) {
        set_error("b2c_admm_solve: a required array is NULL");
        return B2C_EARG;
    }
    if (a->n_env == 0) return B2C_OK;
    const size_t smem = badmm::env_bytes(a->nc, a->nv);
    static bool attr_set[B2C_ADMM_MAX_CONTACTS + 1] = {};
    switch (a->nc) {
#define B2C_ADMM_CASE(n)                                                                                  \
    case n:                                                                                               \
        if (!attr_set[n]) {                                                                               \
            cudaFuncSetAttribute(badmm::k_admm<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024); \
            attr_set[n] = true;                                                                           \
        }                                                                                                 \
        badmm::k_admm<n><<<a->n_env, 32, smem, stream_of(st)>>>(*a, *p);                                 \
        break;
        B2C_ADMM_CASE(1)
        B2C_ADMM_CASE(2)
        B2C_ADMM_CASE(3)
        B2C_ADMM_CASE(4)
        B2C_ADMM_CASE(5)
        B2C_ADMM_CASE(6)
        B2C_ADMM_CASE(7)
        B2C_ADMM_CASE(8)
#undef B2C_ADMM_CASE
    }
    return check_launch("admm");
}
