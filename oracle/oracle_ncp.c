/*
 * oracle_ncp.c -- TEST INFRASTRUCTURE (the oracle), not the product.  Only tests/, smoke() and
 * bench.py's cpu_baseline leg may call it, as the checker.
 *
 * A CPU restatement of the reference's exact-cone NCP solve, the coloured projected
 * Gauss-Seidel of src/motion_engine/ncp/ncp_gpu.py:361-781 (NCPSolverGPU.solve, :974-1063):
 *   - per contact the step rho_c = 1 / lambda_max(W_cc), W_cc = Ja Minv_a Ja^T + Jb Minv_b Jb^T
 *     (k_rho, :441-459; lambda_max by Newton's method on the characteristic polynomial from the
 *     Gershgorin bound instead of the reference's trigonometric closed form f_eigmax, :399-415 --
 *     rho is only the step of the fixed-point map, whose fixed points do not depend on it);
 *   - contacts coloured so that no two contacts of a colour share a dynamic body, by
 *     Jones-Plassmann rounds (k_claim / k_win, :682-722) with a priority that is a pure function
 *     of the canonical key (body_a, body_b, feature) (:656-676; here a 64-bit bijective hash of
 *     the key instead of a hash of its rank, so no sort is needed);
 *   - a sweep over the colours: u = bias + Ja v_a + Jb v_b, lambda <- proj_K(lambda - rho (u +
 *     Gamma(u))) with the de Saxce term Gamma = (mu |u_t|, 0, 0) (k_sweep, :485-568, including
 *     the soft-step branch), the exact projection onto the Coulomb cone (f_proj, :382-397);
 *   - the int64 accumulator holding sum_c round(1e10 Minv J_c^T lambda_c) per body, each update
 *     swapping its own rounded contribution (f_swap, :425-438), and v = v_free + acc / 1e10
 *     (k_apply / k_apply_c, :570-599);
 *   - the natural-map residual max_c |lambda_c - proj_K(lambda_c - rho_c (u_c + Gamma))|
 *     (k_resid, :601-649; ncp_ref.natural_residual, src/motion_engine/ncp/ncp_ref.py:224-234).
 * Sums run in index order, separately rounded (no fused multiply-add), as the CUDA kernels do.
 *
 * Compiled twice: REAL=float SUF=_f SQRT=sqrtf ABS=fabsf and REAL=double SUF=_d SQRT=sqrt ABS=fabs.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_API __attribute__((visibility("default")))
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)

typedef REAL real;

static const double kScale = 1.0e10;

/* splitmix64's output function: a bijection of 64-bit integers */
static uint64_t FN(mix64)(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

/* largest eigenvalue of a symmetric positive semi-definite 3x3: Newton's method on
 * p(x) = x^3 - c2 x^2 + c1 x - c0 from the Gershgorin upper bound; the iterates decrease
 * monotonically to the largest root (p is increasing and convex right of it) */
static double FN(eigmax3)(const double W[3][3])
{
    double c2 = W[0][0] + W[1][1] + W[2][2];
    double c1 = (W[0][0] * W[1][1] - W[0][1] * W[1][0]) + (W[0][0] * W[2][2] - W[0][2] * W[2][0]) +
                (W[1][1] * W[2][2] - W[1][2] * W[2][1]);
    double c0 = W[0][0] * (W[1][1] * W[2][2] - W[1][2] * W[2][1]) - W[0][1] * (W[1][0] * W[2][2] - W[1][2] * W[2][0]) +
                W[0][2] * (W[1][0] * W[2][1] - W[1][1] * W[2][0]);
    double x = 0.0;
    for (int i = 0; i < 3; ++i) {
        double r = W[i][i] + fabs(W[i][(i + 1) % 3]) + fabs(W[i][(i + 2) % 3]);
        if (r > x) x = r;
    }
    if (!(x > 0.0)) return 0.0;
    for (int it = 0; it < 100; ++it) {
        double p = ((x - c2) * x + c1) * x - c0;
        double dp = (3.0 * x - 2.0 * c2) * x + c1;
        if (!(dp > 0.0)) break;
        double xn = x - p / dp;
        if (!(xn < x)) break;
        x = xn;
    }
    return x;
}

/* W += J Minv J^T (3x6, 6x6), sums in index order */
static void FN(add_jmjt)(real W[3][3], const real *J, const real *M)
{
    real T[3][6];
    for (int i = 0; i < 3; ++i)
        for (int l = 0; l < 6; ++l) {
            real s = J[i * 6 + 0] * M[0 * 6 + l];
            for (int k = 1; k < 6; ++k) s = s + J[i * 6 + k] * M[k * 6 + l];
            T[i][l] = s;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            real s = T[i][0] * J[j * 6 + 0];
            for (int l = 1; l < 6; ++l) s = s + T[i][l] * J[j * 6 + l];
            W[i][j] = W[i][j] + s;
        }
}

static real FN(rho_of)(const real *Ja, const real *Jb, const real *Ma, const real *Mb)
{
    real W[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (Ma) FN(add_jmjt)(W, Ja, Ma);
    if (Mb) FN(add_jmjt)(W, Jb, Mb);
    double Wd[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Wd[i][j] = (double)W[i][j];
    double lm = FN(eigmax3)(Wd);
    return lm > 1e-14 ? (real)(1.0 / lm) : (real)0;
}

/* exact projection onto K_mu = {|z_t| <= mu z_n} (f_proj) */
static void FN(proj)(const real z[3], real mu, real out[3])
{
    real zn = z[0], zt = SQRT(z[1] * z[1] + z[2] * z[2]);
    if (zt <= mu * zn) {
        out[0] = z[0]; out[1] = z[1]; out[2] = z[2];
    } else if (mu * zt <= -zn) {
        out[0] = 0; out[1] = 0; out[2] = 0;
    } else {
        real s = (zn + mu * zt) / ((real)1 + mu * mu);
        real f = mu * s / zt;
        out[0] = s; out[1] = f * z[1]; out[2] = f * z[2];
    }
}

/* d = Minv (J^T l) */
static void FN(minv_jt)(const real *J, const real *M, const real l[3], real d[6])
{
    real t[6];
    for (int j = 0; j < 6; ++j) {
        real s = J[0 * 6 + j] * l[0];
        s = s + J[1 * 6 + j] * l[1];
        s = s + J[2 * 6 + j] * l[2];
        t[j] = s;
    }
    for (int k = 0; k < 6; ++k) {
        real s = M[k * 6 + 0] * t[0];
        for (int j = 1; j < 6; ++j) s = s + M[k * 6 + j] * t[j];
        d[k] = s;
    }
}

static int64_t FN(q)(real x) { return (int64_t)llround((double)x * kScale); }

static void FN(contact_u)(int c, const real *Ja, const real *Jb, const int *pa, const int *pb, const real *bias,
                          const real *v, real u[3])
{
    int a = pa[c], b = pb[c];
    for (int i = 0; i < 3; ++i) {
        real ui = bias[3 * c + i];
        if (a >= 0) {
            const real *J = Ja + 18 * c + 6 * i;
            real s = J[0] * v[6 * a + 0];
            for (int j = 1; j < 6; ++j) s = s + J[j] * v[6 * a + j];
            ui = ui + s;
        }
        if (b >= 0) {
            const real *J = Jb + 18 * c + 6 * i;
            real s = J[0] * v[6 * b + 0];
            for (int j = 1; j < 6; ++j) s = s + J[j] * v[6 * b + j];
            ui = ui + s;
        }
        u[i] = ui;
    }
}

/* the argument of the projection for contact c (k_sweep / k_resid) */
static void FN(contact_z)(const real u[3], const real lo[3], real mu, real rho, int desaxce, const real *softp,
                          int use_bias, real sp, real z[3])
{
    if (softp) {
        real vb = 0, ms = 1, isc = 0;
        if (sp > (real)0) {
            vb = sp * softp[3];
        } else if (use_bias) {
            real t = softp[1] * softp[0] * sp;
            vb = t > -softp[4] ? t : -softp[4];
            ms = softp[1];
            isc = softp[2];
        }
        real rn = u[0];
        if (desaxce) rn = rn + mu * SQRT(u[1] * u[1] + u[2] * u[2]);
        z[0] = ((real)1 - isc) * lo[0] - rho * (ms * rn + vb);
        z[1] = lo[1] - rho * u[1];
        z[2] = lo[2] - rho * u[2];
    } else {
        real s0 = u[0];
        if (desaxce) s0 = u[0] + mu * SQRT(u[1] * u[1] + u[2] * u[2]);
        z[0] = lo[0] - rho * s0;
        z[1] = lo[1] - rho * u[1];
        z[2] = lo[2] - rho * u[2];
    }
}

static int FN(is_dyn)(const real *M)
{
    for (int k = 0; k < 36; ++k)
        if (M[k] != (real)0) return 1;
    return 0;
}

/* Jones-Plassmann colouring of the contacts; returns the number of colours, fills col */
static int FN(color)(int nc, int nb, const int *pa, const int *pb, const int *feat, const int *dyn, int *col)
{
    uint64_t *prio = malloc(sizeof(uint64_t) * (nc > 0 ? nc : 1));
    uint64_t *claim = malloc(sizeof(uint64_t) * (nb > 0 ? nb : 1));
    int *won = malloc(sizeof(int) * (nc > 0 ? nc : 1));
    for (int c = 0; c < nc; ++c) {
        uint64_t key = ((uint64_t)(pa[c] + 1) * (uint64_t)(nb + 1) + (uint64_t)(pb[c] + 1)) * 1048576ULL +
                       (uint64_t)(uint32_t)feat[c];
        prio[c] = FN(mix64)(key);
        col[c] = -1;
    }
    int r = 0;
    for (;; ++r) {
        for (int i = 0; i < nb; ++i) claim[i] = UINT64_MAX;
        for (int c = 0; c < nc; ++c) {
            if (col[c] >= 0) continue;
            if (pa[c] >= 0 && dyn[pa[c]] && prio[c] < claim[pa[c]]) claim[pa[c]] = prio[c];
            if (pb[c] >= 0 && dyn[pb[c]] && prio[c] < claim[pb[c]]) claim[pb[c]] = prio[c];
        }
        int left = 0;
        for (int c = 0; c < nc; ++c) {
            won[c] = 0;
            if (col[c] >= 0) continue;
            int ok = 1;
            if (pa[c] >= 0 && dyn[pa[c]] && claim[pa[c]] != prio[c]) ok = 0;
            if (pb[c] >= 0 && dyn[pb[c]] && claim[pb[c]] != prio[c]) ok = 0;
            if (ok) won[c] = 1;
            else left++;
        }
        for (int c = 0; c < nc; ++c)
            if (won[c]) col[c] = r;
        if (left == 0 || r > nc) break;
    }
    free(prio); free(claim); free(won);
    return nc > 0 ? r + 1 : 0;
}

/*
 * Solve: setup (rho, acc from the warm lambda, v), colouring, `iters` sweeps over the colours,
 * then the residual.  lam holds the warm start on entry when warm != 0 (else it is zeroed) and
 * the solution on return; v the velocity; res the per-contact residual.  Returns the residual.
 */
OR_API double FN(or_ncp_solve)(int nc, int nb, const real *Ja, const real *Jb, const real *Minv, const real *vfree,
                               const real *mu, const int *pa, const int *pb, const int *feat, const real *bias,
                               const real *sep, const real *softp, int use_bias, int desaxce, int iters, int warm,
                               real *lam, real *v, real *res, int *col, int *ncol_out)
{
    int *dyn = malloc(sizeof(int) * (nb > 0 ? nb : 1));
    real *rho = malloc(sizeof(real) * (nc > 0 ? nc : 1));
    int64_t *acc = calloc((size_t)(nb > 0 ? nb : 1) * 6, sizeof(int64_t));
    for (int i = 0; i < nb; ++i) dyn[i] = FN(is_dyn)(Minv + 36 * i);
    for (int c = 0; c < nc; ++c)
        rho[c] = FN(rho_of)(Ja + 18 * c, Jb + 18 * c, pa[c] >= 0 ? Minv + 36 * pa[c] : NULL,
                            pb[c] >= 0 ? Minv + 36 * pb[c] : NULL);
    if (!warm) memset(lam, 0, sizeof(real) * 3 * (size_t)nc);
    else
        for (int c = 0; c < nc; ++c) {
            real d[6];
            if (pa[c] >= 0) {
                FN(minv_jt)(Ja + 18 * c, Minv + 36 * pa[c], lam + 3 * c, d);
                for (int k = 0; k < 6; ++k) acc[6 * pa[c] + k] += FN(q)(d[k]);
            }
            if (pb[c] >= 0) {
                FN(minv_jt)(Jb + 18 * c, Minv + 36 * pb[c], lam + 3 * c, d);
                for (int k = 0; k < 6; ++k) acc[6 * pb[c] + k] += FN(q)(d[k]);
            }
        }
    for (int i = 0; i < nb; ++i)
        for (int k = 0; k < 6; ++k) v[6 * i + k] = vfree[6 * i + k] + (real)((double)acc[6 * i + k] / kScale);
    int ncol = FN(color)(nc, nb, pa, pb, feat, dyn, col);
    *ncol_out = ncol;
    for (int it = 0; it < iters; ++it)
        for (int ci = 0; ci < ncol; ++ci)
            for (int c = 0; c < nc; ++c) {
                if (col[c] != ci) continue;
                real u[3], z[3], zn[3], lo[3] = {lam[3 * c], lam[3 * c + 1], lam[3 * c + 2]};
                FN(contact_u)(c, Ja, Jb, pa, pb, bias, v, u);
                FN(contact_z)(u, lo, mu[c], rho[c], desaxce, softp, use_bias, sep ? sep[c] : (real)0, z);
                FN(proj)(z, mu[c], zn);
                lam[3 * c] = zn[0]; lam[3 * c + 1] = zn[1]; lam[3 * c + 2] = zn[2];
                for (int side = 0; side < 2; ++side) {
                    int bdy = side == 0 ? pa[c] : pb[c];
                    if (bdy < 0) continue;
                    const real *J = (side == 0 ? Ja : Jb) + 18 * c;
                    real dn[6], dold[6];
                    FN(minv_jt)(J, Minv + 36 * bdy, zn, dn);
                    FN(minv_jt)(J, Minv + 36 * bdy, lo, dold);
                    for (int k = 0; k < 6; ++k) acc[6 * bdy + k] += FN(q)(dn[k]) - FN(q)(dold[k]);
                    if (dyn[bdy])
                        for (int k = 0; k < 6; ++k)
                            v[6 * bdy + k] = vfree[6 * bdy + k] + (real)((double)acc[6 * bdy + k] / kScale);
                }
            }
    double rmax = 0.0;
    for (int c = 0; c < nc; ++c) {
        real u[3], z[3], zn[3], lo[3] = {lam[3 * c], lam[3 * c + 1], lam[3 * c + 2]};
        FN(contact_u)(c, Ja, Jb, pa, pb, bias, v, u);
        FN(contact_z)(u, lo, mu[c], rho[c], desaxce, softp, use_bias, sep ? sep[c] : (real)0, z);
        FN(proj)(z, mu[c], zn);
        real m = 0;
        for (int i = 0; i < 3; ++i) {
            real d = ABS(lo[i] - zn[i]);
            if (d > m) m = d;
        }
        res[c] = m;
        if ((double)m > rmax) rmax = (double)m;
    }
    free(dyn); free(rho); free(acc);
    return rmax;
}
