// Batched exact-cone NCP in Delassus form with its implicit sensitivity (the reference's
// batched adjoint, src/motion_engine/ncp/ncp_batch_gpu.py:918-1313, and the CPU
// implicit-function response of src/motion_engine/ncp/ncp_ref.py:786-959).
//
// Every environment e holds a small contact problem: G_e (n x n, n = 3 n_c <= 48), b_e, mu_e.
// One warp owns one environment, with G in shared memory:
//
//   solve     projected Gauss-Seidel over the contacts, lambda_c <- proj_K(lambda_c - rho_c
//             (u_c + Gamma(u_c))), u = G lambda + b, rho_c = 1 / lambda_max(G_cc) (the sweep of
//             ncp_gpu.py:485-568 on the Delassus operator), until the natural residual
//             max_c |lambda_c - proj_K(...)| is below tol (checked every `check` sweeps; the
//             convergence mask of the batched solver) or max_iters;
//   adjoint   the contacts labelled open / stick / slip from lambda (ncp_ref.classify,
//             :251-274), the fixed-branch residual Jacobian A and the parameter maps Bmu, Bb
//             (ncp_ref._active_system, :786-842), LU with partial pivoting, then either the full
//             responses X = -A^-1 [Bmu Bb] (ncp_ref.sensitivity) or the vector-Jacobian product
//             y = A^-T g, dL/db = -Bb^T y, dL/dmu = -Bmu^T y.  A pivot below 1e-12 max|A| marks
//             the branch singular and, like a branch boundary, returns NaN (the reference's
//             guarded_response without a selection).
//
// Sums over a row are warp reductions in a fixed butterfly order, so results are bit-identical
// run to run.
#include "b2c_common.cuh"

namespace b2c {
namespace bncp {

constexpr int kMaxN = 48;  // 3 x 16 contacts

struct Env {
    int n, nc;
    const double *G, *b, *mu;
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ double eigmax3(const double W[3][3])
{
    const double c2 = W[0][0] + W[1][1] + W[2][2];
    const double c1 = (W[0][0] * W[1][1] - W[0][1] * W[1][0]) + (W[0][0] * W[2][2] - W[0][2] * W[2][0]) +
                      (W[1][1] * W[2][2] - W[1][2] * W[2][1]);
    const double c0 = W[0][0] * (W[1][1] * W[2][2] - W[1][2] * W[2][1]) -
                      W[0][1] * (W[1][0] * W[2][2] - W[1][2] * W[2][0]) +
                      W[0][2] * (W[1][0] * W[2][1] - W[1][1] * W[2][0]);
    double x = 0.0;
    for (int i = 0; i < 3; ++i) {
        const double r = W[i][i] + fabs(W[i][(i + 1) % 3]) + fabs(W[i][(i + 2) % 3]);
        if (r > x) x = r;
    }
    if (!(x > 0.0)) return 0.0;
    for (int it = 0; it < 100; ++it) {
        const double p = ((x - c2) * x + c1) * x - c0;
        const double dp = (3.0 * x - 2.0 * c2) * x + c1;
        if (!(dp > 0.0)) break;
        const double xn = x - p / dp;
        if (!(xn < x)) break;
        x = xn;
    }
    return x;
}

__device__ __forceinline__ void proj(const double z[3], double mu, double out[3])
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

// u_r = b_r + sum_j G[r][j] lam[j] for the warp, every lane returns it
__device__ __forceinline__ double row_u(const double *G, const double *lam, const double *b, int n, int r, int lane)
{
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += G[r * n + j] * lam[j];
    return warp_sum(s) + b[r];
}

// the projection argument of contact c with the de Saxce term
__device__ __forceinline__ void zarg(const double u[3], const double lo[3], double mu, double rho, double z[3])
{
    const double s0 = u[0] + mu * sqrt(u[1] * u[1] + u[2] * u[2]);
    z[0] = lo[0] - rho * s0;
    z[1] = lo[1] - rho * u[1];
    z[2] = lo[2] - rho * u[2];
}

__global__ void __launch_bounds__(32) k_solve(int n_env, int n_max, const int *__restrict__ ncs,
                                              const double *__restrict__ G, const double *__restrict__ b,
                                              const double *__restrict__ mu, double *__restrict__ lam_io,
                                              double *__restrict__ res_out, int *__restrict__ iters_out,
                                              int max_iters, double tol, int check)
{
    extern __shared__ double sm[];
    const int e = blockIdx.x, lane = threadIdx.x;
    if (e >= n_env) return;
    const int nc = ncs[e], n = 3 * nc;
    double *Gs = sm, *bs = Gs + n_max * n_max, *lam = bs + n_max, *rho = lam + n_max, *mus = rho + n_max / 3;
    const double *Ge = G + (size_t)e * n_max * n_max;
    for (int i = lane; i < n * n; i += 32) Gs[i] = Ge[(i / n) * n_max + (i % n)];
    for (int i = lane; i < n; i += 32) {
        bs[i] = b[(size_t)e * n_max + i];
        lam[i] = lam_io[(size_t)e * n_max + i];
    }
    for (int c = lane; c < nc; c += 32) {
        mus[c] = mu[(size_t)e * (n_max / 3) + c];
        double W[3][3];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) W[i][j] = Ge[(3 * c + i) * n_max + 3 * c + j];
        const double lm = eigmax3(W);
        rho[c] = lm > 1e-300 ? 1.0 / lm : 0.0;
    }
    __syncwarp();
    double res = 0.0;
    int it = 0;
    for (; it < max_iters; ++it) {
        if (check > 0 && it % check == 0) {
            double r = 0.0;
            for (int c = 0; c < nc; ++c) {
                double u[3], z[3], p[3];
                for (int k = 0; k < 3; ++k) u[k] = row_u(Gs, lam, bs, n, 3 * c + k, lane);
                const double lo[3] = {lam[3 * c], lam[3 * c + 1], lam[3 * c + 2]};
                zarg(u, lo, mus[c], rho[c], z);
                proj(z, mus[c], p);
                for (int k = 0; k < 3; ++k) r = fmax(r, fabs(lo[k] - p[k]));
            }
            res = r;
            if (r < tol) break;
        }
        for (int c = 0; c < nc; ++c) {
            double u[3], z[3], p[3];
            for (int k = 0; k < 3; ++k) u[k] = row_u(Gs, lam, bs, n, 3 * c + k, lane);
            const double lo[3] = {lam[3 * c], lam[3 * c + 1], lam[3 * c + 2]};
            zarg(u, lo, mus[c], rho[c], z);
            proj(z, mus[c], p);
            __syncwarp();
            if (lane == 0) {
                lam[3 * c] = p[0];
                lam[3 * c + 1] = p[1];
                lam[3 * c + 2] = p[2];
            }
            __syncwarp();
        }
    }
    if (it == max_iters || check <= 0) {  // residual of the final iterate
        double r = 0.0;
        for (int c = 0; c < nc; ++c) {
            double u[3], z[3], p[3];
            for (int k = 0; k < 3; ++k) u[k] = row_u(Gs, lam, bs, n, 3 * c + k, lane);
            const double lo[3] = {lam[3 * c], lam[3 * c + 1], lam[3 * c + 2]};
            zarg(u, lo, mus[c], rho[c], z);
            proj(z, mus[c], p);
            for (int k = 0; k < 3; ++k) r = fmax(r, fabs(lo[k] - p[k]));
        }
        res = r;
    }
    for (int i = lane; i < n_max; i += 32) lam_io[(size_t)e * n_max + i] = i < n ? lam[i] : 0.0;
    if (lane == 0) {
        res_out[e] = res;
        iters_out[e] = it;
    }
}

// Fixed-branch system of one environment into shared memory: A (n x n), Bmu (n x nc), Bb (n x n).
// Returns the status bits (2 = a branch boundary); labels written per contact.
__device__ int assemble(const double *Gs, const double *bs, const double *lam, const double *mus, int n, int nc,
                        double *A, double *Bmu, double *Bb, int *labels, int lane)
{
    __shared__ double s_u[kMaxN];
    for (int r = 0; r < n; ++r) {
        const double u = row_u(Gs, lam, bs, n, r, lane);
        if (lane == 0) s_u[r] = u;
    }
    for (int i = lane; i < n * n; i += 32) {
        A[i] = 0.0;
        Bb[i] = 0.0;
    }
    for (int i = lane; i < n * nc; i += 32) Bmu[i] = 0.0;
    __syncwarp();
    int status = 0;
    if (lane == 0) {
        double scale = 0.0;
        for (int i = 0; i < n; ++i) scale = fmax(scale, fabs(lam[i]));
        scale = fmax(scale, 1e-30);
        for (int c = 0; c < nc; ++c) {
            const int i = 3 * c;
            const double ln = lam[i], lt = sqrt(lam[i + 1] * lam[i + 1] + lam[i + 2] * lam[i + 2]);
            const double m = mus[c];
            int lab;
            if (ln <= 1e-10 + 1e-6 * scale) lab = 0;
            else if (lt >= m * ln * (1.0 - 1e-6) - 1e-10) lab = 2;
            else lab = 1;
            labels[c] = lab;
            if (lab == 0) {
                for (int k = 0; k < 3; ++k) A[(i + k) * n + i + k] = 1.0;
                if (fabs(s_u[i]) < 1e-9) status |= 2;
            } else if (lab == 1) {
                for (int k = 0; k < 3; ++k) {
                    for (int j = 0; j < n; ++j) A[(i + k) * n + j] = Gs[(i + k) * n + j];
                    Bb[(i + k) * n + i + k] = 1.0;
                }
            } else {
                for (int j = 0; j < n; ++j) A[i * n + j] = Gs[i * n + j];
                Bb[i * n + i] = 1.0;
                const double s0 = s_u[i + 1], s1 = s_u[i + 2];
                double ns = sqrt(s0 * s0 + s1 * s1);
                if (ns < 1e-14) {
                    status |= 2;
                    ns = 1e-14;
                }
                const double h0 = s0 / ns, h1 = s1 / ns;
                const double P[2][2] = {{(1.0 - h0 * h0) / ns, (-h0 * h1) / ns}, {(-h1 * h0) / ns, (1.0 - h1 * h1) / ns}};
                const double ml = m * ln;
                for (int a = 0; a < 2; ++a) {
                    for (int j = 0; j < n; ++j)
                        A[(i + 1 + a) * n + j] = ml * (P[a][0] * Gs[(i + 1) * n + j] + P[a][1] * Gs[(i + 2) * n + j]);
                    A[(i + 1 + a) * n + i] += m * (a == 0 ? h0 : h1);
                    A[(i + 1 + a) * n + i + 1 + a] += 1.0;
                    Bb[(i + 1 + a) * n + i + 1] = ml * P[a][0];
                    Bb[(i + 1 + a) * n + i + 2] = ml * P[a][1];
                    Bmu[(i + 1 + a) * nc + c] = ln * (a == 0 ? h0 : h1);
                }
            }
            const double sc = fmax(fabs(ln), 1e-12);
            if (lab == 1 && fabs(lt - m * ln) < 1e-7 * m * sc) status |= 2;
            if (lab != 0 && ln < 1e-9) status |= 2;
        }
    }
    __syncwarp();
    return __shfl_sync(0xffffffffu, status, 0);
}

// In-place LU with partial pivoting of A (n x n); piv[k] = row swapped with k.  Returns 1 when a
// pivot is below 1e-12 max|A| (the branch is numerically singular).
__device__ int lu(double *A, int *piv, int n, int lane)
{
    double amax = 0.0;
    for (int i = lane; i < n * n; i += 32) amax = fmax(amax, fabs(A[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    for (int k = 0; k < n; ++k) {
        // pivot: the largest |A[r][k]|, r >= k (lowest row on ties)
        double best = -1.0;
        int br = k;
        for (int r = k + lane; r < n; r += 32) {
            const double v = fabs(A[r * n + k]);
            if (v > best) {
                best = v;
                br = r;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > best || (ov == best && orr < br)) {
                best = ov;
                br = orr;
            }
        }
        if (!(best > 1e-12 * amax)) return 1;
        if (lane == 0) piv[k] = br;
        if (br != k)
            for (int j = lane; j < n; j += 32) {
                const double t = A[k * n + j];
                A[k * n + j] = A[br * n + j];
                A[br * n + j] = t;
            }
        __syncwarp();
        const double d = A[k * n + k];
        for (int r = k + 1 + lane; r < n; r += 32) A[r * n + k] /= d;
        __syncwarp();
        for (int idx = lane; idx < (n - k - 1) * (n - k - 1); idx += 32) {
            const int r = k + 1 + idx / (n - k - 1), j = k + 1 + idx % (n - k - 1);
            A[r * n + j] -= A[r * n + k] * A[k * n + j];
        }
        __syncwarp();
    }
    return 0;
}

// X (n x m, row-major) <- A^-1 X with the factors of lu()
__device__ void lu_solve(const double *A, const int *piv, int n, double *X, int m, int lane)
{
    for (int k = 0; k < n; ++k) {
        const int p = piv[k];
        if (p != k)
            for (int j = lane; j < m; j += 32) {
                const double t = X[k * m + j];
                X[k * m + j] = X[p * m + j];
                X[p * m + j] = t;
            }
    }
    __syncwarp();
    for (int j = lane; j < m; j += 32) {
        for (int r = 1; r < n; ++r) {
            double s = X[r * m + j];
            for (int k = 0; k < r; ++k) s -= A[r * n + k] * X[k * m + j];
            X[r * m + j] = s;
        }
        for (int r = n - 1; r >= 0; --r) {
            double s = X[r * m + j];
            for (int k = r + 1; k < n; ++k) s -= A[r * n + k] * X[k * m + j];
            X[r * m + j] = s / A[r * n + r];
        }
    }
    __syncwarp();
}

// y <- A^-T y with the factors of lu() (A = P^T L U, so A^T y = g is U^T L^T P y = g)
__device__ void lu_solve_t(const double *A, const int *piv, int n, double *y, int lane)
{
    if (lane == 0) {
        for (int r = 0; r < n; ++r) {  // U^T z = g
            double s = y[r];
            for (int k = 0; k < r; ++k) s -= A[k * n + r] * y[k];
            y[r] = s / A[r * n + r];
        }
        for (int r = n - 1; r >= 0; --r) {  // L^T w = z (unit diagonal)
            double s = y[r];
            for (int k = r + 1; k < n; ++k) s -= A[k * n + r] * y[k];
            y[r] = s;
        }
        for (int k = n - 1; k >= 0; --k) {  // y = P^T w: undo the swaps in reverse
            const int p = piv[k];
            if (p != k) {
                const double t = y[k];
                y[k] = y[p];
                y[p] = t;
            }
        }
    }
    __syncwarp();
}

// mode 0: full responses dlam/dmu (n x nc) and dlam/db (n x n); mode 1: vector-Jacobian product
__global__ void __launch_bounds__(32) k_adjoint(int n_env, int n_max, const int *__restrict__ ncs,
                                                const double *__restrict__ G, const double *__restrict__ b,
                                                const double *__restrict__ mu, const double *__restrict__ lam_in,
                                                int *__restrict__ labels_out, int *__restrict__ status_out, int mode,
                                                double *__restrict__ dmu, double *__restrict__ db,
                                                const double *__restrict__ glam, double *__restrict__ gb,
                                                double *__restrict__ gmu)
{
    extern __shared__ double sm[];
    const int e = blockIdx.x, lane = threadIdx.x;
    if (e >= n_env) return;
    const int nc = ncs[e], n = 3 * nc, ncm = n_max / 3;
    double *Gs = sm, *A = Gs + kMaxN * kMaxN, *Bb = A + kMaxN * kMaxN, *Bmu = Bb + kMaxN * kMaxN;
    double *bs = Bmu + kMaxN * (kMaxN / 3), *lam = bs + kMaxN, *mus = lam + kMaxN, *y = mus + kMaxN / 3;
    __shared__ int piv[kMaxN];
    __shared__ int labels[kMaxN / 3];
    const double *Ge = G + (size_t)e * n_max * n_max;
    for (int i = lane; i < n * n; i += 32) Gs[i] = Ge[(i / n) * n_max + (i % n)];
    for (int i = lane; i < n; i += 32) {
        bs[i] = b[(size_t)e * n_max + i];
        lam[i] = lam_in[(size_t)e * n_max + i];
    }
    for (int c = lane; c < nc; c += 32) mus[c] = mu[(size_t)e * ncm + c];
    __syncwarp();
    int status = assemble(Gs, bs, lam, mus, n, nc, A, Bmu, Bb, labels, lane);
    if (lu(A, piv, n, lane)) status |= 1;
    for (int c = lane; c < ncm; c += 32) labels_out[(size_t)e * ncm + c] = c < nc ? labels[c] : 0;
    if (lane == 0) status_out[e] = status;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (mode == 0) {
        // X = -A^-1 [Bmu | Bb], columns solved together in Bb-sized chunks
        double *X = Bb;  // n x n, Bb's own storage (Bb is not needed after the copy below)
        if (!status) {
            // Bmu columns first, into y-sized scratch one column at a time
            for (int c = 0; c < nc; ++c) {
                for (int r = lane; r < n; r += 32) y[r] = -Bmu[r * nc + c];
                __syncwarp();
                lu_solve(A, piv, n, y, 1, lane);
                for (int r = lane; r < n; r += 32) dmu[((size_t)e * n_max + r) * ncm + c] = y[r];
                __syncwarp();
            }
            for (int i = lane; i < n * n; i += 32) X[i] = -X[i];
            __syncwarp();
            lu_solve(A, piv, n, X, n, lane);
        }
        for (int i = lane; i < n_max * n_max; i += 32) {
            const int r = i / n_max, j = i % n_max;
            db[(size_t)e * n_max * n_max + i] = (r < n && j < n) ? (status ? nan : X[r * n + j]) : 0.0;
        }
        for (int i = lane; i < n_max * ncm; i += 32) {
            const int r = i / ncm, c = i % ncm;
            if (status || r >= n || c >= nc)
                dmu[(size_t)e * n_max * ncm + i] = (r < n && c < nc) ? nan : 0.0;
        }
    } else {
        for (int r = lane; r < n; r += 32) y[r] = glam[(size_t)e * n_max + r];
        __syncwarp();
        if (!status) lu_solve_t(A, piv, n, y, lane);
        // dL/db = -Bb^T y, dL/dmu = -Bmu^T y
        for (int j = lane; j < n_max; j += 32) {
            double s = 0.0;
            if (j < n)
                for (int r = 0; r < n; ++r) s -= Bb[r * n + j] * y[r];
            gb[(size_t)e * n_max + j] = j < n ? (status ? nan : s) : 0.0;
        }
        for (int c = lane; c < ncm; c += 32) {
            double s = 0.0;
            if (c < nc)
                for (int r = 0; r < n; ++r) s -= Bmu[r * nc + c] * y[r];
            gmu[(size_t)e * ncm + c] = c < nc ? (status ? nan : s) : 0.0;
        }
    }
}

size_t solve_smem(int n_max) { return sizeof(double) * ((size_t)n_max * n_max + 2 * n_max + 2 * (n_max / 3)); }
size_t adjoint_smem()
{
    return sizeof(double) * (3 * (size_t)kMaxN * kMaxN + (size_t)kMaxN * (kMaxN / 3) + 2 * kMaxN + 2 * (kMaxN / 3) +
                             kMaxN);
}

}  // namespace bncp
}  // namespace b2c

static bool bncp_ok(const b2c_bncp *p)
{
    return p && p->n_env >= 0 && p->n_max >= 3 && p->n_max % 3 == 0 && p->n_max <= b2c::bncp::kMaxN && p->nc &&
           p->G && p->b && p->mu && p->lam && p->res && p->iters && p->labels && p->status;
}

extern "C" int32_t b2c_bncp_max_rows(void) { return b2c::bncp::kMaxN; }

extern "C" int32_t b2c_bncp_solve(const b2c_bncp *p, int32_t max_iters, double tol, int32_t check, b2c_stream s)
{
    if (!bncp_ok(p) || max_iters < 0) {
        b2c::set_error("b2c_bncp_solve: bad argument (n_max must be a multiple of 3, at most %d)", b2c::bncp::kMaxN);
        return B2C_EARG;
    }
    if (p->n_env == 0) return B2C_OK;
    const size_t smem = b2c::bncp::solve_smem(p->n_max);
    b2c::bncp::k_solve<<<p->n_env, 32, smem, b2c::stream_of(s)>>>(p->n_env, p->n_max, p->nc, p->G, p->b, p->mu,
                                                                     p->lam, p->res, p->iters, max_iters, tol, check);
    return b2c::check_launch("bncp_solve");
}

static int32_t bncp_adjoint(const b2c_bncp *p, int mode, double *dmu, double *db, const double *glam, double *gb,
                            double *gmu, b2c_stream s)
{
    if (p->n_env == 0) return B2C_OK;
    static bool attr = false;
    const size_t smem = b2c::bncp::adjoint_smem();
    if (!attr) {
        cudaFuncSetAttribute(b2c::bncp::k_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    b2c::bncp::k_adjoint<<<p->n_env, 32, smem, b2c::stream_of(s)>>>(p->n_env, p->n_max, p->nc, p->G, p->b, p->mu,
                                                                      p->lam, p->labels, p->status, mode, dmu, db,
                                                                      glam, gb, gmu);
    return b2c::check_launch("bncp_adjoint");
}

extern "C" int32_t b2c_bncp_sensitivity(const b2c_bncp *p, double *dlam_dmu, double *dlam_db, b2c_stream s)
{
    if (!bncp_ok(p) || !dlam_dmu || !dlam_db) {
        b2c::set_error("b2c_bncp_sensitivity: bad argument");
        return B2C_EARG;
    }
    return bncp_adjoint(p, 0, dlam_dmu, dlam_db, nullptr, nullptr, nullptr, s);
}

extern "C" int32_t b2c_bncp_vjp(const b2c_bncp *p, const double *glam, double *gb, double *gmu, b2c_stream s)
{
    if (!bncp_ok(p) || !glam || !gb || !gmu) {
        b2c::set_error("b2c_bncp_vjp: bad argument");
        return B2C_EARG;
    }
    return bncp_adjoint(p, 1, nullptr, nullptr, glam, gb, gmu, s);
}
