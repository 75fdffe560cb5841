// Exact-cone NCP solve: the coloured projected Gauss-Seidel of the reference's NCPSolverGPU
// (src/motion_engine/ncp/ncp_gpu.py:361-1063) on per-contact 3x6 Jacobian blocks, in float32 or
// float64.
//
//   setup     rho_c = 1 / lambda_max(Ja Minv_a Ja^T + Jb Minv_b Jb^T) (k_rho, :441-459; the
//             largest eigenvalue by Newton's method on the characteristic polynomial from the
//             Gershgorin bound, in float64), acc = sum_c round(1e10 Minv J_c^T lambda_c) of the
//             warm start (k_scatter, :468-483), v = v_free + acc / 1e10 (k_apply, :570-581);
//   colour    Jones-Plassmann over the contacts, claims on dynamic bodies only (k_claim /
//             k_win, :682-722), priority a bijective 64-bit hash of the canonical key
//             (body_a, body_b, feature) (:656-664), so the colouring is a pure function of the
//             contact set and not of its order; cached while pairs, features and masses stay
//             the same (k_cache_cmp, :736-765);
//   sweeps    per colour, per contact: u = bias + Ja v_a + Jb v_b, the de Saxce term, the
//             soft-step branch, lambda <- proj_K(z) (k_sweep, :485-568); acc swaps the contact's
//             old rounded contribution for the new one (f_swap, :425-438) and the velocity of
//             the contact's dynamic bodies is rebuilt from acc at once (k_apply_c, :583-599: a
//             colour holds each dynamic body at most once, so the thread that owns the contact
//             owns those bodies for the phase).  All colours of all iterations run in ONE
//             persistent launch with a barrier between colours (block or cluster);
//   residual  max_c |lambda_c - proj_K(z_c)| of the same map (k_resid, :601-649).
//
// Every sum runs in index order with separately rounded operations (the library is built
// with -fmad=false), so the oracle's C restatement reproduces the results bit for bit.
#include <cooperative_groups.h>

#include "b2c_barrier.cuh"
#include "b2c_common.cuh"

namespace cg = cooperative_groups;

namespace b2c {
namespace ncp {

constexpr double kScale = 1.0e10;
constexpr int kColorThreads = 1024;
constexpr int kSweepThreads = 512;
constexpr int kClusterMax = 16;
constexpr int kMaxColors = 1024;  // the reference's _NCOLMAX

enum Stat { kNColors = 0, kCacheValid = 1, kCachedC = 2, kCacheHit = 3, kHits = 4, kMisses = 5, kRounds = 6,
            kError = 7 };
enum ErrBit { kErrColorOverflow = 1, kErrColorTimeout = 2, kErrBarrier = 4 };

__device__ __forceinline__ float rsq(float x) { return sqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return sqrt(x); }
__device__ __forceinline__ float rab(float x) { return fabsf(x); }
__device__ __forceinline__ double rab(double x) { return fabs(x); }

// splitmix64's output function: a bijection of 64-bit integers
__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

// largest eigenvalue of a symmetric positive semi-definite 3x3: Newton's method on the
// characteristic polynomial p(x) = x^3 - c2 x^2 + c1 x - c0 from the Gershgorin bound; the
// iterates decrease monotonically to the largest root
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

template <typename T>
__device__ void add_jmjt(T W[3][3], const T *__restrict__ J, const T *__restrict__ M)
{
    T Tm[3][6];
    for (int i = 0; i < 3; ++i)
        for (int l = 0; l < 6; ++l) {
            T s = J[i * 6 + 0] * M[0 * 6 + l];
            for (int k = 1; k < 6; ++k) s = s + J[i * 6 + k] * M[k * 6 + l];
            Tm[i][l] = s;
        }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T s = Tm[i][0] * J[j * 6 + 0];
            for (int l = 1; l < 6; ++l) s = s + Tm[i][l] * J[j * 6 + l];
            W[i][j] = W[i][j] + s;
        }
}

template <typename T>
__global__ void k_rho(int nc, const T *__restrict__ Ja, const T *__restrict__ Jb, const T *__restrict__ Minv,
                      const int *__restrict__ pa, const int *__restrict__ pb, T *__restrict__ rho)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    T W[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
    if (pa[c] >= 0) add_jmjt(W, Ja + 18 * (size_t)c, Minv + 36 * (size_t)pa[c]);
    if (pb[c] >= 0) add_jmjt(W, Jb + 18 * (size_t)c, Minv + 36 * (size_t)pb[c]);
    double Wd[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Wd[i][j] = (double)W[i][j];
    const double lm = eigmax3(Wd);
    rho[c] = lm > 1e-14 ? (T)(1.0 / lm) : T(0);
}

template <typename T>
__global__ void k_dyn(int nb, const T *__restrict__ Minv, int *__restrict__ dyn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    int d = 0;
    for (int k = 0; k < 36; ++k) d |= Minv[36 * (size_t)i + k] != T(0);
    dyn[i] = d;
}

// d = Minv (J^T l)
template <typename T>
__device__ __forceinline__ void minv_jt(const T *__restrict__ J, const T *__restrict__ M, const T l[3], T d[6])
{
    T t[6];
    for (int j = 0; j < 6; ++j) {
        T s = J[0 * 6 + j] * l[0];
        s = s + J[1 * 6 + j] * l[1];
        s = s + J[2 * 6 + j] * l[2];
        t[j] = s;
    }
    for (int k = 0; k < 6; ++k) {
        T s = M[k * 6 + 0] * t[0];
        for (int j = 1; j < 6; ++j) s = s + M[k * 6 + j] * t[j];
        d[k] = s;
    }
}

template <typename T>
__device__ __forceinline__ long long quant(T x)
{
    return llround((double)x * kScale);
}

template <typename T>
__global__ void k_scatter(int nc, const T *__restrict__ Ja, const T *__restrict__ Jb, const T *__restrict__ Minv,
                          const int *__restrict__ pa, const int *__restrict__ pb, const T *__restrict__ lam,
                          long long *__restrict__ acc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const T l[3] = {lam[3 * (size_t)c], lam[3 * (size_t)c + 1], lam[3 * (size_t)c + 2]};
    for (int side = 0; side < 2; ++side) {
        const int b = side == 0 ? pa[c] : pb[c];
        if (b < 0) continue;
        T d[6];
        minv_jt((side == 0 ? Ja : Jb) + 18 * (size_t)c, Minv + 36 * (size_t)b, l, d);
        for (int k = 0; k < 6; ++k)
            atomicAdd(reinterpret_cast<unsigned long long *>(acc + 6 * (size_t)b + k), (unsigned long long)quant(d[k]));
    }
}

template <typename T>
__global__ void k_apply(int nb, const T *__restrict__ vfree, const long long *__restrict__ acc, T *__restrict__ v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 6 * nb) return;
    v[i] = vfree[i] + (T)((double)acc[i] / kScale);
}

// u = bias + Ja v_a + Jb v_b (v read through L2: other CTAs of the sweep write it)
template <typename T>
__device__ __forceinline__ void contact_u(int c, const T *__restrict__ Ja, const T *__restrict__ Jb, int a, int b,
                                          const T *__restrict__ bias, const T *v, T u[3])
{
    T va[6], vb[6];
    if (a >= 0)
        for (int j = 0; j < 6; ++j) va[j] = __ldcg(v + 6 * (size_t)a + j);
    if (b >= 0)
        for (int j = 0; j < 6; ++j) vb[j] = __ldcg(v + 6 * (size_t)b + j);
    for (int i = 0; i < 3; ++i) {
        T ui = bias[3 * (size_t)c + i];
        if (a >= 0) {
            const T *J = Ja + 18 * (size_t)c + 6 * i;
            T s = J[0] * va[0];
            for (int j = 1; j < 6; ++j) s = s + J[j] * va[j];
            ui = ui + s;
        }
        if (b >= 0) {
            const T *J = Jb + 18 * (size_t)c + 6 * i;
            T s = J[0] * vb[0];
            for (int j = 1; j < 6; ++j) s = s + J[j] * vb[j];
            ui = ui + s;
        }
        u[i] = ui;
    }
}

struct Soft {
    int on, use_bias;
    double p[5];  // bias_rate, mass_scale, impulse_scale, inv_h, contact_speed
};

// the argument of the projection (k_sweep's two branches)
template <typename T>
__device__ __forceinline__ void contact_z(const T u[3], const T lo[3], T mu, T rho, int desaxce, const Soft &sf, T sp,
                                          T z[3])
{
    if (sf.on) {
        T vb = T(0), ms = T(1), isc = T(0);
        if (sp > T(0)) {
            vb = sp * (T)sf.p[3];
        } else if (sf.use_bias) {
            const T t = (T)sf.p[1] * (T)sf.p[0] * sp;
            vb = t > -(T)sf.p[4] ? t : -(T)sf.p[4];
            ms = (T)sf.p[1];
            isc = (T)sf.p[2];
        }
        T rn = u[0];
        if (desaxce) rn = rn + mu * rsq(u[1] * u[1] + u[2] * u[2]);
        z[0] = (T(1) - isc) * lo[0] - rho * (ms * rn + vb);
        z[1] = lo[1] - rho * u[1];
        z[2] = lo[2] - rho * u[2];
    } else {
        T s0 = u[0];
        if (desaxce) s0 = u[0] + mu * rsq(u[1] * u[1] + u[2] * u[2]);
        z[0] = lo[0] - rho * s0;
        z[1] = lo[1] - rho * u[1];
        z[2] = lo[2] - rho * u[2];
    }
}

// exact projection onto K_mu (f_proj, :382-397)
template <typename T>
__device__ __forceinline__ void proj(const T z[3], T mu, T out[3])
{
    const T zn = z[0], zt = rsq(z[1] * z[1] + z[2] * z[2]);
    if (zt <= mu * zn) {
        out[0] = z[0];
        out[1] = z[1];
        out[2] = z[2];
    } else if (mu * zt <= -zn) {
        out[0] = out[1] = out[2] = T(0);
    } else {
        const T s = (zn + mu * zt) / (T(1) + mu * mu);
        const T f = mu * s / zt;
        out[0] = s;
        out[1] = f * z[1];
        out[2] = f * z[2];
    }
}

template <typename T>
struct SweepArgs {
    int nc;
    const T *Ja, *Jb, *Minv, *vfree, *mu, *bias, *sep, *rho;
    const int *pa, *pb, *order, *cstart, *ccount, *dyn;
    T *lam, *v;
    long long *acc;
    int *stats;
    unsigned int *bar;
    long long timeout_ns;
    int iters, desaxce;
    Soft soft;
};

enum Kind { kBlock = 0, kCluster = 1, kGrid = 2 };

// The barrier between colours.  The grid form (a cooperative launch, every CTA co-resident) is
// the arrival-counter barrier of b2c_barrier.cuh over a.bar[0] (cleared by the host before the
// launch); `epoch` counts the grid barriers of this launch.  Its wait is bounded by
// a.timeout_ns, after which it sets kErrBarrier and every CTA leaves the sweep.
template <int kKind, typename T>
__device__ __forceinline__ bool phase_barrier(const SweepArgs<T> &a, unsigned int &epoch)
{
    if (kKind == kBlock) {
        __syncthreads();
        return true;
    }
    if (kKind == kCluster) {
        cg::this_cluster().sync();
        return true;
    }
    ++epoch;
    grid_arrive(a.bar);
    return grid_wait(a.bar, epoch, a.timeout_ns, a.stats + kError, kErrBarrier);
}

template <typename T>
__device__ __forceinline__ void sweep_contact(const SweepArgs<T> &a, int c)
{
    const int pa = a.pa[c], pb = a.pb[c];
    T u[3], z[3], zn[3];
    const T lo[3] = {a.lam[3 * (size_t)c], a.lam[3 * (size_t)c + 1], a.lam[3 * (size_t)c + 2]};
    contact_u(c, a.Ja, a.Jb, pa, pb, a.bias, a.v, u);
    contact_z(u, lo, a.mu[c], a.rho[c], a.desaxce, a.soft, a.sep ? a.sep[c] : T(0), z);
    proj(z, a.mu[c], zn);
    a.lam[3 * (size_t)c] = zn[0];
    a.lam[3 * (size_t)c + 1] = zn[1];
    a.lam[3 * (size_t)c + 2] = zn[2];
    for (int side = 0; side < 2; ++side) {
        const int b = side == 0 ? pa : pb;
        if (b < 0 || !a.dyn[b]) continue;  // a static body's Minv is zero: nothing to add
        const T *J = (side == 0 ? a.Ja : a.Jb) + 18 * (size_t)c;
        T dn[6], dold[6];
        minv_jt(J, a.Minv + 36 * (size_t)b, zn, dn);
        minv_jt(J, a.Minv + 36 * (size_t)b, lo, dold);
        for (int k = 0; k < 6; ++k) {
            long long *p = a.acc + 6 * (size_t)b + k;
            const long long s = __ldcg(p) + (quant(dn[k]) - quant(dold[k]));
            __stcg(p, s);
            __stcg(a.v + 6 * (size_t)b + k, a.vfree[6 * (size_t)b + k] + (T)((double)s / kScale));
        }
    }
}

template <typename T, int kKind>
__global__ void __launch_bounds__(kSweepThreads) k_sweeps(SweepArgs<T> a)
{
    const int ncol = a.stats[kNColors];
    // Task slot: chunk k = t / 32 of a colour runs on CTA k mod gridDim, so a colour narrower
    // than the launch is spread over every SM of it (contiguous slots would give all of a
    // colour's float64 work to its first CTAs).  A contact keeps its thread in every sweep.
    const int nb = gridDim.x, nth = gridDim.x * blockDim.x;
    const int tid = ((((int)threadIdx.x >> 5) * nb + (int)blockIdx.x) << 5) | ((int)threadIdx.x & 31);
    unsigned int epoch = 0;
    for (int it = 0; it < a.iters; ++it)
        for (int ci = 0; ci < ncol; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = tid; t < cnt; t += nth) sweep_contact(a, a.order[s0 + t]);
            if (!phase_barrier<kKind>(a, epoch)) return;
        }
}

template <typename T>
__global__ void k_resid(SweepArgs<T> a, T *__restrict__ res, T *__restrict__ uout,
                        unsigned long long *__restrict__ res_max)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= a.nc) return;
    T u[3], z[3], zn[3];
    const T lo[3] = {a.lam[3 * (size_t)c], a.lam[3 * (size_t)c + 1], a.lam[3 * (size_t)c + 2]};
    contact_u(c, a.Ja, a.Jb, a.pa[c], a.pb[c], a.bias, a.v, u);
    contact_z(u, lo, a.mu[c], a.rho[c], a.desaxce, a.soft, a.sep ? a.sep[c] : T(0), z);
    proj(z, a.mu[c], zn);
    T m = T(0);
    for (int i = 0; i < 3; ++i) {
        const T d = rab(lo[i] - zn[i]);
        if (d > m) m = d;
    }
    res[c] = m;
    uout[3 * (size_t)c] = u[0];
    uout[3 * (size_t)c + 1] = u[1];
    uout[3 * (size_t)c + 2] = u[2];
    // non-negative reals order like their bit patterns
    atomicMax(res_max, (unsigned long long)__double_as_longlong((double)m));
}

// Colouring behind the cache, one CTA.
template <typename T>
__global__ void __launch_bounds__(kColorThreads)
    k_color(int nc, int nb, const int *__restrict__ pa, const int *__restrict__ pb, const int *__restrict__ feat,
            const T *__restrict__ Minv, const int *__restrict__ dyn, b2c_ncp_state st, int use_cache, int max_colors)
{
    __shared__ int s_flag, s_left;
    __shared__ int s_cnt[kMaxColors];
    const int tid = threadIdx.x;
    int *S = st.stats;
    T *cm = reinterpret_cast<T *>(st.cache_minv);
    if (use_cache && S[kCacheValid] == 1 && S[kCachedC] == nc) {
        if (tid == 0) s_flag = 0;
        __syncthreads();
        int mism = 0;
        for (int c = tid; c < nc; c += kColorThreads)
            mism |= (pa[c] != st.cache_pa[c]) | (pb[c] != st.cache_pb[c]) | (feat[c] != st.cache_feat[c]);
        // the translational block (1/m I) and the dynamic flag (k_cache_cmp, :750-765)
        for (int i = tid; i < nb; i += kColorThreads)
            mism |= (Minv[36 * (size_t)i] != cm[4 * (size_t)i]) | (Minv[36 * (size_t)i + 7] != cm[4 * (size_t)i + 1]) |
                    (Minv[36 * (size_t)i + 14] != cm[4 * (size_t)i + 2]) | ((T)dyn[i] != cm[4 * (size_t)i + 3]);
        if (mism) atomicOr(&s_flag, 1);
        __syncthreads();
        if (s_flag == 0) {
            if (tid == 0) {
                S[kCacheHit] = 1;
                S[kHits] += 1;
            }
            return;
        }
    }
    for (int c = tid; c < nc; c += kColorThreads) st.col[c] = -1;
    int r = 0;
    bool done = nc == 0;
    for (; !done && r <= nc && r < max_colors; ++r) {
        for (int i = tid; i < nb; i += kColorThreads) st.claim[i] = ~0ull;
        __syncthreads();
        if (tid == 0) s_left = 0;
        for (int c = tid; c < nc; c += kColorThreads) {
            if (st.col[c] >= 0) continue;
            const unsigned long long k = mix64(((unsigned long long)(pa[c] + 1) * (unsigned long long)(nb + 1) +
                                                (unsigned long long)(pb[c] + 1)) * 1048576ull +
                                               (unsigned long long)(unsigned)feat[c]);
            unsigned long long *claim = reinterpret_cast<unsigned long long *>(st.claim);
            if (pa[c] >= 0 && dyn[pa[c]]) atomicMin(claim + pa[c], k);
            if (pb[c] >= 0 && dyn[pb[c]]) atomicMin(claim + pb[c], k);
        }
        __syncthreads();
        for (int c = tid; c < nc; c += kColorThreads) {
            if (st.col[c] >= 0) continue;
            const unsigned long long k = mix64(((unsigned long long)(pa[c] + 1) * (unsigned long long)(nb + 1) +
                                                (unsigned long long)(pb[c] + 1)) * 1048576ull +
                                               (unsigned long long)(unsigned)feat[c]);
            bool ok = true;
            if (pa[c] >= 0 && dyn[pa[c]] && st.claim[pa[c]] != k) ok = false;
            if (pb[c] >= 0 && dyn[pb[c]] && st.claim[pb[c]] != k) ok = false;
            if (ok) st.col[c] = r;
            else atomicAdd(&s_left, 1);
        }
        __syncthreads();
        done = s_left == 0;
        __syncthreads();  // every thread has read s_left before the next round resets it
    }
    const int ncol = done ? (nc > 0 ? r : 0) : r;
    if (!done || ncol > max_colors || ncol > kMaxColors) {
        if (tid == 0) {
            S[kError] |= done ? kErrColorOverflow : kErrColorTimeout;
            S[kNColors] = 0;
            S[kCacheValid] = 0;
            S[kRounds] = r;
        }
        return;
    }
    for (int k = tid; k < ncol; k += kColorThreads) s_cnt[k] = 0;
    __syncthreads();
    for (int c = tid; c < nc; c += kColorThreads) atomicAdd(&s_cnt[st.col[c]], 1);
    __syncthreads();
    if (tid == 0) {
        int acc = 0;
        for (int k = 0; k < ncol; ++k) {
            st.cstart[k] = acc;
            st.ccount[k] = s_cnt[k];
            const int t = s_cnt[k];
            s_cnt[k] = acc;
            acc += t;
        }
    }
    __syncthreads();
    for (int c = tid; c < nc; c += kColorThreads) st.order[atomicAdd(&s_cnt[st.col[c]], 1)] = c;
    if (use_cache) {
        for (int c = tid; c < nc; c += kColorThreads) {
            st.cache_pa[c] = pa[c];
            st.cache_pb[c] = pb[c];
            st.cache_feat[c] = feat[c];
        }
        for (int i = tid; i < nb; i += kColorThreads) {
            cm[4 * (size_t)i] = Minv[36 * (size_t)i];
            cm[4 * (size_t)i + 1] = Minv[36 * (size_t)i + 7];
            cm[4 * (size_t)i + 2] = Minv[36 * (size_t)i + 14];
            cm[4 * (size_t)i + 3] = (T)dyn[i];
        }
    }
    if (tid == 0) {
        S[kNColors] = ncol;
        S[kRounds] = r;
        S[kCacheHit] = 0;
        S[kCacheValid] = use_cache ? 1 : 0;
        S[kCachedC] = nc;
        S[kMisses] += 1;
    }
}

// ---------------------------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------------------------
template <typename T>
SweepArgs<T> sweep_args(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, int iters)
{
    SweepArgs<T> a;
    a.nc = sc->n_c;
    a.Ja = (const T *)sc->Ja;
    a.Jb = (const T *)sc->Jb;
    a.Minv = (const T *)sc->Minv;
    a.vfree = (const T *)sc->v_free;
    a.mu = (const T *)sc->mu;
    a.bias = (const T *)sc->bias;
    a.sep = (const T *)sc->sep;
    a.rho = (const T *)st->rho;
    a.pa = sc->pa;
    a.pb = sc->pb;
    a.order = st->order;
    a.cstart = st->cstart;
    a.ccount = st->ccount;
    a.dyn = st->dyn;
    a.lam = (T *)st->lam;
    a.v = (T *)st->v;
    a.acc = reinterpret_cast<long long *>(st->acc);
    a.stats = st->stats;
    a.bar = st->barrier;
    a.timeout_ns = (p && p->barrier_timeout_ns > 0) ? p->barrier_timeout_ns : 1000000000LL;  // default 1 s
    a.iters = iters;
    a.desaxce = p ? p->desaxce : 1;
    a.soft.on = p ? p->soft : 0;
    a.soft.use_bias = p ? p->use_bias : 1;
    for (int k = 0; k < 5; ++k) a.soft.p[k] = p ? p->softp[k] : 0.0;
    return a;
}

template <typename T>
int setup(const b2c_ncp_scene *sc, b2c_ncp_state *st, int warm, cudaStream_t s)
{
    const int nc = sc->n_c, nb = sc->n_b;
    if (nc > 0)
        k_rho<T><<<blocks_for(nc), kThreads, 0, s>>>(nc, (const T *)sc->Ja, (const T *)sc->Jb, (const T *)sc->Minv,
                                                     sc->pa, sc->pb, (T *)st->rho);
    if (nb > 0) k_dyn<T><<<blocks_for(nb), kThreads, 0, s>>>(nb, (const T *)sc->Minv, st->dyn);
    cudaMemsetAsync(st->acc, 0, sizeof(int64_t) * 6 * (size_t)nb, s);
    if (!warm) cudaMemsetAsync(st->lam, 0, sizeof(T) * 3 * (size_t)nc, s);
    else if (nc > 0)
        k_scatter<T><<<blocks_for(nc), kThreads, 0, s>>>(nc, (const T *)sc->Ja, (const T *)sc->Jb,
                                                         (const T *)sc->Minv, sc->pa, sc->pb, (const T *)st->lam,
                                                         reinterpret_cast<long long *>(st->acc));
    if (nb > 0)
        k_apply<T><<<blocks_for(6 * (long long)nb), kThreads, 0, s>>>(
            nb, (const T *)sc->v_free, reinterpret_cast<const long long *>(st->acc), (T *)st->v);
    return check_launch("ncp_setup");
}

template <typename T>
int color(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, cudaStream_t s)
{
    k_color<T><<<1, kColorThreads, 0, s>>>(sc->n_c, sc->n_b, sc->pa, sc->pb, sc->feature, (const T *)sc->Minv, st->dyn,
                                           *st, p->color_cache, std::min(st->max_colors, kMaxColors));
    return check_launch("ncp_color");
}

template <typename T>
int cluster_size()
{
    static int cached = -1;
    if (cached < 0) {
        cudaFuncSetAttribute(k_sweeps<T, kCluster>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterMax);
        cfg.blockDim = dim3(kSweepThreads);
        int cs = 0;
        if (cudaOccupancyMaxPotentialClusterSize(&cs, k_sweeps<T, kCluster>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            cs = 1;
        }
        int p2 = 1;
        for (int c = 1; c <= std::min(cs, kClusterMax); c *= 2) p2 = c;
        cached = p2;
    }
    return cached;
}

// CTAs of the grid sweep the device holds at once (SMs x resident CTAs per SM); cached per type
template <typename T>
int grid_blocks()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sweeps<T, kGrid>, kSweepThreads, 0);
        cached = std::min(kBarrierMaxCTAs, std::max(1, sms * per));
    }
    return cached;
}

template <typename T>
int sweeps(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, int iters, cudaStream_t s)
{
    if (iters <= 0 || sc->n_c == 0) return B2C_OK;
    const SweepArgs<T> a = sweep_args<T>(sc, st, p, iters);
    int mode = p->solve_blocks;
    // auto: one CTA for small scenes; else every SM (the sweep's float64 work needs their issue
    // rate: on the 40 000-contact lattice a grid of 148 CTAs takes 4.6 ms for 40 sweeps, a
    // 16-CTA cluster 6.6 ms)
    if (mode == 0) mode = sc->n_c <= 16384 ? 1 : grid_blocks<T>();
    if (mode > 1) {  // a cooperative grid of at most the co-resident CTAs
        const int nblocks = std::min(mode, grid_blocks<T>());
        if (nblocks > 1) {
            cudaMemsetAsync(st->barrier, 0, sizeof(uint32_t), s);  // the arrival count restarts every launch
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(nblocks);
            cfg.blockDim = dim3(kSweepThreads);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_sweeps<T, kGrid>, a);
            if (e != cudaSuccess) {
                set_error("ncp_sweeps: cooperative launch of %d CTAs: %s", nblocks, cudaGetErrorString(e));
                return B2C_ECUDA;
            }
            return check_launch("ncp_sweeps_grid");
        }
        mode = 1;
    }
    if (mode < 0) {
        const int cs = std::min(-mode, cluster_size<T>());
        if (cs >= 2) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cs);
            cfg.blockDim = dim3(kSweepThreads);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cs;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_sweeps<T, kCluster>, a);
            if (e != cudaSuccess) {
                set_error("ncp_sweeps: cluster launch of %d CTAs: %s", cs, cudaGetErrorString(e));
                return B2C_ECUDA;
            }
            return check_launch("ncp_sweeps_cluster");
        }
    }
    k_sweeps<T, kBlock><<<1, kSweepThreads, 0, s>>>(a);
    return check_launch("ncp_sweeps");
}

template <typename T>
int residual(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, cudaStream_t s)
{
    cudaMemsetAsync(st->res_max, 0, sizeof(uint64_t), s);
    if (sc->n_c == 0) return check_launch("ncp_residual");
    const SweepArgs<T> a = sweep_args<T>(sc, st, p, 0);
    k_resid<T><<<blocks_for(sc->n_c), kThreads, 0, s>>>(a, (T *)st->res, (T *)st->u,
                                                         reinterpret_cast<unsigned long long *>(st->res_max));
    return check_launch("ncp_residual");
}

}  // namespace ncp
}  // namespace b2c

static bool ncp_scene_ok(const b2c_ncp_scene *sc, const b2c_ncp_state *st)
{
    return sc && st && (sc->dtype == 4 || sc->dtype == 8) && sc->n_c >= 0 && sc->n_b >= 0 &&
           sc->n_c <= st->max_contacts && sc->n_b <= st->n_bodies && sc->Ja && sc->Jb && sc->Minv && sc->v_free &&
           sc->mu && sc->bias && sc->pa && sc->pb && sc->feature && st->rho && st->lam && st->v && st->acc &&
           st->res && st->u && st->col && st->order && st->cstart && st->ccount && st->claim && st->dyn &&
           st->cache_pa && st->cache_pb && st->cache_feat && st->cache_minv && st->stats && st->res_max &&
           st->barrier && st->max_colors >= 1;
}

extern "C" int32_t b2c_ncp_setup(const b2c_ncp_scene *sc, b2c_ncp_state *st, int32_t warm, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st)) {
        b2c::set_error("b2c_ncp_setup: bad argument");
        return B2C_EARG;
    }
    return sc->dtype == 4 ? b2c::ncp::setup<float>(sc, st, warm, b2c::stream_of(s))
                          : b2c::ncp::setup<double>(sc, st, warm, b2c::stream_of(s));
}

extern "C" int32_t b2c_ncp_color(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p) {
        b2c::set_error("b2c_ncp_color: bad argument");
        return B2C_EARG;
    }
    return sc->dtype == 4 ? b2c::ncp::color<float>(sc, st, p, b2c::stream_of(s))
                          : b2c::ncp::color<double>(sc, st, p, b2c::stream_of(s));
}

extern "C" int32_t b2c_ncp_sweeps(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                  int32_t iters, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p || iters < 0) {
        b2c::set_error("b2c_ncp_sweeps: bad argument");
        return B2C_EARG;
    }
    return sc->dtype == 4 ? b2c::ncp::sweeps<float>(sc, st, p, iters, b2c::stream_of(s))
                          : b2c::ncp::sweeps<double>(sc, st, p, iters, b2c::stream_of(s));
}

extern "C" int32_t b2c_ncp_residual(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                    b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p) {
        b2c::set_error("b2c_ncp_residual: bad argument");
        return B2C_EARG;
    }
    return sc->dtype == 4 ? b2c::ncp::residual<float>(sc, st, p, b2c::stream_of(s))
                          : b2c::ncp::residual<double>(sc, st, p, b2c::stream_of(s));
}
