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
constexpr int kSweepThreads = 1024;  // 64 groups of 16 lanes: one contact each
constexpr int kAdjThreads = 512;     // the reverse sweeps: one thread per contact
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
    double *trace;  // null, or (iters, nc, kTraceWords): what each contact's update of each sweep started from
    int *stats;
    unsigned int *bar;
    long long timeout_ns;
    int iters, desaxce;
    Soft soft;
};

enum Kind { kBlock = 0, kCluster = 1, kGrid = 2 };

// A recorded update, written by the sweeps: the contact's impulse before it [0, 3), the
// velocities of its bodies a, b [3, 9), [9, 15) (zero where there is no body), the impulse
// change dl [18, 21), the projection's argument z [33, 36) and the contact velocity u [36, 39);
// the reverse sweep adds the update's adjoints: ub [15, 18) and the adjoints of both bodies'
// velocities after the update [21, 27), [27, 33).
constexpr int kTraceWords = 39;

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

// One contact update of k_sweep (:485-568): u = bias + Ja v_a + Jb v_b (contact_u's sums), the
// projection of contact_z's argument, then for each dynamic body the swap of the contact's
// rounded contribution Minv J^T lambda in the int64 accumulator (f_swap, :425-438) and the
// body's velocity rebuilt from it (k_apply_c, :583-599).  It runs on a group of kGroup = 16
// lanes, so that one contact's dependent chain is short: lanes 0..5 form the six 6-term sums of
// u (row i = lane % 3 of side lane / 3); every lane then has u, z and the projection (the same
// bits in each); lanes 0..11 each own one velocity component k of one side: row k of the
// Minv J^T products, the accumulator swap and the velocity rebuild (one division each, in
// parallel).  Every sum runs in the same order as a one-thread update would.
constexpr int kGroup = 16;

template <typename T>
__device__ __forceinline__ T group_get(T x, int src, unsigned mask)
{
    return __shfl_sync(mask, x, src, kGroup);
}

template <typename T>
__device__ __forceinline__ void sweep_contact_group(const SweepArgs<T> &a, int c, int it, int l, unsigned mask)
{
    const int pa = a.pa[c], pb = a.pb[c];
    const T lo[3] = {a.lam[3 * (size_t)c], a.lam[3 * (size_t)c + 1], a.lam[3 * (size_t)c + 2]};
    // the six partial sums of u
    T part = T(0), vs[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
    if (l < 6) {
        const int i = l % 3, side = l / 3, b = side == 0 ? pa : pb;
        if (b >= 0) {
            for (int j = 0; j < 6; ++j) vs[j] = __ldcg(a.v + 6 * (size_t)b + j);
            const T *J = (side == 0 ? a.Ja : a.Jb) + 18 * (size_t)c + 6 * i;
            T sacc = J[0] * vs[0];
            for (int j = 1; j < 6; ++j) sacc = sacc + J[j] * vs[j];
            part = sacc;
        }
    }
    T u[3];
    for (int i = 0; i < 3; ++i) {
        const T sa = group_get(part, i, mask), sb = group_get(part, 3 + i, mask);
        T ui = a.bias[3 * (size_t)c + i];
        if (pa >= 0) ui = ui + sa;
        if (pb >= 0) ui = ui + sb;
        u[i] = ui;
    }
    T z[3], zn[3];
    contact_z(u, lo, a.mu[c], a.rho[c], a.desaxce, a.soft, a.sep ? a.sep[c] : T(0), z);
    proj(z, a.mu[c], zn);
    if (a.trace) {
        double *t = a.trace + kTraceWords * ((size_t)it * a.nc + c);
        if (l == 0)
            for (int k = 0; k < 3; ++k) {
                t[k] = (double)lo[k];
                t[18 + k] = (double)zn[k] - (double)lo[k];
                t[33 + k] = (double)z[k];
                t[36 + k] = (double)u[k];
            }
        if (l == 0 || l == 3)
            for (int k = 0; k < 6; ++k) t[(l == 0 ? 3 : 9) + k] = (double)vs[k];
    }
    if (l == 0) {
        a.lam[3 * (size_t)c] = zn[0];
        a.lam[3 * (size_t)c + 1] = zn[1];
        a.lam[3 * (size_t)c + 2] = zn[2];
    }
    if (l < 12) {
        const int side = l / 6, k = l % 6, b = side == 0 ? pa : pb;
        if (b >= 0 && a.dyn[b]) {
            const T *J = (side == 0 ? a.Ja : a.Jb) + 18 * (size_t)c;
            const T *M = a.Minv + 36 * (size_t)b + 6 * k;
            // row k of Minv (J^T l), minv_jt's order, for the new and the old impulse
            T dn = T(0), dold = T(0);
            for (int j = 0; j < 6; ++j) {
                T tn = J[j] * zn[0];
                tn = tn + J[6 + j] * zn[1];
                tn = tn + J[12 + j] * zn[2];
                T to = J[j] * lo[0];
                to = to + J[6 + j] * lo[1];
                to = to + J[12 + j] * lo[2];
                if (j == 0) {
                    dn = M[0] * tn;
                    dold = M[0] * to;
                } else {
                    dn = dn + M[j] * tn;
                    dold = dold + M[j] * to;
                }
            }
            long long *p = a.acc + 6 * (size_t)b + k;
            const long long sacc = __ldcg(p) + (quant(dn) - quant(dold));
            __stcg(p, sacc);
            __stcg(a.v + 6 * (size_t)b + k, a.vfree[6 * (size_t)b + k] + (T)((double)sacc / kScale));
        }
    }
}

template <typename T, int kKind>
__global__ void __launch_bounds__(kSweepThreads) k_sweeps(SweepArgs<T> a)
{
    const int ncol = a.stats[kNColors];
    // Task slot: one group of kGroup lanes per contact; group g = (group in CTA) x CTAs + CTA,
    // so consecutive contacts of a colour land on different CTAs and a colour narrower than
    // the launch is spread over every SM of it.  A contact keeps its group in every sweep.
    const int nb = gridDim.x, groups = nb * (blockDim.x / kGroup);
    const int g = ((int)threadIdx.x / kGroup) * nb + (int)blockIdx.x, l = (int)threadIdx.x % kGroup;
    const unsigned mask = 0xFFFFu << (((int)threadIdx.x & 31) & ~(kGroup - 1));
    unsigned int epoch = 0;
    for (int it = 0; it < a.iters; ++it)
        for (int ci = 0; ci < ncol; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = g; t < cnt; t += groups) sweep_contact_group(a, a.order[s0 + t], it, l, mask);
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
    a.trace = nullptr;
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

// The same colouring over a cooperative grid: every Jones-Plassmann round is three grid phases
// (reset the claims; claim; win) with the arrival-counter barrier between them, so a round costs
// a few microseconds however many contacts there are (the one-CTA form walks all of them with
// 1024 threads, once per round).  Jones-Plassmann is local -- a contact takes colour r when it
// holds the smallest key at each of its dynamic bodies among the contacts still uncoloured -- so
// the colours are those of k_color exactly; only the order of the contacts inside a colour
// (which thread sweeps which contact) differs, and the sweeps do not depend on it.  Scratch words
// of the barrier buffer: [8], [9] the uncoloured counts of alternate rounds, [10] the cache
// mismatch flag (all zero at launch).
constexpr int kColorGridThreads = 512;

template <typename T>
__global__ void __launch_bounds__(kColorGridThreads)
    k_color_grid(int nc, int nb, const int *__restrict__ pa, const int *__restrict__ pb, const int *__restrict__ feat,
                 const T *__restrict__ Minv, const int *__restrict__ dyn, b2c_ncp_state st, int use_cache,
                 int max_colors, long long timeout_ns)
{
    __shared__ int s_cnt;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const bool lead = gid == 0;
    int *S = st.stats;
    unsigned int *bar = st.barrier;
    unsigned int epoch = 0;
    T *cm = reinterpret_cast<T *>(st.cache_minv);
    auto sync = [&]() -> bool {
        ++epoch;
        grid_arrive(bar);
        return grid_wait(bar, epoch, timeout_ns, S + kError, kErrBarrier);
    };
    auto key_of = [&](int c) -> unsigned long long {
        return mix64(((unsigned long long)(pa[c] + 1) * (unsigned long long)(nb + 1) + (unsigned long long)(pb[c] + 1)) *
                         1048576ull +
                     (unsigned long long)(unsigned)feat[c]);
    };
    if (use_cache && S[kCacheValid] == 1 && S[kCachedC] == nc) {
        int mism = 0;
        for (int c = gid; c < nc; c += nth)
            mism |= (pa[c] != st.cache_pa[c]) | (pb[c] != st.cache_pb[c]) | (feat[c] != st.cache_feat[c]);
        for (int i = gid; i < nb; i += nth)
            mism |= (Minv[36 * (size_t)i] != cm[4 * (size_t)i]) | (Minv[36 * (size_t)i + 7] != cm[4 * (size_t)i + 1]) |
                    (Minv[36 * (size_t)i + 14] != cm[4 * (size_t)i + 2]) | ((T)dyn[i] != cm[4 * (size_t)i + 3]);
        if (mism) atomicOr(bar + 10, 1u);
        if (!sync()) return;
        if (__ldcg(bar + 10) == 0u) {
            if (lead) {
                S[kCacheHit] = 1;
                S[kHits] += 1;
            }
            return;
        }
    }
    for (int c = gid; c < nc; c += nth) st.col[c] = -1;
    unsigned long long *claim = reinterpret_cast<unsigned long long *>(st.claim);
    int r = 0;
    bool done = nc == 0;
    for (; !done && r <= nc && r < max_colors; ++r) {
        for (int i = gid; i < nb; i += nth) claim[i] = ~0ull;
        if (!sync()) return;
        if (lead) bar[8 + ((r + 1) & 1)] = 0u;  // every CTA has read the previous round's count
        for (int c = gid; c < nc; c += nth) {
            if (st.col[c] >= 0) continue;
            const unsigned long long k = key_of(c);
            if (pa[c] >= 0 && dyn[pa[c]]) atomicMin(claim + pa[c], k);
            if (pb[c] >= 0 && dyn[pb[c]]) atomicMin(claim + pb[c], k);
        }
        if (!sync()) return;
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        int left = 0;
        for (int c = gid; c < nc; c += nth) {
            if (st.col[c] >= 0) continue;
            const unsigned long long k = key_of(c);
            bool ok = true;
            if (pa[c] >= 0 && dyn[pa[c]] && __ldcg(claim + pa[c]) != k) ok = false;
            if (pb[c] >= 0 && dyn[pb[c]] && __ldcg(claim + pb[c]) != k) ok = false;
            if (ok) st.col[c] = r;
            else ++left;
        }
        if (left) atomicAdd(&s_cnt, left);
        __syncthreads();
        if (threadIdx.x == 0 && s_cnt) atomicAdd(bar + 8 + (r & 1), (unsigned)s_cnt);
        if (!sync()) return;
        done = __ldcg(bar + 8 + (r & 1)) == 0u;
    }
    const int ncol = done ? (nc > 0 ? r : 0) : r;
    if (!done || ncol > max_colors || ncol > kMaxColors) {
        if (lead) {
            S[kError] |= done ? kErrColorOverflow : kErrColorTimeout;
            S[kNColors] = 0;
            S[kCacheValid] = 0;
            S[kRounds] = r;
        }
        return;
    }
    // counts per colour, then their exclusive scan (one thread), then the scatter with the
    // counts as cursors (they end where they started)
    for (int k = gid; k < ncol; k += nth) st.ccount[k] = 0;
    if (!sync()) return;
    for (int c = gid; c < nc; c += nth) atomicAdd(st.ccount + st.col[c], 1);
    if (!sync()) return;
    if (lead) {
        int acc = 0;
        for (int k = 0; k < ncol; ++k) {
            st.cstart[k] = acc;
            acc += __ldcg(st.ccount + k);
            st.ccount[k] = 0;
        }
    }
    if (!sync()) return;
    for (int c = gid; c < nc; c += nth) {
        const int k = st.col[c];
        st.order[__ldcg(st.cstart + k) + atomicAdd(st.ccount + k, 1)] = c;
    }
    if (use_cache) {
        for (int c = gid; c < nc; c += nth) {
            st.cache_pa[c] = pa[c];
            st.cache_pb[c] = pb[c];
            st.cache_feat[c] = feat[c];
        }
        for (int i = gid; i < nb; i += nth) {
            cm[4 * (size_t)i] = Minv[36 * (size_t)i];
            cm[4 * (size_t)i + 1] = Minv[36 * (size_t)i + 7];
            cm[4 * (size_t)i + 2] = Minv[36 * (size_t)i + 14];
            cm[4 * (size_t)i + 3] = (T)dyn[i];
        }
    }
    if (lead) {
        S[kNColors] = ncol;
        S[kRounds] = r;
        S[kCacheHit] = 0;
        S[kCacheValid] = use_cache ? 1 : 0;
        S[kCachedC] = nc;
        S[kMisses] += 1;
    }
}

template <typename T>
int color(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, cudaStream_t s)
{
    const int maxc = std::min(st->max_colors, kMaxColors);
    int mode = p->solve_blocks;
    if (mode == 0) mode = sc->n_c <= 16384 ? 1 : 2;
    if (mode > 1) {  // a cooperative grid of one CTA per SM (fewer arrivals per barrier)
        static int nblocks = -1;
        if (nblocks < 0) {
            int dev = 0, sms = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_color_grid<T>, kColorGridThreads, 0);
            nblocks = per > 0 ? std::min(kBarrierMaxCTAs, sms) : 1;
        }
        if (nblocks > 1) {
            cudaMemsetAsync(st->barrier, 0, sizeof(uint32_t) * kBarrierWords, s);
            const long long tmo = p->barrier_timeout_ns > 0 ? p->barrier_timeout_ns : 1000000000LL;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(nblocks);
            cfg.blockDim = dim3(kColorGridThreads);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_color_grid<T>, sc->n_c, sc->n_b, sc->pa, sc->pb,
                                                     sc->feature, (const T *)sc->Minv, st->dyn, *st, p->color_cache,
                                                     maxc, tmo);
            if (e != cudaSuccess) {
                set_error("ncp_color: cooperative launch of %d CTAs: %s", nblocks, cudaGetErrorString(e));
                return B2C_ECUDA;
            }
            return check_launch("ncp_color_grid");
        }
    }
    k_color<T><<<1, kColorThreads, 0, s>>>(sc->n_c, sc->n_b, sc->pa, sc->pb, sc->feature, (const T *)sc->Minv, st->dyn,
                                           *st, p->color_cache, maxc);
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
int sweeps(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, int iters, cudaStream_t s,
           double *trace = nullptr)
{
    if (iters <= 0 || sc->n_c == 0) return B2C_OK;
    SweepArgs<T> a = sweep_args<T>(sc, st, p, iters);
    a.trace = trace;
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

// ---------------------------------------------------------------------------------------------
// The adjoint of the sweeps at a fixed point (float64): the implicit-function derivative of the
// converged impulses, as the reverse of `iters` sweeps evaluated at the final iterate.
//
// A forward sweep maps lambda -> Phi(lambda; b, mu) with b = J v_free + bias; at its fixed point
// lambda* the implicit function theorem gives d lambda* = (I - dPhi/dlambda)^-1 dPhi/d(b, mu).
// Its transpose applied to an adjoint g is the limit of the reverse sweeps: starting from g,
// each reverse sweep (colours in reverse order, each contact the transposed derivative of its
// update at lambda*) pushes the adjoint back through one sweep and hands the free velocity, the
// bias and the friction their share; `iters` reverse sweeps sum the first `iters` terms of that
// Neumann series, the same truncation as `iters` forward sweeps from a warm start.
//
// One contact update (forward, in colour order, v the current body velocities):
//   u = J v + bias,  z = lambda - rho (u + (mu |u_t|, 0, 0)),  lambda' = proj_K(z),
//   v += Minv J^T (lambda' - lambda).
// Its reverse, given the adjoints gl of lambda' and Vb of v after it:
//   g  = gl + J Minv Vb;  (zb, mub) = the transposed derivative of proj_K at z applied to g;
//   gl <- zb - J Minv Vb;  ub = -rho (zb + mu zb_n u_t / |u_t| on the tangential rows);
//   Vb += J^T ub;  bias_b += ub;  mu_b += mub - rho |u_t| zb_n.
// After the last (first) colour, the adjoint of v at the sweep's start goes to v_free (v =
// v_free + Minv J^T lambda) and, through J Minv, back onto every gl; Vb restarts at zero.
// Within a colour no two contacts share a dynamic body, so every write is the owner's; the
// adjoint of kinematic and static bodies is not kept (their velocity is prescribed).
// ---------------------------------------------------------------------------------------------
struct AdjArgs {
    int nc, nb, iters, desaxce;
    const double *Ja, *Jb, *Minv, *mu, *rho, *lam, *u;
    double *trace;  // null: every reverse sweep at the final iterate (lam, u); else the recorded sweeps
    const double *bias;
    const int *pa, *pb, *order, *cstart, *ccount, *dyn;
    double *gl, *vb, *vfree_b, *bias_b, *mu_b;
    double *Ja_b, *Jb_b, *Minv_b, *rho_b;  // the recorded form's adjoints of the blocks and step sizes
    int *stats;
    unsigned int *bar;
    long long timeout_ns;
};

// J_side (3x6) Minv_b (6x6) x, x = Vb of body b (6): out[3] += J (Minv x)
__device__ __forceinline__ void add_j_minv(const double *J, const double *M, const double *x, double out[3])
{
    double t[6];
    for (int k = 0; k < 6; ++k) {
        double s = 0.0;
        for (int j = 0; j < 6; ++j) s += M[k * 6 + j] * x[j];
        t[k] = s;
    }
    for (int r = 0; r < 3; ++r) {
        double s = 0.0;
        for (int k = 0; k < 6; ++k) s += J[r * 6 + k] * t[k];
        out[r] += s;
    }
}

// The de Saxce term mu |u_t| has a kink at u_t = 0, where a sticking contact sits: its slip
// speed there is the rounding of the fixed-point velocity sums (1e-10 m/s), whose direction says
// nothing.  Below this speed the adjoints take the term's derivative in u_t as zero (the stick
// rows of the implicit-function system, ncp_ref.py:_active_system, carry no such term either).
constexpr double kStickSpeed = 1e-8;

// transposed derivative of proj_K (the branches of proj) at z, applied to g: zb, and mub
__device__ __forceinline__ void proj_adjoint(const double z[3], double mu, const double g[3], double zb[3],
                                             double &mub)
{
    const double zn = z[0], zt = sqrt(z[1] * z[1] + z[2] * z[2]);
    if (zt <= mu * zn) {
        zb[0] = g[0];
        zb[1] = g[1];
        zb[2] = g[2];
        return;
    }
    if (mu * zt <= -zn) {
        zb[0] = zb[1] = zb[2] = 0.0;
        return;
    }
    // s = (zn + mu zt) / (1 + mu^2), f = mu s / zt, out = (s, f z1, f z2)
    const double den = 1.0 + mu * mu, iden = 1.0 / den, izt = 1.0 / zt;
    const double sv = (zn + mu * zt) * iden;
    const double f = mu * sv * izt;
    const double t1 = z[1] * izt, t2 = z[2] * izt;
    const double ds_dzn = iden;
    const double ds_dt1 = mu * t1 * iden, ds_dt2 = mu * t2 * iden;
    const double ds_dmu = (zt * den - 2.0 * mu * (zn + mu * zt)) * iden * iden;
    const double df_dzn = mu * ds_dzn * izt;
    const double df_dt1 = (mu * ds_dt1 - mu * sv * t1 * izt) * izt;
    const double df_dt2 = (mu * ds_dt2 - mu * sv * t2 * izt) * izt;
    const double df_dmu = (sv + mu * ds_dmu) * izt;
    const double gz = g[1] * z[1] + g[2] * z[2];
    zb[0] = g[0] * ds_dzn + gz * df_dzn;
    zb[1] = g[0] * ds_dt1 + f * g[1] + gz * df_dt1;
    zb[2] = g[0] * ds_dt2 + f * g[2] + gz * df_dt2;
    mub += g[0] * ds_dmu + gz * df_dmu;
}

__device__ void adj_contact(const AdjArgs &a, int c)
{
    const int A = a.pa[c], B = a.pb[c];
    const bool dA = A >= 0 && a.dyn[A], dB = B >= 0 && a.dyn[B];
    double vA[6], vBb[6];
    double jm[3] = {0.0, 0.0, 0.0};
    if (dA) {
        for (int k = 0; k < 6; ++k) vA[k] = __ldcg(a.vb + 6 * (size_t)A + k);
        add_j_minv(a.Ja + 18 * (size_t)c, a.Minv + 36 * (size_t)A, vA, jm);
    }
    if (dB) {
        for (int k = 0; k < 6; ++k) vBb[k] = __ldcg(a.vb + 6 * (size_t)B + k);
        add_j_minv(a.Jb + 18 * (size_t)c, a.Minv + 36 * (size_t)B, vBb, jm);
    }
    double g[3], z[3], u[3], lo[3];
    const double mu = a.mu[c], rho = a.rho[c];
    for (int k = 0; k < 3; ++k) {
        g[k] = a.gl[3 * (size_t)c + k] + jm[k];
        u[k] = a.u[3 * (size_t)c + k];
        lo[k] = a.lam[3 * (size_t)c + k];
    }
    const double ut = sqrt(u[1] * u[1] + u[2] * u[2]);
    const double s0 = a.desaxce ? u[0] + mu * ut : u[0];
    z[0] = lo[0] - rho * s0;
    z[1] = lo[1] - rho * u[1];
    z[2] = lo[2] - rho * u[2];
    double zb[3], mub = 0.0;
    proj_adjoint(z, mu, g, zb, mub);
    double ub[3];
    ub[0] = -rho * zb[0];
    ub[1] = -rho * zb[1];
    ub[2] = -rho * zb[2];
    if (a.desaxce) {
        mub += -rho * ut * zb[0];
        if (ut > kStickSpeed) {
            ub[1] += -rho * mu * (u[1] / ut) * zb[0];
            ub[2] += -rho * mu * (u[2] / ut) * zb[0];
        }
    }
    for (int k = 0; k < 3; ++k) {
        a.gl[3 * (size_t)c + k] = zb[k] - jm[k];
        a.bias_b[3 * (size_t)c + k] += ub[k];
    }
    a.mu_b[c] += mub;
    for (int side = 0; side < 2; ++side) {
        if (!(side == 0 ? dA : dB)) continue;
        const int b = side == 0 ? A : B;
        const double *J = (side == 0 ? a.Ja : a.Jb) + 18 * (size_t)c;
        const double *cur = side == 0 ? vA : vBb;
        for (int k = 0; k < 6; ++k)
            __stcg(a.vb + 6 * (size_t)b + k, cur[k] + ((J[k] * ub[0] + J[6 + k] * ub[1]) + J[12 + k] * ub[2]));
    }
}

// The reverse of one recorded update of contact c in sweep `it` (sweep_contact_group):
//   u = bias + Ja va + Jb vb,  z = lo - rho (u_n + mu |u_t| (de Saxce), u_t),  l = proj(z),
//   v_a += Minv_a Ja^T (l - lo),  v_b likewise,
// with z and u read back from the record.  On entry gl[c] is the adjoint of l and vb the
// adjoint of the velocities after the update; on exit gl[c] is the adjoint of lo and vb that of
// the velocities before it, and bias_b, mu_b, rho_b hold the update's share.  Only vb and gl
// are on the path to the next update; what the blocks' and Minv's adjoints need (ub, the impulse
// change dl, the velocity adjoints) goes back into the trace for adj_start_group.
// It runs on a group of kGroup lanes (the forward's layout): lanes 0..5 the six sums of u,
// lanes 0..11 one velocity component k of one side each (its vbar, row k of Minv vbar, its
// share of J Minv vbar -- summed over the lanes by a fixed butterfly -- and its vbar update),
// every lane the projection and its adjoint.
__device__ void adj_contact_group(const AdjArgs &a, int c, int it, int l, unsigned mask)
{
    const int A = a.pa[c], B = a.pb[c];
    const bool dA = A >= 0 && a.dyn[A], dB = B >= 0 && a.dyn[B];
    double *tr = a.trace + kTraceWords * ((size_t)it * a.nc + c);
    const double *JA = a.Ja + 18 * (size_t)c, *JB = a.Jb + 18 * (size_t)c;
    const int side = l / 6, k = l % 6, b = side == 0 ? A : B;
    const bool mine = l < 12 && (side == 0 ? dA : dB);
    const double *J = side == 0 ? JA : JB;
    // only vbar waits on the previous colour; the record and the per-contact sums do not
    const double w = mine ? __ldcg(a.vb + 6 * (size_t)b + k) : 0.0;
    const double z[3] = {tr[33], tr[34], tr[35]}, u[3] = {tr[36], tr[37], tr[38]};
    const double gl0[3] = {a.gl[3 * (size_t)c], a.gl[3 * (size_t)c + 1], a.gl[3 * (size_t)c + 2]};
    const double mu = a.mu[c], rho = a.rho[c];
    const double ut = sqrt(u[1] * u[1] + u[2] * u[2]);
    const double s0 = a.desaxce ? u[0] + mu * ut : u[0];
    // row k of Minv vbar for this lane's side, then J Minv vbar summed over the lanes
    double mk = 0.0;
    {
        const int base = side * 6;
        double wj[6];
        for (int j = 0; j < 6; ++j) wj[j] = group_get(w, (base + j) & (kGroup - 1), mask);
        if (mine) {
            const double *M = a.Minv + 36 * (size_t)b + 6 * k;
            for (int j = 0; j < 6; ++j) mk += M[j] * wj[j];
        }
    }
    double jm[3];
    for (int r = 0; r < 3; ++r) {
        double x = mine ? J[6 * r + k] * mk : 0.0;
        for (int off = kGroup / 2; off > 0; off >>= 1) x += __shfl_xor_sync(mask, x, off, kGroup);
        jm[r] = x;
    }
    double g[3];
    for (int r = 0; r < 3; ++r) g[r] = gl0[r] + jm[r];
    double zb[3], mub = 0.0;
    proj_adjoint(z, mu, g, zb, mub);
    double ub[3] = {-rho * zb[0], -rho * zb[1], -rho * zb[2]};
    const double rb = -(zb[0] * s0 + zb[1] * u[1] + zb[2] * u[2]);
    if (a.desaxce) {
        mub += -rho * ut * zb[0];
        if (ut > kStickSpeed) {
            const double q = -rho * mu / ut;
            ub[1] += q * u[1] * zb[0];
            ub[2] += q * u[2] * zb[0];
        }
    }
    if (mine) {
        __stcg(a.vb + 6 * (size_t)b + k, w + ((J[k] * ub[0] + J[6 + k] * ub[1]) + J[12 + k] * ub[2]));
        tr[21 + 6 * side + k] = w;
    } else if (l < 12) {
        tr[21 + 6 * side + k] = 0.0;
    }
    if (l == 0) {
        for (int r = 0; r < 3; ++r) {
            a.gl[3 * (size_t)c + r] = zb[r] - jm[r];
            a.bias_b[3 * (size_t)c + r] += ub[r];
            tr[15 + r] = ub[r];
        }
        a.mu_b[c] += mub;
        a.rho_b[c] += rb;
    }
}

// unit eigenvector of the largest eigenvalue lm of a symmetric 3x3 W, from the largest cross
// product of two rows of W - lm I; false when that eigenvalue is not simple (no derivative)
__device__ bool eigvec_max3(const double W[3][3], double lm, double e[3])
{
    double R[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = W[i][j] - (i == j ? lm : 0.0);
    double best = 0.0;
    for (int p = 0; p < 3; ++p) {
        const double *x = R[p], *y = R[(p + 1) % 3];
        const double cr[3] = {x[1] * y[2] - x[2] * y[1], x[2] * y[0] - x[0] * y[2], x[0] * y[1] - x[1] * y[0]};
        const double nn = cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2];
        if (nn > best) {
            best = nn;
            for (int k = 0; k < 3; ++k) e[k] = cr[k];
        }
    }
    if (!(best > 1e-20 * lm * lm * lm * lm)) return false;
    const double inv = 1.0 / sqrt(best);
    for (int k = 0; k < 3; ++k) e[k] *= inv;
    return true;
}

// The derivative of rho_c = 1 / lambda_max(W_c) takes the projector P onto the eigenspace of
// the largest eigenvalue lm, divided by its dimension k: d lm = tr(P dW) / k.  For a simple
// eigenvalue (k = 1) that is the derivative; for a repeated one -- every corner contact of a
// cube on the ground, whose inertia is isotropic, has lm twice -- lm is not differentiable and
// tr(P dW) / k, the derivative of the mean of the k top eigenvalues, is what a central
// difference measures.  Eigenvalues within 1e-6 lm of lm count as repeated.
__device__ void top_projector(const double W[3][3], double lm, double P[3][3])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[i][j] = 0.0;
    const double c2 = W[0][0] + W[1][1] + W[2][2];
    const double c1 = (W[0][0] * W[1][1] - W[0][1] * W[1][0]) + (W[0][0] * W[2][2] - W[0][2] * W[2][0]) +
                      (W[1][1] * W[2][2] - W[1][2] * W[2][1]);
    const double sm = c2 - lm, pr = c1 - lm * sm;  // the other two: sum and product
    const double disc = sqrt(fmax(sm * sm - 4.0 * pr, 0.0));
    const double l2 = 0.5 * (sm + disc), l3 = 0.5 * (sm - disc);
    const double tol = 1e-6 * lm;
    if (lm - l3 <= tol) {
        for (int i = 0; i < 3; ++i) P[i][i] = 1.0 / 3.0;
        return;
    }
    if (lm - l2 <= tol) {  // W - lm I ~ (l3 - lm) e3 e3^T: its largest row is along e3
        int best = 0;
        double bn = -1.0;
        for (int r = 0; r < 3; ++r) {
            double nn = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double x = W[r][k] - (r == k ? lm : 0.0);
                nn += x * x;
            }
            if (nn > bn) {
                bn = nn;
                best = r;
            }
        }
        double e3[3];
        const double inv = 1.0 / sqrt(bn);
        for (int k = 0; k < 3; ++k) e3[k] = (W[best][k] - (best == k ? lm : 0.0)) * inv;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) P[i][j] = 0.5 * ((i == j ? 1.0 : 0.0) - e3[i] * e3[j]);
        return;
    }
    double e[3];
    if (!eigvec_max3(W, lm, e)) return;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) P[i][j] = e[i] * e[j];
}

// After the reverse sweeps, per contact (colour by colour, so that each dynamic body belongs to
// one contact at a time): the blocks' and Minv's adjoints summed over the recorded updates --
// ub (x) v (through u) and dl (x) Minv vbar (through the velocity change) for the blocks,
// vbar (x) J^T dl for Minv -- and the start of the sweeps, v = v_free + Minv sum_c J_c^T lo_c
// (setup, lo the warm start) and rho_c = 1 / lambda_max(W_c), W_c = sum_sides J Minv J^T
// (k_rho): gl[c] += J Minv vbar (the warm start's adjoint), lo (x) Minv vbar and vbar (x) J^T lo,
// and rho_b through Wbar = -rho^2 rho_b P / k (top_projector).  A group of kGroup lanes per
// contact: lane (side, k), k < 6, owns column k of its side's block adjoint (3 entries) and of
// its body's Minv adjoint (6 entries) and walks the sweeps for them.
__device__ void adj_start_group(const AdjArgs &a, int c, int l, unsigned mask)
{
    const int A = a.pa[c], B = a.pb[c];
    const double *tr0 = a.trace + kTraceWords * (size_t)c;  // sweep 0
    const double lo[3] = {tr0[0], tr0[1], tr0[2]};
    const double rho = a.rho[c];
    const double rb = a.rho_b[c];
    double Wb[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    if (rb != 0.0 && rho > 0.0) {
        double W[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        if (A >= 0) add_jmjt(W, a.Ja + 18 * (size_t)c, a.Minv + 36 * (size_t)A);
        if (B >= 0) add_jmjt(W, a.Jb + 18 * (size_t)c, a.Minv + 36 * (size_t)B);
        double P[3][3];
        top_projector(W, eigmax3(W), P);
        const double lmb = -rho * rho * rb;  // rho = 1 / lambda_max
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) Wb[i][j] = lmb * P[i][j];
    }
    const int side = l / 6, k = l % 6, b = side == 0 ? A : B;
    const bool on = l < 12 && b >= 0, d = on && a.dyn[b] != 0;
    double jm[3] = {0.0, 0.0, 0.0};
    if (on) {
        const double *M = a.Minv + 36 * (size_t)b, *J = (side == 0 ? a.Ja : a.Jb) + 18 * (size_t)c;
        const int vo = side == 0 ? 3 : 9, wo = side == 0 ? 21 : 27;
        double Jc[3] = {0.0, 0.0, 0.0}, Mc[6] = {0, 0, 0, 0, 0, 0};
        for (int it = 0; it < a.iters; ++it) {
            const double *tr = a.trace + kTraceWords * ((size_t)it * a.nc + c);
            const double ub[3] = {tr[15], tr[16], tr[17]}, vk = tr[vo + k];
            for (int r = 0; r < 3; ++r) Jc[r] += ub[r] * vk;
            if (!d) continue;
            const double dl[3] = {tr[18], tr[19], tr[20]};
            double w[6], mk = 0.0;
            for (int j = 0; j < 6; ++j) {
                w[j] = tr[wo + j];
                mk += M[6 * k + j] * w[j];
            }
            for (int r = 0; r < 3; ++r) Jc[r] += dl[r] * mk;
            const double jt = (J[k] * dl[0] + J[6 + k] * dl[1]) + J[12 + k] * dl[2];
            for (int i = 0; i < 6; ++i) Mc[i] += w[i] * jt;
        }
        double *Jbar = (side == 0 ? a.Ja_b : a.Jb_b) + 18 * (size_t)c;
        if (d) {
            // the start: vbar of the sweeps' initial velocities
            double w0[6], m0 = 0.0;
            for (int j = 0; j < 6; ++j) {
                w0[j] = __ldcg(a.vb + 6 * (size_t)b + j);
                m0 += M[6 * k + j] * w0[j];
            }
            const double jt0 = (J[k] * lo[0] + J[6 + k] * lo[1]) + J[12 + k] * lo[2];
            for (int r = 0; r < 3; ++r) jm[r] = J[6 * r + k] * m0;
            // WJ = Wbar J (3x6); Jbar += 2 Wbar J Minv, Minv_bar += J^T Wbar J (column k)
            double WJ[3][6];
            for (int r = 0; r < 3; ++r)
                for (int j = 0; j < 6; ++j) WJ[r][j] = (Wb[r][0] * J[j] + Wb[r][1] * J[6 + j]) + Wb[r][2] * J[12 + j];
            for (int r = 0; r < 3; ++r) {
                double sacc = 0.0;
                for (int j = 0; j < 6; ++j) sacc += WJ[r][j] * M[j * 6 + k];
                Jbar[6 * r + k] += Jc[r] + lo[r] * m0 + 2.0 * sacc;
            }
            double *Mb = a.Minv_b + 36 * (size_t)b;
            for (int i = 0; i < 6; ++i) {
                const double jwj = (J[i] * WJ[0][k] + J[6 + i] * WJ[1][k]) + J[12 + i] * WJ[2][k];
                __stcg(Mb + 6 * i + k, __ldcg(Mb + 6 * i + k) + (Mc[i] + w0[i] * jt0 + jwj));
            }
        } else {
            for (int r = 0; r < 3; ++r) Jbar[6 * r + k] += Jc[r];
        }
    }
    for (int r = 0; r < 3; ++r) {
        double x = jm[r];
        for (int off = kGroup / 2; off > 0; off >>= 1) x += __shfl_xor_sync(mask, x, off, kGroup);
        if (l == 0) a.gl[3 * (size_t)c + r] += x;
    }
}

template <int kKind>
__device__ __forceinline__ bool adj_barrier(const AdjArgs &a, unsigned int &epoch)
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

template <int kKind>
__global__ void __launch_bounds__(kAdjThreads) k_adj_sweeps(AdjArgs a)
{
    const int ncol = a.stats[kNColors];
    const int nb = gridDim.x, nth = gridDim.x * blockDim.x;
    const int tid = ((((int)threadIdx.x >> 5) * nb + (int)blockIdx.x) << 5) | ((int)threadIdx.x & 31);
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned int epoch = 0;
    if (a.trace) {
        // the recorded sweeps in reverse (a group of kGroup lanes per contact, the forward's
        // task layout), then their start; vb carries through
        const int groups = nb * (blockDim.x / kGroup);
        const int g = ((int)threadIdx.x / kGroup) * nb + (int)blockIdx.x, l = (int)threadIdx.x % kGroup;
        const unsigned mask = 0xFFFFu << (((int)threadIdx.x & 31) & ~(kGroup - 1));
        for (int it = a.iters - 1; it >= 0; --it)
            for (int ci = ncol - 1; ci >= 0; --ci) {
                const int s0 = a.cstart[ci], cnt = a.ccount[ci];
                for (int t = g; t < cnt; t += groups) adj_contact_group(a, a.order[s0 + t], it, l, mask);
                if (!adj_barrier<kKind>(a, epoch)) return;
            }
        for (int ci = 0; ci < ncol; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = g; t < cnt; t += groups) adj_start_group(a, a.order[s0 + t], l, mask);
            if (!adj_barrier<kKind>(a, epoch)) return;
        }
        for (int i = gid; i < 6 * a.nb; i += nth) {
            a.vfree_b[i] += __ldcg(a.vb + i);
            __stcg(a.vb + i, 0.0);
        }
        return;
    }
    for (int it = 0; it < a.iters; ++it) {
        for (int ci = ncol - 1; ci >= 0; --ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = tid; t < cnt; t += nth) adj_contact(a, a.order[s0 + t]);
            if (!adj_barrier<kKind>(a, epoch)) return;
        }
        // the sweep's start: v = v_free + Minv J^T lambda
        for (int c = gid; c < a.nc; c += nth) {
            const int A = a.pa[c], B = a.pb[c];
            double jm[3] = {0.0, 0.0, 0.0}, x[6];
            if (A >= 0 && a.dyn[A]) {
                for (int k = 0; k < 6; ++k) x[k] = __ldcg(a.vb + 6 * (size_t)A + k);
                add_j_minv(a.Ja + 18 * (size_t)c, a.Minv + 36 * (size_t)A, x, jm);
            }
            if (B >= 0 && a.dyn[B]) {
                for (int k = 0; k < 6; ++k) x[k] = __ldcg(a.vb + 6 * (size_t)B + k);
                add_j_minv(a.Jb + 18 * (size_t)c, a.Minv + 36 * (size_t)B, x, jm);
            }
            for (int k = 0; k < 3; ++k) a.gl[3 * (size_t)c + k] += jm[k];
        }
        if (!adj_barrier<kKind>(a, epoch)) return;
        for (int i = gid; i < 6 * a.nb; i += nth) {
            a.vfree_b[i] += __ldcg(a.vb + i);
            __stcg(a.vb + i, 0.0);
        }
        if (!adj_barrier<kKind>(a, epoch)) return;
    }
}

int adjoint_sweeps(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p, int iters,
                   double *trace, double *gl, double *vb, double *vfree_b, double *bias_b, double *mu_b,
                   double *Ja_b, double *Jb_b, double *Minv_b, cudaStream_t s)
{
    if (iters <= 0 || sc->n_c == 0) return B2C_OK;
    AdjArgs a;
    a.nc = sc->n_c;
    a.nb = sc->n_b;
    a.iters = iters;
    a.desaxce = p->desaxce;
    a.Ja = (const double *)sc->Ja;
    a.Jb = (const double *)sc->Jb;
    a.Minv = (const double *)sc->Minv;
    a.mu = (const double *)sc->mu;
    a.rho = (const double *)st->rho;
    a.lam = (const double *)st->lam;
    a.u = (const double *)st->u;
    a.trace = trace;
    a.bias = (const double *)sc->bias;
    a.Ja_b = Ja_b;
    a.Jb_b = Jb_b;
    a.Minv_b = Minv_b;
    a.rho_b = (double *)st->res;
    a.pa = sc->pa;
    a.pb = sc->pb;
    a.order = st->order;
    a.cstart = st->cstart;
    a.ccount = st->ccount;
    a.dyn = st->dyn;
    a.gl = gl;
    a.vb = vb;
    a.vfree_b = vfree_b;
    a.bias_b = bias_b;
    a.mu_b = mu_b;
    a.stats = st->stats;
    a.bar = st->barrier;
    a.timeout_ns = p->barrier_timeout_ns > 0 ? p->barrier_timeout_ns : 1000000000LL;
    cudaMemsetAsync(vb, 0, sizeof(double) * 6 * (size_t)sc->n_b, s);
    if (trace) cudaMemsetAsync(st->res, 0, sizeof(double) * (size_t)sc->n_c, s);
    int mode = p->solve_blocks;
    if (mode == 0) mode = sc->n_c <= 16384 ? 1 : grid_blocks<double>();
    if (mode > 1) {
        int per = 0, dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_adj_sweeps<kGrid>, kAdjThreads, 0);
        const int nblocks = std::min(std::min(mode, kBarrierMaxCTAs), std::max(1, sms * per));
        if (nblocks > 1) {
            cudaMemsetAsync(st->barrier, 0, sizeof(uint32_t), s);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(nblocks);
            cfg.blockDim = dim3(kAdjThreads);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, k_adj_sweeps<kGrid>, a);
            if (e != cudaSuccess) {
                set_error("ncp_adjoint: cooperative launch of %d CTAs: %s", nblocks, cudaGetErrorString(e));
                return B2C_ECUDA;
            }
            return check_launch("ncp_adjoint_grid");
        }
    }
    k_adj_sweeps<kBlock><<<1, kAdjThreads, 0, s>>>(a);
    return check_launch("ncp_adjoint");
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

extern "C" int32_t b2c_ncp_adjoint(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                   int32_t iters, double *lam_bar, double *v_bar, double *vfree_bar, double *bias_bar,
                                   double *mu_bar, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p || sc->dtype != 8 || iters < 0 || !v_bar || !vfree_bar || p->soft ||
        (sc->n_c > 0 && (!lam_bar || !bias_bar || !mu_bar))) {
        b2c::set_error("b2c_ncp_adjoint: bad argument (float64 scenes only)");
        return B2C_EARG;
    }
    return b2c::ncp::adjoint_sweeps(sc, st, p, iters, nullptr, lam_bar, v_bar, vfree_bar, bias_bar, mu_bar, nullptr,
                                    nullptr, nullptr, b2c::stream_of(s));
}

extern "C" int32_t b2c_ncp_trace_words(void) { return b2c::ncp::kTraceWords; }

extern "C" int32_t b2c_ncp_sweeps_record(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                         int32_t iters, double *trace, int64_t trace_len, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p || sc->dtype != 8 || iters < 0 ||
        (sc->n_c > 0 && iters > 0 && (!trace || trace_len < b2c::ncp::kTraceWords * (int64_t)iters * sc->n_c))) {
        b2c::set_error("b2c_ncp_sweeps_record: bad argument (float64 scenes; trace of b2c_ncp_trace_words() * iters * n_c doubles)");
        return B2C_EARG;
    }
    return b2c::ncp::sweeps<double>(sc, st, p, iters, b2c::stream_of(s), trace);
}

extern "C" int32_t b2c_ncp_adjoint_unrolled(const b2c_ncp_scene *sc, b2c_ncp_state *st, const b2c_ncp_params *p,
                                            int32_t iters, double *trace, int64_t trace_len, double *lam_bar,
                                            double *v_bar, double *vfree_bar, double *bias_bar, double *mu_bar,
                                            double *Ja_bar, double *Jb_bar, double *Minv_bar, b2c_stream s)
{
    if (!ncp_scene_ok(sc, st) || !p || sc->dtype != 8 || iters < 0 || !v_bar || !vfree_bar || p->soft ||
        (sc->n_c > 0 && (!lam_bar || !bias_bar || !mu_bar || !Ja_bar || !Jb_bar || !Minv_bar)) ||
        (sc->n_c > 0 && iters > 0 && (!trace || trace_len < b2c::ncp::kTraceWords * (int64_t)iters * sc->n_c))) {
        b2c::set_error("b2c_ncp_adjoint_unrolled: bad argument (float64 hard-contact scenes; the trace of "
                       "b2c_ncp_sweeps_record)");
        return B2C_EARG;
    }
    return b2c::ncp::adjoint_sweeps(sc, st, p, iters, trace, lam_bar, v_bar, vfree_bar, bias_bar, mu_bar, Ja_bar,
                                    Jb_bar, Minv_bar, b2c::stream_of(s));
}
