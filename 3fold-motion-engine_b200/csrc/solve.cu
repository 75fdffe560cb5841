// The persistent pair-chunk solve of one substep: applied warm start per colour
// (contact_engine_gpu_applied_warm.py:68-75), vit velocity sweeps (k_fixed_frame,
// contact_engine_gpu_fixed_frame.py:7-77, or the slip-basis k_chunk_vel_r, COL:413-490) and pit
// position sweeps (k_chunk_pos_r, COL:510-554) over the colours, in ONE kernel launch.
//
// The reference launches one kernel per colour per sweep ((1 + vit + pit) x ncol launches in a
// graph).  Here the colours are separated by a barrier inside one kernel:
//   * one CTA (small scenes): __syncthreads;
//   * a thread-block cluster of up to 16 CTAs (up to ~32k bodies): the hardware cluster barrier
//     (barrier.cluster arrive.release / wait.acquire) -- no spinning, a few hundred ns;
//   * a cooperative grid (larger scenes): an atomic grid barrier whose wait is bounded by a
//     %globaltimer limit, after which it sets B2C_ERR_BARRIER_TIMEOUT and every CTA returns.
// Body velocities are read and written through L2 (ld.cg / st.cg), since CTAs on other SMs read
// them after a barrier and L1 is not coherent across SMs.
//
// Terms that do not change during a solve (lever arms rA, rB, the fixed tangent frame t1, t2 and
// the effective masses meff, meft1, meft2) are computed once per substep by k_contact_prep with
// exactly the reference's expressions, instead of in every sweep.  Same inputs, same operations:
// the results are bit-identical to recomputing them.
#include <cooperative_groups.h>

#include "b2c_common.cuh"

namespace cg = cooperative_groups;

namespace b2c {

__device__ __forceinline__ float4 ldcg4(const float *p, int i) { return __ldcg(reinterpret_cast<const float4 *>(p) + i); }
__device__ __forceinline__ void stcg4(float *p, int i, float4 v) { __stcg(reinterpret_cast<float4 *>(p) + i, v); }
__device__ __forceinline__ f3 ldcg3(const float *p, int i) { return xyz(ldcg4(p, i)); }

struct SolveArgs {
    const b2c_header *hdr;
    int *err;
    const int *porder, *cstart, *ccount, *pstart, *pcount, *pidx, *pbi, *pbj;
    const float *cpA, *cpB, *cn;
    const float4 *prep;
    float *imp;
    const float *invIw, *invM;
    float *v, *w, *pv, *po;
    float mu, t2d, dt;
    int vit, pit, fixed_frame, apply_warm;
    unsigned int *bar_count, *bar_gen;
    long long timeout_ns;
};

// ---------------------------------------------------------------------------------------------
// per-contact invariants of one solve
// ---------------------------------------------------------------------------------------------
// rA = cpA - xc[bi], rB = cpB - xc[bj]; meff (normal); the axis-derived frame
// t1 = normalize(a - (a.n) n), t2 = n x t1 with a = x (y when |n.x| >= 0.9) and its effective
// masses meft1, meft2 -- the expressions of k_fixed_frame / apply_warm / k_chunk_pos_r.
__global__ void k_contact_prep(const b2c_header *__restrict__ hdr, const int *__restrict__ kbi,
                               const int *__restrict__ kbj, const float *__restrict__ cpA,
                               const float *__restrict__ cpB, const float *__restrict__ cn,
                               const float *__restrict__ xc, const float *__restrict__ invIw,
                               const float *__restrict__ invM, float4 *__restrict__ prep)
{
    const int Ck = hdr->n_contacts > 0 ? hdr->n_kept : 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < Ck; c += gridDim.x * blockDim.x) {
        const int bi = kbi[c], bj = kbj[c];
        const f3 nrm = ld3(cn, c);
        const f3 rA = sub3(ld3(cpA, c), ld3(xc, bi));
        const m3 IA = ldm(invIw, bi);
        const float iMA = invM[bi];
        f3 rB{0.0f, 0.0f, 0.0f};
        m3 IB = IA;
        float iMB = 0.0f;
        if (bj >= 0) {
            rB = sub3(ld3(cpB, c), ld3(xc, bj));
            IB = ldm(invIw, bj);
            iMB = invM[bj];
        }
        f3 aa{1.0f, 0.0f, 0.0f};
        if (fabsf(nrm.x) >= 0.9f) aa = f3{0.0f, 1.0f, 0.0f};
        const float dd = dot3(aa, nrm);
        const f3 t1 = normalize3(f3{fmaf(-dd, nrm.x, aa.x), fmaf(-dd, nrm.y, aa.y), fmaf(-dd, nrm.z, aa.z)});
        const f3 t2 = cross3(nrm, t1);
        const f3 rnA = cross3(rA, nrm);
        float meff = iMA + dot3(rnA, matvec(IA, rnA));
        const f3 rtA1 = cross3(rA, t1);
        float meft1 = iMA + dot3(rtA1, matvec(IA, rtA1));
        const f3 rtA2 = cross3(rA, t2);
        float meft2 = iMA + dot3(rtA2, matvec(IA, rtA2));
        if (bj >= 0) {
            const f3 rnB = cross3(rB, nrm);
            meff = (meff + iMB) + dot3(rnB, matvec(IB, rnB));
            const f3 rtB1 = cross3(rB, t1);
            meft1 = (meft1 + iMB) + dot3(rtB1, matvec(IB, rtB1));
            const f3 rtB2 = cross3(rB, t2);
            meft2 = (meft2 + iMB) + dot3(rtB2, matvec(IB, rtB2));
        }
        prep[4 * c + 0] = f4(rA, meff);
        prep[4 * c + 1] = f4(rB, meft1);
        prep[4 * c + 2] = f4(t1, meft2);
        prep[4 * c + 3] = f4(t2, 0.0f);
    }
}

// ---------------------------------------------------------------------------------------------
// barriers
// ---------------------------------------------------------------------------------------------
enum BarrierKind { kBlock = 0, kCluster = 1, kGrid = 2 };

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <int kKind>
__device__ __forceinline__ bool solve_barrier(const SolveArgs &a)
{
    if (kKind == kBlock) {
        __syncthreads();
        return true;
    }
    if (kKind == kCluster) {
        cg::this_cluster().sync();
        return true;
    }
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned int *gen = a.bar_gen;
        const unsigned int my_gen = *gen;
        __threadfence();
        const unsigned int prev = atomicAdd(a.bar_count, 1u);
        if (prev == gridDim.x - 1) {
            atomicExch(a.bar_count, 0u);
            __threadfence();
            atomicAdd(a.bar_gen, 1u);
        } else {
            const unsigned long long t0 = global_ns();
            while (*gen == my_gen) {
                if (global_ns() - t0 > (unsigned long long)a.timeout_ns) {
                    atomicOr(a.err, B2C_ERR_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        if (*(volatile int *)a.err & B2C_ERR_BARRIER_TIMEOUT) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------------------------------------
// one pair of a colour
// ---------------------------------------------------------------------------------------------
// apply_warm, contact_engine_gpu_applied_warm.py:5-54
__device__ void pair_apply_warm(const SolveArgs &a, int p)
{
    const int A = a.pbi[p], B = a.pbj[p];
    const float iMA = a.invM[A], iMB = B >= 0 ? a.invM[B] : 0.0f;
    f3 va = ldcg3(a.v, A), wa = ldcg3(a.w, A), vb{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
    const m3 IA = ldm(a.invIw, A);
    m3 IB = IA;
    if (B >= 0) {
        vb = ldcg3(a.v, B);
        wb = ldcg3(a.w, B);
        IB = ldm(a.invIw, B);
    }
    const int st = a.pstart[p], n = a.pcount[p];
    for (int k = 0; k < n; ++k) {
        const int c = a.pidx[st + k];
        const f3 nrm = ld3(a.cn, c);
        const float4 p0 = a.prep[4 * c + 0], p1 = a.prep[4 * c + 1], p2 = a.prep[4 * c + 2], p3 = a.prep[4 * c + 3];
        const f3 t1 = xyz(p2), t2 = xyz(p3);
        const float4 im = ldcg4(a.imp, c);
        const f3 J{fmaf(im.z, t2.x, fmaf(im.x, nrm.x, im.y * t1.x)), fmaf(im.z, t2.y, fmaf(im.x, nrm.y, im.y * t1.y)),
                   fmaf(im.z, t2.z, fmaf(im.x, nrm.z, im.y * t1.z))};
        if (iMA > 0.0f) {
            va = f3{fmaf(iMA, J.x, va.x), fmaf(iMA, J.y, va.y), fmaf(iMA, J.z, va.z)};
            wa = add3(wa, matvec(IA, cross3(xyz(p0), J)));
        }
        if (B >= 0 && iMB > 0.0f) {
            vb = f3{fmaf(-iMB, J.x, vb.x), fmaf(-iMB, J.y, vb.y), fmaf(-iMB, J.z, vb.z)};
            wb = sub3(wb, matvec(IB, cross3(xyz(p1), J)));
        }
    }
    if (iMA > 0.0f) {
        stcg4(a.v, A, f4(va, 0.0f));
        stcg4(a.w, A, f4(wa, 0.0f));
    }
    if (B >= 0 && iMB > 0.0f) {
        stcg4(a.v, B, f4(vb, 0.0f));
        stcg4(a.w, B, f4(wb, 0.0f));
    }
}

// velocity chunk: k_fixed_frame (fixed_frame.py:7-77) or k_chunk_vel_r (COL:413-490)
__device__ void pair_velocity(const SolveArgs &a, int p)
{
    const int bi = a.pbi[p], bj = a.pbj[p];
    const float iMA = a.invM[bi];
    const m3 IA = ldm(a.invIw, bi);
    m3 IB = IA;
    f3 vA = ldcg3(a.v, bi), wA = ldcg3(a.w, bi);
    float iMB = 0.0f;
    f3 vB{0.0f, 0.0f, 0.0f}, wB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        iMB = a.invM[bj];
        IB = ldm(a.invIw, bj);
        vB = ldcg3(a.v, bj);
        wB = ldcg3(a.w, bj);
    }
    const int st = a.pstart[p], n = a.pcount[p];
    for (int k = 0; k < n; ++k) {
        const int c = a.pidx[st + k];
        const f3 nrm = ld3(a.cn, c);
        const float4 p0 = a.prep[4 * c + 0], p1 = a.prep[4 * c + 1];
        const f3 rA = xyz(p0), rB = xyz(p1);
        const float meff = p0.w;
        f3 va = add3(vA, cross3(wA, rA));
        f3 vb{0.0f, 0.0f, 0.0f};
        if (bj >= 0) vb = add3(vB, cross3(wB, rB));
        f3 vrel = sub3(va, vb);
        const float vn = dot3(vrel, nrm);
        f3 t1, t2;
        float meft1, meft2;
        bool axis_frame = a.fixed_frame;
        if (!a.fixed_frame) {
            const f3 vt{fmaf(-vn, nrm.x, vrel.x), fmaf(-vn, nrm.y, vrel.y), fmaf(-vn, nrm.z, vrel.z)};
            const float mt = len3(vt);
            t1 = div3(vt, mt);
            axis_frame = mt <= 5e-3f;
        }
        if (axis_frame) {
            const float4 p2 = a.prep[4 * c + 2], p3 = a.prep[4 * c + 3];
            t1 = xyz(p2);
            t2 = xyz(p3);
            meft1 = p1.w;
            meft2 = p2.w;
        } else {
            t2 = cross3(nrm, t1);
            const f3 rtA1 = cross3(rA, t1);
            meft1 = iMA + dot3(rtA1, matvec(IA, rtA1));
            const f3 rtA2 = cross3(rA, t2);
            meft2 = iMA + dot3(rtA2, matvec(IA, rtA2));
            if (bj >= 0) {
                const f3 rtB1 = cross3(rB, t1);
                meft1 = (meft1 + iMB) + dot3(rtB1, matvec(IB, rtB1));
                const f3 rtB2 = cross3(rB, t2);
                meft2 = (meft2 + iMB) + dot3(rtB2, matvec(IB, rtB2));
            }
        }
        if (!(meff >= 1e-12f)) continue;
        float4 im = ldcg4(a.imp, c);
        float dj = -vn / meff;
        const float nw = fmaxf(0.0f, im.x + dj);
        dj = nw - im.x;
        im.x = nw;
        const f3 Jn = scale3(nrm, dj);
        if (iMA > 0.0f) {
            vA = f3{fmaf(Jn.x, iMA, vA.x), fmaf(Jn.y, iMA, vA.y), fmaf(Jn.z, iMA, vA.z)};
            wA = add3(wA, matvec(IA, cross3(rA, Jn)));
        }
        if (bj >= 0 && iMB > 0.0f) {
            vB = f3{fmaf(-Jn.x, iMB, vB.x), fmaf(-Jn.y, iMB, vB.y), fmaf(-Jn.z, iMB, vB.z)};
            wB = sub3(wB, matvec(IB, cross3(rB, Jn)));
        }
        va = add3(vA, cross3(wA, rA));
        vb = f3{0.0f, 0.0f, 0.0f};
        if (bj >= 0) vb = add3(vB, cross3(wB, rB));
        vrel = sub3(va, vb);
        if (meft1 >= 1e-12f && meft2 >= 1e-12f) {
            const float o1 = im.y, o2 = im.z;
            float a1 = o1 - dot3(vrel, t1) / meft1;
            float a2 = o2 - dot3(vrel, t2) / meft2;
            const float mag = sqrtf(fmaf(a1, a1, a2 * a2));
            const float lim = a.mu * im.x;
            if (mag > lim && mag > 1e-12f) {
                a1 = a1 * lim / mag;
                a2 = a2 * lim / mag;
            }
            im.y = a1;
            im.z = a2;
            const float e1 = a1 - o1, e2 = a.t2d * (a2 - o2);
            const f3 Jt{fmaf(e1, t1.x, e2 * t2.x), fmaf(e1, t1.y, e2 * t2.y), fmaf(e1, t1.z, e2 * t2.z)};
            if (iMA > 0.0f) {
                vA = f3{fmaf(Jt.x, iMA, vA.x), fmaf(Jt.y, iMA, vA.y), fmaf(Jt.z, iMA, vA.z)};
                wA = add3(wA, matvec(IA, cross3(rA, Jt)));
            }
            if (bj >= 0 && iMB > 0.0f) {
                vB = f3{fmaf(-Jt.x, iMB, vB.x), fmaf(-Jt.y, iMB, vB.y), fmaf(-Jt.z, iMB, vB.z)};
                wB = sub3(wB, matvec(IB, cross3(rB, Jt)));
            }
        }
        stcg4(a.imp, c, im);
    }
    if (iMA > 0.0f) {
        stcg4(a.v, bi, f4(vA, 0.0f));
        stcg4(a.w, bi, f4(wA, 0.0f));
    }
    if (bj >= 0 && iMB > 0.0f) {
        stcg4(a.v, bj, f4(vB, 0.0f));
        stcg4(a.w, bj, f4(wB, 0.0f));
    }
}

// position chunk, k_chunk_pos_r (COL:510-554)
__device__ void pair_position(const SolveArgs &a, int p)
{
    const int bi = a.pbi[p], bj = a.pbj[p];
    const float iMA = a.invM[bi];
    const m3 IA = ldm(a.invIw, bi);
    m3 IB = IA;
    f3 pvA = ldcg3(a.pv, bi), poA = ldcg3(a.po, bi);
    float iMB = 0.0f;
    f3 pvB{0.0f, 0.0f, 0.0f}, poB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        iMB = a.invM[bj];
        IB = ldm(a.invIw, bj);
        pvB = ldcg3(a.pv, bj);
        poB = ldcg3(a.po, bj);
    }
    const int st = a.pstart[p], n = a.pcount[p];
    for (int k = 0; k < n; ++k) {
        const int c = a.pidx[st + k];
        const f3 nrm = ld3(a.cn, c);
        const float pen = a.cpA[4 * c + 3];
        const float4 p0 = a.prep[4 * c + 0], p1 = a.prep[4 * c + 1];
        const f3 rA = xyz(p0), rB = xyz(p1);
        f3 rel = add3(pvA, cross3(poA, rA));
        if (bj >= 0) rel = sub3(rel, add3(pvB, cross3(poB, rB)));
        const float meff = p0.w;
        if (!(meff >= 1e-12f)) continue;
        const float bias = B2C_BETA * fmaxf(pen - B2C_SLOP, 0.0f) / a.dt;
        float dj = (bias - dot3(rel, nrm)) / meff;
        const float jp = __ldcg(a.imp + 4 * c + 3);
        const float nw = fmaxf(0.0f, jp + dj);
        dj = nw - jp;
        __stcg(a.imp + 4 * c + 3, nw);
        const f3 Jn = scale3(nrm, dj);
        if (iMA > 0.0f) {
            pvA = f3{fmaf(Jn.x, iMA, pvA.x), fmaf(Jn.y, iMA, pvA.y), fmaf(Jn.z, iMA, pvA.z)};
            poA = add3(poA, matvec(IA, cross3(rA, Jn)));
        }
        if (bj >= 0 && iMB > 0.0f) {
            pvB = f3{fmaf(-Jn.x, iMB, pvB.x), fmaf(-Jn.y, iMB, pvB.y), fmaf(-Jn.z, iMB, pvB.z)};
            poB = sub3(poB, matvec(IB, cross3(rB, Jn)));
        }
    }
    if (iMA > 0.0f) {
        stcg4(a.pv, bi, f4(pvA, 0.0f));
        stcg4(a.po, bi, f4(poA, 0.0f));
    }
    if (bj >= 0 && iMB > 0.0f) {
        stcg4(a.pv, bj, f4(pvB, 0.0f));
        stcg4(a.po, bj, f4(poB, 0.0f));
    }
}

// ---------------------------------------------------------------------------------------------
// the persistent kernel
// ---------------------------------------------------------------------------------------------
template <int kKind>
__device__ __forceinline__ void solve_body(const SolveArgs &a)
{
    const int nc = a.hdr->n_colors;
    if (a.hdr->n_pairs == 0 || nc == 0) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (a.apply_warm) {
        for (int ci = 0; ci < nc; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = tid; t < cnt; t += nth) pair_apply_warm(a, a.porder[s0 + t]);
            if (!solve_barrier<kKind>(a)) return;
        }
    }
    for (int it = 0; it < a.vit; ++it)
        for (int ci = 0; ci < nc; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = tid; t < cnt; t += nth) pair_velocity(a, a.porder[s0 + t]);
            if (!solve_barrier<kKind>(a)) return;
        }
    for (int it = 0; it < a.pit; ++it)
        for (int ci = 0; ci < nc; ++ci) {
            const int s0 = a.cstart[ci], cnt = a.ccount[ci];
            for (int t = tid; t < cnt; t += nth) pair_position(a, a.porder[s0 + t]);
            if (!solve_barrier<kKind>(a)) return;
        }
}

__global__ void __launch_bounds__(256) k_color_solve_block(SolveArgs a) { solve_body<kBlock>(a); }
__global__ void __launch_bounds__(512) k_color_solve_cluster(SolveArgs a) { solve_body<kCluster>(a); }
__global__ void __launch_bounds__(256) k_color_solve_grid(SolveArgs a) { solve_body<kGrid>(a); }

constexpr int kClusterThreads = 512;
constexpr int kClusterMax = 16;

static int max_coresident_grid_blocks()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_color_solve_grid, 256, 0);
        cached = std::max(1, sms * std::max(per, 1));
    }
    return cached;
}

// largest cluster (<= 16) of k_color_solve_cluster CTAs the device can co-schedule; 0 if none.
// A host-side occupancy query, done once (the first step of an engine runs eagerly, before any
// graph capture).
static int max_cluster_size()
{
    static int cached = -1;
    if (cached < 0) {
        cudaFuncSetAttribute(k_color_solve_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterMax);
        cfg.blockDim = dim3(kClusterThreads);
        int cs = 0;
        if (cudaOccupancyMaxPotentialClusterSize(&cs, k_color_solve_cluster, &cfg) != cudaSuccess) {
            cudaGetLastError();
            cs = 0;
        }
        int p2 = 0;
        for (int c = 1; c <= std::min(cs, kClusterMax); c *= 2) p2 = c;
        cached = p2 >= 2 ? p2 : 0;
    }
    return cached;
}

static int launch_cluster(const SolveArgs &a, int csize, cudaStream_t s)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_color_solve_cluster, a);
    if (e != cudaSuccess) {
        set_error("color_solve: cluster launch of %d CTAs: %s", csize, cudaGetErrorString(e));
        return B2C_ECUDA;
    }
    return check_launch("color_solve_cluster");
}

int color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                float dt, cudaStream_t s)
{
    SolveArgs a;
    a.hdr = hdr;
    a.err = &hdr->error;
    a.porder = pr->porder;
    a.cstart = pr->cstart;
    a.ccount = pr->ccount;
    a.pstart = pr->pstart;
    a.pcount = pr->kcount;
    a.pidx = pr->pidx;
    a.pbi = pr->pbi;
    a.pbj = pr->pbj;
    a.cpA = kept->pA;
    a.cpB = kept->pB;
    a.cn = kept->n;
    a.prep = reinterpret_cast<const float4 *>(pr->prep);
    a.imp = kept->imp;
    a.invIw = b->invIw;
    a.invM = b->invM;
    a.v = b->v;
    a.w = b->w;
    a.pv = b->pv;
    a.po = b->po;
    a.mu = p->mu;
    a.t2d = p->t2d;
    a.dt = dt;
    a.vit = p->vit;
    a.pit = p->pit;
    a.fixed_frame = (p->flags & B2C_COLOR_FIXED_FRAME) ? 1 : 0;
    a.apply_warm = (p->flags & B2C_COLOR_APPLY_WARM) ? 1 : 0;
    a.bar_count = pr->barrier;
    a.bar_gen = pr->barrier + 1;
    a.timeout_ns = p->barrier_timeout_ns > 0 ? p->barrier_timeout_ns : 1000000000LL;

    k_contact_prep<<<std::min(blocks_for(kept->capacity), kSMs * 8), kThreads, 0, s>>>(
        hdr, kept->bi, kept->bj, kept->pA, kept->pB, kept->n, b->xc, b->invIw, b->invM, reinterpret_cast<float4 *>(pr->prep));
    int rc = check_launch("contact_prep");
    if (rc) return rc;

    int mode = p->solve_blocks;
    if (mode == 0) {  // auto: one CTA for small scenes, a cluster up to ~32k bodies, else a grid
        if (b->n <= 256) mode = 1;
        else if (b->n <= 2 * kClusterMax * kClusterThreads * 2) mode = -kClusterMax;
        else mode = std::min((b->n + 255) / 256, max_coresident_grid_blocks());
    }
    if (mode < 0) {
        const int cs = std::min(-mode, max_cluster_size());
        if (cs >= 2) return launch_cluster(a, cs, s);
        mode = std::min((b->n + 255) / 256, max_coresident_grid_blocks());  // no cluster possible
    }
    const int nblocks = std::max(1, std::min(mode, max_coresident_grid_blocks()));
    if (nblocks == 1) {
        k_color_solve_block<<<1, 256, 0, s>>>(a);
        return check_launch("color_solve_block");
    }
    cudaMemsetAsync(pr->barrier, 0, sizeof(uint32_t), s);  // arrival count (the generation keeps counting)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(256);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_color_solve_grid, a);
    if (e != cudaSuccess) {
        set_error("color_solve: cooperative launch of %d blocks: %s", nblocks, cudaGetErrorString(e));
        return B2C_ECUDA;
    }
    return check_launch("color_solve_grid");
}

}  // namespace b2c
