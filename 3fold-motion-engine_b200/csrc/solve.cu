// The persistent pair-chunk solve of one substep: applied warm start per colour
// (contact_engine_gpu_applied_warm.py:68-75), vit velocity sweeps (k_fixed_frame,
// contact_engine_gpu_fixed_frame.py:7-77, or the slip-basis k_chunk_vel_r, COL:413-490) and pit
// position sweeps (k_chunk_pos_r, COL:510-554) over the colours, in ONE kernel launch.
//
// The reference launches one kernel per colour per sweep ((1 + vit + pit) x ncol launches in a
// graph).  Here the colours are separated by a barrier inside one kernel:
//   * one CTA (tiny scenes): __syncthreads (~0.04 us measured on B200);
//   * a thread-block cluster of up to 16 CTAs: the hardware cluster barrier
//     (barrier.cluster arrive.release / wait.acquire; ~0.25 us measured);
//   * a cooperative grid: the arrival-counter barrier of b2c_barrier.cuh (~1.3 us measured),
//     whose wait is bounded by a %globaltimer limit, after which it sets B2C_ERR_BARRIER_TIMEOUT
//     and every CTA returns.
//
// Data layout.  The sweeps are bound by the latency of dependent loads, not by arithmetic or
// bandwidth: following porder -> pair -> pidx -> contact -> body costs several L2 round trips
// per pair and per phase.  So once per substep k_pair_gather writes every pair into a
// colour-major record (slot s = position in porder): a header (bodies, contact count), both
// bodies' inverse inertia rows and inverse masses, and per contact its normal|depth, the terms
// that stay fixed during the solve (rA|meff, rB|meft1, t1|meft2 -- computed with exactly the
// reference's expressions, so bit-identical to recomputing them every sweep) and its impulses.
// A phase then needs one batch of independent 128-bit loads for the record and one for the two
// bodies' velocities.  Records are structure-of-arrays by field, so consecutive threads read
// consecutive 16-byte words.  After the solve k_imp_scatter returns the impulses to the kept
// contacts (the warm store reads them there).
//
// Body velocities are read and written through L2 (ld.cg / st.cg): CTAs on other SMs read them
// after a barrier, and L1 is not coherent across SMs.
#include <cooperative_groups.h>

#include "b2c_barrier.cuh"
#include "b2c_common.cuh"

namespace cg = cooperative_groups;

namespace b2c {

__device__ __forceinline__ float4 ldcg4(const float *p, int i) { return __ldcg(reinterpret_cast<const float4 *>(p) + i); }
__device__ __forceinline__ void stcg4(float *p, int i, float4 v) { __stcg(reinterpret_cast<float4 *>(p) + i, v); }
__device__ __forceinline__ f3 ldcg3(const float *p, int i) { return xyz(ldcg4(p, i)); }

// record fields (float4 units)
enum { kRecBody = 7, kRecContact = 5 };
enum { kCN = 0, kCRA = 1, kCRB = 2, kCT1 = 3, kCImp = 4 };
// row form (B2C_COLOR_ROW_FORM): the reference form's header and inverse-inertia rows, and per
// contact n|inv_n, rA|bias, rB|inv_2, t1|inv_1 and the impulses.  The second tangent t2 = n x t1
// and the angular responses k = I^-1 (r x d) are not stored: the sweeps recompute them with the
// gather's own expressions (row_responses), which gives the same bits, and do so off the
// velocity chain.  Five words per contact let a pair's first kRowBatch contacts load in one
// batch of independent 128-bit loads.
enum { kRecContactRow = 5 };
enum { kRN = 0, kRRA = 1, kRRB = 2, kRT1 = 3, kRImp = 4 };
constexpr int kRowBatch = 4;

// the angular responses of one contact's three rows on one body: I^-1 (r x n), I^-1 (r x t1),
// I^-1 (r x t2)
struct RowResp {
    f3 n, t1, t2;
};
__device__ __forceinline__ RowResp row_responses(const m3 &I, f3 r, f3 nrm, f3 t1, f3 t2)
{
    return RowResp{matvec(I, cross3(r, nrm)), matvec(I, cross3(r, t1)), matvec(I, cross3(r, t2))};
}

struct Records {
    float4 *base;
    int cap, K;
    __device__ __forceinline__ int4 *hdr() const { return reinterpret_cast<int4 *>(base); }
    __device__ __forceinline__ float4 *body(int f) const { return base + (size_t)(1 + f) * cap; }
    __device__ __forceinline__ float4 *contact(int f, int j) const
    {
        return base + (size_t)(1 + kRecBody) * cap + ((size_t)f * K + j) * cap;
    }
};

struct SolveArgs {
    const b2c_header *hdr;
    int *err;
    const int *cstart, *ccount;
    Records rec;
    float *v, *w, *pv, *po;
    float mu, t2d, dt;
    int vit, pit, fixed_frame, apply_warm, row;
    unsigned int *bar_count;  // the grid barrier's arrival counter
    long long timeout_ns;
    const int *island_info;   // the island partition's statistics (B2C_COLOR_ISLANDS) or NULL
};

// The island solve ran this substep (its partition has no island above B2C_ISLAND_MAX_PAIRS
// pairs): the persistent forms have nothing to do.  Every thread of every CTA reads the same
// word, written by an earlier launch, so the early return is uniform.
__device__ __forceinline__ bool islands_took_solve(const SolveArgs &a)
{
    return a.island_info && a.island_info[1] <= B2C_ISLAND_MAX_PAIRS;
}

// ---------------------------------------------------------------------------------------------
// gather (once per substep) and scatter
// ---------------------------------------------------------------------------------------------
__global__ void k_pair_gather(const b2c_header *__restrict__ hdr, const int *__restrict__ porder,
                              const int *__restrict__ pstart, const int *__restrict__ pcount,
                              const int *__restrict__ pidx, const int *__restrict__ pbi, const int *__restrict__ pbj,
                              b2c_contacts kept, const float *__restrict__ xc, const float *__restrict__ invIw,
                              const float *__restrict__ invM, const float *__restrict__ body_mu, float mu, Records R,
                              b2c_header *hdr_w)
{
    const int P = (hdr->n_pairs > 0 && hdr->n_colors > 0) ? hdr->n_pairs : 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P; s += gridDim.x * blockDim.x) {
        const int p = porder[s];
        const int bi = pbi[p], bj = pbj[p];
        int n = pcount[p];
        if (n > R.K) {
            atomicOr(&hdr_w->error, B2C_ERR_CHUNK_OVERFLOW);
            n = R.K;
        }
        R.hdr()[s] = make_int4(bi, bj, n, p);
        const m3 IA = ldm(invIw, bi);
        const float iMA = invM[bi];
        m3 IB = IA;
        float iMB = 0.0f;
        if (bj >= 0) {
            IB = ldm(invIw, bj);
            iMB = invM[bj];
        }
        R.body(0)[s] = f4(IA.r0, 0.0f);
        R.body(1)[s] = f4(IA.r1, 0.0f);
        R.body(2)[s] = f4(IA.r2, 0.0f);
        R.body(3)[s] = f4(IB.r0, 0.0f);
        R.body(4)[s] = f4(IB.r1, 0.0f);
        R.body(5)[s] = f4(IB.r2, 0.0f);
        // friction of the pair: the scalar mu, or sqrt(mu_a mu_b) (ground pair: mu_a) per body
        float mu_p = mu;
        if (body_mu) mu_p = bj >= 0 ? sqrtf(body_mu[bi] * body_mu[bj]) : body_mu[bi];
        R.body(6)[s] = make_float4(iMA, iMB, mu_p, 0.0f);
        const f3 xA = ld3(xc, bi);
        f3 xB{0.0f, 0.0f, 0.0f};
        if (bj >= 0) xB = ld3(xc, bj);
        const int st = pstart[p];
        for (int j = 0; j < n; ++j) {
            const int c = pidx[st + j];
            const float4 pA4 = ld4(kept.pA, c);
            const f3 nrm = ld3(kept.n, c);
            // the invariants of k_fixed_frame / apply_warm / k_chunk_pos_r, reference expressions
            const f3 rA = sub3(xyz(pA4), xA);
            f3 rB{0.0f, 0.0f, 0.0f};
            if (bj >= 0) rB = sub3(ld3(kept.pB, c), xB);
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
            R.contact(kCN, j)[s] = f4(nrm, pA4.w);
            R.contact(kCRA, j)[s] = f4(rA, meff);
            R.contact(kCRB, j)[s] = f4(rB, meft1);
            R.contact(kCT1, j)[s] = f4(t1, meft2);
            R.contact(kCImp, j)[s] = ld4(kept.imp, c);
        }
    }
}

// row form: the reference form's header, inertia rows and masses, and per contact the constants
// of the substep
__global__ void k_pair_gather_row(const b2c_header *__restrict__ hdr, const int *__restrict__ porder,
                                  const int *__restrict__ pstart, const int *__restrict__ pcount,
                                  const int *__restrict__ pidx, const int *__restrict__ pbi,
                                  const int *__restrict__ pbj, b2c_contacts kept, const float *__restrict__ xc,
                                  const float *__restrict__ invIw, const float *__restrict__ invM,
                                  const float *__restrict__ body_mu, float mu, float dt, Records R, b2c_header *hdr_w,
                                  const int *__restrict__ col, int *__restrict__ body_slots,
                                  int *__restrict__ pair_slot)
{
    const int P = (hdr->n_pairs > 0 && hdr->n_colors > 0) ? hdr->n_pairs : 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P; s += gridDim.x * blockDim.x) {
        const int p = porder[s];
        if (pair_slot) pair_slot[p] = s;  // the scene schedule's map from pair to record slot
        const int bi = pbi[p], bj = pbj[p];
        int n = pcount[p];
        if (n > R.K) {
            atomicOr(&hdr_w->error, B2C_ERR_CHUNK_OVERFLOW);
            n = R.K;
        }
        R.hdr()[s] = make_int4(bi, bj, n, p);
        const m3 IA = ldm(invIw, bi);
        const float iMA = invM[bi];
        m3 IB = IA;
        float iMB = 0.0f;
        if (bj >= 0) {
            IB = ldm(invIw, bj);
            iMB = invM[bj];
        }
        float mu_p = mu;
        if (body_mu) mu_p = bj >= 0 ? sqrtf(body_mu[bi] * body_mu[bj]) : body_mu[bi];
        if (body_slots) {  // this pair's slot under its colour, for each dynamic side
            const int c = col[p];
            if (c >= 0 && c < 64) {
                if (iMA > 0.0f) body_slots[64 * bi + c] = 2 * s;
                if (bj >= 0 && iMB > 0.0f) body_slots[64 * bj + c] = 2 * s + 1;
            }
        }
        R.body(0)[s] = f4(IA.r0, 0.0f);
        R.body(1)[s] = f4(IA.r1, 0.0f);
        R.body(2)[s] = f4(IA.r2, 0.0f);
        R.body(3)[s] = f4(IB.r0, 0.0f);
        R.body(4)[s] = f4(IB.r1, 0.0f);
        R.body(5)[s] = f4(IB.r2, 0.0f);
        R.body(6)[s] = make_float4(iMA, iMB, mu_p, 0.0f);
        const f3 xA = ld3(xc, bi);
        f3 xB{0.0f, 0.0f, 0.0f};
        if (bj >= 0) xB = ld3(xc, bj);
        const int st = pstart[p];
        for (int j = 0; j < n; ++j) {
            const int c = pidx[st + j];
            const float4 pA4 = ld4(kept.pA, c);
            const f3 nrm = ld3(kept.n, c);
            const f3 rA = sub3(xyz(pA4), xA);
            f3 rB{0.0f, 0.0f, 0.0f};
            if (bj >= 0) rB = sub3(ld3(kept.pB, c), xB);
            f3 aa{1.0f, 0.0f, 0.0f};
            if (fabsf(nrm.x) >= 0.9f) aa = f3{0.0f, 1.0f, 0.0f};
            const float dd = dot3(aa, nrm);
            const f3 t1 = normalize3(f3{fmaf(-dd, nrm.x, aa.x), fmaf(-dd, nrm.y, aa.y), fmaf(-dd, nrm.z, aa.z)});
            const f3 t2 = cross3(nrm, t1);
            const f3 rnA = cross3(rA, nrm), rtA1 = cross3(rA, t1), rtA2 = cross3(rA, t2);
            const RowResp kA = row_responses(IA, rA, nrm, t1, t2);
            float meff = iMA + dot3(rnA, kA.n), meft1 = iMA + dot3(rtA1, kA.t1), meft2 = iMA + dot3(rtA2, kA.t2);
            if (bj >= 0) {
                const f3 rnB = cross3(rB, nrm), rtB1 = cross3(rB, t1), rtB2 = cross3(rB, t2);
                const RowResp kB = row_responses(IB, rB, nrm, t1, t2);
                meff = (meff + iMB) + dot3(rnB, kB.n);
                meft1 = (meft1 + iMB) + dot3(rtB1, kB.t1);
                meft2 = (meft2 + iMB) + dot3(rtB2, kB.t2);
            }
            const float inv_n = meff >= 1e-12f ? 1.0f / meff : 0.0f;
            const float inv_1 = meft1 >= 1e-12f ? 1.0f / meft1 : 0.0f;
            const float inv_2 = meft2 >= 1e-12f ? 1.0f / meft2 : 0.0f;
            const float bias = B2C_BETA * fmaxf(pA4.w - B2C_SLOP, 0.0f) / dt;
            R.contact(kRN, j)[s] = f4(nrm, inv_n);
            R.contact(kRRA, j)[s] = f4(rA, bias);
            R.contact(kRRB, j)[s] = f4(rB, inv_2);
            R.contact(kRT1, j)[s] = f4(t1, inv_1);
            R.contact(kRImp, j)[s] = ld4(kept.imp, c);
        }
    }
}

__global__ void k_imp_scatter(const b2c_header *__restrict__ hdr, const int *__restrict__ pstart,
                              const int *__restrict__ pidx, Records R, int imp_field, float *__restrict__ imp)
{
    const int P = (hdr->n_pairs > 0 && hdr->n_colors > 0) ? hdr->n_pairs : 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P; s += gridDim.x * blockDim.x) {
        const int4 h = R.hdr()[s];
        const int st = pstart[h.w];
        for (int j = 0; j < h.z; ++j) st4(imp, pidx[st + j], R.contact(imp_field, j)[s]);
    }
}

// ---------------------------------------------------------------------------------------------
// barriers
// ---------------------------------------------------------------------------------------------
enum BarrierKind { kBlock = 0, kCluster = 1, kGrid = 2 };

// The barrier between colour phases, split into an arrive and a wait, so that a thread can
// issue loads that do not depend on the other CTAs' work of the phase (its next task's fixed
// record words) in between.  The grid form counts its barriers in `epoch` (uniform over the
// CTA): barrier k waits for k arrivals of every CTA (b2c_barrier.cuh).
struct BarTok {
    unsigned int epoch;
};
template <int kKind>
__device__ __forceinline__ BarTok bar_arrive(const SolveArgs &a, unsigned int &epoch)
{
    BarTok tok{0u};
    if (kKind == kCluster) {
        asm volatile("barrier.cluster.arrive.release;\n" ::: "memory");
    } else if (kKind == kGrid) {
        tok.epoch = ++epoch;
        grid_arrive(a.bar_count);
    }
    return tok;
}
template <int kKind>
__device__ __forceinline__ bool bar_wait(const SolveArgs &a, BarTok tok)
{
    if (kKind == kBlock) {
        __syncthreads();
        return true;
    }
    if (kKind == kCluster) {
        asm volatile("barrier.cluster.wait.acquire;\n" ::: "memory");
        return true;
    }
    return grid_wait(a.bar_count, tok.epoch, a.timeout_ns, a.err, B2C_ERR_BARRIER_TIMEOUT);
}

// ---------------------------------------------------------------------------------------------
// pair tasks
// ---------------------------------------------------------------------------------------------
// Body state access through L2 (a policy class, so the pair physics is written once).
struct GlobalBodies {
    float *v, *w, *pv, *po;
    __device__ __forceinline__ f3 get(int b, int k) const
    {
        const float *p = k == 0 ? v : k == 1 ? w : k == 2 ? pv : po;
        return ldcg3(p, b);
    }
    __device__ __forceinline__ void set(int b, int k, f3 x) const
    {
        float *p = k == 0 ? v : k == 1 ? w : k == 2 ? pv : po;
        stcg4(p, b, f4(x, 0.0f));
    }
};

// The impulse word of a contact is (jn, jt1, jt2, jp).  A phase can run the velocity chunk and
// the position chunk of the same pair on two threads (they read and write disjoint state), so the
// velocity chunk stores only x, y, z and the position chunk only w.
__device__ __forceinline__ void store_imp_xyz(float4 *p, float4 im)
{
    float *f = reinterpret_cast<float *>(p);
    *reinterpret_cast<float2 *>(f) = make_float2(im.x, im.y);
    f[2] = im.z;
}
__device__ __forceinline__ void store_imp_w(float4 *p, float jp) { reinterpret_cast<float *>(p)[3] = jp; }

// ---------------------------------------------------------------------------------------------
// row form of the three chunks (B2C_COLOR_ROW_FORM; not in the reference): the same sweep with
// the substep constants of k_pair_gather_row.  A pair's contacts are loaded kRowBatch at a time,
// the first batch together with the pair's header (without waiting for it: the slots exist
// whatever the pair's count), so a pair of up to kRowBatch contacts pays two dependent round
// trips (record, then the bodies' velocities) however many contacts it has.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ f3 fma3s(float s, f3 a, f3 b) { return f3{fmaf(s, a.x, b.x), fmaf(s, a.y, b.y), fmaf(s, a.z, b.z)}; }
__device__ __forceinline__ f3 sel3(bool c, f3 a, f3 b) { return f3{c ? a.x : b.x, c ? a.y : b.y, c ? a.z : b.z}; }

struct RowC {
    float4 n, ra, rb, t1, im;
};

// Staging.  A batch of a pair's contact records is copied into this thread's part of the
// dynamic shared memory with cp.async (no registers held while the copies are in flight), and
// each contact is read from there when its turn comes: field f of batch contact j sits at
// s_stage[(f * kRowBatch + j) * blockDim.x + threadIdx.x], so a warp's reads are consecutive.
// A thread only ever reads its own words after its own cp.async.wait_group, so no block-level
// synchronisation is involved.
extern __shared__ float4 s_stage[];
constexpr int kStageBytesPerThread = kRecContactRow * kRowBatch * 16;

__device__ __forceinline__ float4 *stage_word(int f, int j)
{
    return s_stage + ((f * kRowBatch + j) * (int)blockDim.x + (int)threadIdx.x);
}
// kL1: the copy allocates in L1 (cp.async.ca), for a kernel whose thread re-reads the same
// records many times and is the only one that writes them (the island solve); otherwise L2 only.
template <bool kL1 = false>
__device__ __forceinline__ void cp_async16(float4 *dst, const float4 *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (kL1) asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
// issue the copies of contacts k0 .. k0 + kRowBatch - 1 of slot s (those below the slot count
// K; a slot beyond the pair's count holds stale words that are never read); the position chunk
// skips t1
template <bool kL1 = false>
__device__ __forceinline__ void stage_rows(const Records &R, int s, int k0, bool pos)
{
#pragma unroll
    for (int j = 0; j < kRowBatch; ++j) {
        if (k0 + j < R.K) {
            cp_async16<kL1>(stage_word(kRN, j), &R.contact(kRN, k0 + j)[s]);
            cp_async16<kL1>(stage_word(kRRA, j), &R.contact(kRRA, k0 + j)[s]);
            cp_async16<kL1>(stage_word(kRRB, j), &R.contact(kRRB, k0 + j)[s]);
            if (!pos) cp_async16<kL1>(stage_word(kRT1, j), &R.contact(kRT1, k0 + j)[s]);
            cp_async16<kL1>(stage_word(kRImp, j), &R.contact(kRImp, k0 + j)[s]);
        }
    }
}
__device__ __forceinline__ RowC staged_row(int j)
{
    return RowC{*stage_word(kRN, j), *stage_word(kRRA, j), *stage_word(kRRB, j), *stage_word(kRT1, j),
                *stage_word(kRImp, j)};
}
__device__ __forceinline__ m3 load_inertia(const Records &R, int s, int f0)
{
    return m3{xyz(R.body(f0)[s]), xyz(R.body(f0 + 1)[s]), xyz(R.body(f0 + 2)[s])};
}
// The words of a task that stay fixed during the solve (header, masses, inertia rows) in
// registers, and its first kRowBatch contacts on their way into the staging area.  Issued either
// at the start of the task or, for a thread's first task of the next phase, between the arrive
// and the wait of the barrier before it.
struct RowPre {
    int4 h;
    float4 mm;
    m3 IA, IB;
};
template <bool kL1 = false>
__device__ __forceinline__ RowPre row_pre(const Records &R, int s, bool pos)
{
    stage_rows<kL1>(R, s, 0, pos);
    RowPre q;
    q.h = R.hdr()[s];
    q.mm = R.body(6)[s];
    q.IA = load_inertia(R, s, 0);
    q.IB = load_inertia(R, s, 3);
    return q;
}

// apply_warm, contact_engine_gpu_applied_warm.py:5-54.  The reference form's chunks take the
// pair's fixed words from a RowPre and its contacts from the staging area, as the row form's do
// (the record layouts share the header, the inertia rows, the masses and the five-word contact).
template <class BA>
__device__ void pair_apply_warm(const SolveArgs &a, int s, const BA &BS, const RowPre &pre)
{
    const int A = pre.h.x, B = pre.h.y, n = pre.h.z;
    const float iMA = pre.mm.x, iMB = pre.mm.y;
    f3 va = BS.get(A, 0), wa = BS.get(A, 1), vb{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
    if (B >= 0) {
        vb = BS.get(B, 0);
        wb = BS.get(B, 1);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, false);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const RowC cur = staged_row(j);
            const f3 nrm = xyz(cur.n), rA = xyz(cur.ra), rB = xyz(cur.rb), t1 = xyz(cur.t1);
            const f3 t2 = cross3(nrm, t1);
            const float4 im = cur.im;
            const f3 J{fmaf(im.z, t2.x, fmaf(im.x, nrm.x, im.y * t1.x)),
                       fmaf(im.z, t2.y, fmaf(im.x, nrm.y, im.y * t1.y)),
                       fmaf(im.z, t2.z, fmaf(im.x, nrm.z, im.y * t1.z))};
            if (iMA > 0.0f) {
                va = f3{fmaf(iMA, J.x, va.x), fmaf(iMA, J.y, va.y), fmaf(iMA, J.z, va.z)};
                wa = add3(wa, matvec(pre.IA, cross3(rA, J)));
            }
            if (B >= 0 && iMB > 0.0f) {
                vb = f3{fmaf(-iMB, J.x, vb.x), fmaf(-iMB, J.y, vb.y), fmaf(-iMB, J.z, vb.z)};
                wb = sub3(wb, matvec(pre.IB, cross3(rB, J)));
            }
        }
    }
    if (iMA > 0.0f) {
        BS.set(A, 0, va);
        BS.set(A, 1, wa);
    }
    if (B >= 0 && iMB > 0.0f) {
        BS.set(B, 0, vb);
        BS.set(B, 1, wb);
    }
}

// velocity chunk: k_fixed_frame (fixed_frame.py:7-77) or k_chunk_vel_r (COL:413-490)
template <class BA, bool kFixed>
__device__ void pair_velocity(const SolveArgs &a, int s, const BA &B, const RowPre &pre)
{
    const int bi = pre.h.x, bj = pre.h.y, n = pre.h.z;
    const float iMA = pre.mm.x, iMB = pre.mm.y, mu = pre.mm.z;
    const m3 &IA = pre.IA, &IB = pre.IB;
    f3 vA = B.get(bi, 0), wA = B.get(bi, 1);
    f3 vB{0.0f, 0.0f, 0.0f}, wB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        vB = B.get(bj, 0);
        wB = B.get(bj, 1);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, false);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const RowC cur = staged_row(j);
            const f3 nrm = xyz(cur.n), rA = xyz(cur.ra), rB = xyz(cur.rb);
            const float meff = cur.ra.w;
            f3 va = add3(vA, cross3(wA, rA));
            f3 vb{0.0f, 0.0f, 0.0f};
            if (bj >= 0) vb = add3(vB, cross3(wB, rB));
            f3 vrel = sub3(va, vb);
            const float vn = dot3(vrel, nrm);
            f3 t1 = xyz(cur.t1);
            f3 t2 = cross3(nrm, t1);
            float meft1 = cur.rb.w, meft2 = cur.t1.w;
            if (!kFixed) {
                const f3 vt{fmaf(-vn, nrm.x, vrel.x), fmaf(-vn, nrm.y, vrel.y), fmaf(-vn, nrm.z, vrel.z)};
                const float mt = len3(vt);
                if (!(mt <= 5e-3f)) {  // slip basis t1 = vt / |vt|; otherwise the axis frame of the record
                    t1 = div3(vt, mt);
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
            }
            if (meff >= 1e-12f) {
                float4 im = cur.im;
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
                    const float lim = mu * im.x;
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
                store_imp_xyz(&a.rec.contact(kCImp, k0 + j)[s], im);
            }
        }
    }
    if (iMA > 0.0f) {
        B.set(bi, 0, vA);
        B.set(bi, 1, wA);
    }
    if (bj >= 0 && iMB > 0.0f) {
        B.set(bj, 0, vB);
        B.set(bj, 1, wB);
    }
}

// position chunk, k_chunk_pos_r (COL:510-554)
template <class BA>
__device__ void pair_position(const SolveArgs &a, int s, const BA &B, const RowPre &pre)
{
    const int bi = pre.h.x, bj = pre.h.y, n = pre.h.z;
    const float iMA = pre.mm.x, iMB = pre.mm.y;
    f3 pvA = B.get(bi, 2), poA = B.get(bi, 3);
    f3 pvB{0.0f, 0.0f, 0.0f}, poB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        pvB = B.get(bj, 2);
        poB = B.get(bj, 3);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, true);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const float4 wn = *stage_word(kCN, j), wa = *stage_word(kCRA, j), wb = *stage_word(kCRB, j);
            const float jp = stage_word(kCImp, j)->w;
            const f3 nrm = xyz(wn), rA = xyz(wa), rB = xyz(wb);
            f3 rel = add3(pvA, cross3(poA, rA));
            if (bj >= 0) rel = sub3(rel, add3(pvB, cross3(poB, rB)));
            const float meff = wa.w;
            if (meff >= 1e-12f) {
                const float bias = B2C_BETA * fmaxf(wn.w - B2C_SLOP, 0.0f) / a.dt;
                float dj = (bias - dot3(rel, nrm)) / meff;
                const float nw = fmaxf(0.0f, jp + dj);
                dj = nw - jp;
                store_imp_w(&a.rec.contact(kCImp, k0 + j)[s], nw);
                const f3 Jn = scale3(nrm, dj);
                if (iMA > 0.0f) {
                    pvA = f3{fmaf(Jn.x, iMA, pvA.x), fmaf(Jn.y, iMA, pvA.y), fmaf(Jn.z, iMA, pvA.z)};
                    poA = add3(poA, matvec(pre.IA, cross3(rA, Jn)));
                }
                if (bj >= 0 && iMB > 0.0f) {
                    pvB = f3{fmaf(-Jn.x, iMB, pvB.x), fmaf(-Jn.y, iMB, pvB.y), fmaf(-Jn.z, iMB, pvB.z)};
                    poB = sub3(poB, matvec(pre.IB, cross3(rB, Jn)));
                }
            }
        }
    }
    if (iMA > 0.0f) {
        B.set(bi, 2, pvA);
        B.set(bi, 3, poA);
    }
    if (bj >= 0 && iMB > 0.0f) {
        B.set(bj, 2, pvB);
        B.set(bj, 3, poB);
    }
}

template <class BA>
__device__ void pair_apply_warm_row(const SolveArgs &a, int s, const BA &BS, const RowPre &pre)
{
    const int4 h = pre.h;
    const float4 mm = pre.mm;
    const m3 &IA = pre.IA, &IB = pre.IB;
    const int A = h.x, B = h.y, n = h.z;
    const float iMA = mm.x, iMB = mm.y;
    f3 va = BS.get(A, 0), wa = BS.get(A, 1), vb{0.0f, 0.0f, 0.0f}, wb{0.0f, 0.0f, 0.0f};
    if (B >= 0) {
        vb = BS.get(B, 0);
        wb = BS.get(B, 1);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, false);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const RowC cur = staged_row(j);
            const f3 nrm = xyz(cur.n), t1 = xyz(cur.t1), t2 = cross3(nrm, t1);
            const float jn = cur.im.x, j1 = cur.im.y, j2 = cur.im.z;
            const f3 J{fmaf(j2, t2.x, fmaf(jn, nrm.x, j1 * t1.x)), fmaf(j2, t2.y, fmaf(jn, nrm.y, j1 * t1.y)),
                       fmaf(j2, t2.z, fmaf(jn, nrm.z, j1 * t1.z))};
            if (iMA > 0.0f) {
                const RowResp k = row_responses(IA, xyz(cur.ra), nrm, t1, t2);
                va = f3{fmaf(iMA, J.x, va.x), fmaf(iMA, J.y, va.y), fmaf(iMA, J.z, va.z)};
                wa = add3(wa, f3{fmaf(j2, k.t2.x, fmaf(jn, k.n.x, j1 * k.t1.x)),
                                 fmaf(j2, k.t2.y, fmaf(jn, k.n.y, j1 * k.t1.y)),
                                 fmaf(j2, k.t2.z, fmaf(jn, k.n.z, j1 * k.t1.z))});
            }
            if (B >= 0 && iMB > 0.0f) {
                const RowResp k = row_responses(IB, xyz(cur.rb), nrm, t1, t2);
                vb = f3{fmaf(-iMB, J.x, vb.x), fmaf(-iMB, J.y, vb.y), fmaf(-iMB, J.z, vb.z)};
                wb = sub3(wb, f3{fmaf(j2, k.t2.x, fmaf(jn, k.n.x, j1 * k.t1.x)),
                                 fmaf(j2, k.t2.y, fmaf(jn, k.n.y, j1 * k.t1.y)),
                                 fmaf(j2, k.t2.z, fmaf(jn, k.n.z, j1 * k.t1.z))});
            }
        }
    }
    if (iMA > 0.0f) {
        BS.set(A, 0, va);
        BS.set(A, 1, wa);
    }
    if (B >= 0 && iMB > 0.0f) {
        BS.set(B, 0, vb);
        BS.set(B, 1, wb);
    }
}

// The row form's warm start applied body by body: each dynamic body walks its pairs in colour
// order (the set bits of its first-fit colour mask, the slots from body_slots) and applies
// every contact of each with pair_apply_warm_row's expressions for its side.  A body's pairs
// have distinct colours and the colour phases visit them in colour order, so the result is
// the same bits as the warm pass of colour phases, in one launch.
__global__ void k_warm_gather_row(const b2c_header *__restrict__ hdr, int nbodies,
                                  const unsigned long long *__restrict__ body_colors,
                                  const int *__restrict__ body_slots, Records R, float *v, float *w)
{
    if (hdr->n_pairs == 0 || hdr->n_colors == 0) return;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nbodies; b += gridDim.x * blockDim.x) {
        unsigned long long m = body_colors[b];
        if (!m) continue;
        f3 vv = ld3(v, b), ww = ld3(w, b);
        int e = body_slots[64 * b + (__ffsll((long long)m) - 1)];
        m &= m - 1;
        // The loads run ahead of the arithmetic: the next pair's slot while a pair is applied,
        // a pair's first contact with its header, the next contact's words while a contact is
        // applied.  The first contact's words are read before the count arrives: they lie inside
        // the slot's record whatever its count (and every pair has at least one contact).  The
        // arithmetic and its order are those of the colour phases.
        for (;;) {
            const int s = e >> 1;
            const bool sideB = (e & 1) != 0;
            const int rf = sideB ? kRRB : kRRA;
            int e_next = -1;
            if (m) {
                e_next = body_slots[64 * b + (__ffsll((long long)m) - 1)];
                m &= m - 1;
            }
            const int4 h = R.hdr()[s];
            const float4 mm = R.body(6)[s];
            const m3 I = load_inertia(R, s, sideB ? 3 : 0);
            const float iM = sideB ? mm.y : mm.x;
            float4 n_cn = R.contact(kRN, 0)[s], n_ct1 = R.contact(kRT1, 0)[s], n_im = R.contact(kRImp, 0)[s];
            float4 n_r = R.contact(rf, 0)[s];
            for (int k = 0; k < h.z; ++k) {
                const float4 cn = n_cn, ct1 = n_ct1, im = n_im, rr = n_r;
                if (k + 1 < h.z) {
                    n_cn = R.contact(kRN, k + 1)[s];
                    n_ct1 = R.contact(kRT1, k + 1)[s];
                    n_im = R.contact(kRImp, k + 1)[s];
                    n_r = R.contact(rf, k + 1)[s];
                }
                const f3 nrm = xyz(cn), t1 = xyz(ct1), t2 = cross3(nrm, t1);
                const f3 r = xyz(rr);
                const float jn = im.x, j1 = im.y, j2 = im.z;
                const f3 J{fmaf(j2, t2.x, fmaf(jn, nrm.x, j1 * t1.x)), fmaf(j2, t2.y, fmaf(jn, nrm.y, j1 * t1.y)),
                           fmaf(j2, t2.z, fmaf(jn, nrm.z, j1 * t1.z))};
                const RowResp kr = row_responses(I, r, nrm, t1, t2);
                const f3 dw{fmaf(j2, kr.t2.x, fmaf(jn, kr.n.x, j1 * kr.t1.x)),
                            fmaf(j2, kr.t2.y, fmaf(jn, kr.n.y, j1 * kr.t1.y)),
                            fmaf(j2, kr.t2.z, fmaf(jn, kr.n.z, j1 * kr.t1.z))};
                if (!sideB) {
                    vv = f3{fmaf(iM, J.x, vv.x), fmaf(iM, J.y, vv.y), fmaf(iM, J.z, vv.z)};
                    ww = add3(ww, dw);
                } else {
                    vv = f3{fmaf(-iM, J.x, vv.x), fmaf(-iM, J.y, vv.y), fmaf(-iM, J.z, vv.z)};
                    ww = sub3(ww, dw);
                }
            }
            if (e_next < 0) break;
            e = e_next;
        }
        st4(v, b, f4(vv, 0.0f));
        st4(w, b, f4(ww, 0.0f));
    }
}

template <class BA>
__device__ void pair_velocity_row(const SolveArgs &a, int s, const BA &B, const RowPre &pre)
{
    const int4 h = pre.h;
    const float4 mm = pre.mm;
    const m3 &IA = pre.IA, &IB = pre.IB;
    const int bi = h.x, bj = h.y, n = h.z;
    const float iMA = mm.x, iMB = mm.y, mu = mm.z;
    f3 vA = B.get(bi, 0), wA = B.get(bi, 1);
    f3 vB{0.0f, 0.0f, 0.0f}, wB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        vB = B.get(bj, 0);
        wB = B.get(bj, 1);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, false);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const RowC cur = staged_row(j);
            const f3 nrm = xyz(cur.n), rA = xyz(cur.ra), rB = xyz(cur.rb), t1 = xyz(cur.t1), t2 = cross3(nrm, t1);
            // the responses depend on the record only, so they are computed off the velocity chain
            const RowResp kA = row_responses(IA, rA, nrm, t1, t2);
            RowResp kB{};
            if (bj >= 0) kB = row_responses(IB, rB, nrm, t1, t2);
            // The guarded updates below are written as selects of the updated and the old value
            // (exactly the values of the branches they replace), so the chain has no branches
            // but the friction clamp's.
            const bool hasB = bj >= 0, dynA = iMA > 0.0f, dynB = hasB && iMB > 0.0f;
            const bool act = cur.n.w > 0.0f, fric = cur.t1.w > 0.0f && cur.rb.w > 0.0f;
            const f3 zero{0.0f, 0.0f, 0.0f};
            f3 va = add3(vA, cross3(wA, rA));
            f3 vb = sel3(hasB, add3(vB, cross3(wB, rB)), zero);
            f3 vrel = sub3(va, vb);
            const float vn = dot3(vrel, nrm);
            float4 im = cur.im;
            float dj = -vn * cur.n.w;
            const float nw = fmaxf(0.0f, im.x + dj);
            dj = nw - im.x;
            im.x = nw;
            const f3 Jn = scale3(nrm, dj);
            const f3 vA1 = sel3(dynA, f3{fmaf(Jn.x, iMA, vA.x), fmaf(Jn.y, iMA, vA.y), fmaf(Jn.z, iMA, vA.z)}, vA);
            const f3 wA1 = sel3(dynA, fma3s(dj, kA.n, wA), wA);
            const f3 vB1 = sel3(dynB, f3{fmaf(-Jn.x, iMB, vB.x), fmaf(-Jn.y, iMB, vB.y), fmaf(-Jn.z, iMB, vB.z)}, vB);
            const f3 wB1 = sel3(dynB, fma3s(-dj, kB.n, wB), wB);
            va = add3(vA1, cross3(wA1, rA));
            vb = sel3(hasB, add3(vB1, cross3(wB1, rB)), zero);
            vrel = sub3(va, vb);
            const float o1 = im.y, o2 = im.z;
            float a1 = o1 - dot3(vrel, t1) * cur.t1.w;
            float a2 = o2 - dot3(vrel, t2) * cur.rb.w;
            const float mag = sqrtf(fmaf(a1, a1, a2 * a2));
            const float lim = mu * im.x;
            if (fric && mag > lim && mag > 1e-12f) {
                const float sc = lim / mag;
                a1 = a1 * sc;
                a2 = a2 * sc;
            }
            const float e1 = a1 - o1, e2 = a.t2d * (a2 - o2);
            const f3 Jt{fmaf(e1, t1.x, e2 * t2.x), fmaf(e1, t1.y, e2 * t2.y), fmaf(e1, t1.z, e2 * t2.z)};
            const bool fA = fric && dynA, fB = fric && dynB;
            const f3 vA2 = sel3(fA, f3{fmaf(Jt.x, iMA, vA1.x), fmaf(Jt.y, iMA, vA1.y), fmaf(Jt.z, iMA, vA1.z)}, vA1);
            const f3 wA2 = sel3(fA, fma3s(e1, kA.t1, fma3s(e2, kA.t2, wA1)), wA1);
            const f3 vB2 = sel3(fB, f3{fmaf(-Jt.x, iMB, vB1.x), fmaf(-Jt.y, iMB, vB1.y), fmaf(-Jt.z, iMB, vB1.z)}, vB1);
            const f3 wB2 = sel3(fB, fma3s(-e1, kB.t1, fma3s(-e2, kB.t2, wB1)), wB1);
            if (fric) {
                im.y = a1;
                im.z = a2;
            }
            vA = sel3(act, vA2, vA);
            wA = sel3(act, wA2, wA);
            vB = sel3(act, vB2, vB);
            wB = sel3(act, wB2, wB);
            if (act) store_imp_xyz(&a.rec.contact(kRImp, k0 + j)[s], im);
        }
    }
    if (iMA > 0.0f) {
        B.set(bi, 0, vA);
        B.set(bi, 1, wA);
    }
    if (bj >= 0 && iMB > 0.0f) {
        B.set(bj, 0, vB);
        B.set(bj, 1, wB);
    }
}

template <class BA>
__device__ void pair_position_row(const SolveArgs &a, int s, const BA &B, const RowPre &pre)
{
    const int4 h = pre.h;
    const float4 mm = pre.mm;
    const m3 &IA = pre.IA, &IB = pre.IB;
    const int bi = h.x, bj = h.y, n = h.z;
    const float iMA = mm.x, iMB = mm.y;
    f3 pvA = B.get(bi, 2), poA = B.get(bi, 3);
    f3 pvB{0.0f, 0.0f, 0.0f}, poB{0.0f, 0.0f, 0.0f};
    if (bj >= 0) {
        pvB = B.get(bj, 2);
        poB = B.get(bj, 3);
    }
    cp_async_wait_all();
    for (int k0 = 0; k0 < n; k0 += kRowBatch) {
        if (k0 > 0) {
            stage_rows(a.rec, s, k0, true);
            cp_async_wait_all();
        }
        for (int j = 0; j < kRowBatch; ++j) {
            if (k0 + j >= n) break;
            const float4 wn = *stage_word(kRN, j), wa = *stage_word(kRRA, j), wb = *stage_word(kRRB, j);
            const float jp = stage_word(kRImp, j)->w;
            const f3 nrm = xyz(wn), rA = xyz(wa), rB = xyz(wb);
            const f3 kAn = matvec(IA, cross3(rA, nrm));
            f3 kBn{0.0f, 0.0f, 0.0f};
            if (bj >= 0) kBn = matvec(IB, cross3(rB, nrm));
            // selects of the updated and the old values, as in the velocity chunk
            const bool hasB = bj >= 0, act = wn.w > 0.0f;
            const bool uA = act && iMA > 0.0f, uB = act && hasB && iMB > 0.0f;
            f3 rel = add3(pvA, cross3(poA, rA));
            rel = sel3(hasB, sub3(rel, add3(pvB, cross3(poB, rB))), rel);
            float dj = (wa.w - dot3(rel, nrm)) * wn.w;
            const float nw = fmaxf(0.0f, jp + dj);
            dj = nw - jp;
            if (act) store_imp_w(&a.rec.contact(kRImp, k0 + j)[s], nw);
            const f3 Jn = scale3(nrm, dj);
            pvA = sel3(uA, f3{fmaf(Jn.x, iMA, pvA.x), fmaf(Jn.y, iMA, pvA.y), fmaf(Jn.z, iMA, pvA.z)}, pvA);
            poA = sel3(uA, fma3s(dj, kAn, poA), poA);
            pvB = sel3(uB, f3{fmaf(-Jn.x, iMB, pvB.x), fmaf(-Jn.y, iMB, pvB.y), fmaf(-Jn.z, iMB, pvB.z)}, pvB);
            poB = sel3(uB, fma3s(-dj, kBn, poB), poB);
        }
    }
    if (iMA > 0.0f) {
        B.set(bi, 2, pvA);
        B.set(bi, 3, poA);
    }
    if (bj >= 0 && iMB > 0.0f) {
        B.set(bj, 2, pvB);
        B.set(bj, 3, poB);
    }
}

// ---------------------------------------------------------------------------------------------
// the persistent kernels
//
// Phase schedule.  The position sweeps read and write only pv, po and the contacts' jp, which no
// velocity sweep or warm application touches, and the velocity sweeps never read them; so
// position sweep k runs in the same phase as the k-th (warm application, velocity sweep 0,
// velocity sweep 1, ...) pass over the colours, on other threads.  Every pair still sees the
// same values in the same order as in the sequential schedule (warm; vit velocity sweeps; pit
// position sweeps), so the results are identical, with (warm + max(vit, pit)) x colours phases
// instead of (warm + vit + pit) x colours.
//
// Task t of a phase (velocity/warm tasks first, then position tasks) runs on lane t mod 32 of
// warp chunk c = t div 32, and chunk c on CTA c mod CTAs: a warp reads 32 consecutive record
// slots (coalesced), and a colour narrower than the launch is spread over all of its SMs.
// ---------------------------------------------------------------------------------------------
constexpr int kMaxSolveColors = 512;  // the colouring's cap (kMaxColorsCap)

// The phases of the persistent solve (both forms).  Task layout of a colour of cnt pairs: velocity (or warm) tasks
// [0, cnt) and position tasks [P0, P0 + cnt) with P0 = cnt rounded up to a warp, in every pass
// (a pass without the velocity sweep leaves [0, P0) idle).  So no warp mixes the two kinds,
// and a pair's velocity task and its position task each stay on one thread in every pass: the
// impulse words a task reads are written only by the thread that runs it.  A thread's first
// task of the next phase has its fixed words loaded between the barrier's arrive and wait.
// Those words do not change during the solve, and its contact words were last written by this
// same thread.  With a single colour the next phase revisits this phase's pairs, so nothing is
// prefetched then.
template <int kKind, bool kRow, bool kFixed, class BA>
__device__ __forceinline__ void solve_phases(const SolveArgs &a, const BA &B)
{
    const int nc = a.hdr->n_colors;
    if (a.hdr->n_pairs == 0 || nc == 0 || islands_took_solve(a)) return;  // uniform over all CTAs
    __shared__ int s_cstart[kMaxSolveColors], s_ccount[kMaxSolveColors];
    for (int c = threadIdx.x; c < nc && c < kMaxSolveColors; c += blockDim.x) {
        s_cstart[c] = a.cstart[c];
        s_ccount[c] = a.ccount[c];
    }
    __syncthreads();
    const int nb = gridDim.x, nth = gridDim.x * blockDim.x;
    const int me = ((((int)threadIdx.x >> 5) * nb + (int)blockIdx.x) << 5) | ((int)threadIdx.x & 31);  // task slot
    const int vpasses = (a.apply_warm ? 1 : 0) + a.vit;
    const int passes = vpasses > a.pit ? vpasses : a.pit;
    // task t of phase (pass, ci): its record slot, or -1 for none; pos tells the kind
    auto task_slot = [&](int pass, int ci, int t, bool &pos) -> int {
        const int cnt = s_ccount[ci], p0 = (cnt + 31) & ~31;
        if (t < cnt) {
            pos = false;
            return pass < vpasses ? s_cstart[ci] + t : -1;
        }
        pos = true;
        return (pass < a.pit && t >= p0 && t < p0 + cnt) ? s_cstart[ci] + (t - p0) : -1;
    };
    RowPre pre;
    int pre_t = -1;
    bool pos;
    unsigned int epoch = 0;  // grid barriers passed in this launch
    {
        const int sl = task_slot(0, 0, me, pos);
        if (sl >= 0) {
            pre = row_pre(a.rec, sl, pos);
            pre_t = me;
        }
    }
    for (int pass = 0; pass < passes; ++pass) {
        const bool warm = a.apply_warm && pass == 0;
        for (int ci = 0; ci < nc; ++ci) {
            const int cnt = s_ccount[ci], ntask = ((cnt + 31) & ~31) + cnt;
            for (int t = me; t < ntask; t += nth) {
                const int sl = task_slot(pass, ci, t, pos);
                if (sl < 0) continue;
                const RowPre q = (t == pre_t) ? pre : row_pre(a.rec, sl, pos);
                if (kRow) {
                    if (!pos) {
                        if (warm) pair_apply_warm_row(a, sl, B, q);
                        else pair_velocity_row(a, sl, B, q);
                    } else {
                        pair_position_row(a, sl, B, q);
                    }
                } else {
                    if (!pos) {
                        if (warm) pair_apply_warm(a, sl, B, q);
                        else pair_velocity<BA, kFixed>(a, sl, B, q);
                    } else {
                        pair_position(a, sl, B, q);
                    }
                }
            }
            pre_t = -1;
            const BarTok tok = bar_arrive<kKind>(a, epoch);
            const int np = ci + 1 < nc ? pass : pass + 1, nci = ci + 1 < nc ? ci + 1 : 0;
            if (nc > 1 && np < passes) {
                const int sl = task_slot(np, nci, me, pos);
                if (sl >= 0) {
                    pre = row_pre(a.rec, sl, pos);
                    pre_t = me;
                }
            }
            if (!bar_wait<kKind>(a, tok)) return;
        }
    }
}

constexpr int kClusterThreads = 384;     // reference form (contact staging as the row form)
constexpr int kClusterThreadsRow = 384;  // row form (123 registers; 120 KB of contact staging)
constexpr int kClusterMax = 16;

__global__ void __launch_bounds__(256, 1) k_color_solve_block(SolveArgs a)
{
    const GlobalBodies B{a.v, a.w, a.pv, a.po};
    if (a.row) solve_phases<kBlock, true, true>(a, B);
    else if (a.fixed_frame) solve_phases<kBlock, false, true>(a, B);
    else solve_phases<kBlock, false, false>(a, B);
}
__global__ void __launch_bounds__(256, 1) k_color_solve_grid(SolveArgs a)
{
    const GlobalBodies B{a.v, a.w, a.pv, a.po};
    if (a.row) solve_phases<kGrid, true, true>(a, B);
    else if (a.fixed_frame) solve_phases<kGrid, false, true>(a, B);
    else solve_phases<kGrid, false, false>(a, B);
}
// Cluster solve, one kernel per form so each gets the registers it needs.  (Holding the body
// state in distributed shared memory instead measured slower on B200 for this access pattern:
// 1.25 ms against 0.78 ms on the 10k-box lattice.)
__global__ void __launch_bounds__(kClusterThreads) k_color_solve_cluster(SolveArgs a)
{
    const GlobalBodies B{a.v, a.w, a.pv, a.po};
    if (a.fixed_frame) solve_phases<kCluster, false, true>(a, B);
    else solve_phases<kCluster, false, false>(a, B);
}
__global__ void __launch_bounds__(kClusterThreadsRow) k_color_solve_cluster_row(SolveArgs a)
{
    const GlobalBodies B{a.v, a.w, a.pv, a.po};
    solve_phases<kCluster, true, true>(a, B);
}

// ---------------------------------------------------------------------------------------------
// Scene schedule: one CTA per scene of a batch.  Scenes share no bodies, so each scene's colour
// phases only have to wait for the scene's own pairs: the CTA barrier replaces the barrier over
// all scenes, and a scene's phase lasts as long as its own heaviest pair.  The pair tasks, the
// passes and the colour order inside a scene are those of solve_phases, so the bits are too.
// ---------------------------------------------------------------------------------------------
struct SceneSched {
    const int *pbi, *col, *body_start, *order, *pair_slot;
    int *slots;
};

// first index in [0, n) whose pbi is >= body (pbi is sorted)
__device__ __forceinline__ int first_pair_of(const int *pbi, int n, int body)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pbi[mid] < body) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

template <class BA>
__device__ __forceinline__ void solve_phases_scene(const SolveArgs &a, const SceneSched &sc, const BA &B)
{
    const int P = a.hdr->n_pairs, ncg = a.hdr->n_colors;
    if (P == 0 || ncg == 0 || islands_took_solve(a)) return;  // uniform over all CTAs
    __shared__ int s_cstart[kMaxSolveColors], s_ccount[kMaxSolveColors], s_cur[kMaxSolveColors];
    __shared__ int s_pa, s_pb, s_nc;
    const int scene = sc.order ? sc.order[blockIdx.x] : (int)blockIdx.x;
    if (threadIdx.x == 0) {
        s_pa = first_pair_of(sc.pbi, P, sc.body_start[scene]);
        s_pb = first_pair_of(sc.pbi, P, sc.body_start[scene + 1]);
    }
    for (int c = threadIdx.x; c < kMaxSolveColors; c += blockDim.x) s_ccount[c] = 0;
    __syncthreads();
    const int pa = s_pa, pb = s_pb;
    // this scene's pairs by colour: counts, offsets, then its record slots in colour order
    for (int p = pa + (int)threadIdx.x; p < pb; p += blockDim.x) atomicAdd(&s_ccount[sc.col[p]], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0, nc = 0;
        for (int c = 0; c < ncg && c < kMaxSolveColors; ++c) {
            s_cstart[c] = acc;
            s_cur[c] = acc;
            acc += s_ccount[c];
            if (s_ccount[c]) nc = c + 1;
        }
        s_nc = nc;
    }
    __syncthreads();
    for (int p = pa + (int)threadIdx.x; p < pb; p += blockDim.x)
        sc.slots[pa + atomicAdd(&s_cur[sc.col[p]], 1)] = sc.pair_slot[p];
    __syncthreads();
    const int nc = s_nc;
    if (nc == 0) return;  // uniform within the CTA
    const int *slots = sc.slots + pa;
    const int me = (int)threadIdx.x, nth = (int)blockDim.x;
    const int vpasses = (a.apply_warm ? 1 : 0) + a.vit;
    const int passes = vpasses > a.pit ? vpasses : a.pit;
    auto task_slot = [&](int pass, int ci, int t, bool &pos) -> int {
        const int cnt = s_ccount[ci], p0 = (cnt + 31) & ~31;
        if (t < cnt) {
            pos = false;
            return pass < vpasses ? slots[s_cstart[ci] + t] : -1;
        }
        pos = true;
        return (pass < a.pit && t >= p0 && t < p0 + cnt) ? slots[s_cstart[ci] + (t - p0)] : -1;
    };
    RowPre pre;
    int pre_t = -1;
    bool pos;
    {
        const int sl = task_slot(0, 0, me, pos);
        if (sl >= 0) {
            pre = row_pre(a.rec, sl, pos);
            pre_t = me;
        }
    }
    for (int pass = 0; pass < passes; ++pass) {
        const bool warm = a.apply_warm && pass == 0;
        for (int ci = 0; ci < nc; ++ci) {
            const int cnt = s_ccount[ci], ntask = ((cnt + 31) & ~31) + cnt;
            for (int t = me; t < ntask; t += nth) {
                const int sl = task_slot(pass, ci, t, pos);
                if (sl < 0) continue;
                const RowPre q = (t == pre_t) ? pre : row_pre(a.rec, sl, pos);
                if (!pos) {
                    if (warm) pair_apply_warm_row(a, sl, B, q);
                    else pair_velocity_row(a, sl, B, q);
                } else {
                    pair_position_row(a, sl, B, q);
                }
            }
            pre_t = -1;
            const int np = ci + 1 < nc ? pass : pass + 1, nci = ci + 1 < nc ? ci + 1 : 0;
            if (nc > 1 && np < passes) {
                const int sl = task_slot(np, nci, me, pos);
                if (sl >= 0) {
                    pre = row_pre(a.rec, sl, pos);
                    pre_t = me;
                }
            }
            __syncthreads();
        }
    }
}

constexpr int kSceneThreads = 256;
__global__ void __launch_bounds__(kSceneThreads, 2) k_color_solve_scenes(SolveArgs a, SceneSched sc)
{
    const GlobalBodies B{a.v, a.w, a.pv, a.po};
    solve_phases_scene(a, sc, B);
}

// ---------------------------------------------------------------------------------------------
// Island solve (IslandSolveContactEngine's solve kernel, contact_engine_gpu_island_solve.py:230-249):
// one thread runs the warm start and the velocity sweeps of one island, pair after pair in
// colour order, and another thread its position sweeps.  An island's pairs share no dynamic
// body with any other island's, so no other thread reads or writes its bodies' velocities, and
// every pair sees the values it sees in the colour phases: the same bits, with no barrier.
// The bodies are read and written with ordinary (L1-cached) accesses: each body's v, w (or pv,
// po) belong to one thread for the whole launch, and static bodies are only read.  Task t of
// the velocity range [0, P) is the island that starts at position t of the island-ordered slot
// list (isl_at[t] > 0); the position range follows at P rounded up to a warp.
// ---------------------------------------------------------------------------------------------
struct IslandBodies {
    float *v, *w, *pv, *po;
    __device__ __forceinline__ f3 get(int b, int k) const
    {
        const float *p = k == 0 ? v : k == 1 ? w : k == 2 ? pv : po;
        return xyz(reinterpret_cast<const float4 *>(p)[b]);
    }
    __device__ __forceinline__ void set(int b, int k, f3 x) const
    {
        float *p = k == 0 ? v : k == 1 ? w : k == 2 ? pv : po;
        reinterpret_cast<float4 *>(p)[b] = f4(x, 0.0f);
    }
};

template <bool kRow, bool kFixed>
__device__ __forceinline__ void island_tasks(const SolveArgs &a, const int *__restrict__ slots,
                                             const int *__restrict__ isl_at)
{
    const int P = a.hdr->n_pairs;
    if (P == 0 || a.hdr->n_colors == 0 || !(a.island_info[1] <= B2C_ISLAND_MAX_PAIRS)) return;
    const IslandBodies B{a.v, a.w, a.pv, a.po};
    const int p32 = (P + 31) & ~31;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < p32 + P; t += gridDim.x * blockDim.x) {
        const bool pos = t >= p32;
        const int at = pos ? t - p32 : t;
        if (at >= P) continue;
        const int cnt = isl_at[at];
        if (cnt == 0) continue;
        const int *sl = slots + at;
        // A pair's impulses, stored by this thread in one sweep, are read back by the staging
        // copies of the next: the fence orders the stores before the copies.
        if (!pos) {
            if (a.apply_warm) {
                for (int j = 0; j < cnt; ++j) {
                    const int s = sl[j];
                    const RowPre q = row_pre<true>(a.rec, s, false);
                    if (kRow) pair_apply_warm_row(a, s, B, q);
                    else pair_apply_warm(a, s, B, q);
                }
            }
            for (int it = 0; it < a.vit; ++it) {
                for (int j = 0; j < cnt; ++j) {
                    const int s = sl[j];
                    __threadfence_block();
                    const RowPre q = row_pre<true>(a.rec, s, false);
                    if (kRow) pair_velocity_row(a, s, B, q);
                    else pair_velocity<IslandBodies, kFixed>(a, s, B, q);
                }
            }
        } else {
            for (int it = 0; it < a.pit; ++it) {
                for (int j = 0; j < cnt; ++j) {
                    const int s = sl[j];
                    __threadfence_block();
                    const RowPre q = row_pre<true>(a.rec, s, true);
                    if (kRow) pair_position_row(a, s, B, q);
                    else pair_position(a, s, B, q);
                }
            }
        }
    }
}

constexpr int kIslandThreads = 128;
__global__ void __launch_bounds__(kIslandThreads) k_island_solve(SolveArgs a, const int *slots, const int *isl_at)
{
    if (a.row) island_tasks<true, true>(a, slots, isl_at);
    else if (a.fixed_frame) island_tasks<false, true>(a, slots, isl_at);
    else island_tasks<false, false>(a, slots, isl_at);
}

int island_partition_engine(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const int **info,
                            const int **slots, const int **isl_at, cudaStream_t s);

// dynamic shared memory of a solve launch: the contact staging of its threads
static size_t stage_bytes(int threads) { return (size_t)kStageBytesPerThread * threads; }

// the solve kernels' dynamic shared memory exceeds the 48 KB default: opt in once
static void allow_stage_smem()
{
    static bool done = false;
    if (done) return;
    cudaFuncSetAttribute(k_color_solve_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes(256));
    cudaFuncSetAttribute(k_color_solve_grid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes(256));
    cudaFuncSetAttribute(k_color_solve_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)stage_bytes(kClusterThreads));
    cudaFuncSetAttribute(k_color_solve_cluster_row, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)stage_bytes(kClusterThreadsRow));
    cudaFuncSetAttribute(k_color_solve_scenes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)stage_bytes(kSceneThreads));
    cudaFuncSetAttribute(k_island_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)stage_bytes(kIslandThreads));
    done = true;
}

static int max_coresident_grid_blocks()
{
    static int cached = -1;
    if (cached < 0) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        allow_stage_smem();
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_color_solve_grid, 256, stage_bytes(256));
        cached = std::min(kBarrierMaxCTAs, std::max(1, sms * std::max(per, 1)));
    }
    return cached;
}

// largest power-of-two cluster (<= 16) of a cluster-solve kernel that the device can
// co-schedule; a host-side occupancy query, cached per form (an engine's first step runs
// eagerly, before any graph capture)
static int max_cluster_size(int row)
{
    static int cached[2] = {-1, -1};
    if (cached[row] < 0) {
        const void *fn = row ? (const void *)k_color_solve_cluster_row : (const void *)k_color_solve_cluster;
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        allow_stage_smem();
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kClusterMax);
        cfg.blockDim = dim3(row ? kClusterThreadsRow : kClusterThreads);
        cfg.dynamicSmemBytes = stage_bytes(row ? kClusterThreadsRow : kClusterThreads);
        int cs = 0;
        if (cudaOccupancyMaxPotentialClusterSize(&cs, fn, &cfg) != cudaSuccess) {
            cudaGetLastError();
            cs = 0;
        }
        int p2 = 0;
        for (int c = 1; c <= std::min(cs, kClusterMax); c *= 2) p2 = c;
        cached[row] = p2 >= 2 ? p2 : 0;
    }
    return cached[row];
}

int color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                float dt, cudaStream_t s)
{
    SolveArgs a;
    a.hdr = hdr;
    a.err = &hdr->error;
    a.cstart = pr->cstart;
    a.ccount = pr->ccount;
    a.rec = Records{reinterpret_cast<float4 *>(pr->rec), pr->capacity, pr->kslots};
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
    a.row = (p->flags & B2C_COLOR_ROW_FORM) ? 1 : 0;
    if (a.row && !a.fixed_frame) {
        set_error("color_solve: B2C_COLOR_ROW_FORM needs B2C_COLOR_FIXED_FRAME");
        return B2C_EARG;
    }
    a.bar_count = pr->barrier;
    a.timeout_ns = p->barrier_timeout_ns > 0 ? p->barrier_timeout_ns : 1000000000LL;
    a.island_info = nullptr;
    const bool islands = (p->flags & B2C_COLOR_ISLANDS) != 0;
    if (islands && !pr->isl_work) {
        set_error("color_solve: B2C_COLOR_ISLANDS needs b2c_pairs.isl_work");
        return B2C_EARG;
    }

    const int pgrid = std::min(blocks_for(pr->capacity), kSMs * 8);
    const bool scenes = p->solve_blocks == B2C_SOLVE_SCENES;
    if (scenes && !(a.row && pr->n_scenes > 0 && pr->scene_body_start && pr->pair_slot && pr->scene_slots)) {
        set_error("color_solve: the scene schedule needs the row form and b2c_pairs' scene arrays");
        return B2C_EARG;
    }
    // the warm start body by body (one launch) instead of a pass of colour phases
    const bool warm_bodies = a.row && a.apply_warm && (p->flags & B2C_COLOR_FIRST_FIT) && pr->body_slots &&
                             pr->body_colors;
    if (a.row)
        k_pair_gather_row<<<pgrid, kThreads, 0, s>>>(hdr, pr->porder, pr->pstart, pr->kcount, pr->pidx, pr->pbi,
                                                     pr->pbj, *kept, b->xc, b->invIw, b->invM, p->body_mu, p->mu, dt,
                                                     a.rec, hdr, pr->col, warm_bodies ? pr->body_slots : nullptr,
                                                     scenes ? pr->pair_slot : nullptr);
    else
        k_pair_gather<<<pgrid, kThreads, 0, s>>>(hdr, pr->porder, pr->pstart, pr->kcount, pr->pidx, pr->pbi, pr->pbj,
                                                 *kept, b->xc, b->invIw, b->invM, p->body_mu, p->mu, a.rec, hdr);
    int rc = check_launch("pair_gather");
    if (rc) return rc;
    if (warm_bodies) {
        k_warm_gather_row<<<std::min(blocks_for(b->n), kSMs * 8), kThreads, 0, s>>>(
            hdr, b->n, reinterpret_cast<const unsigned long long *>(pr->body_colors), pr->body_slots, a.rec, b->v,
            b->w);
        if ((rc = check_launch("warm_gather"))) return rc;
        a.apply_warm = 0;
    }

    if (islands) {
        const int *isl_slots = nullptr, *isl_at = nullptr;
        if ((rc = island_partition_engine(b, pr, hdr, &a.island_info, &isl_slots, &isl_at, s))) return rc;
        allow_stage_smem();
        k_island_solve<<<std::min(blocks_for(2LL * pr->capacity + 32, kIslandThreads), kSMs * 4), kIslandThreads,
                         stage_bytes(kIslandThreads), s>>>(a, isl_slots, isl_at);
        if ((rc = check_launch("island_solve"))) return rc;
    }
    int mode = p->solve_blocks;
    if (scenes) {
        allow_stage_smem();
        const SceneSched sc{pr->pbi, pr->col, pr->scene_body_start, pr->scene_order, pr->pair_slot,
                            pr->scene_slots};
        k_color_solve_scenes<<<pr->n_scenes, kSceneThreads, stage_bytes(kSceneThreads), s>>>(a, sc);
        if ((rc = check_launch("color_solve_scenes"))) return rc;
        mode = 0;
    } else if (mode == 0) {  // auto: one CTA for tiny scenes, else a cluster (colours wider than it loop)
        if (b->n <= 64) mode = 1;
        else mode = -kClusterMax;
    }
    if (mode < 0) {
        const int cs = std::min(-mode, max_cluster_size(a.row));
        if (cs >= 2) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(cs);
            cfg.blockDim = dim3(a.row ? kClusterThreadsRow : kClusterThreads);
            cfg.dynamicSmemBytes = stage_bytes(a.row ? kClusterThreadsRow : kClusterThreads);
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = cs;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            cudaError_t e = a.row ? cudaLaunchKernelEx(&cfg, k_color_solve_cluster_row, a)
                                  : cudaLaunchKernelEx(&cfg, k_color_solve_cluster, a);
            if (e != cudaSuccess) {
                set_error("color_solve: cluster launch of %d CTAs: %s", cs, cudaGetErrorString(e));
                return B2C_ECUDA;
            }
            if ((rc = check_launch("color_solve_cluster"))) return rc;
        } else {
            mode = std::min((b->n + 255) / 256, max_coresident_grid_blocks());
        }
    }
    if (mode > 0) {
        allow_stage_smem();
        const int nblocks = std::max(1, std::min(mode, max_coresident_grid_blocks()));
        if (nblocks == 1) {
            k_color_solve_block<<<1, 256, stage_bytes(256), s>>>(a);
            if ((rc = check_launch("color_solve_block"))) return rc;
        } else {
            cudaMemsetAsync(a.bar_count, 0, sizeof(uint32_t), s);  // the arrival count restarts every launch
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(nblocks);
            cfg.blockDim = dim3(256);
            cfg.dynamicSmemBytes = stage_bytes(256);
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
            if ((rc = check_launch("color_solve_grid"))) return rc;
        }
    }
    k_imp_scatter<<<pgrid, kThreads, 0, s>>>(hdr, pr->pstart, pr->pidx, a.rec, a.row ? (int)kRImp : (int)kCImp,
                                             kept->imp);
    return check_launch("imp_scatter");
}

}  // namespace b2c

extern "C" int64_t b2c_pair_record_floats(int32_t pair_capacity, int32_t kslots)
{
    if (pair_capacity < 0 || kslots < 1) return -1;
    // room for either layout: the reference form (kRecContact fields per contact) or the row form
    const int64_t per_contact = (int)b2c::kRecContact > (int)b2c::kRecContactRow ? (int)b2c::kRecContact : (int)b2c::kRecContactRow;
    return 4LL * (int64_t)pair_capacity * (1 + b2c::kRecBody + per_contact * (int64_t)kslots);
}
