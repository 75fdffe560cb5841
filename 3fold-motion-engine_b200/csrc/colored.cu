// Coloured Gauss-Seidel pair-chunk chain: GraphColoredContactEngine(manifold_reduce,
// pair_chunks) and its ColorCache descendant (contact_engine_gpu_colored.py,
// contact_engine_gpu_fixed_frame.py, _applied_warm.py, _deferred_force.py, _color_cache.py).
//
// B200 layout of a substep, with no host read-back anywhere:
//   1. contacts in feature-key order by construction: per-bead counts, a scan, then every bead
//      writes its ground contact and its neighbours sorted by bead id at its offset (replaces
//      the atomic append + feature-key radix sort + gather of the reference);
//   2. pair grouping: beads are body-major, so the contacts owned by a body A are contiguous and
//      one warp per body groups them by partner (replaces the pair-key radix sort);
//   3. warm start (binary search), float64 E-optimal selection per pair, compaction, kept pairs;
//   4. Jones-Plassmann colouring of the pair graph in one CTA behind the device-side colour cache;
//   5. the whole chunk solve (applied warm start, vit velocity and pit position sweeps over the
//      colours) in ONE persistent kernel with a bounded grid barrier between colours;
//   6. warm store.
// Every float32 expression follows the reference kernels with the contraction pattern of
// b2c_math.cuh; the selection is float64 without contraction, as the reference compiled it.
#include <cooperative_groups.h>

#include "b2c_grid.cuh"

namespace b2c {

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s);
int body_predict_substep(const b2c_bodies *b, float dt, float *vgrav, bool clear_pseudo, cudaStream_t s);
int body_integrate(const b2c_bodies *b, float dt, cudaStream_t s);
int bead_world(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, cudaStream_t s);
int grid_build(const b2c_beads *beads, b2c_grid *g, cudaStream_t s);

constexpr int kMaxNeighbors = 64;

// ---------------------------------------------------------------------------------------------
// 1. contact generation in feature order (k_gen_fid COL:102-122 + k_fkey/radix sort/k_gather)
// ---------------------------------------------------------------------------------------------
__global__ void k_bead_count(int nb, const float *__restrict__ world, const int *__restrict__ owner,
                             const int *__restrict__ start, const int *__restrict__ sorted,
                             const float4 *__restrict__ spos, GridView g, int *__restrict__ count, b2c_header *hdr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) count[nb] = 0;
    if (i >= nb) return;
    const f3 xi = ld3(world, i);
    const int bi = owner[i];
    int nn = 0;
    for_each_bead_neighbor(i, xi, bi, spos, start, sorted, g, [&](int, f3, f3, float) { ++nn; });
    if (nn > kMaxNeighbors) {
        atomicOr(&hdr->error, B2C_ERR_NEIGHBOR_OVERFLOW);
        nn = kMaxNeighbors;
    }
    count[i] = nn + ((xi.z - B2C_R) < 0.0f ? 1 : 0);
}

__device__ __forceinline__ void put_contact(b2c_contacts &c, int k, int bi, int bj, f3 pA, f3 pB, f3 nrm, float pen,
                                            int fa, int fb)
{
    c.bi[k] = bi;
    c.bj[k] = bj;
    st4(c.pA, k, f4(pA, pen));
    st4(c.pB, k, f4(pB, 0.0f));
    st4(c.n, k, f4(nrm, 0.0f));
    c.fa[k] = fa;
    c.fb[k] = fb;
}

__global__ void k_bead_emit(int nb, const float *__restrict__ world, const int *__restrict__ owner,
                            const int *__restrict__ start, const int *__restrict__ sorted,
                            const float4 *__restrict__ spos, GridView g, const int *__restrict__ offset,
                            b2c_contacts c, b2c_header *hdr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        const int total = offset[nb];
        hdr->n_raw = total;
        hdr->n_contacts = total < c.capacity ? total : c.capacity;
        if (total > c.capacity) atomicOr(&hdr->error, B2C_ERR_CONTACT_OVERFLOW);
    }
    if (i >= nb) return;
    int k = offset[i];
    if (k >= c.capacity) return;
    const f3 xi = ld3(world, i);
    const int bi = owner[i];
    const float s = xi.z - B2C_R;
    if (s < 0.0f) {
        put_contact(c, k, bi, -1, xi, f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 1.0f}, -s, i, -1);
        if (++k >= c.capacity) return;
    }
    if (offset[i + 1] == k) return;  // no bead neighbours
    int js[kMaxNeighbors];
    int n = 0;
    for_each_bead_neighbor(i, xi, bi, spos, start, sorted, g, [&](int j, f3, f3, float) {
        if (n < kMaxNeighbors) {  // insertion into ascending order of bead id
            int t = n++;
            while (t > 0 && js[t - 1] > j) {
                js[t] = js[t - 1];
                --t;
            }
            js[t] = j;
        }
    });
    for (int t = 0; t < n && k < c.capacity; ++t, ++k) {
        const int j = js[t];
        const f3 xj = ld3(world, j);
        const f3 dvec = sub3(xi, xj);
        const float dist = len3(dvec);
        put_contact(c, k, bi, owner[j], xi, xj, div3(dvec, dist), B2C_2R - dist, i, j);
    }
}

// ---------------------------------------------------------------------------------------------
// 2. pair grouping: stable pair-key order (COL:628-649) per body, one warp per body A
// ---------------------------------------------------------------------------------------------
__global__ void k_body_pairs(int nbodies, const int *__restrict__ bead_start, const int *__restrict__ offset, int cap,
                             const int *__restrict__ cbj, int *__restrict__ pair_local, int2 *__restrict__ pair_first,
                             int *__restrict__ gorder, int *__restrict__ body_npairs)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nbodies) return;
    const int lo = min(offset[bead_start[w]], cap), hi = min(offset[bead_start[w + 1]], cap);
    const int L = hi - lo;
    int firsts = 0;
    for (int e = lane; e < L; e += 32) {
        const int v = cbj[lo + e];
        int less = 0, before = 0, same = 0;
        for (int f = 0; f < L; ++f) {
            const int u = cbj[lo + f];
            less += (u < v);
            same += (u == v);
            before += (u == v && f < e);
        }
        gorder[lo + less + before] = lo + e;
        pair_first[lo + e] = before == 0 ? make_int2(lo + less, same) : make_int2(-1, 0);
        firsts += (before == 0);
    }
    __syncwarp();
    for (int e = lane; e < L; e += 32) {
        const int v = cbj[lo + e];
        int dl = 0;
        for (int f = 0; f < L; ++f) dl += (pair_first[lo + f].x >= 0 && cbj[lo + f] < v);
        pair_local[lo + e] = dl;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) firsts += __shfl_xor_sync(0xffffffffu, firsts, o);
    if (lane == 0) body_npairs[w] = firsts;
    if (w == 0 && lane == 0) body_npairs[nbodies] = 0;
}

__global__ void k_pairs_write(const b2c_header *__restrict__ hdr_c, int nbodies, const int *__restrict__ cbi,
                              const int *__restrict__ cbj, const int *__restrict__ pair_local,
                              const int2 *__restrict__ pair_first, const int *__restrict__ pair_base, int pcap,
                              int *__restrict__ pbi, int *__restrict__ pbj, int *__restrict__ praw_start,
                              int *__restrict__ praw_count, b2c_header *hdr)
{
    const int C = hdr_c->n_contacts;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        const int P = pair_base[nbodies];
        hdr->n_pairs = P < pcap ? P : pcap;
        if (P > pcap) atomicOr(&hdr->error, B2C_ERR_PAIR_OVERFLOW);
    }
    for (int e = tid; e < C; e += gridDim.x * blockDim.x) {
        const int2 pf = pair_first[e];
        if (pf.x < 0) continue;
        const int A = cbi[e];
        const int p = pair_base[A] + pair_local[e];
        if (p >= pcap) continue;
        pbi[p] = A;
        pbj[p] = cbj[e];
        praw_start[p] = pf.x;
        praw_count[p] = pf.y;
    }
}

// ---------------------------------------------------------------------------------------------
// 3. warm start, selection, compaction, kept pairs (COL:601-626, 651-751, 1158-1176)
// ---------------------------------------------------------------------------------------------
__global__ void k_warm(const b2c_header *__restrict__ hdr, const int *__restrict__ fa, const int *__restrict__ fb,
                       long long stride, int use_warm, const long long *__restrict__ wkeys,
                       const float *__restrict__ wimp, const int *__restrict__ wn_ptr, double *__restrict__ jn_in,
                       float2 *__restrict__ jt_in)
{
    const int C = hdr->n_contacts;
    const int wn = use_warm ? *wn_ptr : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        double jn = 0.0;
        float2 jt = make_float2(0.0f, 0.0f);
        if (wn > 0) {
            const long long k = (long long)fa[i] * stride + (long long)fb[i] + 1;
            int lo = 0, hi = wn - 1, hit = -1;
            while (lo <= hi) {
                const int mid = (lo + hi) / 2;
                const long long km = wkeys[mid];
                if (km == k) {
                    hit = mid;
                    lo = hi + 1;
                } else if (km < k) {
                    lo = mid + 1;
                } else {
                    hi = mid - 1;
                }
            }
            if (hit >= 0) {
                const float4 w4 = ld4(wimp, hit);
                jn = (double)w4.x;
                jt = make_float2(w4.y, w4.z);
            }
        }
        jn_in[i] = jn;
        jt_in[i] = jt;
    }
}

// _planar, COL:585-590: float32 difference promoted to float64
__device__ __forceinline__ void planar(const float *__restrict__ cpA, int g, f3 ref, const double *u, const double *w,
                                       double *r)
{
    const float4 p = ld4(cpA, g);
    const float dx = p.x - ref.x, dy = p.y - ref.y, dz = p.z - ref.z;
    const double ax = dx, ay = dy, az = dz;
    r[0] = (ax * u[0] + ay * u[1]) + az * u[2];
    r[1] = (ax * w[0] + ay * w[1]) + az * w[2];
}

// k_select, COL:651-728: one thread per body pair
__global__ void k_select(const b2c_header *__restrict__ hdr, int mx, const int *__restrict__ praw_start,
                         const int *__restrict__ praw_count, const int *__restrict__ gorder,
                         const int *__restrict__ cbi, const float *__restrict__ cpA, const float *__restrict__ cn,
                         const float *__restrict__ xc, const double *__restrict__ jn_in, int *__restrict__ keep,
                         double *__restrict__ jn_out, int *__restrict__ kcount, b2c_header *hdr_w)
{
    const int P = hdr->n_pairs;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int i = praw_start[p], L = praw_count[p];
        if (L <= mx || L > 1024 || mx > 8) {
            if (L > mx) atomicOr(&hdr_w->error, B2C_ERR_SEGMENT_OVERFLOW);
            for (int t = 0; t < L; ++t) {
                const int g = gorder[i + t];
                keep[g] = 1;
                jn_out[g] = jn_in[g];
            }
            kcount[p] = L;
            continue;
        }
        int deep = 0;
        float dbest = cpA[4 * gorder[i] + 3];
        for (int t = 1; t < L; ++t) {
            const float pn = cpA[4 * gorder[i + t] + 3];
            if (pn > dbest) {
                dbest = pn;
                deep = t;
            }
        }
        const int gd = gorder[i + deep];
        const f3 nr = ld3(cn, gd);
        double ax = 1.0, ay = 0.0, az = 0.0;
        if (fabsf(nr.x) >= 0.9f) {
            ax = 0.0;
            ay = 1.0;
            az = 0.0;
        }
        const double n0 = nr.x, n1 = nr.y, n2 = nr.z;
        const double dn = (ax * n0 + ay * n1) + az * n2;
        const double u0 = ax - dn * n0, u1 = ay - dn * n1, u2 = az - dn * n2;
        const double ln = sqrt((u0 * u0 + u1 * u1) + u2 * u2);
        const double u[3] = {u0 / ln, u1 / ln, u2 / ln};
        const double w[3] = {n1 * u[2] - n2 * u[1], n2 * u[0] - n0 * u[2], n0 * u[1] - n1 * u[0]};
        const f3 ref = ld3(xc, cbi[gd]);
        double rd[2];
        planar(cpA, gd, ref, u, w, rd);
        double S00 = rd[0] * rd[0], S01 = rd[0] * rd[1], S10 = rd[1] * rd[0], S11 = rd[1] * rd[1];
        int pick[8];
        pick[0] = deep;
        for (int k = 1; k < mx; ++k) {
            double sbest = -1.0e300;
            int tbest = -1;
            double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
            for (int t = 0; t < L; ++t) {
                bool taken = false;
                for (int q = 0; q < k; ++q) taken |= (pick[q] == t);
                if (taken) continue;
                double rt[2];
                planar(cpA, gorder[i + t], ref, u, w, rt);
                const double a00 = S00 + rt[0] * rt[0], a01 = S01 + rt[0] * rt[1];
                const double a10 = S10 + rt[1] * rt[0], a11 = S11 + rt[1] * rt[1];
                const double tr = a00 + a11;
                const double det = a00 * a11 - a01 * a10;
                const double disc = fmax(tr * tr / 4.0 - det, 0.0);
                const double lam = tr / 2.0 - sqrt(disc);
                const double sc = fmin((double)(k + 1), lam);
                if (sc > sbest) {
                    sbest = sc;
                    tbest = t;
                    c00 = a00;
                    c01 = a01;
                    c10 = a10;
                    c11 = a11;
                }
            }
            if (tbest < 0) {  // only with non-finite scores: take the first free point, never index -1
                for (int t = L - 1; t >= 0; --t) {
                    bool taken = false;
                    for (int q = 0; q < k; ++q) taken |= (pick[q] == t);
                    if (!taken) tbest = t;
                }
            }
            pick[k] = tbest;
            S00 = c00;
            S01 = c01;
            S10 = c10;
            S11 = c11;
        }
        for (int t = 0; t < L; ++t) keep[gorder[i + t]] = 0;
        for (int k = 0; k < mx; ++k) {
            const int g = gorder[i + pick[k]];
            keep[g] = 1;
            jn_out[g] = 0.0;
        }
        for (int t = 0; t < L; ++t) {
            double rt[2];
            planar(cpA, gorder[i + t], ref, u, w, rt);
            double dbest2 = 1.0e300;
            int kbest = 0;
            for (int k = 0; k < mx; ++k) {
                double rk[2];
                planar(cpA, gorder[i + pick[k]], ref, u, w, rk);
                const double e0 = rt[0] - rk[0], e1 = rt[1] - rk[1], d2 = e0 * e0 + e1 * e1;
                if (d2 < dbest2) {
                    dbest2 = d2;
                    kbest = k;
                }
            }
            const int gk = gorder[i + pick[kbest]];
            jn_out[gk] = jn_out[gk] + jn_in[gorder[i + t]];
        }
        kcount[p] = mx;
    }
}

__global__ void k_set_kept(b2c_header *hdr, const int *__restrict__ kidx) { hdr->n_kept = kidx[hdr->n_contacts]; }

// The reduced set coloured contact by contact (COL:1105-1113 with the device manifold's priority,
// k_prio_manifold, COL:776-787): every kept contact is a chunk of one, and runs of consecutive
// kept contacts (feature order) of the same body pair are flagged for the priority.
__global__ void k_kept_chunks(b2c_header *hdr, int cap, int pcap, b2c_contacts kept, int *__restrict__ pbi,
                              int *__restrict__ pbj, int *__restrict__ kcount, int *__restrict__ pstart,
                              int *__restrict__ pidx, int *__restrict__ runflag)
{
    const int Ck = hdr->n_kept;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        hdr->n_pairs = Ck < pcap ? Ck : pcap;
        if (Ck > pcap) atomicOr(&hdr->error, B2C_ERR_PAIR_OVERFLOW);
    }
    for (int i = tid; i <= cap; i += gridDim.x * blockDim.x) {
        if (i >= Ck || i >= pcap) {
            runflag[i] = 0;
            continue;
        }
        const int a = kept.bi[i], b = kept.bj[i];
        pbi[i] = a;
        pbj[i] = b;
        kcount[i] = 1;
        pstart[i] = i;
        pidx[i] = i;
        runflag[i] = (i == 0 || a != kept.bi[i - 1] || b != kept.bj[i - 1]) ? 1 : 0;
    }
}

// first kept contact of each run (runs counted by the exclusive scan of the flags)
__global__ void k_kept_runstart(const b2c_header *__restrict__ hdr, int pcap, const int *__restrict__ runflag,
                                const int *__restrict__ runscan, int *__restrict__ runstart)
{
    const int Ck = min(hdr->n_kept, pcap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Ck; i += gridDim.x * blockDim.x)
        if (runflag[i]) runstart[runscan[i]] = i;
}

// priority high part: the slot inside the run (at most 255), then the run's parity; the pair
// index (= the kept rank) follows in claim_key, so the order is k_prio_manifold's
__global__ void k_kept_prio(const b2c_header *__restrict__ hdr, int pcap, const int *__restrict__ runflag,
                            const int *__restrict__ runscan, const int *__restrict__ runstart, int *__restrict__ prio_hi)
{
    const int Ck = min(hdr->n_kept, pcap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Ck; i += gridDim.x * blockDim.x) {
        const int g = runscan[i] + runflag[i] - 1;
        const int slot = min(i - runstart[g], 255);
        prio_hi[i] = (slot << 19) | ((g & 1) << 18);
    }
}

// plain coloured engine (COL:903-936, 1105-1137): every contact kept, one contact per chunk,
// warm impulses uploaded as float32 (COL:931-936)
__global__ void k_per_contact(b2c_header *hdr, long long stride, b2c_contacts c, const double *__restrict__ jn_in,
                              const float2 *__restrict__ jt_in, b2c_contacts kept, long long *__restrict__ kept_keys,
                              int pcap, int *__restrict__ pbi, int *__restrict__ pbj, int *__restrict__ kcount,
                              int *__restrict__ pstart, int *__restrict__ pidx)
{
    const int C = hdr->n_contacts;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        hdr->n_kept = C;
        hdr->n_pairs = C < pcap ? C : pcap;
        if (C > pcap) atomicOr(&hdr->error, B2C_ERR_PAIR_OVERFLOW);
    }
    for (int i = tid; i < C && i < pcap; i += gridDim.x * blockDim.x) {
        kept_keys[i] = (long long)c.fa[i] * stride + (long long)c.fb[i] + 1;
        kept.bi[i] = c.bi[i];
        kept.bj[i] = c.bj[i];
        st4(kept.pA, i, ld4(c.pA, i));
        st4(kept.pB, i, ld4(c.pB, i));
        st4(kept.n, i, ld4(c.n, i));
        kept.fa[i] = c.fa[i];
        kept.fb[i] = c.fb[i];
        const float2 jt = jt_in[i];
        st4(kept.imp, i, make_float4((float)jn_in[i], jt.x, jt.y, 0.0f));
        pbi[i] = c.bi[i];
        pbj[i] = c.bj[i];
        kcount[i] = 1;
        pstart[i] = i;
        pidx[i] = i;
    }
}

// k_compact, COL:730-751: kept contacts in feature order, jn cast to float32
__global__ void k_compact(const b2c_header *__restrict__ hdr, long long stride, b2c_contacts c,
                          const int *__restrict__ keep, const int *__restrict__ kidx, const double *__restrict__ jn_red,
                          const float2 *__restrict__ jt_in, b2c_contacts kept, long long *__restrict__ kept_keys)
{
    const int C = hdr->n_contacts;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        if (!keep[i]) continue;
        const int d = kidx[i];
        kept_keys[d] = (long long)c.fa[i] * stride + (long long)c.fb[i] + 1;
        kept.bi[d] = c.bi[i];
        kept.bj[d] = c.bj[i];
        st4(kept.pA, d, ld4(c.pA, i));
        st4(kept.pB, d, ld4(c.pB, i));
        st4(kept.n, d, ld4(c.n, i));
        kept.fa[d] = c.fa[i];
        kept.fb[d] = c.fb[i];
        const float2 jt = jt_in[i];
        st4(kept.imp, d, make_float4((float)jn_red[i], jt.x, jt.y, 0.0f));
    }
}

// pair-sorted kept list (k_pairkey + radix sort + k_pairbuild, COL:341-389, 1158-1176)
__global__ void k_pair_kept(const b2c_header *__restrict__ hdr, const int *__restrict__ praw_start,
                            const int *__restrict__ praw_count, const int *__restrict__ gorder,
                            const int *__restrict__ keep, const int *__restrict__ kidx, const int *__restrict__ pstart,
                            int *__restrict__ pidx, int *__restrict__ kcount, b2c_header *hdr_w)
{
    const int P = hdr->n_pairs;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int i = praw_start[p], L = praw_count[p], base = pstart[p];
        int r = 0;
        for (int t = 0; t < L; ++t) {
            const int e = gorder[i + t];
            if (keep[e]) pidx[base + r++] = kidx[e];
        }
        if (r > 8) {  // _MAXCHUNK, COL:384-386
            atomicOr(&hdr_w->error, B2C_ERR_CHUNK_OVERFLOW);
            kcount[p] = 8;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// 4. colouring behind the colour cache (COL:136-185, 1178-1208; color_cache.py:5-54), one CTA
// ---------------------------------------------------------------------------------------------
// Warp's rand_init / randi: the PCG-RXS-M-XS 32-bit output permutation used as a hash
// (Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020).
__device__ __forceinline__ uint32_t pcg_hash(uint32_t state)
{
    const uint32_t b = state * 747796405u + 2891336453u;
    const uint32_t c = ((b >> ((b >> 28u) + 4u)) ^ b) * 277803737u;
    return (c >> 22u) ^ c;
}

constexpr int kColorThreads = 1024;
constexpr int kMaxColorsCap = 512;
constexpr int kColorSub = 16;  // buckets inside a colour: 8 contact counts (descending) x ground / box pair
constexpr int kColorClusterMax = 16;
constexpr int kPrioPairBits = 22;  // pair index bits of the compact priority (capacity <= 4M pairs)
constexpr int kJPRegPairs = 4;     // pairs per colouring thread whose round state lives in registers

// Round-tagged claim of pair p in round r: a larger key wins atomicMax.  The priority of a pair
// is k_prio's (COL:136-148) |int32(randi(rand_init(7919, p)))| << 32 | p, the smaller first; it is
// packed here as |h| << 22 | p (the same order while p < 2^22).  The round tag makes the claims
// of earlier rounds lose without clearing them; inside a round the smaller priority gives the
// larger key.
__device__ __forceinline__ unsigned long long claim_key(int p, int r, unsigned long long h)
{
    const unsigned long long prio = (h << kPrioPairBits) | (unsigned long long)p;  // < 2^54
    return ((unsigned long long)(r + 1) << 54) | ((1ull << 54) - 1ull - prio);
}
// The hash part of a pair's priority (<= 2^31).  Without body_local: k_prio's hash of the pair
// index.  With body_local (the box engine): a hash of the pair's two scene-local body indices,
// so the colouring of a scene does not depend on where its pairs sit in a batch of scenes (ties
// fall back to the pair index, whose order inside a scene is the same either way).
__device__ __forceinline__ unsigned long long pair_hash(int p, int a, int b, const int *__restrict__ body_local,
                                                        const int *__restrict__ prio_hi)
{
    if (prio_hi) return (unsigned long long)(unsigned)prio_hi[p];  // B2C_COLOR_REDUCED_CONTACTS
    if (body_local) {
        const unsigned long long key = ((unsigned long long)(unsigned)(body_local[a] + 1) << 32) |
                                       (unsigned long long)(unsigned)(b >= 0 ? body_local[b] + 1 : 0);
        unsigned long long z = key;
        z ^= z >> 30;
        z *= 0xbf58476d1ce4e5b9ULL;
        z ^= z >> 27;
        z *= 0x94d049bb133111ebULL;
        z ^= z >> 31;
        return z >> 33;
    }
    const uint32_t st = pcg_hash(pcg_hash(7919u + pcg_hash((uint32_t)p)));
    long long h = (long long)(int32_t)st;
    if (h < 0) h = -h;  // <= 2^31: 32 bits
    return (unsigned long long)h;
}

// One pair's part in the Jones-Plassmann rounds: the bodies it claims (the dynamic ones; -1
// for a static or absent body), its colour (-1 while uncoloured) and the low 54 bits of its
// claim key, which carry the priority (the round tag sits above them).
struct JPPair {
    int bi, bj, col;
    unsigned long long low;
};
__device__ __forceinline__ JPPair jp_pair(int p, const b2c_pairs &pr, const float *__restrict__ invM)
{
    const int a = pr.pbi[p], b = pr.pbj[p];
    const unsigned long long h = pair_hash(p, a, b, pr.body_local, pr.prio_hi);
    JPPair q;
    q.bi = invM[a] > 0.0f ? a : -1;
    q.bj = (b >= 0 && invM[b] > 0.0f) ? b : -1;
    q.col = -1;
    q.low = claim_key(p, -1, h);  // round tag 0: the low bits alone
    return q;
}
__device__ __forceinline__ unsigned long long jp_key(const JPPair &q, int r)
{
    return ((unsigned long long)(r + 1) << 54) | q.low;
}
__device__ __forceinline__ void jp_claim(const JPPair &q, int r, unsigned long long *claim)
{
    const unsigned long long k = jp_key(q, r);
    if (q.bi >= 0) atomicMax(claim + q.bi, k);
    if (q.bj >= 0) atomicMax(claim + q.bj, k);
}
// Pair q's turn in round r: it wins if it holds every claim it made in `cur`, and then takes
// the round number or, with first_fit, the smallest colour not used around its bodies (the
// masks are read together with the claims: the winners of a round share no dynamic body, so a
// winner's masks hold exactly the colours of the earlier rounds).  A pair that loses claims
// its bodies for round r + 1 in `nxt`.  Returns 1 while the pair is uncoloured; `ncol` keeps
// the thread's colour count.
__device__ __forceinline__ int jp_turn(JPPair &q, int p, int r, const unsigned long long *cur,
                                       unsigned long long *nxt, unsigned long long *used, int first_fit,
                                       int *__restrict__ col, int &ncol)
{
    if (q.col >= 0) return 0;
    const unsigned long long k = jp_key(q, r);
    unsigned long long ca = k, cb = k, ua = 0ull, ub = 0ull;
    if (q.bi >= 0) {
        ca = __ldcg(cur + q.bi);
        if (first_fit) ua = __ldcg(used + q.bi);
    }
    if (q.bj >= 0) {
        cb = __ldcg(cur + q.bj);
        if (first_fit) ub = __ldcg(used + q.bj);
    }
    if (ca != k || cb != k) {
        jp_claim(q, r + 1, nxt);
        return 1;
    }
    int c = r;
    if (first_fit) {
        const unsigned long long m = ua | ub;
        c = (~m == 0ull) ? 64 : __ffsll((long long)~m) - 1;
        if (c < 64) {
            if (q.bi >= 0) __stcg(used + q.bi, ua | (1ull << c));
            if (q.bj >= 0) __stcg(used + q.bj, ub | (1ull << c));
        }
        ncol = max(ncol, c + 1);
    }
    q.col = c;
    col[p] = c;
    return 0;
}

// exclusive scan of a[0, E) in shared memory by the whole CTA (E <= 8 x blockDim.x); ends with a
// __syncthreads
__device__ void block_exclusive_scan(int *a, int E)
{
    __shared__ int s_w[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int per = (E + (int)blockDim.x - 1) / (int)blockDim.x, b0 = (int)threadIdx.x * per;
    int sum = 0;
    for (int i = 0; i < per; ++i)
        if (b0 + i < E) sum += a[b0 + i];
    int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? s_w[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        s_w[lane] = w;
    }
    __syncthreads();
    int base = x - sum + (warp > 0 ? s_w[warp - 1] : 0);
    for (int i = 0; i < per; ++i)
        if (b0 + i < E) {
            const int v = a[b0 + i];
            a[b0 + i] = base;
            base += v;
        }
    __syncthreads();
}
__device__ __forceinline__ int color_bucket(const b2c_pairs &pr, int p)
{
    const int n = min(max(pr.kcount[p], 1), 8);
    return pr.col[p] * kColorSub + (8 - n) * 2 + (pr.pbj[p] >= 0 ? 1 : 0);
}
constexpr int kColorDynSmem = 2 * kMaxColorsCap * kColorSub * (int)sizeof(int);  // counts + cursors

// Jones-Plassmann colouring of the pair graph behind the colour cache, on one thread-block
// cluster (CTAs synchronised by cluster barriers, sums and histograms in distributed shared
// memory).  Every round: each uncoloured pair claims its dynamic bodies (atomicMax of the
// round-tagged key); a pair that holds all its claims takes the round number as its colour
// (k_win, COL:163-181) or, with first_fit, the smallest colour not used around its bodies.  The
// pairs are then grouped by colour, inside a colour by contact count (descending) and ground
// pairs first, so the lanes of a warp of the solve run similar code.
//
// A round costs one cluster barrier.  The claims alternate between two body arrays (pr.claim
// holds 2 x bodies): the pairs that lose round r claim for round r + 1 in the other array in the
// same pass, and a round's winners are decided only after the barrier that follows every claim
// of that round.  Each thread's pairs are fixed (p = thread + k x threads), and their static
// part (claimed bodies, priority) is computed once: in registers for the first kJPRegPairs of
// them, and in the record buffer's header words beyond that (scratch until the solve's gather
// rewrites them).  The winners and colours of every round are those of the two-barrier form.
__global__ void __launch_bounds__(kColorThreads) k_color_pairs(b2c_header *hdr, int nbodies,
                                                                const float *__restrict__ invM, b2c_pairs pr,
                                                                int use_cache, int color_cap, int max_rounds,
                                                                int first_fit)
{
    namespace cgc = cooperative_groups;
    cgc::cluster_group cluster = cgc::this_cluster();
    __shared__ int s_flag;
    __shared__ int s_left[3];
    __shared__ int s_total[2];
    __shared__ int s_ncol;
    extern __shared__ int s_dyn[];  // this CTA's bucket counts, then its cursors
    const int rank = (int)cluster.block_rank(), nrank = (int)cluster.num_blocks();
    const int tid = rank * kColorThreads + threadIdx.x, nth = nrank * kColorThreads;
    const int P = hdr->n_pairs;
    if (P == 0) {
        if (tid == 0) {
            hdr->n_colors = 0;
            hdr->cache_hit = 0;
        }
        return;
    }
    // colour cache: reuse while the pair count, pbi, pbj and invM are unchanged
    if (use_cache && pr.cache_state[2] == 1 && pr.cache_state[0] == P) {
        if (threadIdx.x == 0) s_flag = 0;
        __syncthreads();
        int mism = 0;
        for (int p = tid; p < P; p += nth) mism |= (pr.pbi[p] != pr.cached_a[p]) | (pr.pbj[p] != pr.cached_b[p]);
        for (int i = tid; i < nbodies; i += nth) mism |= (invM[i] != pr.cached_mass[i]);
        if (mism) atomicOr(&s_flag, 1);
        cluster.sync();
        int any = 0;
        for (int r = 0; r < nrank; ++r) any |= *cluster.map_shared_rank(&s_flag, r);
        cluster.sync();  // no CTA leaves while another still reads its shared memory
        if (!any) {
            if (tid == 0) {
                hdr->n_colors = pr.cache_state[1];
                pr.cache_state[3] += 1;
                hdr->cache_hit = 1;
            }
            return;
        }
    }
    unsigned long long *claim0 = reinterpret_cast<unsigned long long *>(pr.claim);
    unsigned long long *claim1 = claim0 + nbodies;
    unsigned long long *used = reinterpret_cast<unsigned long long *>(pr.body_colors);
    int4 *pstate = reinterpret_cast<int4 *>(pr.rec);
    JPPair rq[kJPRegPairs];
#pragma unroll
    for (int k = 0; k < kJPRegPairs; ++k) {
        const int p = tid + k * nth;
        if (p < P) rq[k] = jp_pair(p, pr, invM);
    }
    for (int p = tid + kJPRegPairs * nth; p < P; p += nth) {
        const JPPair q = jp_pair(p, pr, invM);
        pstate[p] = make_int4(q.bi, q.bj, (int)(unsigned)q.low, (int)(unsigned)(q.low >> 32));
    }
    for (int p = tid; p < P; p += nth) pr.col[p] = -1;
    for (int i = tid; i < nbodies; i += nth) {
        claim0[i] = 0ull;
        claim1[i] = 0ull;
        if (first_fit) used[i] = 0ull;
    }
    if (threadIdx.x == 0) {
        s_ncol = 0;
        s_left[0] = 0;
    }
    cluster.sync();
    // the claims of round 0
#pragma unroll
    for (int k = 0; k < kJPRegPairs; ++k)
        if (tid + k * nth < P) jp_claim(rq[k], 0, claim0);
    for (int p = tid + kJPRegPairs * nth; p < P; p += nth) {
        const int4 st = pstate[p];
        jp_claim(JPPair{st.x, st.y, -1, (unsigned long long)(unsigned)st.z | ((unsigned long long)(unsigned)st.w << 32)},
                 0, claim0);
    }
    cluster.sync();
    int r = 0, my_ncol = 0;
    bool done = false;
    for (; r < max_rounds; ++r) {
        const unsigned long long *cur = (r & 1) ? claim1 : claim0;
        unsigned long long *nxt = (r & 1) ? claim0 : claim1;
        // s_left[r % 3] counts this round; the next round's counter is cleared here (every CTA
        // read it two barriers ago)
        if (threadIdx.x == 0) s_left[(r + 1) % 3] = 0;
        int left = 0;
#pragma unroll
        for (int k = 0; k < kJPRegPairs; ++k) {
            const int p = tid + k * nth;
            if (p < P) left += jp_turn(rq[k], p, r, cur, nxt, used, first_fit, pr.col, my_ncol);
        }
        for (int p = tid + kJPRegPairs * nth; p < P; p += nth) {
            if (pr.col[p] >= 0) continue;
            const int4 st = pstate[p];
            JPPair q{st.x, st.y, -1, (unsigned long long)(unsigned)st.z | ((unsigned long long)(unsigned)st.w << 32)};
            left += jp_turn(q, p, r, cur, nxt, used, first_fit, pr.col, my_ncol);
        }
        // one shared-memory atomic per warp for the count and the colour number
        left = __reduce_add_sync(0xffffffffu, left);
        const int wcol = __reduce_max_sync(0xffffffffu, my_ncol);
        if ((threadIdx.x & 31) == 0) {
            if (left) atomicAdd(&s_left[r % 3], left);
            if (wcol > 0) atomicMax(&s_ncol, wcol);
        }
        cluster.sync();
        // the cluster-wide count: one warp reads the CTAs' counters and shares the sum
        if (threadIdx.x < 32) {
            int v = (int)threadIdx.x < nrank ? *cluster.map_shared_rank(&s_left[r % 3], (int)threadIdx.x) : 0;
            v = __reduce_add_sync(0xffffffffu, v);
            if (threadIdx.x == 0) s_total[r & 1] = v;
        }
        __syncthreads();
        if (s_total[r & 1] == 0) {
            done = true;
            break;
        }
    }
    int ncol = done ? r + 1 : r;
    if (first_fit) {
        ncol = 0;
        for (int q = 0; q < nrank; ++q) ncol = max(ncol, *cluster.map_shared_rank(&s_ncol, q));
    }
    cluster.sync();  // every CTA has read the others' s_left and s_ncol
    if (!done || ncol > color_cap || ncol > pr.max_colors || ncol > kMaxColorsCap) {
        if (tid == 0) {
            atomicOr(&hdr->error, done ? B2C_ERR_COLOR_OVERFLOW : B2C_ERR_COLOR_TIMEOUT);
            hdr->n_colors = 0;
            hdr->cache_hit = 0;
            hdr->rounds = r;
            pr.cache_state[2] = 0;
        }
        return;
    }
    // group by (colour, bucket).  Each CTA counts its own pairs in its shared memory; the bucket
    // starts are a scan of the cluster-wide totals, and a CTA's cursors start after the pairs of
    // the same bucket held by the lower ranks.  (The order inside a bucket is free: the pairs of
    // a colour share no dynamic body.)
    const int E = ncol * kColorSub;
    int *s_hist = s_dyn, *s_cur = s_dyn + kMaxColorsCap * kColorSub;
    for (int k = threadIdx.x; k < E; k += kColorThreads) s_hist[k] = 0;
    __syncthreads();
    for (int p = tid; p < P; p += nth) atomicAdd(&s_hist[color_bucket(pr, p)], 1);
    cluster.sync();
    for (int k = threadIdx.x; k < E; k += kColorThreads) {
        int t = 0;
        for (int q = 0; q < nrank; ++q) t += cluster.map_shared_rank(s_hist, q)[k];
        s_cur[k] = t;
    }
    __syncthreads();
    block_exclusive_scan(s_cur, E);
    if (rank == 0)
        for (int c = threadIdx.x; c < ncol; c += kColorThreads) {
            const int st = s_cur[c * kColorSub];
            pr.cstart[c] = st;
            pr.ccount[c] = (c + 1 < ncol ? s_cur[(c + 1) * kColorSub] : P) - st;
        }
    __syncthreads();
    for (int k = threadIdx.x; k < E; k += kColorThreads) {
        int t = 0;
        for (int q = 0; q < rank; ++q) t += cluster.map_shared_rank(s_hist, q)[k];
        s_cur[k] += t;
    }
    __syncthreads();
    for (int p = tid; p < P; p += nth) pr.porder[atomicAdd(&s_cur[color_bucket(pr, p)], 1)] = p;
    if (use_cache) {
        for (int p = tid; p < P; p += nth) {
            pr.cached_a[p] = pr.pbi[p];
            pr.cached_b[p] = pr.pbj[p];
        }
        for (int i = tid; i < nbodies; i += nth) pr.cached_mass[i] = invM[i];
    }
    if (tid == 0) {
        hdr->n_colors = ncol;
        hdr->cache_hit = 0;
        hdr->rounds = r + 1;
        pr.cache_state[0] = P;
        pr.cache_state[1] = ncol;
        pr.cache_state[2] = 1;
        if (use_cache) pr.cache_state[4] += 1;  // cumulative misses ([3] counts hits)
    }
    cluster.sync();  // every CTA's counts stay alive until the others are done reading them
}

// largest power-of-two cluster (<= 16) of colouring CTAs the device co-schedules; cached
static int color_cluster_size()
{
    static int cached = -1;
    if (cached < 0) {
        cudaFuncSetAttribute(k_color_pairs, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        cudaFuncSetAttribute(k_color_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize, kColorDynSmem);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kColorClusterMax);
        cfg.blockDim = dim3(kColorThreads);
        cfg.dynamicSmemBytes = kColorDynSmem;
        int cs = 0;
        if (cudaOccupancyMaxPotentialClusterSize(&cs, k_color_pairs, &cfg) != cudaSuccess) {
            cudaGetLastError();
            cs = 1;
        }
        int p2 = 1;
        for (int c = 1; c <= std::min(cs, kColorClusterMax); c *= 2) p2 = c;
        cached = p2;
    }
    return cached;
}

int color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                float dt, cudaStream_t s);

// ---------------------------------------------------------------------------------------------
// 6. warm store (COL:1089-1093)
// ---------------------------------------------------------------------------------------------
__global__ void k_warm_store(const b2c_header *__restrict__ hdr, const long long *__restrict__ kept_keys,
                             const float *__restrict__ imp, int use_warm, long long *__restrict__ wkeys,
                             float *__restrict__ wimp, int *__restrict__ wn)
{
    const int Ck = hdr->n_contacts > 0 ? hdr->n_kept : 0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) *wn = use_warm ? Ck : 0;
    if (!use_warm) return;
    for (int d = tid; d < Ck; d += gridDim.x * blockDim.x) {
        wkeys[d] = kept_keys[d];
        const float4 v = ld4(imp, d);
        st4(wimp, d, make_float4(v.x, v.y, v.z, 0.0f));
    }
}

// ---------------------------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------------------------
int bead_contacts_sorted(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c, b2c_manifold *m,
                         b2c_header *hdr, cudaStream_t s)
{
    const int nb = beads->n;
    const float4 *spos = reinterpret_cast<const float4 *>(g->sorted_pos);
    k_bead_count<<<blocks_for(nb + 1, 128), 128, 0, s>>>(nb, beads->world, beads->owner, g->start, g->sorted, spos,
                                                         view_of(g), m->bead_count, hdr);
    int rc = check_launch("bead_count");
    if (rc) return rc;
    rc = exclusive_scan(m->bead_count, m->bead_offset, nb + 1, nullptr, m->scan_tmp, s);
    if (rc) return rc;
    k_bead_emit<<<blocks_for(nb + 1, 128), 128, 0, s>>>(nb, beads->world, beads->owner, g->start, g->sorted, spos,
                                                        view_of(g), m->bead_offset, *c, hdr);
    return check_launch("bead_emit");
}

int manifold_reduce(const b2c_bodies *b, const b2c_beads *beads, const b2c_contacts *c, b2c_manifold *m,
                    b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr, const b2c_warm *warm, b2c_header *hdr,
                    const b2c_color_params *p, cudaStream_t s)
{
    const int N = b->n, cap = c->capacity, pcap = pr->capacity;
    const long long stride = (long long)beads->n + 1;
    const int cgrid = std::min(blocks_for(cap), kSMs * 8);
    const int pgrid = std::min(blocks_for(pcap), kSMs * 8);
    int rc;
    if (p->flags & B2C_COLOR_PER_CONTACT) {
        k_warm<<<cgrid, kThreads, 0, s>>>(hdr, c->fa, c->fb, stride, (p->flags & B2C_COLOR_WARM_START) ? 1 : 0,
                                          reinterpret_cast<const long long *>(warm->keys), warm->imp, warm->n,
                                          m->jn_in, reinterpret_cast<float2 *>(m->jt_in));
        k_per_contact<<<cgrid, kThreads, 0, s>>>(hdr, stride, *c, m->jn_in, reinterpret_cast<const float2 *>(m->jt_in),
                                                 *kept, reinterpret_cast<long long *>(kept_keys), pcap, pr->pbi,
                                                 pr->pbj, pr->kcount, pr->pstart, pr->pidx);
        return check_launch("per_contact");
    }
    k_body_pairs<<<blocks_for((long long)N * 32, 256), 256, 0, s>>>(
        N, beads->bead_start, m->bead_offset, cap, c->bj, m->pair_local, reinterpret_cast<int2 *>(m->pair_first),
        m->gorder, m->body_npairs);
    rc = check_launch("body_pairs");
    if (rc) return rc;
    if ((rc = exclusive_scan(m->body_npairs, m->pair_base, N + 1, nullptr, m->scan_tmp, s))) return rc;
    k_pairs_write<<<cgrid, kThreads, 0, s>>>(hdr, N, c->bi, c->bj, m->pair_local,
                                             reinterpret_cast<const int2 *>(m->pair_first), m->pair_base, pcap, pr->pbi,
                                             pr->pbj, m->praw_start, m->praw_count, hdr);
    k_warm<<<cgrid, kThreads, 0, s>>>(hdr, c->fa, c->fb, stride, (p->flags & B2C_COLOR_WARM_START) ? 1 : 0,
                                      reinterpret_cast<const long long *>(warm->keys), warm->imp, warm->n, m->jn_in,
                                      reinterpret_cast<float2 *>(m->jt_in));
    k_select<<<pgrid, 128, 0, s>>>(hdr, p->max_points, m->praw_start, m->praw_count, m->gorder, c->bi, c->pA, c->n,
                                   b->xc, m->jn_in, m->keep, m->jn_red, pr->kcount, hdr);
    if ((rc = check_launch("select"))) return rc;
    if ((rc = exclusive_scan(m->keep, m->kidx, cap + 1, &hdr->n_contacts, m->scan_tmp, s))) return rc;
    k_set_kept<<<1, 1, 0, s>>>(hdr, m->kidx);
    k_compact<<<cgrid, kThreads, 0, s>>>(hdr, stride, *c, m->keep, m->kidx, m->jn_red,
                                         reinterpret_cast<const float2 *>(m->jt_in), *kept,
                                         reinterpret_cast<long long *>(kept_keys));
    if (p->flags & B2C_COLOR_REDUCED_CONTACTS) {
        // every kept contact its own chunk; keep / kidx / gorder are free after the compaction
        if (!pr->prio_hi || pcap < cap) {
            set_error("manifold_reduce: B2C_COLOR_REDUCED_CONTACTS needs pairs->prio_hi and a pair capacity of "
                      "one per contact");
            return B2C_EARG;
        }
        k_kept_chunks<<<cgrid, kThreads, 0, s>>>(hdr, cap, pcap, *kept, pr->pbi, pr->pbj, pr->kcount, pr->pstart,
                                                 pr->pidx, m->keep);
        if ((rc = check_launch("kept_chunks"))) return rc;
        if ((rc = exclusive_scan(m->keep, m->kidx, cap + 1, nullptr, m->scan_tmp, s))) return rc;
        k_kept_runstart<<<cgrid, kThreads, 0, s>>>(hdr, pcap, m->keep, m->kidx, m->gorder);
        k_kept_prio<<<cgrid, kThreads, 0, s>>>(hdr, pcap, m->keep, m->kidx, m->gorder, pr->prio_hi);
        return check_launch("manifold_reduce");
    }
    if ((rc = exclusive_scan(pr->kcount, pr->pstart, pcap + 1, &hdr->n_pairs, m->scan_tmp, s))) return rc;
    k_pair_kept<<<pgrid, kThreads, 0, s>>>(hdr, m->praw_start, m->praw_count, m->gorder, m->keep, m->kidx,
                                           pr->pstart, pr->pidx, pr->kcount, hdr);
    return check_launch("manifold_reduce");
}

int color_pairs(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p, cudaStream_t s)
{
    const int cap = std::min(p->color_cap, std::min(pr->max_colors, kMaxColorsCap));
    const int first_fit = (p->flags & B2C_COLOR_FIRST_FIT) ? 1 : 0;
    if (first_fit && !pr->body_colors) {
        set_error("color_pairs: B2C_COLOR_FIRST_FIT needs pairs->body_colors");
        return B2C_EARG;
    }
    if (!pr->claim || !pr->rec || !pr->col || !pr->porder) {
        set_error("color_pairs: pairs->claim, rec, col and porder are required");
        return B2C_EARG;
    }
    if (pr->capacity > (1 << kPrioPairBits)) {
        set_error("color_pairs: pair capacity %d above %d", pr->capacity, 1 << kPrioPairBits);
        return B2C_EARG;
    }
    const int cs = color_cluster_size();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(kColorThreads);
    cfg.dynamicSmemBytes = kColorDynSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_color_pairs, hdr, b->n, (const float *)b->invM, *pr,
                                       (p->flags & B2C_COLOR_CACHE) ? 1 : 0, first_fit ? std::min(cap, 64) : cap,
                                       kMaxColorsCap + 1, first_fit);
    if (e != cudaSuccess) {
        set_error("color_pairs: cluster launch of %d CTAs: %s", cs, cudaGetErrorString(e));
        return B2C_ECUDA;
    }
    return check_launch("color_pairs");
}


int warm_store(const b2c_contacts *kept, const int64_t *kept_keys, b2c_warm *warm, const b2c_header *hdr, int use,
               cudaStream_t s)
{
    k_warm_store<<<std::min(blocks_for(kept->capacity), kSMs * 8), kThreads, 0, s>>>(
        hdr, reinterpret_cast<const long long *>(kept_keys), kept->imp, use, reinterpret_cast<long long *>(warm->keys),
        warm->imp, warm->n);
    return check_launch("warm_store");
}

}  // namespace b2c

// ---------------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------------
static bool color_params_ok(const b2c_color_params *p)
{
    return p && p->vit >= 0 && p->pit >= 0 && p->max_points >= 1 && p->max_points <= 8 && p->color_cap >= 1;
}

extern "C" int32_t b2c_bead_contacts_sorted(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c,
                                            b2c_manifold *m, b2c_header *hdr, b2c_stream s)
{
    if (!beads || !b2c::grid_valid(g) || !c || !m || !hdr || !m->bead_count || !m->bead_offset) {
        b2c::set_error("b2c_bead_contacts_sorted: bad argument");
        return B2C_EARG;
    }
    return b2c::bead_contacts_sorted(beads, g, c, m, hdr, b2c::stream_of(s));
}

extern "C" int32_t b2c_manifold_reduce(const b2c_bodies *b, const b2c_beads *beads, const b2c_contacts *c,
                                       b2c_manifold *m, b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr,
                                       const b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, b2c_stream s)
{
    if (!b || !beads || !beads->bead_start || !c || !m || !kept || !kept_keys || !pr || !warm || !hdr ||
        !color_params_ok(p) || kept->capacity < c->capacity) {
        b2c::set_error("b2c_manifold_reduce: bad argument");
        return B2C_EARG;
    }
    return b2c::manifold_reduce(b, beads, c, m, kept, kept_keys, pr, warm, hdr, p, b2c::stream_of(s));
}

extern "C" int32_t b2c_color_pairs(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                                   b2c_stream s)
{
    if (!b || !pr || !hdr || !color_params_ok(p) || pr->max_colors < 1) {
        b2c::set_error("b2c_color_pairs: bad argument");
        return B2C_EARG;
    }
    return b2c::color_pairs(b, pr, hdr, p, b2c::stream_of(s));
}

extern "C" int32_t b2c_color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr,
                                   const b2c_color_params *p, float dt, b2c_stream s)
{
    if (!b || !kept || !pr || !hdr || !color_params_ok(p) || !(dt > 0.0f) || !pr->barrier || !pr->rec || pr->kslots < 1) {
        b2c::set_error("b2c_color_solve: bad argument");
        return B2C_EARG;
    }
    return b2c::color_solve(b, kept, pr, hdr, p, dt, b2c::stream_of(s));
}

extern "C" int32_t b2c_warm_store(const b2c_contacts *kept, const int64_t *kept_keys, b2c_warm *warm,
                                  const b2c_header *hdr, b2c_stream s)
{
    if (!kept || !kept_keys || !warm || !hdr || warm->capacity < kept->capacity) {
        b2c::set_error("b2c_warm_store: bad argument");
        return B2C_EARG;
    }
    return b2c::warm_store(kept, kept_keys, warm, hdr, 1, b2c::stream_of(s));
}

extern "C" int32_t b2c_color_substep(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_contacts *c,
                                     b2c_manifold *m, b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr,
                                     b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, float dt,
                                     float *vgrav, b2c_stream s)
{
    if (!b || !beads || !beads->bead_start || !b2c::grid_valid(g) || !c || !m || !kept || !kept_keys || !pr ||
        !warm || !hdr ||
        !color_params_ok(p) || !vgrav || !(dt > 0.0f) || kept->capacity < c->capacity ||
        warm->capacity < kept->capacity || !pr->barrier || !pr->rec || pr->kslots < 1) {
        b2c::set_error("b2c_color_substep: bad argument");
        return B2C_EARG;
    }
    cudaStream_t st = b2c::stream_of(s);
    int rc;
    // predict, vgrav, and pv / po cleared for the substep (deferred_force.py:37-38, 54-55)
    if ((rc = b2c::body_predict_substep(b, dt, vgrav, true, st))) return rc;
    if ((rc = b2c::bead_world(b, beads, g, st))) return rc;
    if ((rc = b2c::grid_build(beads, g, st))) return rc;
    if ((rc = b2c::bead_contacts_sorted(beads, g, c, m, hdr, st))) return rc;
    if ((rc = b2c::manifold_reduce(b, beads, c, m, kept, kept_keys, pr, warm, hdr, p, st))) return rc;
    if ((rc = b2c::color_pairs(b, pr, hdr, p, st))) return rc;
    if ((rc = b2c::color_solve(b, kept, pr, hdr, p, dt, st))) return rc;
    if ((rc = b2c::warm_store(kept, kept_keys, warm, hdr, (p->flags & B2C_COLOR_WARM_START) ? 1 : 0, st))) return rc;
    return b2c::body_integrate(b, dt, st);
}
