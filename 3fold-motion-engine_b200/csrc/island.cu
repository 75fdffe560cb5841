// Island partition of the pair graph (contact_engine_gpu_island_solve.py:7-34, partition_pairs),
// on the device.
//
// Two bodies belong to one island when a chain of pairs joins them through dynamic bodies only
// (a pair couples its bodies when both have inverse mass > 0); static and kinematic bodies, and
// the ground, join nothing.  A pair belongs to the island of its first dynamic body; a pair
// without a dynamic body is an island of its own.  The islands' pairs are listed in the order of
// `order` (the colour-major record slots), so that one thread can run an island's sweeps colour
// by colour (solve.cu, k_island_solve).
//
// Steps, all on the device with no host read-back (a captured step replays them):
//  1. init: parent[b] = b, counters cleared;
//  2. union: every coupling pair hooks the larger of its two roots under the smaller with
//     atomicCAS (lock-free union-find with path halving).  Every hook points to a smaller index,
//     so the root of an island is its smallest body, whatever order the hooks ran in;
//  3. key: each slot's island key (the root of its first dynamic body, or bodies + pair for a pair
//     without one, the reference's len(mass) + p), and the pairs per key;
//  4. scan of the counts: each key's first position;
//  5. fill: each slot's position inside its key's range; the first slot of a key writes the
//     island's pair count at the island's first position (isl_at), and the island statistics;
//  6. order: each island's slots ascending (engine form: islands of <= B2C_ISLAND_MAX_PAIRS pairs,
//     the only ones the island solve runs, sorted by one thread; API form: a stable fill instead).
#include <algorithm>

#include "b2c_common.cuh"

namespace b2c {

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s);
int scan_scratch_ints(int n);

// The island workspace inside one int32 buffer (b2c_pairs.isl_work), each part on a 256-byte
// boundary.  K = bodies + pair capacity keys.
struct IslandWork {
    int *info;    // [0] islands, [1] most pairs of one island, [2] partitioned (1), [3] pairs,
                  // [4] this substep reuses the last partition (engine form)
    int *parent;  // (bodies) union-find forest
    int *count;   // (K) pairs per key
    int *start;   // (K) first position of each key (exclusive scan of count)
    int *fill;    // (K) slots placed per key
    int *key;     // (cap) island key of each slot
    int *slots;   // (cap) record slots grouped by island
    int *isl_at;  // (cap) pair count of the island that starts at a position, 0 elsewhere
    int *scan_tmp;
    int nb, cap, K;
};

static long long seg_ints(long long n) { return (n + 63) / 64 * 64; }

static long long island_work_layout(int nb, int cap, int *base, IslandWork *W)
{
    const long long K = (long long)nb + cap;
    long long o = 0;
    auto take = [&](long long n) -> int * {
        int *p = base ? base + o : nullptr;
        o += seg_ints(n > 0 ? n : 1);
        return p;
    };
    IslandWork w;
    w.info = take(8);
    w.parent = take(nb);
    w.count = take(K);
    w.start = take(K);
    w.fill = take(K);
    w.key = take(cap);
    w.slots = take(cap);
    w.isl_at = take(cap);
    w.scan_tmp = take(scan_scratch_ints((int)K) + 1);
    w.nb = nb;
    w.cap = cap;
    w.K = (int)K;
    if (W) *W = w;
    return o;
}

__device__ __forceinline__ int ld_parent(const int *parent, int x) { return *(volatile const int *)(parent + x); }

// root of x with path halving: x's parent becomes its grandparent on the way up.  Roots change
// only by the CAS in unite (at the root's own entry), and every entry points to a smaller index,
// so a grandparent read at any time is still an ancestor.
__device__ __forceinline__ int isl_find(int *parent, int x)
{
    int p = ld_parent(parent, x);
    while (p != x) {
        const int g = ld_parent(parent, p);
        if (g != p) *(volatile int *)(parent + x) = g;
        x = p;
        p = g;
    }
    return x;
}

__device__ __forceinline__ int pairs_of(const int *np_dev, int np_host, int cap)
{
    const int n = np_dev ? *np_dev : np_host;
    return n < 0 ? 0 : (n > cap ? cap : n);
}

// On a colour-cache hit the pairs, their bodies' masses and the colour order are those of the
// previous substep, and so is the partition: the engine form skips the steps then.  The decision
// is taken once per substep (k_isl_begin) and read by every later step of the partition.
__device__ __forceinline__ bool skip_partition(const b2c_header *hdr, const IslandWork &W)
{
    return hdr && W.info[4] == 1;
}

__global__ void k_isl_init(IslandWork W, const b2c_header *hdr)
{
    if (skip_partition(hdr, W)) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < W.K; i += stride) {
        W.count[i] = 0;
        W.fill[i] = 0;
        if (i < W.nb) W.parent[i] = (int)i;
        if (i < W.cap) W.isl_at[i] = 0;
    }
}

__global__ void k_isl_union(IslandWork W, const b2c_header *hdr, const int *np_dev, int np_host,
                            const int *__restrict__ pbi, const int *__restrict__ pbj, const float *__restrict__ invM)
{
    if (skip_partition(hdr, W)) return;
    const int P = pairs_of(np_dev, np_host, W.cap);
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const int a = pbi[p], b = pbj[p];
        if (b < 0 || !(invM[a] > 0.0f) || !(invM[b] > 0.0f)) continue;
        for (;;) {
            const int ra = isl_find(W.parent, a), rb = isl_find(W.parent, b);
            if (ra == rb) break;
            const int lo = ra < rb ? ra : rb, hi = ra < rb ? rb : ra;
            if (atomicCAS(&W.parent[hi], hi, lo) == hi) break;
        }
    }
}

__global__ void k_isl_key(IslandWork W, const b2c_header *hdr, const int *np_dev, int np_host,
                          const int *__restrict__ order, const int *__restrict__ pbi, const int *__restrict__ pbj,
                          const float *__restrict__ invM)
{
    if (skip_partition(hdr, W)) return;
    const int P = pairs_of(np_dev, np_host, W.cap);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P; s += gridDim.x * blockDim.x) {
        const int p = order ? order[s] : s;
        const int a = pbi[p], b = pbj[p];
        int k;
        if (invM[a] > 0.0f) k = isl_find(W.parent, a);
        else if (b >= 0 && invM[b] > 0.0f) k = isl_find(W.parent, b);
        else k = W.nb + p;
        W.key[s] = k;
        atomicAdd(&W.count[k], 1);
    }
}

__device__ __forceinline__ void note_island(IslandWork &W, int k)
{
    const int c = W.count[k];
    W.isl_at[W.start[k]] = c;
    atomicAdd(&W.info[0], 1);
    atomicMax(&W.info[1], c);
}

// engine form: positions inside a key's range in arrival order (ordered afterwards)
__global__ void k_isl_fill(IslandWork W, const b2c_header *hdr, const int *np_dev, int np_host)
{
    if (skip_partition(hdr, W)) return;
    const int P = pairs_of(np_dev, np_host, W.cap);
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < P; s += gridDim.x * blockDim.x) {
        const int k = W.key[s];
        const int r = atomicAdd(&W.fill[k], 1);
        W.slots[W.start[k] + r] = s;
        if (r == 0) note_island(W, k);
    }
}

// API form: one warp walks the slots in order, so each key's slots land in ascending order
// (__match_any_sync groups the lanes of one key; the lowest lane advances the key's count).
__global__ void k_isl_fill_stable(IslandWork W, const int *np_dev, int np_host)
{
    const int P = pairs_of(np_dev, np_host, W.cap);
    const int lane = threadIdx.x & 31;
    for (int base = 0; base < P; base += 32) {
        const int s = base + lane;
        const int k = s < P ? W.key[s] : -1;
        const unsigned m = __match_any_sync(0xffffffffu, k);
        const int rank = __popc(m & ((1u << lane) - 1u));
        const int filled = s < P ? W.fill[k] : 0;
        __syncwarp();
        if (s < P) {
            W.slots[W.start[k] + filled + rank] = s;
            if (filled + rank == 0) note_island(W, k);
            if (rank == 0) W.fill[k] = filled + __popc(m);
        }
        __syncwarp();
    }
}

// engine form: each island the island solve can run (<= B2C_ISLAND_MAX_PAIRS pairs) sorted by
// slot, i.e. colour-major; then the partition is marked done
__global__ void k_isl_order(IslandWork W, const b2c_header *hdr, const int *np_dev, int np_host)
{
    if (skip_partition(hdr, W)) return;
    const int P = pairs_of(np_dev, np_host, W.cap);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P; t += gridDim.x * blockDim.x) {
        const int c = W.isl_at[t];
        if (c < 2 || c > B2C_ISLAND_MAX_PAIRS) continue;
        int *v = W.slots + t;
        for (int i = 1; i < c; ++i) {
            const int x = v[i];
            int j = i - 1;
            while (j >= 0 && v[j] > x) {
                v[j + 1] = v[j];
                --j;
            }
            v[j + 1] = x;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        W.info[2] = 1;
        W.info[3] = P;
    }
}

// the steps shared by both forms; hdr non-null = engine form (header-counted pairs, skipped on a
// colour-cache hit)
static int island_partition_steps(IslandWork &W, const b2c_header *hdr, const int *np_dev, int np_host,
                                  const int *order, const int *pbi, const int *pbj, const float *invM, bool stable,
                                  cudaStream_t s)
{
    const int gk = std::min(blocks_for(W.K), kSMs * 8), gp = std::min(blocks_for(W.cap), kSMs * 8);
    k_isl_init<<<gk, kThreads, 0, s>>>(W, hdr);
    k_isl_union<<<gp, kThreads, 0, s>>>(W, hdr, np_dev, np_host, pbi, pbj, invM);
    k_isl_key<<<gp, kThreads, 0, s>>>(W, hdr, np_dev, np_host, order, pbi, pbj, invM);
    int rc = check_launch("island_init_union_key");
    if (rc) return rc;
    if ((rc = exclusive_scan(W.count, W.start, W.K, nullptr, W.scan_tmp, s))) return rc;
    if (stable) {
        k_isl_fill_stable<<<1, 32, 0, s>>>(W, np_dev, np_host);
        return check_launch("island_fill_stable");
    }
    k_isl_fill<<<gp, kThreads, 0, s>>>(W, hdr, np_dev, np_host);
    k_isl_order<<<gp, kThreads, 0, s>>>(W, hdr, np_dev, np_host);
    return check_launch("island_fill_order");
}

// engine form: decide whether this substep reuses the last partition; if not, restart the
// island statistics
__global__ void k_isl_begin(IslandWork W, const b2c_header *hdr)
{
    const int reuse = (hdr->cache_hit && W.info[2] == 1) ? 1 : 0;
    W.info[4] = reuse;
    if (!reuse) {
        W.info[0] = 0;
        W.info[1] = 0;
    }
}

// engine form, called by the solve (b2c_pairs.isl_work, B2C_COLOR_ISLANDS)
int island_partition_engine(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const int **info,
                            const int **slots, const int **isl_at, cudaStream_t s)
{
    IslandWork W;
    island_work_layout(b->n, pr->capacity, pr->isl_work, &W);
    k_isl_begin<<<1, 1, 0, s>>>(W, hdr);
    int rc = check_launch("island_begin");
    if (rc) return rc;
    if ((rc = island_partition_steps(W, hdr, &hdr->n_pairs, 0, pr->porder, pr->pbi, pr->pbj, b->invM, false, s)))
        return rc;
    *info = W.info;
    *slots = W.slots;
    *isl_at = W.isl_at;
    return B2C_OK;
}

// API form: the islands in key order, compacted
__global__ void k_isl_compact(IslandWork W, int P, const int *__restrict__ order, const int *__restrict__ flag_scan,
                              int *__restrict__ packed, int *__restrict__ starts, int *__restrict__ counts)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P; t += gridDim.x * blockDim.x) {
        const int sl = W.slots[t];
        packed[t] = order ? order[sl] : sl;
        const int c = W.isl_at[t];
        if (c > 0) {
            const int i = flag_scan[t];
            starts[i] = t;
            counts[i] = c;
        }
    }
}
__global__ void k_isl_flags(IslandWork W, int P, int *__restrict__ flag)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P; t += gridDim.x * blockDim.x)
        flag[t] = W.isl_at[t] > 0 ? 1 : 0;
}

}  // namespace b2c

extern "C" int64_t b2c_island_work_ints(int32_t n_bodies, int32_t pair_capacity)
{
    if (n_bodies < 0 || pair_capacity < 0) return -1;
    return b2c::island_work_layout(n_bodies, pair_capacity, nullptr, nullptr);
}

extern "C" int32_t b2c_island_partition(const int32_t *pbi, const int32_t *pbj, const float *inv_mass,
                                        const int32_t *order, int32_t n_pairs, int32_t n_bodies, int32_t *work,
                                        int32_t *packed, int32_t *starts, int32_t *counts, int32_t *info,
                                        b2c_stream st)
{
    using namespace b2c;
    const bool arrays = n_pairs == 0 || (pbi && pbj && packed && starts && counts);
    if (n_pairs < 0 || n_bodies < 0 || !arrays || !work || !info || (n_bodies > 0 && !inv_mass)) {
        set_error("b2c_island_partition: bad argument (n_pairs %d, n_bodies %d)", n_pairs, n_bodies);
        return B2C_EARG;
    }
    cudaStream_t s = stream_of(st);
    IslandWork W;
    island_work_layout(n_bodies, n_pairs, work, &W);
    cudaMemsetAsync(W.info, 0, 8 * sizeof(int), s);
    int rc = island_partition_steps(W, nullptr, nullptr, n_pairs, order, pbi, pbj, inv_mass, true, s);
    if (rc) return rc;
    if (n_pairs > 0) {
        // flags of the island starts (into the key array, no longer needed), scanned into the
        // fill counters (likewise): each island's index in key order
        const int gp = std::min(blocks_for(n_pairs), kSMs * 8);
        k_isl_flags<<<gp, kThreads, 0, s>>>(W, n_pairs, W.key);
        if ((rc = check_launch("island_flags"))) return rc;
        if ((rc = exclusive_scan(W.key, W.fill, n_pairs, nullptr, W.scan_tmp, s))) return rc;
        k_isl_compact<<<gp, kThreads, 0, s>>>(W, n_pairs, order, W.fill, packed, starts, counts);
        if ((rc = check_launch("island_compact"))) return rc;
    }
    cudaMemcpyAsync(info, W.info, 4 * sizeof(int32_t), cudaMemcpyDeviceToDevice, s);
    return check_launch("island_info");
}
