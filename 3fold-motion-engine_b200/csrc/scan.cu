// Exclusive prefix sum over int32, three-phase (tile scan, scan of tile totals, add back),
// recursive over the tile totals.  Used for bucket offsets of the hash grid, the emission
// offsets of contact generation and the compaction of kept contacts.  The element count can
// be read from the device (`dn`), so a scan inside a captured step needs no host read-back:
// elements at or beyond *dn read as zero.
#include <mutex>

#include "b2c_common.cuh"

namespace b2c {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int warp_incl_scan(int v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// block-wide exclusive scan of one int per thread; returns the exclusive prefix, *total the sum
__device__ __forceinline__ int block_excl_scan(int v, int *total)
{
    __shared__ int warp_sums[kScanThreads / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = warp_incl_scan(v);
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int s = lane < kScanThreads / 32 ? warp_sums[lane] : 0;
        int si = warp_incl_scan(s);
        if (lane < kScanThreads / 32) warp_sums[lane] = si - s;
    }
    __syncthreads();
    int excl = warp_sums[wid] + inc - v;
    __shared__ int tot;
    if (threadIdx.x == kScanThreads - 1) tot = excl + v;
    __syncthreads();
    *total = tot;
    return excl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int *__restrict__ in, int *__restrict__ out, int n,
                                                              const int *__restrict__ dn, int *__restrict__ tile_sums)
{
    const int ne = dn ? min(*dn, n) : n;
    const long long base = (long long)blockIdx.x * kScanTile + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        v[k] = (i < ne) ? in[i] : 0;
        s += v[k];
    }
    int total;
    int ex = block_excl_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
    }
    if (threadIdx.x == 0 && tile_sums) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_add(int *__restrict__ out, int n, const int *__restrict__ tile_off)
{
    const long long i = (long long)blockIdx.x * kScanTile + threadIdx.x;
    const int add = tile_off[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        long long j = i + (long long)k * kScanThreads;
        if (j < n) out[j] += add;
    }
}

int scan_scratch_ints(int n)
{
    if (n <= kScanTile) return 0;
    int nt = (n + kScanTile - 1) / kScanTile;
    return 2 * nt + scan_scratch_ints(nt);
}

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s)
{
    if (n <= 0) return B2C_OK;
    int nt = (n + kScanTile - 1) / kScanTile;
    if (nt == 1) {
        k_scan_tiles<<<1, kScanThreads, 0, s>>>(in, out, n, dn, nullptr);
        return check_launch("scan");
    }
    int *sums = scratch, *offs = scratch + nt;
    k_scan_tiles<<<nt, kScanThreads, 0, s>>>(in, out, n, dn, sums);
    int rc = exclusive_scan(sums, offs, nt, nullptr, scratch + 2 * nt, s);
    if (rc) return rc;
    k_scan_add<<<nt, kScanThreads, 0, s>>>(out, n, offs);
    return check_launch("scan_add");
}

// Scratch of b2c_exclusive_scan_noalloc: one file-scope device array, sized for the largest
// scan it accepts (kNoAllocMaxN elements: 2 x 8192 tile sums and offsets plus 8 for the second
// level = 16,392 ints, 64 KiB).  It keeps its contents between calls; nothing in it has to
// start at zero (every tile sum is written before it is read).
constexpr int kNoAllocMaxN = 1 << 24;
constexpr int noalloc_scratch_ints(int n)
{
    return n <= kScanTile ? 0 : 2 * ((n + kScanTile - 1) / kScanTile) + noalloc_scratch_ints((n + kScanTile - 1) / kScanTile);
}
constexpr int kNoAllocScratchInts = noalloc_scratch_ints(kNoAllocMaxN);
static __device__ __align__(256) int g_noalloc_scan_scratch[kNoAllocScratchInts];

// Identifier of the calling thread's current CUDA context, 0 when there is none or it cannot be
// read.  The driver's cuCtxGetCurrent / cuCtxGetId are reached through the runtime's entry-point
// query, so the library does not link the driver library itself.
typedef int (*ctx_current_fn)(void **);
typedef int (*ctx_id_fn)(void *, unsigned long long *);
static unsigned long long current_context_id()
{
    static ctx_current_fn get_cur = nullptr;
    static ctx_id_fn get_id = nullptr;
    static bool tried = false;
    if (!tried) {  // the callers hold the scratch mutex
        tried = true;
        void *f = nullptr, *g = nullptr;
        cudaDriverEntryPointQueryResult q1 = cudaDriverEntryPointSymbolNotFound, q2 = q1;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &g, 12000, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_cur = reinterpret_cast<ctx_current_fn>(f);
            get_id = reinterpret_cast<ctx_id_fn>(g);
        }
        cudaGetLastError();  // a failed query leaves no sticky error behind
    }
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (!get_cur || !get_id || get_cur(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array for the current device.  It is looked up with that
// device current and cached per device together with the context it belongs to; a call from
// another context of the device (after cudaDeviceReset the runtime makes a new one and loads the
// library's module again) looks it up again instead of reusing an address of a context that is
// gone.
static int noalloc_scratch(int **out)
{
    static std::mutex mu;
    static int *addr[64] = {};
    static unsigned long long ctx_of[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("b2c_exclusive_scan_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return B2C_ECUDA;
    }
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_context_id();
    if (!addr[dev] || ctx == 0 || ctx != ctx_of[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch);
        if (e != cudaSuccess || !p) {
            set_error("b2c_exclusive_scan_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return B2C_ECUDA;
        }
        addr[dev] = static_cast<int *>(p);
        ctx_of[dev] = current_context_id();  // the lookup made the device's context current
    }
    *out = addr[dev];
    return B2C_OK;
}

}  // namespace b2c

extern "C" int32_t b2c_scan_noalloc_max_n(void) { return b2c::kNoAllocMaxN; }

extern "C" int32_t b2c_exclusive_scan_noalloc(const int32_t *in, int32_t *out, int32_t n, b2c_stream s)
{
    if (n < 0 || (n > 0 && (!in || !out))) {
        b2c::set_error("b2c_exclusive_scan_noalloc: bad argument");
        return B2C_EARG;
    }
    if (n > b2c::kNoAllocMaxN) {
        b2c::set_error("b2c_exclusive_scan_noalloc: n = %d exceeds the maximum %d of its built-in scratch; "
                       "use b2c_exclusive_scan with a caller scratch buffer",
                       n, b2c::kNoAllocMaxN);
        return B2C_EARG;
    }
    int *scratch = nullptr;
    const int rc = b2c::noalloc_scratch(&scratch);  // also the whole of a call with n = 0
    if (rc || n == 0) return rc;
    return b2c::exclusive_scan(in, out, n, nullptr, scratch, b2c::stream_of(s));
}

extern "C" int32_t b2c_scan_scratch_ints(int32_t n) { return b2c::scan_scratch_ints(n); }

extern "C" int32_t b2c_exclusive_scan(const int32_t *in, int32_t *out, int32_t n, int32_t *scratch, b2c_stream s)
{
    if (!in || !out || n < 0 || (n > b2c::kScanTile && !scratch)) {
        b2c::set_error("b2c_exclusive_scan: bad argument");
        return B2C_EARG;
    }
    return b2c::exclusive_scan(in, out, n, nullptr, scratch, b2c::stream_of(s));
}
