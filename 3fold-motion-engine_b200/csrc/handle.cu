// Engine handle: the ContactEngine protocol (contact_engine.py:48-55) over the box engine as C
// calls, with the device memory owned by the library.
//
// The build mirrors the Python BoxContactEngine._build: the same host arithmetic for the body
// arrays (float64, rounded once to float32), the same broadphase grid and capacities, the same
// structs handed to b2c_box_substep.  A step is that launch sequence per substep, captured into a
// CUDA graph after its first eager run (as the Python engine's torch graph), then a header
// read-back into pinned memory; the next step checks the error bits before launching.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>

#include "b2c_barrier.cuh"
#include "b2c_common.cuh"

namespace {

constexpr int kMaxColors = 512;    // per-colour arrays (the reference's _NCOLMAX)
constexpr int kRecSlots = 8;       // contact slots of a pair record (<= 8 corners on the ground)
constexpr int kMaxGraphs = 8;      // captured (dt, substeps) keys kept at once
constexpr size_t kAlign = 256;

struct Graph {
    double sdt;
    int substeps;
    cudaGraphExec_t exec;
};

struct Engine {
    b2c_config cfg;
    // bodies as added (host, float64 as the reference's setup)
    std::vector<double> center, dims, dens, mu;
    std::vector<int32_t> kin, scene;
    // after the build
    bool built = false;
    int N = 0, nbk = 0, cand_cap = 0, kept_cap = 0, pcap = 0;
    std::vector<double> M;            // masses, for contact_forces (inf once made kinematic)
    std::vector<double> M0;           // every body's mass from its box and density, kinematic or not
    std::vector<int32_t> kinarr;
    char *arena = nullptr;
    size_t arena_bytes = 0;
    float *state = nullptr, *pv = nullptr, *po = nullptr, *vgrav = nullptr, *invM = nullptr, *IbInv = nullptr,
          *invIw = nullptr, *half = nullptr, *body_mu = nullptr, *stage = nullptr;
    int32_t *kin_d = nullptr, *local = nullptr, *scene_d = nullptr, *header = nullptr;
    int64_t *kept_keys = nullptr;
    b2c_bodies bodies{};
    b2c_boxes boxes{};
    b2c_contacts kept{};
    b2c_pairs pairs{};
    b2c_warm warm{};
    b2c_color_params params{};
    int32_t *hdr_host = nullptr;      // pinned: header of the last step, then [hits, misses]
    cudaEvent_t hdr_event = nullptr;
    bool hdr_pending = false;
    cudaStream_t capture = nullptr;
    cudaStream_t last = nullptr;
    std::vector<Graph> graphs;
    int graph_captures = 0, kernels_per_step = 0;
    double force_dt = 0.0;
    bool has_force = false;
};

struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int d)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        ok = cudaSetDevice(d) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int cuda_fail(const char *what, cudaError_t e)
{
    b2c::set_error("%s: %s", what, cudaGetErrorString(e));
    return B2C_ECUDA;
}

bool finite3(const double *p) { return std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]); }

// Box.Ib (ncp_gpu.py:1105-1109) as BoxContactEngine's box_body_arrays computes it: mass =
// density x 8 hx hy hz, Ib = m / 12 diag(ey^2 + ez^2, ex^2 + ez^2, ex^2 + ey^2) over the full
// edges e = 2 h, all float64; the inverse of the diagonal is 1 / Ib; one rounding to float32.
int box_setup(int n, const double *center3, const double *half3, const double *density, const int32_t *kin,
              float *xc4, float *invM, float *IbInv12, double *M)
{
    for (int i = 0; i < n; ++i) {
        const double *h = half3 + 3 * i;
        const double m = density[i] * 8.0 * h[0] * h[1] * h[2];
        const double ex = 2.0 * h[0], ey = 2.0 * h[1], ez = 2.0 * h[2];
        const double m12 = m / 12.0;
        const double Ib[3] = {m12 * (ey * ey + ez * ez), m12 * (ex * ex + ez * ez), m12 * (ex * ex + ey * ey)};
        const bool k = kin && kin[i] != 0;
        double inv[3];
        for (int a = 0; a < 3; ++a) inv[a] = k ? 1.0 : 1.0 / Ib[a];
        if (!(m > 0.0) || !std::isfinite(inv[0]) || !std::isfinite(inv[1]) || !std::isfinite(inv[2])) {
            b2c::set_error("box engine: degenerate box mass / inertia (body %d)", i);
            return B2C_EARG;
        }
        if (xc4)
            for (int a = 0; a < 4; ++a) xc4[4 * i + a] = a < 3 ? (float)center3[3 * i + a] : 0.0f;
        if (invM) invM[i] = k ? 0.0f : (float)(1.0 / m);
        if (IbInv12)
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 4; ++c) IbInv12[12 * i + 4 * r + c] = (r == c) ? (float)inv[r] : 0.0f;
        if (M) M[i] = m;
    }
    return B2C_OK;
}

__global__ void k_state_unpack(int n, const float4 *__restrict__ st, float *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 x = st[i], q = st[n + i], v = st[2 * n + i], w = st[3 * n + i];
    float *ox = out + 3 * i, *oq = out + 3 * n + 4 * i, *ov = out + 7 * n + 3 * i, *ow = out + 10 * n + 3 * i;
    ox[0] = x.x, ox[1] = x.y, ox[2] = x.z;
    oq[0] = q.x, oq[1] = q.y, oq[2] = q.z, oq[3] = q.w;
    ov[0] = v.x, ov[1] = v.y, ov[2] = v.z;
    ow[0] = w.x, ow[1] = w.y, ow[2] = w.z;
}

void drop_graphs(Engine *e)
{
    for (Graph &g : e->graphs) cudaGraphExecDestroy(g.exec);
    e->graphs.clear();
}

void release(Engine *e)
{
    drop_graphs(e);
    if (e->arena) cudaFree(e->arena);
    if (e->hdr_host) cudaFreeHost(e->hdr_host);
    if (e->hdr_event) cudaEventDestroy(e->hdr_event);
    if (e->capture) cudaStreamDestroy(e->capture);
    e->arena = nullptr;
    e->hdr_host = nullptr;
    e->hdr_event = nullptr;
    e->capture = nullptr;
    e->hdr_pending = false;
    e->built = false;
    e->has_force = false;
}

// The device arrays in one allocation: `carve` runs twice, first to size the arena, then to
// hand out 256-byte-aligned pieces of it.
template <class F>
size_t carve(Engine *e, char *base, F &&take_all)
{
    size_t off = 0;
    auto take = [&](auto *&ptr, size_t count) {
        using T = std::remove_reference_t<decltype(*ptr)>;
        const size_t bytes = sizeof(T) * (count > 0 ? count : 1);
        off = (off + kAlign - 1) / kAlign * kAlign;
        ptr = base ? reinterpret_cast<T *>(base + off) : nullptr;
        off += bytes;
    };
    take_all(take);
    (void)e;
    return off;
}

int build(Engine *e)
{
    const int N = (int)e->mu.size();  // bodies (centre and edge arrays hold three doubles each)
    // host body arrays
    std::vector<double> half(3 * (size_t)N);
    for (size_t k = 0; k < half.size(); ++k) half[k] = 0.5 * e->dims[k];
    std::vector<float> xc4(4 * (size_t)N), invM(N), IbInv(12 * (size_t)N), half4(4 * (size_t)N, 0.0f),
        mus(N);
    std::vector<double> M(N);
    int rc = box_setup(N, e->center.data(), half.data(), e->dens.data(), e->kin.data(), xc4.data(), invM.data(),
                       IbInv.data(), M.data());
    if (rc) return rc;
    float hmax = 0.0f;
    for (int i = 0; i < N; ++i) {
        float h[3];
        for (int a = 0; a < 3; ++a) half4[4 * i + a] = h[a] = (float)half[3 * i + a];
        const float r = sqrtf((h[0] * h[0] + h[1] * h[1]) + h[2] * h[2]);
        hmax = (i == 0 || r > hmax) ? r : hmax;
        mus[i] = (float)e->mu[i];
    }
    const double hm = N ? (double)hmax : 0.5;
    const float cell = (float)(1.01 * (2.0 * hm + e->cfg.margin));  // every sphere-test pair in adjacent cells
    int dims[3];
    if (N <= 2000) dims[0] = 16, dims[1] = 16, dims[2] = 8;
    else if (N <= 20000) dims[0] = 32, dims[1] = 32, dims[2] = 16;
    else if (N <= 500000) dims[0] = 64, dims[1] = 64, dims[2] = 32;
    else dims[0] = 128, dims[1] = 128, dims[2] = 64;
    // scenes: each body's index among its scene's bodies (the colouring priority)
    int n_scenes = 0;
    for (int s : e->scene) n_scenes = s + 1 > n_scenes ? s + 1 : n_scenes;
    std::vector<int32_t> local(N), seen(n_scenes > 0 ? n_scenes : 1, 0);
    for (int i = 0; i < N; ++i) local[i] = seen[e->scene[i]]++;
    bool per_body_mu = false;
    for (int i = 0; i < N; ++i) per_body_mu |= mus[i] != (float)e->cfg.mu;

    const int nbk = dims[0] * dims[1] * dims[2];
    const int cand_cap = (int)std::max<long long>((long long)e->cfg.cand_per_body * N + N, 64);
    const int kept_cap = 4 * cand_cap + 8 * N;
    const int pcap = cand_cap;
    const int scan_ints = b2c_scan_scratch_ints(std::max(std::max(nbk, N), cand_cap) + 1);
    const long long rec_floats = b2c_pair_record_floats(pcap, kRecSlots);
    if (scan_ints <= 0 || rec_floats <= 0) {
        b2c::set_error("box engine: capacity out of range (%d bodies)", N);
        return B2C_EARG;
    }

    e->N = N, e->nbk = nbk, e->cand_cap = cand_cap, e->kept_cap = kept_cap, e->pcap = pcap;
    b2c_boxes &bx = e->boxes;
    b2c_contacts &kc = e->kept;
    b2c_pairs &pr = e->pairs;
    b2c_warm &wm = e->warm;
    float *slot_p, *slot_n, *kpA, *kpB, *kn, *kimp, *wimp, *rec, *cached_mass;
    int32_t *bucket, *start, *cursor, *sorted, *cand_count, *cand_offset, *cand_a, *cand_b, *cont_count, *cont_offset,
        *pair_flag, *pair_offset, *slot_f, *scan_tmp, *kbi, *kbj, *kfa, *kfb, *pbi, *pbj, *kcount, *pstart, *pidx,
        *col, *porder, *cstart, *ccount, *cached_a, *cached_b, *cache_state, *body_slots, *wn;
    int64_t *claim, *wkeys;
    uint64_t *body_colors;
    uint32_t *barrier;
    auto layout = [&](auto &take) {
        take(e->state, 16 * (size_t)N);
        take(e->pv, 4 * (size_t)N), take(e->po, 4 * (size_t)N), take(e->vgrav, 4 * (size_t)N);
        take(e->invM, N), take(e->IbInv, 12 * (size_t)N), take(e->invIw, 12 * (size_t)N);
        take(e->kin_d, N), take(e->half, 4 * (size_t)N), take(e->body_mu, N);
        take(e->local, N), take(e->scene_d, N), take(e->header, 8);
        take(e->stage, 13 * (size_t)N);
        take(bucket, N), take(start, nbk + 1), take(cursor, nbk + 1), take(sorted, N);
        take(cand_count, N + 1), take(cand_offset, N + 1), take(cand_a, cand_cap), take(cand_b, cand_cap);
        take(cont_count, cand_cap + 1), take(cont_offset, cand_cap + 1);
        take(pair_flag, cand_cap + 1), take(pair_offset, cand_cap + 1);
        take(slot_p, 32 * (size_t)cand_cap), take(slot_n, 4 * (size_t)cand_cap), take(slot_f, 8 * (size_t)cand_cap);
        take(scan_tmp, scan_ints);
        take(kbi, kept_cap), take(kbj, kept_cap), take(kfa, kept_cap), take(kfb, kept_cap);
        take(kpA, 4 * (size_t)kept_cap), take(kpB, 4 * (size_t)kept_cap), take(kn, 4 * (size_t)kept_cap);
        take(kimp, 4 * (size_t)kept_cap), take(e->kept_keys, kept_cap);
        take(pbi, pcap), take(pbj, pcap), take(kcount, pcap + 1), take(pstart, pcap + 1), take(pidx, kept_cap);
        take(col, pcap), take(porder, pcap), take(cstart, kMaxColors), take(ccount, kMaxColors);
        take(claim, 2 * (size_t)N), take(cached_a, pcap), take(cached_b, pcap), take(cached_mass, N);
        take(cache_state, 8), take(body_colors, N), take(body_slots, 64 * (size_t)N), take(barrier, b2c::kBarrierWords);
        take(rec, (size_t)rec_floats);
        take(wkeys, kept_cap), take(wimp, 4 * (size_t)kept_cap), take(wn, 1);
    };
    const size_t bytes = carve(e, nullptr, layout);
    cudaError_t ce;
    if ((ce = cudaMalloc(&e->arena, bytes)) != cudaSuccess) {
        e->arena = nullptr;
        return cuda_fail("box engine: device allocation", ce);
    }
    e->arena_bytes = bytes;
    carve(e, e->arena, layout);
    if ((ce = cudaMemset(e->arena, 0, bytes)) != cudaSuccess) return cuda_fail("box engine: clear", ce);
    if ((ce = cudaMallocHost(&e->hdr_host, 16 * sizeof(int32_t))) != cudaSuccess) {
        e->hdr_host = nullptr;
        return cuda_fail("box engine: pinned header", ce);
    }
    std::memset(e->hdr_host, 0, 16 * sizeof(int32_t));
    if ((ce = cudaEventCreateWithFlags(&e->hdr_event, cudaEventDisableTiming)) != cudaSuccess) {
        e->hdr_event = nullptr;
        return cuda_fail("box engine: event", ce);
    }
    if ((ce = cudaStreamCreateWithFlags(&e->capture, cudaStreamNonBlocking)) != cudaSuccess) {
        e->capture = nullptr;
        return cuda_fail("box engine: capture stream", ce);
    }
    // initial state: centres, identity quaternions (x, y, z, w), zero velocities
    std::vector<float> st(16 * (size_t)N, 0.0f);
    std::memcpy(st.data(), xc4.data(), sizeof(float) * 4 * (size_t)N);
    for (int i = 0; i < N; ++i) st[4 * (size_t)N + 4 * i + 3] = 1.0f;
    auto up = [&](void *dst, const void *src, size_t b) {
        return b ? cudaMemcpy(dst, src, b, cudaMemcpyHostToDevice) : cudaSuccess;
    };
    if ((ce = up(e->state, st.data(), sizeof(float) * st.size())) != cudaSuccess ||
        (ce = up(e->invM, invM.data(), sizeof(float) * N)) != cudaSuccess ||
        (ce = up(e->IbInv, IbInv.data(), sizeof(float) * IbInv.size())) != cudaSuccess ||
        (ce = up(e->kin_d, e->kin.data(), sizeof(int32_t) * N)) != cudaSuccess ||
        (ce = up(e->half, half4.data(), sizeof(float) * half4.size())) != cudaSuccess ||
        (ce = up(e->body_mu, mus.data(), sizeof(float) * N)) != cudaSuccess ||
        (ce = up(e->local, local.data(), sizeof(int32_t) * N)) != cudaSuccess ||
        (ce = up(e->scene_d, e->scene.data(), sizeof(int32_t) * N)) != cudaSuccess)
        return cuda_fail("box engine: upload", ce);

    e->bodies = b2c_bodies{N, e->state, e->state + 4 * (size_t)N, e->state + 8 * (size_t)N, e->state + 12 * (size_t)N,
                           e->pv, e->po, e->invM, e->IbInv, e->kin_d, e->invIw};
    bx = b2c_boxes{};
    bx.n = N, bx.half = e->half, bx.mu = e->body_mu, bx.margin = (float)e->cfg.margin, bx.cell = cell;
    bx.dim_x = dims[0], bx.dim_y = dims[1], bx.dim_z = dims[2], bx.cand_capacity = cand_cap;
    bx.bucket = bucket, bx.start = start, bx.cursor = cursor, bx.sorted = sorted;
    bx.cand_count = cand_count, bx.cand_offset = cand_offset, bx.cand_a = cand_a, bx.cand_b = cand_b;
    bx.cont_count = cont_count, bx.cont_offset = cont_offset, bx.pair_flag = pair_flag, bx.pair_offset = pair_offset;
    bx.slot_p = slot_p, bx.slot_n = slot_n, bx.slot_f = slot_f, bx.scan_tmp = scan_tmp;
    bx.scene = n_scenes > 1 ? e->scene_d : nullptr;
    kc = b2c_contacts{kept_cap, kbi, kbj, kpA, kpB, kn, kfa, kfb, kimp};
    pr = b2c_pairs{};
    pr.capacity = pcap, pr.max_colors = kMaxColors, pr.pbi = pbi, pr.pbj = pbj, pr.kcount = kcount;
    pr.pstart = pstart, pr.pidx = pidx, pr.col = col, pr.porder = porder, pr.cstart = cstart, pr.ccount = ccount;
    pr.claim = claim, pr.cached_a = cached_a, pr.cached_b = cached_b, pr.cached_mass = cached_mass;
    pr.cache_state = cache_state, pr.barrier = barrier, pr.rec = rec, pr.kslots = kRecSlots;
    pr.body_colors = body_colors, pr.body_local = e->local, pr.body_slots = body_slots;
    wm = b2c_warm{kept_cap, wkeys, wimp, wn};
    b2c_color_params &p = e->params;
    p.vit = e->cfg.vit, p.pit = e->cfg.pit, p.max_points = 8, p.flags = e->cfg.flags, p.mu = (float)e->cfg.mu;
    p.t2d = 1.0f, p.color_cap = std::min(e->cfg.color_cap, kMaxColors), p.solve_blocks = e->cfg.solve_blocks;
    p.barrier_timeout_ns = e->cfg.barrier_timeout_ns > 0 ? e->cfg.barrier_timeout_ns : 1000000000LL;
    p.body_mu = per_body_mu ? e->body_mu : nullptr;
    e->M0 = M;
    e->M = M;
    e->kinarr = e->kin;
    e->built = true;
    return B2C_OK;
}

int ensure_built(Engine *e)
{
    if (e->built) return B2C_OK;
    int rc = build(e);
    if (rc) release(e);
    return rc;
}

int launch(Engine *e, float sdt, int substeps, cudaStream_t s)
{
    for (int k = 0; k < substeps; ++k) {
        int rc = b2c_box_substep(&e->bodies, &e->boxes, &e->kept, e->kept_keys, &e->pairs, &e->warm,
                                 reinterpret_cast<b2c_header *>(e->header), &e->params, sdt, e->vgrav, s);
        if (rc) return rc;
    }
    return B2C_OK;
}

// one captured graph per (dt, substeps): the capture runs on a side stream ordered after s
int capture_graph(Engine *e, float sdt, int substeps, cudaStream_t s, cudaGraphExec_t *out)
{
    cudaEvent_t ev;
    cudaError_t ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (ce != cudaSuccess) return cuda_fail("box engine: capture", ce);
    cudaEventRecord(ev, s);
    cudaStreamWaitEvent(e->capture, ev, 0);
    cudaGraph_t g = nullptr;
    if ((ce = cudaStreamBeginCapture(e->capture, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        cudaEventDestroy(ev);
        return cuda_fail("box engine: begin capture", ce);
    }
    int rc = launch(e, sdt, substeps, e->capture);
    ce = cudaStreamEndCapture(e->capture, &g);
    if (rc == B2C_OK && ce != cudaSuccess) rc = cuda_fail("box engine: end capture", ce);
    if (rc == B2C_OK) {
        const int nk = b2c_graph_kernel_nodes(g);
        ce = cudaGraphInstantiate(out, g, 0);
        if (ce != cudaSuccess) rc = cuda_fail("box engine: instantiate", ce);
        else e->kernels_per_step = nk;
    }
    if (g) cudaGraphDestroy(g);
    cudaEventRecord(ev, e->capture);
    cudaStreamWaitEvent(s, ev, 0);
    cudaEventDestroy(ev);
    return rc;
}

int header_wait(Engine *e)
{
    if (!e->hdr_pending) return B2C_OK;
    cudaError_t ce = cudaEventSynchronize(e->hdr_event);
    if (ce != cudaSuccess) return cuda_fail("box engine: step", ce);
    e->hdr_pending = false;
    return B2C_OK;
}

int sync_last(Engine *e, const char *what)
{
    cudaError_t ce = cudaStreamSynchronize(e->last);
    return ce == cudaSuccess ? B2C_OK : cuda_fail(what, ce);
}

Engine *engine(void *h) { return reinterpret_cast<Engine *>(h); }

// the device arrays a checkpoint holds, in blob order
struct Section {
    void *ptr;
    size_t bytes;
};

std::vector<Section> sections(Engine *e)
{
    const size_t N = (size_t)e->N, K = (size_t)e->kept_cap, P = (size_t)e->pcap;
    b2c_pairs &pr = e->pairs;
    return {{e->state, 64 * N},         {e->vgrav, 16 * N},         {e->invM, 4 * N},
            {e->kin_d, 4 * N},          {e->header, 32},            {e->warm.keys, 8 * K},
            {e->warm.imp, 16 * K},      {e->warm.n, 4},             {pr.col, 4 * P},
            {pr.porder, 4 * P},         {pr.cstart, 4 * kMaxColors}, {pr.ccount, 4 * kMaxColors},
            {pr.cached_a, 4 * P},       {pr.cached_b, 4 * P},       {pr.cached_mass, 4 * N},
            {pr.cache_state, 32},       {pr.barrier, 8}};
}

struct BlobHead {
    char magic[8];
    int32_t version, n, cand_cap, kept_cap, pcap, kslots;
    int32_t has_force, pad;
    double force_dt;
    uint64_t bytes;
};
constexpr char kMagic[8] = {'b', '2', 'c', 'b', 'o', 'x', 'e', 's'};

}  // namespace

extern "C" void b2c_config_init(b2c_config *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->kind = B2C_ENGINE_BOX;
    c->device = 0;
    c->vit = 16, c->pit = 10;
    c->mu = 0.5;
    c->dims[0] = 0.3, c->dims[1] = 0.3, c->dims[2] = 0.2;
    c->margin = 2e-3;
    c->flags = B2C_COLOR_FIXED_FRAME | B2C_COLOR_APPLY_WARM | B2C_COLOR_CACHE | B2C_COLOR_WARM_START |
               B2C_COLOR_FIRST_FIT | B2C_COLOR_ROW_FORM;
    c->color_cap = kMaxColors;
    c->solve_blocks = 0;
    c->cand_per_body = 16;
    c->barrier_timeout_ns = 1000000000LL;
    c->graph = 1;
}

extern "C" int32_t b2c_box_body_setup(int32_t n, const double *center3, const double *dims3, const double *density,
                                      const int32_t *kin, float *xc4, float *invM, float *IbInv12, double *M)
{
    if (n < 0 || (n > 0 && (!center3 || !dims3 || !density))) {
        b2c::set_error("b2c_box_body_setup: bad argument");
        return B2C_EARG;
    }
    std::vector<double> half(3 * (size_t)n);
    for (size_t k = 0; k < half.size(); ++k) half[k] = 0.5 * dims3[k];
    return box_setup(n, center3, half.data(), density, kin, xc4, invM, IbInv12, M);
}

extern "C" int32_t b2c_create(const b2c_config *c, void **h)
{
    if (!c || !h) {
        b2c::set_error("b2c_create: bad argument");
        return B2C_EARG;
    }
    *h = nullptr;
    if (c->kind != B2C_ENGINE_BOX) {
        b2c::set_error("b2c_create: engine kind %d is not built on the handle interface (B2C_ENGINE_BOX = %d)",
                       c->kind, B2C_ENGINE_BOX);
        return B2C_EARG;
    }
    if (c->flags & B2C_COLOR_ISLANDS) {
        b2c::set_error("b2c_create: B2C_COLOR_ISLANDS is not available on the handle interface (the stage calls "
                       "take it with b2c_pairs.isl_work)");
        return B2C_EARG;
    }
    const bool dims_ok = c->dims[0] > 0.0 && c->dims[1] > 0.0 && c->dims[2] > 0.0 && finite3(c->dims);
    const bool frame_ok = !(c->flags & B2C_COLOR_ROW_FORM) || (c->flags & B2C_COLOR_FIXED_FRAME);
    if (c->vit < 0 || c->pit < 0 || !(c->mu >= 0.0) || !std::isfinite(c->mu) || !dims_ok || !(c->margin >= 0.0) ||
        !std::isfinite(c->margin) || c->color_cap < 1 || c->cand_per_body < 1 || c->device < 0 ||
        (c->flags & B2C_COLOR_PER_CONTACT) || !frame_ok) {
        b2c::set_error("b2c_create: bad configuration");
        return B2C_EARG;
    }
    Engine *e = new (std::nothrow) Engine;
    if (!e) {
        b2c::set_error("b2c_create: out of host memory");
        return B2C_EARG;
    }
    e->cfg = *c;
    *h = e;
    return B2C_OK;
}

extern "C" int32_t b2c_add_bodies(void *h, int32_t n, const double *center3, const double *density, const double *dims3,
                                  const int32_t *kin)
{
    Engine *e = engine(h);
    if (!e || n < 0 || (n > 0 && !center3)) {
        b2c::set_error("b2c_add_bodies: bad argument");
        return B2C_EARG;
    }
    for (int i = 0; i < n; ++i) {
        const double *d = dims3 ? dims3 + 3 * i : e->cfg.dims;
        const double rho = density ? density[i] : 1000.0;
        if (!finite3(center3 + 3 * i) || !finite3(d) || !(d[0] > 0.0 && d[1] > 0.0 && d[2] > 0.0) ||
            !(rho > 0.0) || !std::isfinite(rho)) {
            b2c::set_error("b2c_add_bodies: body %d: non-finite centre or non-positive size / density", i);
            return B2C_EARG;
        }
    }
    for (int i = 0; i < n; ++i) {
        const double *d = dims3 ? dims3 + 3 * i : e->cfg.dims;
        for (int a = 0; a < 3; ++a) e->center.push_back(center3[3 * i + a]), e->dims.push_back(d[a]);
        e->dens.push_back(density ? density[i] : 1000.0);
        e->mu.push_back(e->cfg.mu);
        e->kin.push_back(kin && kin[i] ? 1 : 0);
        e->scene.push_back(0);
    }
    if (n > 0 && e->built) {  // a new body rebuilds from the added centres at the next step
        DeviceGuard dg(e->cfg.device);
        if (e->last) cudaStreamSynchronize(e->last);
        release(e);
    }
    return B2C_OK;
}

extern "C" int32_t b2c_set_body_mu(void *h, int32_t first, int32_t n, const double *mu)
{
    Engine *e = engine(h);
    if (!e || first < 0 || n < 0 || (long long)first + n > (long long)e->mu.size() || (n > 0 && !mu) || e->built) {
        b2c::set_error("b2c_set_body_mu: bad argument (bodies out of range, or set after the first step)");
        return B2C_EARG;
    }
    for (int i = 0; i < n; ++i)
        if (!(mu[i] >= 0.0) || !std::isfinite(mu[i])) {
            b2c::set_error("b2c_set_body_mu: friction must be finite and >= 0");
            return B2C_EARG;
        }
    for (int i = 0; i < n; ++i) e->mu[first + i] = mu[i];
    return B2C_OK;
}

extern "C" int32_t b2c_set_body_scene(void *h, int32_t first, int32_t n, const int32_t *scene)
{
    Engine *e = engine(h);
    if (!e || first < 0 || n < 0 || (long long)first + n > (long long)e->scene.size() || (n > 0 && !scene) ||
        e->built) {
        b2c::set_error("b2c_set_body_scene: bad argument (bodies out of range, or set after the first step)");
        return B2C_EARG;
    }
    for (int i = 0; i < n; ++i)
        if (scene[i] < 0) {
            b2c::set_error("b2c_set_body_scene: scene ids are >= 0");
            return B2C_EARG;
        }
    for (int i = 0; i < n; ++i) e->scene[first + i] = scene[i];
    return B2C_OK;
}

extern "C" int32_t b2c_body_count(const void *h)
{
    const Engine *e = reinterpret_cast<const Engine *>(h);
    return e ? (int32_t)e->mu.size() : -1;
}

extern "C" int32_t b2c_set_kinematic(void *h, int32_t i, const double *xc3)
{
    Engine *e = engine(h);
    if (!e || i < 0 || i >= (int32_t)e->mu.size() || !xc3 || !finite3(xc3)) {
        b2c::set_error("b2c_set_kinematic: bad argument");
        return B2C_EARG;
    }
    e->kin[i] = 1;
    for (int a = 0; a < 3; ++a) e->center[3 * (size_t)i + a] = xc3[a];
    if (!e->built) return B2C_OK;
    DeviceGuard dg(e->cfg.device);
    const float x[3] = {(float)xc3[0], (float)xc3[1], (float)xc3[2]};
    const float zero4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const int32_t one = 1;
    const size_t N = (size_t)e->N;
    cudaStream_t s = e->last;
    cudaMemcpyAsync(e->state + 4 * (size_t)i, x, sizeof(x), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(e->invM + i, zero4, sizeof(float), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(e->state + 8 * N + 4 * (size_t)i, zero4, sizeof(zero4), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(e->state + 12 * N + 4 * (size_t)i, zero4, sizeof(zero4), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(e->kin_d + i, &one, sizeof(one), cudaMemcpyHostToDevice, s);
    e->kinarr[i] = 1;
    e->M[i] = INFINITY;
    return sync_last(e, "b2c_set_kinematic");
}

extern "C" int32_t b2c_step(void *h, double dt, int32_t substeps, b2c_stream stream)
{
    Engine *e = engine(h);
    if (!e || !(dt > 0.0) || !std::isfinite(dt) || substeps < 1) {
        b2c::set_error("b2c_step: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    if (!dg.ok) {
        b2c::set_error("b2c_step: CUDA device %d is not available", e->cfg.device);
        return B2C_ECUDA;
    }
    int rc = ensure_built(e);
    if (rc) return rc;
    // the previous step's error bits (check_errors before every step)
    if ((rc = header_wait(e))) return rc;
    const int32_t err = e->hdr_host[6];
    if (err) {
        e->hdr_host[6] = 0;
        cudaMemsetAsync(e->header, 0, 8 * sizeof(int32_t), e->last);
        cudaStreamSynchronize(e->last);
        const bool timeout = err & (B2C_ERR_COLOR_TIMEOUT | B2C_ERR_BARRIER_TIMEOUT);
        static const char *const names[8] = {"contact capacity overflow",
                                             "a body pair carries more than 1024 contacts",
                                             "a body pair carries more than 8 kept contacts",
                                             "colour count exceeds the colour cap",
                                             "colouring did not finish in its round budget",
                                             "a bead has more than 64 neighbours within 2R",
                                             "pair capacity overflow",
                                             "a grid barrier of the persistent solve gave up waiting"};
        char msg[400];
        size_t len = 0;
        for (int b = 0; b < 8; ++b)
            if (err & (1 << b))
                len += (size_t)snprintf(msg + len, sizeof(msg) - std::min(len, sizeof(msg)), "%s%s",
                                        len ? "; " : "", names[b]);
        b2c::set_error("box engine: device error of the previous step (cleared): %s", msg);
        return timeout ? B2C_ETIMEOUT : B2C_ECAPACITY;
    }
    cudaStream_t s = b2c::stream_of(stream);
    const double sdt = dt / substeps;
    const float sdt_f = (float)sdt;
    if (!e->cfg.graph) {
        rc = launch(e, sdt_f, substeps, s);
    } else {
        cudaGraphExec_t exec = nullptr;
        for (const Graph &g : e->graphs)
            if (g.sdt == sdt && g.substeps == substeps) exec = g.exec;
        if (exec) {
            cudaError_t ce = cudaGraphLaunch(exec, s);
            if (ce != cudaSuccess) rc = cuda_fail("b2c_step: graph launch", ce);
        } else if ((rc = launch(e, sdt_f, substeps, s)) == B2C_OK &&
                   (rc = capture_graph(e, sdt_f, substeps, s, &exec)) == B2C_OK) {
            if ((int)e->graphs.size() >= kMaxGraphs) drop_graphs(e);
            e->graphs.push_back(Graph{sdt, substeps, exec});
            e->graph_captures += 1;
        }
    }
    if (rc) return rc;
    cudaMemcpyAsync(e->hdr_host, e->header, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaEventRecord(e->hdr_event, s);
    e->hdr_pending = true;
    e->last = s;
    e->force_dt = sdt;
    e->has_force = true;
    return b2c::check_launch("b2c_step");
}

extern "C" int32_t b2c_sync_header(void *h, b2c_step_header *out)
{
    Engine *e = engine(h);
    if (!e || !out) {
        b2c::set_error("b2c_sync_header: bad argument");
        return B2C_EARG;
    }
    std::memset(out, 0, sizeof(*out));
    out->bodies = (int32_t)e->mu.size();
    out->graph_captures = e->graph_captures;
    out->kernels_per_step = e->kernels_per_step;
    out->built = e->built ? 1 : 0;
    if (!e->built) return B2C_OK;
    DeviceGuard dg(e->cfg.device);
    int rc = header_wait(e);
    if (rc) return rc;
    std::memcpy(&out->last, e->hdr_host, sizeof(b2c_header));
    cudaMemcpyAsync(e->hdr_host + 8, e->pairs.cache_state + 3, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, e->last);
    if ((rc = sync_last(e, "b2c_sync_header"))) return rc;
    out->color_cache_hits = e->hdr_host[8];
    out->color_cache_misses = e->hdr_host[9];
    return B2C_OK;
}

extern "C" int32_t b2c_get_state(void *h, float *xc, float *q, float *v, float *w)
{
    Engine *e = engine(h);
    if (!e) {
        b2c::set_error("b2c_get_state: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    int rc = ensure_built(e);
    if (rc || e->N == 0) return rc;
    const size_t N = (size_t)e->N;
    k_state_unpack<<<b2c::blocks_for(e->N), b2c::kThreads, 0, e->last>>>(e->N, reinterpret_cast<float4 *>(e->state),
                                                                          e->stage);
    if ((rc = b2c::check_launch("b2c_get_state"))) return rc;
    float *dst[4] = {xc, q, v, w};
    const size_t off[4] = {0, 3 * N, 7 * N, 10 * N}, len[4] = {3 * N, 4 * N, 3 * N, 3 * N};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) cudaMemcpyAsync(dst[k], e->stage + off[k], sizeof(float) * len[k], cudaMemcpyDefault, e->last);
    return sync_last(e, "b2c_get_state");
}

extern "C" int32_t b2c_get_state_packed(void *h, float *state, b2c_stream s)
{
    Engine *e = engine(h);
    if (!e || !state) {
        b2c::set_error("b2c_get_state_packed: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    int rc = ensure_built(e);
    if (rc || e->N == 0) return rc;
    cudaError_t ce = cudaMemcpyAsync(state, e->state, 64 * (size_t)e->N, cudaMemcpyDefault, b2c::stream_of(s));
    return ce == cudaSuccess ? B2C_OK : cuda_fail("b2c_get_state_packed", ce);
}

extern "C" int32_t b2c_set_state_packed(void *h, const float *state, b2c_stream s)
{
    Engine *e = engine(h);
    if (!e || !state) {
        b2c::set_error("b2c_set_state_packed: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    int rc = ensure_built(e);
    if (rc || e->N == 0) return rc;
    cudaError_t ce = cudaMemcpyAsync(e->state, state, 64 * (size_t)e->N, cudaMemcpyDefault, b2c::stream_of(s));
    return ce == cudaSuccess ? B2C_OK : cuda_fail("b2c_set_state_packed", ce);
}

extern "C" int32_t b2c_contact_forces(void *h, double *f3)
{
    Engine *e = engine(h);
    if (!e || (!f3 && !e->mu.empty())) {
        b2c::set_error("b2c_contact_forces: bad argument");
        return B2C_EARG;
    }
    const size_t n = e->mu.size();
    std::fill(f3, f3 + 3 * n, 0.0);
    if (!e->built || !e->has_force || e->N == 0) return B2C_OK;
    DeviceGuard dg(e->cfg.device);
    const size_t N = (size_t)e->N;
    std::vector<float> after(4 * N), before(4 * N);
    int rc = sync_last(e, "b2c_contact_forces");
    if (rc) return rc;
    cudaError_t ce;
    if ((ce = cudaMemcpy(after.data(), e->state + 8 * N, 16 * N, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (ce = cudaMemcpy(before.data(), e->vgrav, 16 * N, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail("b2c_contact_forces", ce);
    // M (v_after - v_before) / dt with the velocity difference taken in float32, as the engine's
    // host arithmetic does (float32 arrays subtracted, then scaled in float64)
    for (size_t i = 0; i < N; ++i) {
        if (e->kinarr[i]) continue;
        for (int a = 0; a < 3; ++a) {
            const float dv = after[4 * i + a] - before[4 * i + a];
            f3[3 * i + a] = e->M[i] * (double)dv / e->force_dt;
        }
    }
    return B2C_OK;
}

extern "C" int32_t b2c_state_save(void *h, void *blob, size_t *size)
{
    Engine *e = engine(h);
    if (!e || !size) {
        b2c::set_error("b2c_state_save: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    int rc = ensure_built(e);
    if (rc) return rc;
    const std::vector<Section> secs = sections(e);
    size_t need = sizeof(BlobHead);
    for (const Section &s : secs) need += s.bytes;
    if (!blob) {
        *size = need;
        return B2C_OK;
    }
    if (*size < need) {
        b2c::set_error("b2c_state_save: blob of %zu bytes, %zu needed", *size, need);
        *size = need;
        return B2C_EARG;
    }
    if ((rc = sync_last(e, "b2c_state_save"))) return rc;
    BlobHead hd{};
    std::memcpy(hd.magic, kMagic, 8);
    hd.version = 1, hd.n = e->N, hd.cand_cap = e->cand_cap, hd.kept_cap = e->kept_cap, hd.pcap = e->pcap;
    hd.kslots = kRecSlots, hd.has_force = e->has_force ? 1 : 0, hd.force_dt = e->force_dt, hd.bytes = need;
    char *p = static_cast<char *>(blob);
    std::memcpy(p, &hd, sizeof(hd));
    p += sizeof(hd);
    for (const Section &s : secs) {
        cudaError_t ce = cudaMemcpy(p, s.ptr, s.bytes, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return cuda_fail("b2c_state_save", ce);
        p += s.bytes;
    }
    *size = need;
    return B2C_OK;
}

extern "C" int32_t b2c_state_load(void *h, const void *blob, size_t size)
{
    Engine *e = engine(h);
    if (!e || !blob || size < sizeof(BlobHead)) {
        b2c::set_error("b2c_state_load: bad argument");
        return B2C_EARG;
    }
    DeviceGuard dg(e->cfg.device);
    int rc = ensure_built(e);
    if (rc) return rc;
    BlobHead hd;
    std::memcpy(&hd, blob, sizeof(hd));
    const std::vector<Section> secs = sections(e);
    size_t need = sizeof(BlobHead);
    for (const Section &s : secs) need += s.bytes;
    if (std::memcmp(hd.magic, kMagic, 8) != 0 || hd.version != 1 || hd.n != e->N || hd.cand_cap != e->cand_cap ||
        hd.kept_cap != e->kept_cap || hd.pcap != e->pcap || hd.kslots != kRecSlots || hd.bytes != need ||
        size < need) {
        b2c::set_error("b2c_state_load: the blob does not match this engine's bodies and capacities");
        return B2C_EARG;
    }
    if ((rc = header_wait(e)) || (rc = sync_last(e, "b2c_state_load"))) return rc;
    const char *p = static_cast<const char *>(blob) + sizeof(hd);
    for (const Section &s : secs) {
        cudaError_t ce = cudaMemcpy(s.ptr, p, s.bytes, cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return cuda_fail("b2c_state_load", ce);
        p += s.bytes;
    }
    // host mirrors of the kinematic flags and the header
    std::vector<int32_t> kin(e->N);
    cudaError_t ce;
    if (e->N && (ce = cudaMemcpy(kin.data(), e->kin_d, 4 * (size_t)e->N, cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail("b2c_state_load", ce);
    if ((ce = cudaMemcpy(e->hdr_host, e->header, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail("b2c_state_load", ce);
    // the blob's flags hold in both directions: a body made kinematic after the save is dynamic
    // again, with its mass from the build
    for (int i = 0; i < e->N; ++i) {
        e->kinarr[i] = e->kin[i] = kin[i] ? 1 : 0;
        e->M[i] = kin[i] ? INFINITY : e->M0[i];
    }
    e->has_force = hd.has_force != 0;
    e->force_dt = hd.force_dt;
    return B2C_OK;
}

extern "C" int32_t b2c_destroy(void **h)
{
    if (!h) {
        b2c::set_error("b2c_destroy: bad argument");
        return B2C_EARG;
    }
    Engine *e = engine(*h);
    if (e) {
        if (e->built) {
            DeviceGuard dg(e->cfg.device);
            if (e->last) cudaStreamSynchronize(e->last);
            release(e);
        }
        delete e;
    }
    *h = nullptr;
    return B2C_OK;
}
