// Box engine contact generation: body-AABB broadphase and the box/plane + box/box narrowphase
// of the reference's BoxWorld (src/motion_engine/ncp/ncp_gpu.py:1097-1227, 1273-1280), feeding
// the coloured pair-chunk solve.
//
// The narrowphase runs in float64, one thread per candidate pair, in the reference's order of
// operations (quaternion -> matrix, 6 face axes with the face-preference tolerances, 9 edge
// axes, edge-edge single point or reference/incident face clipping with Sutherland-Hodgman,
// <= 4 deepest points).  Contacts are written to fixed per-candidate slots, so their order --
// pairs ascending in (a, b), the ground first, feature order inside a pair -- is a pure
// function of the state: no sort is needed and the step is deterministic.
#include "b2c_common.cuh"
#include "b2c_sat.cuh"

namespace b2c {

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s);
int body_predict_substep(const b2c_bodies *b, float dt, float *vgrav, bool clear_pseudo, cudaStream_t s);
int body_integrate(const b2c_bodies *b, float dt, cudaStream_t s);
int color_pairs(const b2c_bodies *b, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p, cudaStream_t s);
int color_solve(const b2c_bodies *b, b2c_contacts *kept, b2c_pairs *pr, b2c_header *hdr, const b2c_color_params *p,
                float dt, cudaStream_t s);
int warm_store(const b2c_contacts *kept, const int64_t *kept_keys, b2c_warm *warm, const b2c_header *hdr, int use,
               cudaStream_t s);

constexpr int kMaxBoxCandidates = 64;  // candidate partners of one body
constexpr int kSlots = 8;              // contacts of one candidate (a box on the ground: <= 8 corners)

// the float64 narrowphase (box_plane, box_box) lives in b2c_sat.cuh; here its float32 inputs
// ---------------------------------------------------------------------------------------------
// broadphase
// ---------------------------------------------------------------------------------------------
struct BoxGrid {
    int dx, dy, dz;
    float inv;
    const int *scene;  // scene of each body (NULL: one scene)
};
__device__ __forceinline__ int bwrap(int a, int m)
{
    int r = a % m;
    return r < 0 ? r + m : r;
}
__device__ __forceinline__ int bcell(float x, float inv) { return (int)floorf(x * inv); }
// bucket of a cell; in a batch the scene shifts it (the 27 buckets of a query stay distinct, and
// scenes that overlap in space mostly fall into different buckets)
__device__ __forceinline__ int bbucket(const BoxGrid &g, int ix, int iy, int iz, int sc)
{
    const int nb = g.dx * g.dy * g.dz;
    const int b = (bwrap(ix, g.dx) * g.dy + bwrap(iy, g.dy)) * g.dz + bwrap(iz, g.dz);
    return sc ? (int)(((long long)b + (long long)sc * 40503LL) % nb) : b;
}
__device__ __forceinline__ int scene_of(const BoxGrid &g, int i) { return g.scene ? g.scene[i] : 0; }
// bounding-sphere radius of a box, float64 from the float32 half extents
__device__ __forceinline__ double bound_radius(float4 hf)
{
    const double x = hf.x, y = hf.y, z = hf.z;
    return sqrt((x * x + y * y) + z * z);
}
// the pair test of the box engine: a pair is a candidate when its bounding spheres are at most
// the margin apart, |xb - xa|^2 <= (ra + rb + margin)^2 in float64.  Every face contact passes
// it (a kept face point is a point of B at distance < margin from A); it leaves out the
// edge-edge points that the 15-axis test alone can report for boxes whose closest features are
// two vertices farther than the margin apart.
__device__ __forceinline__ bool sphere_pair(f3 xa, double ra, f3 xb, double rb, double margin)
{
    const double dx = (double)xb.x - (double)xa.x, dy = (double)xb.y - (double)xa.y, dz = (double)xb.z - (double)xa.z;
    const double rr = (ra + rb) + margin;
    return (dx * dx + dy * dy) + dz * dz <= rr * rr;
}

__global__ void k_box_cells(int n, const float *__restrict__ xc, BoxGrid g, int *__restrict__ bucket,
                            int *__restrict__ count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const f3 x = ld3(xc, i);
    const int b = bbucket(g, bcell(x.x, g.inv), bcell(x.y, g.inv), bcell(x.z, g.inv), scene_of(g, i));
    bucket[i] = b;
    atomicAdd(count + b, 1);
}
__global__ void k_box_scatter(int n, const int *__restrict__ bucket, const int *__restrict__ start,
                              int *__restrict__ cursor, int *__restrict__ sorted)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int b = bucket[i];
    sorted[start[b] + atomicAdd(cursor + b, 1)] = i;
}

// a box can touch the ground only if its lowest bounding-sphere point is below the margin
// (box_plane decides; this test only has to keep every box that has a corner below it)
__device__ __forceinline__ bool ground_candidate(int i, const float *__restrict__ xc, const float *__restrict__ half,
                                                 float margin)
{
    return (double)ld3(xc, i).z - bound_radius(ld4(half, i)) < (double)margin + 1e-9;
}

// One warp per body i: lane l < 27 holds the bucket range of neighbour cell l; the ranges are
// flattened by a warp prefix sum, and the lanes walk the flat list 32 entries at a time, so the
// dependent loads of one body's candidates overlap.  f(j, pass) is called by every lane of every
// iteration (pass = j is a partner of i: j > i and the sphere test holds), uniformly per warp.
template <class F>
__device__ __forceinline__ void warp_box_neighbors(int i, const float *__restrict__ xc, const float *__restrict__ half,
                                                   const int *__restrict__ start, const int *__restrict__ sorted,
                                                   const BoxGrid &g, float margin, F &&f)
{
    const int lane = threadIdx.x & 31;
    const f3 xi = ld3(xc, i);
    const double ri = bound_radius(ld4(half, i));
    const int cx = bcell(xi.x, g.inv), cy = bcell(xi.y, g.inv), cz = bcell(xi.z, g.inv);
    const int si = scene_of(g, i);
    int lo = 0, cnt = 0;
    if (lane < 27) {
        const int b = bbucket(g, cx + lane % 3 - 1, cy + (lane / 3) % 3 - 1, cz + lane / 9 - 1, si);
        lo = start[b];
        cnt = start[b + 1] - lo;
    }
    int incl = cnt;  // inclusive prefix over lanes
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - cnt;
    for (int base = 0; base < total; base += 32) {
        const int k = base + lane;
        // the cell of flat entry k: the last lane whose exclusive prefix is <= k
        int cell = 0;
        for (int l = 1; l < 27; ++l) cell = (__shfl_sync(0xffffffffu, excl, l) <= k) ? l : cell;
        const int t = __shfl_sync(0xffffffffu, lo, cell) + (k - __shfl_sync(0xffffffffu, excl, cell));
        bool pass = false;
        int j = -1;
        if (k < total) {
            j = sorted[t];
            pass = j > i && scene_of(g, j) == si && sphere_pair(xi, ri, ld3(xc, j), bound_radius(ld4(half, j)), margin);
        }
        f(j, pass);
    }
}

constexpr int kBroadWarps = 4;  // warps (bodies) per CTA of the broadphase kernels

__global__ void __launch_bounds__(32 * kBroadWarps)
    k_box_cand_count(int n, const float *__restrict__ xc, const float *__restrict__ half,
                     const int *__restrict__ start, const int *__restrict__ sorted, BoxGrid g, float margin,
                     int *__restrict__ count, b2c_header *hdr)
{
    const int i = blockIdx.x * kBroadWarps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (blockIdx.x == 0 && threadIdx.x == 0) count[n] = 0;
    if (i >= n) return;  // warp-uniform
    int c = 0;
    warp_box_neighbors(i, xc, half, start, sorted, g, margin,
                       [&](int, bool pass) { c += __popc(__ballot_sync(0xffffffffu, pass)); });
    if (lane == 0) {
        if (c > kMaxBoxCandidates) {
            atomicOr(&hdr->error, B2C_ERR_NEIGHBOR_OVERFLOW);
            c = kMaxBoxCandidates;
        }
        count[i] = c + (ground_candidate(i, xc, half, margin) ? 1 : 0);
    }
}

__global__ void __launch_bounds__(32 * kBroadWarps)
    k_box_cand_emit(int n, const float *__restrict__ xc, const float *__restrict__ half,
                    const int *__restrict__ start, const int *__restrict__ sorted, BoxGrid g, float margin,
                    const int *__restrict__ offset, int cap, int *__restrict__ ca, int *__restrict__ cb,
                    b2c_header *hdr)
{
    __shared__ int s_js[kBroadWarps][kMaxBoxCandidates];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kBroadWarps + w;
    if (blockIdx.x == 0 && threadIdx.x == 0 && offset[n] > cap) atomicOr(&hdr->error, B2C_ERR_PAIR_OVERFLOW);
    if (i >= n) return;  // warp-uniform
    int m = 0;  // partners collected so far (warp-uniform)
    warp_box_neighbors(i, xc, half, start, sorted, g, margin, [&](int j, bool pass) {
        const unsigned bal = __ballot_sync(0xffffffffu, pass);
        const int pos = m + __popc(bal & ((1u << lane) - 1u));
        if (pass && pos < kMaxBoxCandidates) s_js[w][pos] = j;
        m += __popc(bal);
    });
    __syncwarp();
    m = min(m, kMaxBoxCandidates);
    int k = offset[i];
    if (ground_candidate(i, xc, half, margin)) {
        if (lane == 0 && k < cap) {
            ca[k] = i;
            cb[k] = -1;
        }
        ++k;
    }
    // ascending partner order: each entry's rank is the number of smaller entries (ids are unique)
    for (int e = lane; e < m; e += 32) {
        const int j = s_js[w][e];
        int rank = 0;
        for (int q = 0; q < m; ++q) rank += s_js[w][q] < j ? 1 : 0;
        if (k + rank < cap) {
            ca[k + rank] = i;
            cb[k + rank] = j;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// narrowphase per candidate, compaction into kept contacts and pairs
// ---------------------------------------------------------------------------------------------
__global__ void k_box_narrow(const int *__restrict__ cand_offset, int nbodies, int cap, const int *__restrict__ ca,
                             const int *__restrict__ cb, const float *__restrict__ xc, const float *__restrict__ q,
                             const float *__restrict__ half, float margin, float *__restrict__ slot_p,
                             float *__restrict__ slot_n, int *__restrict__ slot_f, int *__restrict__ cont_count,
                             int *__restrict__ pair_flag)
{
    const int nc = min(cand_offset[nbodies], cap);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        cont_count[nc] = 0;
        pair_flag[nc] = 0;
    }
    for (int c = tid; c < nc; c += gridDim.x * blockDim.x) {
        const int a = ca[c], b = cb[c];
        double4 pts[kSlots];
        int fid[kSlots];
        d3 nrm = D3(0.0, 0.0, 1.0);
        int m;
        if (b < 0) m = box_plane(ld4(half, a), ld4(xc, a), ld4(q, a), margin, pts, fid);
        else m = box_box(ld4(half, a), ld4(xc, a), ld4(q, a), ld4(half, b), ld4(xc, b), ld4(q, b), margin, pts, nrm, fid);
        for (int k = 0; k < m; ++k) {
            st4(slot_p, c * kSlots + k, make_float4((float)pts[k].x, (float)pts[k].y, (float)pts[k].z, (float)pts[k].w));
            slot_f[c * kSlots + k] = fid[k];
        }
        st4(slot_n, c, make_float4((float)nrm.x, (float)nrm.y, (float)nrm.z, 0.0f));
        cont_count[c] = m;
        pair_flag[c] = m > 0 ? 1 : 0;
    }
}

// feature key of a box contact: pair key (a, b+1) then the feature id; ascending in pair order,
// then in feature order, as the kept contacts are laid out
__device__ __forceinline__ long long box_key(int a, int b, int f, int nbodies)
{
    return ((long long)a * (nbodies + 1) + (long long)(b + 1)) * 256 + f;
}

__global__ void k_box_compact(const int *__restrict__ cand_offset, int nbodies, int cap, const int *__restrict__ ca,
                              const int *__restrict__ cb, const float *__restrict__ slot_p,
                              const float *__restrict__ slot_n, const int *__restrict__ slot_f,
                              const int *__restrict__ cont_count, const int *__restrict__ cont_offset,
                              const int *__restrict__ pair_offset, b2c_contacts kept, long long *__restrict__ keys,
                              b2c_pairs pr, int use_warm, const long long *__restrict__ wkeys,
                              const float *__restrict__ wimp, const int *__restrict__ wn_ptr, b2c_header *hdr)
{
    const int nc = min(cand_offset[nbodies], cap);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) {
        const int C = cont_offset[nc], P = pair_offset[nc];
        const int Cs = C < kept.capacity ? C : kept.capacity, Ps = P < pr.capacity ? P : pr.capacity;
        hdr->n_raw = C;
        hdr->n_contacts = Cs;
        hdr->n_kept = Cs;
        hdr->n_pairs = Ps;
        if (C > kept.capacity) atomicOr(&hdr->error, B2C_ERR_CONTACT_OVERFLOW);
        if (P > pr.capacity) atomicOr(&hdr->error, B2C_ERR_PAIR_OVERFLOW);
    }
    const int wn = use_warm ? *wn_ptr : 0;
    for (int c = tid; c < nc; c += gridDim.x * blockDim.x) {
        const int m = cont_count[c];
        if (m == 0) continue;
        const int a = ca[c], b = cb[c];
        const int p = pair_offset[c], base = cont_offset[c];
        if (p >= pr.capacity || base + m > kept.capacity) continue;
        pr.pbi[p] = a;
        pr.pbj[p] = b;
        pr.kcount[p] = m;
        const float4 n4 = ld4(slot_n, c);
        for (int k = 0; k < m; ++k) {
            const int d = base + k;
            const float4 ps = ld4(slot_p, c * kSlots + k);
            const int f = slot_f[c * kSlots + k];
            const long long key = box_key(a, b, f, nbodies);
            kept.bi[d] = a;
            kept.bj[d] = b;
            st4(kept.pA, d, make_float4(ps.x, ps.y, ps.z, -ps.w));  // depth = -gap
            st4(kept.pB, d, make_float4(ps.x, ps.y, ps.z, 0.0f));
            st4(kept.n, d, n4);
            kept.fa[d] = a;
            kept.fb[d] = f;
            keys[d] = key;
            pr.pidx[d] = d;
            float4 im = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (wn > 0) {  // warm start: binary search in the previous step's (sorted) keys
                int lo = 0, hi = wn - 1;
                while (lo <= hi) {
                    const int mid = (lo + hi) / 2;
                    const long long km = wkeys[mid];
                    if (km == key) {
                        const float4 w4 = ld4(wimp, mid);
                        im = make_float4(w4.x, w4.y, w4.z, 0.0f);
                        break;
                    }
                    if (km < key) lo = mid + 1;
                    else hi = mid - 1;
                }
            }
            st4(kept.imp, d, im);
        }
    }
}

__global__ void k_pstart_from_offsets(const int *__restrict__ cand_offset, int nbodies, int cap,
                                      const int *__restrict__ cont_count, const int *__restrict__ cont_offset,
                                      const int *__restrict__ pair_offset, int *__restrict__ pstart, int pcap)
{
    const int nc = min(cand_offset[nbodies], cap);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x)
        if (cont_count[c] > 0 && pair_offset[c] < pcap) pstart[pair_offset[c]] = cont_offset[c];
}

// ---------------------------------------------------------------------------------------------
// host drivers
// ---------------------------------------------------------------------------------------------
static BoxGrid box_grid_of(const b2c_boxes *bx)
{
    return BoxGrid{bx->dim_x, bx->dim_y, bx->dim_z, 1.0f / bx->cell, bx->scene};
}

int box_candidates(const b2c_bodies *b, b2c_boxes *bx, b2c_header *hdr, cudaStream_t s)
{
    const int n = b->n;
    const int nbk = bx->dim_x * bx->dim_y * bx->dim_z;
    const BoxGrid g = box_grid_of(bx);
    cudaMemsetAsync(bx->cursor, 0, sizeof(int) * (size_t)(nbk + 1), s);
    if (n > 0) k_box_cells<<<blocks_for(n), kThreads, 0, s>>>(n, b->xc, g, bx->bucket, bx->cursor);
    int rc = check_launch("box_cells");
    if (rc) return rc;
    if ((rc = exclusive_scan(bx->cursor, bx->start, nbk + 1, nullptr, bx->scan_tmp, s))) return rc;
    cudaMemsetAsync(bx->cursor, 0, sizeof(int) * (size_t)nbk, s);
    if (n > 0) k_box_scatter<<<blocks_for(n), kThreads, 0, s>>>(n, bx->bucket, bx->start, bx->cursor, bx->sorted);
    const int bgrid = std::max(1, (n + kBroadWarps - 1) / kBroadWarps);
    k_box_cand_count<<<bgrid, 32 * kBroadWarps, 0, s>>>(n, b->xc, bx->half, bx->start, bx->sorted, g, bx->margin,
                                                         bx->cand_count, hdr);
    if ((rc = check_launch("box_cand_count"))) return rc;
    if ((rc = exclusive_scan(bx->cand_count, bx->cand_offset, n + 1, nullptr, bx->scan_tmp, s))) return rc;
    k_box_cand_emit<<<bgrid, 32 * kBroadWarps, 0, s>>>(n, b->xc, bx->half, bx->start, bx->sorted, g, bx->margin,
                                                        bx->cand_offset, bx->cand_capacity, bx->cand_a, bx->cand_b,
                                                        hdr);
    return check_launch("box_cand_emit");
}

int box_contacts(const b2c_bodies *b, b2c_boxes *bx, b2c_contacts *kept, int64_t *kept_keys, b2c_pairs *pr,
                 const b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, cudaStream_t s)
{
    const int n = b->n, cap = bx->cand_capacity;
    const int cgrid = std::min(blocks_for(cap, 128), kSMs * 16);
    k_box_narrow<<<cgrid, 128, 0, s>>>(bx->cand_offset, n, cap, bx->cand_a, bx->cand_b, b->xc, b->q, bx->half,
                                       bx->margin, bx->slot_p, bx->slot_n, bx->slot_f, bx->cont_count, bx->pair_flag);
    int rc = check_launch("box_narrow");
    if (rc) return rc;
    // candidate counts beyond the live candidates read as zero (dn)
    if ((rc = exclusive_scan(bx->cont_count, bx->cont_offset, cap + 1, bx->cand_offset + n, bx->scan_tmp, s)))
        return rc;
    if ((rc = exclusive_scan(bx->pair_flag, bx->pair_offset, cap + 1, bx->cand_offset + n, bx->scan_tmp, s)))
        return rc;
    k_box_compact<<<cgrid, kThreads, 0, s>>>(bx->cand_offset, n, cap, bx->cand_a, bx->cand_b, bx->slot_p, bx->slot_n,
                                             bx->slot_f, bx->cont_count, bx->cont_offset, bx->pair_offset, *kept,
                                             reinterpret_cast<long long *>(kept_keys), *pr,
                                             (p->flags & B2C_COLOR_WARM_START) ? 1 : 0,
                                             reinterpret_cast<const long long *>(warm->keys), warm->imp, warm->n, hdr);
    k_pstart_from_offsets<<<cgrid, kThreads, 0, s>>>(bx->cand_offset, n, cap, bx->cont_count, bx->cont_offset,
                                                     bx->pair_offset, pr->pstart, pr->capacity);
    return check_launch("box_contacts");
}

__global__ void k_narrow_test(int n, const float *a_half, const float *a_x, const float *a_q, const float *b_half,
                              const float *b_x, const float *b_q, float margin, double *pts, double *nrm, int *fid,
                              int *count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double4 p[kSlots];
    int f[kSlots];
    d3 nn = D3(0.0, 0.0, 1.0);
    int m;
    if (!b_half) m = box_plane(ld4(a_half, i), ld4(a_x, i), ld4(a_q, i), margin, p, f);
    else m = box_box(ld4(a_half, i), ld4(a_x, i), ld4(a_q, i), ld4(b_half, i), ld4(b_x, i), ld4(b_q, i), margin, p,
                     nn, f);
    for (int k = 0; k < m; ++k) {
        pts[(i * kSlots + k) * 4 + 0] = p[k].x;
        pts[(i * kSlots + k) * 4 + 1] = p[k].y;
        pts[(i * kSlots + k) * 4 + 2] = p[k].z;
        pts[(i * kSlots + k) * 4 + 3] = p[k].w;
        fid[i * kSlots + k] = f[k];
    }
    nrm[4 * i + 0] = nn.x;
    nrm[4 * i + 1] = nn.y;
    nrm[4 * i + 2] = nn.z;
    nrm[4 * i + 3] = 0.0;
    count[i] = m;
}

}  // namespace b2c

static bool boxes_ok(const b2c_boxes *bx, int n)
{
    return bx && bx->n == n && bx->half && bx->dim_x >= 8 && bx->dim_y >= 8 && bx->dim_z >= 8 && bx->cell > 0.0f &&
           bx->cand_capacity >= 0 && bx->bucket && bx->start && bx->cursor && bx->sorted && bx->cand_count &&
           bx->cand_offset && bx->cand_a && bx->cand_b && bx->cont_count && bx->cont_offset && bx->pair_flag &&
           bx->pair_offset && bx->slot_p && bx->slot_n && bx->slot_f && bx->scan_tmp;
}

extern "C" int32_t b2c_box_candidates(const b2c_bodies *b, b2c_boxes *bx, b2c_header *hdr, b2c_stream s)
{
    if (!b || !hdr || !boxes_ok(bx, b->n)) {
        b2c::set_error("b2c_box_candidates: bad argument");
        return B2C_EARG;
    }
    return b2c::box_candidates(b, bx, hdr, b2c::stream_of(s));
}

extern "C" int32_t b2c_box_contacts(const b2c_bodies *b, b2c_boxes *bx, b2c_contacts *kept, int64_t *kept_keys,
                                    b2c_pairs *pr, const b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p,
                                    b2c_stream s)
{
    if (!b || !hdr || !boxes_ok(bx, b->n) || !kept || !kept_keys || !pr || !warm || !p) {
        b2c::set_error("b2c_box_contacts: bad argument");
        return B2C_EARG;
    }
    return b2c::box_contacts(b, bx, kept, kept_keys, pr, warm, hdr, p, b2c::stream_of(s));
}

extern "C" int32_t b2c_box_substep(const b2c_bodies *b, b2c_boxes *bx, b2c_contacts *kept, int64_t *kept_keys,
                                   b2c_pairs *pr, b2c_warm *warm, b2c_header *hdr, const b2c_color_params *p, float dt,
                                   float *vgrav, b2c_stream s)
{
    if (!b || !hdr || !boxes_ok(bx, b->n) || !kept || !kept_keys || !pr || !warm || !p || !vgrav || !(dt > 0.0f) ||
        !pr->barrier || !pr->rec || pr->kslots < b2c::kSlots || warm->capacity < kept->capacity) {
        b2c::set_error("b2c_box_substep: bad argument");
        return B2C_EARG;
    }
    cudaStream_t st = b2c::stream_of(s);
    int rc;
    if ((rc = b2c::body_predict_substep(b, dt, vgrav, true, st))) return rc;
    if ((rc = b2c::box_candidates(b, bx, hdr, st))) return rc;
    if ((rc = b2c::box_contacts(b, bx, kept, kept_keys, pr, warm, hdr, p, st))) return rc;
    if ((rc = b2c::color_pairs(b, pr, hdr, p, st))) return rc;
    if ((rc = b2c::color_solve(b, kept, pr, hdr, p, dt, st))) return rc;
    if ((rc = b2c::warm_store(kept, kept_keys, warm, hdr, (p->flags & B2C_COLOR_WARM_START) ? 1 : 0, st))) return rc;
    return b2c::body_integrate(b, dt, st);
}

extern "C" int32_t b2c_box_narrowphase_test(int32_t n, const float *a_half, const float *a_x, const float *a_q,
                                            const float *b_half, const float *b_x, const float *b_q, float margin,
                                            double *pts, double *nrm, int32_t *fid, int32_t *count, b2c_stream s)
{
    if (n < 0 || !a_half || !a_x || !a_q || (b_half && (!b_x || !b_q)) || !pts || !nrm || !fid || !count) {
        b2c::set_error("b2c_box_narrowphase_test: bad argument");
        return B2C_EARG;
    }
    if (n == 0) return B2C_OK;
    b2c::k_narrow_test<<<b2c::blocks_for(n, 64), 64, 0, b2c::stream_of(s)>>>(n, a_half, a_x, a_q, b_half, b_x, b_q,
                                                                             margin, pts, nrm, fid, count);
    return b2c::check_launch("box_narrowphase_test");
}
