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

// ---------------------------------------------------------------------------------------------
// float64 narrowphase
// ---------------------------------------------------------------------------------------------
struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 D3(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 dadd(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 dsub(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 dscale(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double ddot(d3 a, d3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ d3 dcross(d3 a, d3 b)
{
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dget(d3 a, int i) { return i == 0 ? a.x : i == 1 ? a.y : a.z; }

struct dR {  // rotation by columns R[:, i]
    d3 col[3];
};
// _quat_to_R, ncp_gpu.py:1089-1093
__device__ dR dquat_R(float4 qf)
{
    const double x = qf.x, y = qf.y, z = qf.z, w = qf.w;
    const double r00 = 1 - 2 * (y * y + z * z), r01 = 2 * (x * y - z * w), r02 = 2 * (x * z + y * w);
    const double r10 = 2 * (x * y + z * w), r11 = 1 - 2 * (x * x + z * z), r12 = 2 * (y * z - x * w);
    const double r20 = 2 * (x * z - y * w), r21 = 2 * (y * z + x * w), r22 = 1 - 2 * (x * x + y * y);
    dR R;
    R.col[0] = D3(r00, r10, r20);
    R.col[1] = D3(r01, r11, r21);
    R.col[2] = D3(r02, r12, r22);
    return R;
}
__device__ __forceinline__ d3 dR_apply(const dR &R, d3 a)
{
    return D3((R.col[0].x * a.x + R.col[1].x * a.y) + R.col[2].x * a.z,
              (R.col[0].y * a.x + R.col[1].y * a.y) + R.col[2].y * a.z,
              (R.col[0].z * a.x + R.col[1].z * a.y) + R.col[2].z * a.z);
}
__device__ __forceinline__ d3 dRT_apply(const dR &R, d3 a) { return D3(ddot(R.col[0], a), ddot(R.col[1], a), ddot(R.col[2], a)); }
// _corners, ncp_gpu.py:1112-1117: corner k = x + R (s * half), s from k = 4 ix + 2 iy + iz
__device__ __forceinline__ d3 dcorner(d3 half, d3 x, const dR &R, int k)
{
    const d3 s = D3((k & 4) ? 1.0 : -1.0, (k & 2) ? 1.0 : -1.0, (k & 1) ? 1.0 : -1.0);
    return dadd(x, dR_apply(R, D3(s.x * half.x, s.y * half.y, s.z * half.z)));
}
// _face_corners, ncp_gpu.py:1120-1126
__device__ void dface(d3 half, d3 x, const dR &R, int axis, double sgn, d3 *poly, d3 &n, d3 &c)
{
    const int i = axis, j = (axis + 1) % 3, k = (axis + 2) % 3;
    n = dscale(R.col[i], sgn);
    c = dadd(x, dscale(n, dget(half, i)));
    const d3 u = dscale(R.col[j], dget(half, j)), v = dscale(R.col[k], dget(half, k));
    poly[0] = dadd(dadd(c, u), v);
    poly[1] = dadd(dsub(c, u), v);
    poly[2] = dsub(dsub(c, u), v);
    poly[3] = dsub(dadd(c, u), v);
}
// _clip, ncp_gpu.py:1129-1145: Sutherland-Hodgman against |(p - c).ax| <= ha; poly holds 16
__device__ int dclip(d3 *poly, int n, d3 c, d3 ax, double ha)
{
    d3 out[16];
    for (int si = 0; si < 2; ++si) {
        const double s = si == 0 ? 1.0 : -1.0;
        int m = 0;
        for (int i = 0; i < n; ++i) {
            const d3 p = poly[i], q = poly[(i + 1) % n];
            const double dp = s * ddot(dsub(p, c), ax) - ha;
            const double dq = s * ddot(dsub(q, c), ax) - ha;
            if (dp <= 0 && m < 16) out[m++] = p;
            if (dp * dq < 0 && m < 16) out[m++] = dadd(p, dscale(dsub(q, p), dp / (dp - dq)));
        }
        for (int i = 0; i < m; ++i) poly[i] = out[i];
        n = m;
        if (n == 0) return 0;
    }
    return n;
}
// sep_of, ncp_gpu.py:1166-1170
__device__ __forceinline__ double dsep(d3 ax, d3 d, const dR &Ra, d3 ha, const dR &Rb, d3 hb, d3 &axo)
{
    const d3 a = dRT_apply(Ra, ax), b = dRT_apply(Rb, ax);
    const double ra = (fabs(a.x) * ha.x + fabs(a.y) * ha.y) + fabs(a.z) * ha.z;
    const double rb = (fabs(b.x) * hb.x + fabs(b.y) * hb.y) + fabs(b.z) * hb.z;
    const double proj = ddot(d, ax);
    axo = proj >= 0 ? ax : dscale(ax, -1.0);
    return fabs(proj) - (ra + rb);
}

// box_plane_contacts, ncp_gpu.py:1148-1154: corners below z = margin; normal +z, gap = z
__device__ int box_plane(float4 hf, float4 xf, float4 qf, double margin, double4 *pts, int *fid)
{
    const dR R = dquat_R(qf);
    const d3 half = D3(hf.x, hf.y, hf.z), x = D3(xf.x, xf.y, xf.z);
    int m = 0;
    for (int k = 0; k < 8; ++k) {
        const d3 c = dcorner(half, x, R, k);
        if (c.z < margin) {
            pts[m] = make_double4(c.x, c.y, c.z, c.z);
            fid[m] = k;
            ++m;
        }
    }
    return m;
}

// box_box_contacts, ncp_gpu.py:1157-1227: normal from B to A, <= 4 points
__device__ int box_box(float4 haf, float4 xaf, float4 qaf, float4 hbf, float4 xbf, float4 qbf, double margin,
                       double4 *pts, d3 &nrm, int *fid)
{
    const d3 ha = D3(haf.x, haf.y, haf.z), hb = D3(hbf.x, hbf.y, hbf.z);
    const d3 xa = D3(xaf.x, xaf.y, xaf.z), xb = D3(xbf.x, xbf.y, xbf.z);
    const dR Ra = dquat_R(qaf), Rb = dquat_R(qbf);
    const d3 d = dsub(xb, xa);
    bool fset = false, eset = false;
    double fsp = 0.0, esp = 0.0;
    int fkind = 0, fidx = 0, eidx = 0;
    d3 fax = D3(0, 0, 0), eax = D3(0, 0, 0);
    for (int kind = 0; kind < 2; ++kind) {
        const dR &R = kind == 0 ? Ra : Rb;
        for (int i = 0; i < 3; ++i) {
            d3 ax;
            const double sp = dsep(R.col[i], d, Ra, ha, Rb, hb, ax);
            if (sp > margin) return 0;
            const double better = (fset && kind == 1 && fkind == 0) ? 1e-4 : 1e-12;
            if (!fset || sp > fsp + better) {
                fsp = sp;
                fkind = kind;
                fidx = i;
                fax = ax;
                fset = true;
            }
        }
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const d3 cr = dcross(Ra.col[i], Rb.col[j]);
            const double nn = sqrt(ddot(cr, cr));
            if (nn <= 1e-6) continue;
            d3 ax;
            const double sp = dsep(dscale(cr, 1.0 / nn), d, Ra, ha, Rb, hb, ax);
            if (sp > margin) return 0;
            if (!eset || sp > esp + 1e-12) {
                esp = sp;
                eidx = 3 * i + j;
                eax = ax;
                eset = true;
            }
        }
    if (eset && esp > fsp + 1e-3) {  // genuine edge-edge: one point
        int ka = 0, kb = 0;
        double best_a = ddot(dcorner(ha, xa, Ra, 0), eax), best_b = ddot(dcorner(hb, xb, Rb, 0), eax);
        for (int k = 1; k < 8; ++k) {
            const double da = ddot(dcorner(ha, xa, Ra, k), eax), db = ddot(dcorner(hb, xb, Rb, k), eax);
            if (da > best_a) {
                best_a = da;
                ka = k;
            }
            if (db < best_b) {
                best_b = db;
                kb = k;
            }
        }
        const d3 p = dscale(dadd(dcorner(ha, xa, Ra, ka), dcorner(hb, xb, Rb, kb)), 0.5);
        pts[0] = make_double4(p.x, p.y, p.z, esp);
        nrm = dscale(eax, -1.0);
        fid[0] = 100 + eidx;
        return 1;
    }
    d3 rhalf, rx, ihalf, ix, nBA;
    const int raxis = fidx;
    double rsgn;
    const bool refA = fkind == 0;
    const dR &rR = refA ? Ra : Rb;
    const dR &iR = refA ? Rb : Ra;
    if (refA) {
        rhalf = ha;
        rx = xa;
        ihalf = hb;
        ix = xb;
        rsgn = ddot(Ra.col[raxis], fax) >= 0 ? 1.0 : -1.0;
        nBA = dscale(fax, -1.0);
    } else {
        rhalf = hb;
        rx = xb;
        ihalf = ha;
        ix = xa;
        rsgn = ddot(Rb.col[raxis], dscale(fax, -1.0)) >= 0 ? 1.0 : -1.0;
        nBA = fax;
    }
    d3 rpoly[4], rn, rc;
    dface(rhalf, rx, rR, raxis, rsgn, rpoly, rn, rc);
    int mmin = 0;
    double dmin = 0.0;
    for (int a = 0; a < 3; ++a)
        for (int sg = 0; sg < 2; ++sg) {
            const double v = ddot(dscale(iR.col[a], sg == 0 ? 1.0 : -1.0), rn);
            const int k = 2 * a + sg;
            if (k == 0 || v < dmin) {
                dmin = v;
                mmin = k;
            }
        }
    d3 poly[16], in_n, in_c;
    dface(ihalf, ix, iR, mmin / 2, (mmin % 2 == 0) ? 1.0 : -1.0, poly, in_n, in_c);
    const int j = (raxis + 1) % 3, k = (raxis + 2) % 3;
    int np_ = dclip(poly, 4, rc, rR.col[j], dget(rhalf, j));
    if (!np_) return 0;
    np_ = dclip(poly, np_, rc, rR.col[k], dget(rhalf, k));
    if (!np_) return 0;
    double gs[16];
    d3 ps[16];
    int m = 0;
    for (int i = 0; i < np_; ++i) {
        const double g = ddot(dsub(poly[i], rc), rn);
        if (g < margin) {
            gs[m] = g;
            ps[m] = poly[i];
            ++m;
        }
    }
    if (m == 0) return 0;
    if (m > 4) {  // stable sort by gap, keep the 4 deepest (sorted(...)[:4])
        for (int a = 1; a < m; ++a) {
            const double gv = gs[a];
            const d3 pv = ps[a];
            int b = a - 1;
            while (b >= 0 && gs[b] > gv) {
                gs[b + 1] = gs[b];
                ps[b + 1] = ps[b];
                --b;
            }
            gs[b + 1] = gv;
            ps[b + 1] = pv;
        }
        m = 4;
    }
    const int base = (raxis * 2 + (rsgn > 0 ? 0 : 1)) * 8;
    for (int i = 0; i < m; ++i) {
        pts[i] = make_double4(ps[i].x, ps[i].y, ps[i].z, gs[i]);
        fid[i] = base + i;
    }
    nrm = nBA;
    return m;
}

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
