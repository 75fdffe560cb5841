// The float64 narrowphase of the box engines: box/plane and box/box contacts of the reference's
// BoxWorld (src/motion_engine/ncp/ncp_gpu.py:1089-1227), one candidate pair per call.
//
// The entry points take the boxes' half extents, centres and quaternions (x, y, z, w) as float4
// (the box engine's float32 state) or double4 (the float64 box world); either is widened to
// float64 on entry, so the float4 form gives the same bits as before it was a template.
#pragma once

#include "b2c_common.cuh"

namespace b2c {

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
template <class V4>
__device__ dR dquat_R(V4 qf)
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
__device__ inline void dface(d3 half, d3 x, const dR &R, int axis, double sgn, d3 *poly, d3 &n, d3 &c)
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
// _clip, ncp_gpu.py:1129-1145: Sutherland-Hodgman against |(p - c).ax| <= ha; poly holds 16.
// planes (optional): per vertex, the bit set of the three planes it lies on; a vertex made on
// the side s of this axis lies on the two planes its edge's ends share and on plane code0 + si.
__device__ inline int dclip(d3 *poly, int n, d3 c, d3 ax, double ha, int *planes = nullptr, int code0 = 0)
{
    d3 out[16];
    int pout[16];
    for (int si = 0; si < 2; ++si) {
        const double s = si == 0 ? 1.0 : -1.0;
        int m = 0;
        for (int i = 0; i < n; ++i) {
            const d3 p = poly[i], q = poly[(i + 1) % n];
            const double dp = s * ddot(dsub(p, c), ax) - ha;
            const double dq = s * ddot(dsub(q, c), ax) - ha;
            if (dp <= 0 && m < 16) {
                if (planes) pout[m] = planes[i];
                out[m++] = p;
            }
            if (dp * dq < 0 && m < 16) {
                if (planes) pout[m] = (planes[i] & planes[(i + 1) % n]) | (1 << (code0 + si));
                out[m++] = dadd(p, dscale(dsub(q, p), dp / (dp - dq)));
            }
        }
        for (int i = 0; i < m; ++i) {
            poly[i] = out[i];
            if (planes) planes[i] = pout[i];
        }
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
template <class V4>
__device__ int box_plane(V4 hf, V4 xf, V4 qf, double margin, double4 *pts, int *fid)
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
// attach (optional, one per point): what the contacts move with -- bits 0-1 the points (0: box A,
// 1: box B, 2: halfway between a corner of each), bits 2-3 the normal (1: box A, 2: box B); for a
// face contact also the three planes the point lies on (bits 4-13, kAttachPlane*: the incident
// box's faces 2 a + (sign < 0), the reference face's sides 6 + 2 (0: axis j, 1: axis k) +
// (sign < 0)), the reference axis (bits 14-15) and bit 16 set when A is the reference box.
constexpr int kAttachPlaneShift = 4, kAttachAxisShift = 14, kAttachRefA = 1 << 16;
template <class V4>
__device__ int box_box(V4 haf, V4 xaf, V4 qaf, V4 hbf, V4 xbf, V4 qbf, double margin, double4 *pts, d3 &nrm, int *fid,
                       int *attach = nullptr)
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
        if (attach) attach[0] = 2;
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
    const int ia = mmin / 2, isg = mmin % 2;
    dface(ihalf, ix, iR, ia, isg == 0 ? 1.0 : -1.0, poly, in_n, in_c);
    // the incident face's corners c +-u +-v (dface) lie on the face and on two of its sides
    const int ja = (ia + 1) % 3, ka = (ia + 2) % 3, fbit = 1 << (2 * ia + isg);
    int planes[16] = {fbit | (1 << (2 * ja)) | (1 << (2 * ka)), fbit | (1 << (2 * ja + 1)) | (1 << (2 * ka)),
                      fbit | (1 << (2 * ja + 1)) | (1 << (2 * ka + 1)), fbit | (1 << (2 * ja)) | (1 << (2 * ka + 1))};
    const int j = (raxis + 1) % 3, k = (raxis + 2) % 3;
    int np_ = dclip(poly, 4, rc, rR.col[j], dget(rhalf, j), planes, 6);
    if (!np_) return 0;
    np_ = dclip(poly, np_, rc, rR.col[k], dget(rhalf, k), planes, 8);
    if (!np_) return 0;
    double gs[16];
    d3 ps[16];
    int pl[16];
    int m = 0;
    for (int i = 0; i < np_; ++i) {
        const double g = ddot(dsub(poly[i], rc), rn);
        if (g < margin) {
            gs[m] = g;
            ps[m] = poly[i];
            pl[m] = planes[i];
            ++m;
        }
    }
    if (m == 0) return 0;
    if (m > 4) {  // stable sort by gap, keep the 4 deepest (sorted(...)[:4])
        for (int a = 1; a < m; ++a) {
            const double gv = gs[a];
            const d3 pv = ps[a];
            const int lv = pl[a];
            int b = a - 1;
            while (b >= 0 && gs[b] > gv) {
                gs[b + 1] = gs[b];
                ps[b + 1] = ps[b];
                pl[b + 1] = pl[b];
                --b;
            }
            gs[b + 1] = gv;
            ps[b + 1] = pv;
            pl[b + 1] = lv;
        }
        m = 4;
    }
    const int base = (raxis * 2 + (rsgn > 0 ? 0 : 1)) * 8;
    for (int i = 0; i < m; ++i) {
        pts[i] = make_double4(ps[i].x, ps[i].y, ps[i].z, gs[i]);
        fid[i] = base + i;
        // points on the incident box, the normal on the reference box
        if (attach)
            attach[i] = (refA ? (1 | (1 << 2)) : (0 | (2 << 2))) | (pl[i] << kAttachPlaneShift) |
                        (raxis << kAttachAxisShift) | (refA ? kAttachRefA : 0);
    }
    nrm = nBA;
    return m;
}

}  // namespace b2c
