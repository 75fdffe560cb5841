// The exact-cone box world on the device: the reference's BoxWorld substep
// (src/motion_engine/ncp/ncp_gpu.py:1237-1413) -- SAT contacts, build_scene, the NCP solve,
// integration -- for many independent scenes at once, in float64.
//
//   contacts   the box engine's broadphase (b2c_box_candidates, on a float32 mirror of the
//              centres: it only proposes candidate pairs, within the margin of their bounding
//              spheres) and the float64 narrowphase of b2c_sat.cuh on the float64 state, one
//              thread per candidate; contacts land in per-candidate slots and are compacted in
//              candidate order ((a, b) ascending, the ground first, feature order inside a pair),
//              so their keys ((a (N + 1) + b + 1) 256 + feature) ascend;
//   scene      build_scene (:1291-1330): the frame (n, t1, t2) of _basis (:1230-1234), the 3x6
//              blocks Ja = [D, r_a x D], Jb = -[D, r_b x D], the Baumgarte bias on the normal row
//              (gap / dt when open, -beta max(-gap - slop, 0) / dt when penetrating), per-body
//              Minv = [I / m, R Ib^-1 R^T] and v_free = [v + g dt, w] (kinematic bodies: zero
//              Minv, their prescribed velocity);
//   solve      the exact-cone NCP of ncp.cu on those arrays (b2c_ncp_setup / _color / _sweeps),
//              warm-started by contact key from the previous substep when asked;
//   integrate  x += v dt, q <- normalize(q + 0.5 (w, 0) q dt) (:1393-1398); kinematic bodies move
//              with their prescribed velocity.
//
// The adjoint of a substep (world_adjoint below) runs the same pieces backwards.
#include "b2c_common.cuh"
#include "b2c_sat.cuh"

namespace b2c {

int exclusive_scan(const int *in, int *out, int n, const int *dn, int *scratch, cudaStream_t s);
int box_candidates(const b2c_bodies *b, b2c_boxes *bx, b2c_header *hdr, cudaStream_t s);

namespace world {

constexpr int kSlots = 8;
constexpr double kG = 9.81, kBeta = 0.2, kSlop = 1e-4;

__device__ __forceinline__ double4 ld4d(const double *p, int i) { return reinterpret_cast<const double4 *>(p)[i]; }
__device__ __forceinline__ d3 ld3d(const double *p, int i) { return D3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st3d(double *p, int i, d3 v)
{
    p[3 * i] = v.x;
    p[3 * i + 1] = v.y;
    p[3 * i + 2] = v.z;
}

__global__ void k_mirror(int n, const double *__restrict__ x, float *__restrict__ xc32, double *__restrict__ x4,
                         const double *__restrict__ half, double *__restrict__ half4)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const d3 p = ld3d(x, i), h = ld3d(half, i);
    reinterpret_cast<float4 *>(xc32)[i] = make_float4((float)p.x, (float)p.y, (float)p.z, 0.0f);
    reinterpret_cast<double4 *>(x4)[i] = make_double4(p.x, p.y, p.z, 0.0);
    reinterpret_cast<double4 *>(half4)[i] = make_double4(h.x, h.y, h.z, 0.0);
}

__global__ void k_narrow(const int *__restrict__ cand_offset, int n, int cap, const int *__restrict__ ca,
                         const int *__restrict__ cb, const double *__restrict__ x4, const double *__restrict__ q,
                         const double *__restrict__ half4, double margin, double *__restrict__ slot_p,
                         double *__restrict__ slot_n, int *__restrict__ slot_f, int *__restrict__ cont_count)
{
    const int nc = min(cand_offset[n], cap);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) cont_count[nc] = 0;
    for (int c = tid; c < nc; c += gridDim.x * blockDim.x) {
        const int a = ca[c], b = cb[c];
        double4 pts[kSlots];
        int fid[kSlots], att[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0};  // ground: corners of box a, fixed normal
        d3 nrm = D3(0.0, 0.0, 1.0);
        int m;
        if (b < 0) m = box_plane(ld4d(half4, a), ld4d(x4, a), ld4d(q, a), margin, pts, fid);
        else m = box_box(ld4d(half4, a), ld4d(x4, a), ld4d(q, a), ld4d(half4, b), ld4d(x4, b), ld4d(q, b), margin, pts,
                         nrm, fid, att);
        for (int k = 0; k < m; ++k) {
            reinterpret_cast<double4 *>(slot_p)[c * kSlots + k] = pts[k];
            slot_f[c * kSlots + k] = fid[k] | (att[k] << 8);  // fid < 256
        }
        reinterpret_cast<double4 *>(slot_n)[c] = make_double4(nrm.x, nrm.y, nrm.z, 0.0);
        cont_count[c] = m;
    }
}

__global__ void k_emit(const int *__restrict__ cand_offset, int n, int cap, int max_contacts, const int *__restrict__ ca,
                       const int *__restrict__ cb, const double *__restrict__ slot_p, const double *__restrict__ slot_n,
                       const int *__restrict__ slot_f, const int *__restrict__ cont_count,
                       const int *__restrict__ cont_offset, int *__restrict__ pa, int *__restrict__ pb,
                       int *__restrict__ fid, long long *__restrict__ key, double *__restrict__ p,
                       double *__restrict__ nrm, double *__restrict__ gap, int *__restrict__ attach,
                       int *__restrict__ count)
{
    const int nc = min(cand_offset[n], cap);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid == 0) *count = cont_offset[nc];
    for (int c = tid; c < nc; c += gridDim.x * blockDim.x) {
        const int a = ca[c], b = cb[c], m = cont_count[c], o = cont_offset[c];
        const double4 n4 = reinterpret_cast<const double4 *>(slot_n)[c];
        for (int k = 0; k < m; ++k) {
            const int d = o + k;
            if (d >= max_contacts) break;
            const double4 ps = reinterpret_cast<const double4 *>(slot_p)[c * kSlots + k];
            const int f = slot_f[c * kSlots + k] & 255, at = slot_f[c * kSlots + k] >> 8;
            pa[d] = a;
            pb[d] = b;
            fid[d] = f;
            key[d] = ((long long)a * (n + 1) + (long long)(b + 1)) * 256 + f;
            st3d(p, d, D3(ps.x, ps.y, ps.z));
            st3d(nrm, d, D3(n4.x, n4.y, n4.z));
            gap[d] = ps.w;
            attach[d] = at;
        }
    }
}

// _basis, ncp_gpu.py:1230-1234
__device__ __forceinline__ void basis(d3 n, d3 &t1, d3 &t2)
{
    const d3 a = fabs(n.x) < 0.9 ? D3(1.0, 0.0, 0.0) : D3(0.0, 1.0, 0.0);
    const d3 t = dsub(a, dscale(n, ddot(a, n)));
    t1 = dscale(t, 1.0 / sqrt(ddot(t, t)));
    t2 = dcross(n, t1);
}

// world inverse inertia R Ib^-1 R^T of a box of principal inertia Ib (diagonal)
__device__ __forceinline__ void world_inv_inertia(double4 qd, d3 Ib, double Iw[3][3])
{
    const dR R = dquat_R(qd);
    const double inv[3] = {1.0 / Ib.x, 1.0 / Ib.y, 1.0 / Ib.z};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += dget(R.col[k], r) * inv[k] * dget(R.col[k], c);
            Iw[r][c] = s;
        }
}

// per body: Minv (6x6) and v_free (6)
__global__ void k_bodies(int n, const double *__restrict__ q, const double *__restrict__ v,
                         const double *__restrict__ w, const double *__restrict__ mass,
                         const double *__restrict__ Ib, const int *__restrict__ kin, const double *__restrict__ vkin,
                         double dt, int gravity, double *__restrict__ Minv, double *__restrict__ vfree)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *M = Minv + 36 * (size_t)i;
    for (int k = 0; k < 36; ++k) M[k] = 0.0;
    double *vf = vfree + 6 * (size_t)i;
    if (kin[i]) {
        for (int k = 0; k < 6; ++k) vf[k] = vkin[6 * (size_t)i + k];
        return;
    }
    const double im = 1.0 / mass[i];
    M[0] = M[7] = M[14] = im;
    double Iw[3][3];
    world_inv_inertia(ld4d(q, i), ld3d(Ib, i), Iw);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[(3 + r) * 6 + 3 + c] = Iw[r][c];
    const d3 vv = ld3d(v, i), ww = ld3d(w, i);
    vf[0] = vv.x;
    vf[1] = vv.y;
    vf[2] = gravity ? vv.z + dt * (im * (-kG * mass[i])) : vv.z;
    vf[3] = ww.x;
    vf[4] = ww.y;
    vf[5] = ww.z;
}

// per contact: the 3x6 blocks, bias, friction and feature (build_scene, :1310-1325)
__global__ void k_contacts(int nc, const int *__restrict__ pa, const int *__restrict__ pb,
                           const int *__restrict__ fid, const double *__restrict__ p, const double *__restrict__ nrm,
                           const double *__restrict__ gap, const double *__restrict__ x,
                           const double *__restrict__ body_mu, double mu0, double dt, double *__restrict__ Ja,
                           double *__restrict__ Jb, double *__restrict__ bias, double *__restrict__ mu,
                           int *__restrict__ feature)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int a = pa[c], b = pb[c];
    const d3 n = ld3d(nrm, c), pc = ld3d(p, c);
    d3 t1, t2;
    basis(n, t1, t2);
    const d3 D[3] = {n, t1, t2};
    const d3 ra = dsub(pc, ld3d(x, a));
    double *A = Ja + 18 * (size_t)c, *B = Jb + 18 * (size_t)c;
    for (int k = 0; k < 3; ++k) {
        const d3 ang = dcross(ra, D[k]);
        A[6 * k + 0] = D[k].x;
        A[6 * k + 1] = D[k].y;
        A[6 * k + 2] = D[k].z;
        A[6 * k + 3] = ang.x;
        A[6 * k + 4] = ang.y;
        A[6 * k + 5] = ang.z;
    }
    if (b >= 0) {
        const d3 rb = dsub(pc, ld3d(x, b));
        for (int k = 0; k < 3; ++k) {
            const d3 ang = dcross(rb, D[k]);
            B[6 * k + 0] = -D[k].x;
            B[6 * k + 1] = -D[k].y;
            B[6 * k + 2] = -D[k].z;
            B[6 * k + 3] = -ang.x;
            B[6 * k + 4] = -ang.y;
            B[6 * k + 5] = -ang.z;
        }
    } else {
        for (int k = 0; k < 18; ++k) B[k] = 0.0;
    }
    const double g = gap[c];
    bias[3 * (size_t)c] = g > 0.0 ? g / dt : -kBeta * fmax(-g - kSlop, 0.0) / dt;
    bias[3 * (size_t)c + 1] = 0.0;
    bias[3 * (size_t)c + 2] = 0.0;
    mu[c] = body_mu ? (b >= 0 ? sqrt(body_mu[a] * body_mu[b]) : body_mu[a]) : mu0;
    feature[c] = fid[c];
}

// warm start: the previous substep's impulse of the same contact key (binary search), else 0
// lam[c] (kAdd: +)= wlam of the store entry whose key is key[c] (the keys ascend), else 0
template <bool kAdd>
__global__ void k_warm(int nc, const long long *__restrict__ key, const long long *__restrict__ wkeys,
                       const double *__restrict__ wlam, const int *__restrict__ wn, double *__restrict__ lam)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const long long k = key[c];
    int lo = 0, hi = *wn - 1;
    double l0 = 0.0, l1 = 0.0, l2 = 0.0;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        const long long km = wkeys[mid];
        if (km == k) {
            l0 = wlam[3 * (size_t)mid];
            l1 = wlam[3 * (size_t)mid + 1];
            l2 = wlam[3 * (size_t)mid + 2];
            break;
        }
        if (km < k) lo = mid + 1;
        else hi = mid - 1;
    }
    if (kAdd) {
        lam[3 * (size_t)c] += l0;
        lam[3 * (size_t)c + 1] += l1;
        lam[3 * (size_t)c + 2] += l2;
    } else {
        lam[3 * (size_t)c] = l0;
        lam[3 * (size_t)c + 1] = l1;
        lam[3 * (size_t)c + 2] = l2;
    }
}

__global__ void k_store(int nc, const long long *__restrict__ key, const double *__restrict__ lam,
                        long long *__restrict__ wkeys, double *__restrict__ wlam, int *__restrict__ wn)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) *wn = nc;
    if (c >= nc) return;
    wkeys[c] = key[c];
    for (int k = 0; k < 3; ++k) wlam[3 * (size_t)c + k] = lam[3 * (size_t)c + k];
}

// q <- normalize(q + 0.5 (w, 0) (x) q dt), _qmul (ncp_gpu.py:1416-1422) with a = (w, 0)
__device__ __forceinline__ double4 quat_step(double4 q, d3 w, double dt)
{
    const double x1 = w.x, y1 = w.y, z1 = w.z;  // w1 = 0
    const double x2 = q.x, y2 = q.y, z2 = q.z, w2 = q.w;
    const double px = x1 * w2 + y1 * z2 - z1 * y2;
    const double py = -x1 * z2 + y1 * w2 + z1 * x2;
    const double pz = x1 * y2 - y1 * x2 + z1 * w2;
    const double pw = -x1 * x2 - y1 * y2 - z1 * z2;
    double4 r = make_double4(q.x + 0.5 * px * dt, q.y + 0.5 * py * dt, q.z + 0.5 * pz * dt, q.w + 0.5 * pw * dt);
    const double s = 1.0 / sqrt(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
    return make_double4(r.x * s, r.y * s, r.z * s, r.w * s);
}

__global__ void k_integrate(int n, const double *__restrict__ v6, double dt, double *__restrict__ x,
                            double *__restrict__ q, double *__restrict__ v, double *__restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *V = v6 + 6 * (size_t)i;
    const d3 vv = D3(V[0], V[1], V[2]), ww = D3(V[3], V[4], V[5]);
    st3d(v, i, vv);
    st3d(w, i, ww);
    st3d(x, i, dadd(ld3d(x, i), dscale(vv, dt)));
    reinterpret_cast<double4 *>(q)[i] = quat_step(ld4d(q, i), ww, dt);
}

// ---------------------------------------------------------------------------------------------
// The adjoint of a substep (reverse mode), float64.  With x' = x + v' h, q' = normalize(r),
// r = q + 0.5 h (w', 0) q, V' = v_free + Minv J^T lambda and lambda the NCP's, the adjoints
// (xb', qb', vb', wb') of the substep's result give, in this order:
//   adj_integrate  xb = xb'; Vb' = (vb' + h xb', wb' + 0.5 h (d(w' q)/dw')^T rb) with
//                  rb = (qb' - q' (q' . qb')) / |r|; qb = rb + 0.5 h (d(w' q)/dq)^T rb;
//   adj_lambda     lb_c = J_c Minv Vb' (the solve's result through V'), vfree_b = Vb';
//   b2c_ncp_adjoint_unrolled  (ncp.cu) the recorded sweeps in reverse: lb -> the warm start's
//                  adjoint, vfree_b, bias_b, mu_b per contact, and the adjoints of the blocks
//                  Ja, Jb and of Minv;
//   adj_contacts   the bias's normal row is the gap's function (gap / h open, -beta max(-gap -
//                  slop, 0) / h penetrating), and the gap moves with the bodies to first order as
//                  n . (dx_a + dth_a x r_a - dx_b - dth_b x r_b): the pose adjoints xb, thb of
//                  both bodies; mu_c = sqrt(mu_a mu_b) (ground: mu_a) hands mu_b to the bodies;
//   adj_geom       the blocks' adjoints to the poses: lever arms, contact point, frame;
//   adj_finish     vb, wb = vfree_b (v_free = [v + g h, w]); the world inertia's turn;
//                  qb += 2 P(q) thb, where P(q) = d((w, 0) q)/dw maps a rotation vector to the
//                  quaternion change.
// Held at the substep's values: the contact set, the clipping of the manifold, the colouring.
// Several contacts meet at one body: the per-body sums are float64 atomics (an adjoint's range
// -- 1e-9 to 1e7 in one rollout of colliding boxes -- overflows any fixed-point scale; the order
// of the additions can move the last bits).  Kinematic bodies get no adjoint (their motion is
// prescribed).
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ void qmul_w_partials(double4 q, d3 w, double dq[4][4], double dw[4][3])
{
    // p = (w, 0) (x) q: rows px, py, pz, pw; columns qx, qy, qz, qw and wx, wy, wz
    const double Dq[4][4] = {{0.0, -w.z, w.y, w.x}, {w.z, 0.0, -w.x, w.y}, {-w.y, w.x, 0.0, w.z},
                             {-w.x, -w.y, -w.z, 0.0}};
    const double Dw[4][3] = {{q.w, q.z, -q.y}, {-q.z, q.w, q.x}, {q.y, -q.x, q.w}, {-q.x, -q.y, -q.z}};
    for (int r = 0; r < 4; ++r) {
        for (int c = 0; c < 4; ++c) dq[r][c] = Dq[r][c];
        for (int c = 0; c < 3; ++c) dw[r][c] = Dw[r][c];
    }
}

__global__ void k_adj_integrate(int n, const double *__restrict__ q, const double *__restrict__ V6,
                                const int *__restrict__ kin, double h, const double *__restrict__ xb_out,
                                const double *__restrict__ qb_out, const double *__restrict__ vb_out,
                                const double *__restrict__ wb_out, double *__restrict__ xb_in,
                                double *__restrict__ qb_in, double *__restrict__ Vb, double *__restrict__ vfree_b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *V = Vb + 6 * (size_t)i, *F = vfree_b + 6 * (size_t)i;
    if (kin[i]) {
        for (int k = 0; k < 3; ++k) xb_in[3 * (size_t)i + k] = 0.0;
        for (int k = 0; k < 4; ++k) qb_in[4 * (size_t)i + k] = 0.0;
        for (int k = 0; k < 6; ++k) V[k] = F[k] = 0.0;
        return;
    }
    const double4 q0 = ld4d(q, i);
    const d3 w1 = D3(V6[6 * (size_t)i + 3], V6[6 * (size_t)i + 4], V6[6 * (size_t)i + 5]);
    double dq[4][4], dw[4][3];
    qmul_w_partials(q0, w1, dq, dw);
    const double q4[4] = {q0.x, q0.y, q0.z, q0.w};
    double r[4];
    for (int k = 0; k < 4; ++k) {
        double pk = 0.0;
        for (int c = 0; c < 3; ++c) pk += dw[k][c] * dget(w1, c);
        r[k] = q4[k] + 0.5 * h * pk;
    }
    const double nr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
    double qn[4], qbo[4], rb[4];
    for (int k = 0; k < 4; ++k) {
        qn[k] = r[k] / nr;
        qbo[k] = qb_out[4 * (size_t)i + k];
    }
    const double dotq = qn[0] * qbo[0] + qn[1] * qbo[1] + qn[2] * qbo[2] + qn[3] * qbo[3];
    for (int k = 0; k < 4; ++k) rb[k] = (qbo[k] - qn[k] * dotq) / nr;
    for (int c = 0; c < 4; ++c) {
        double sacc = 0.0;
        for (int k = 0; k < 4; ++k) sacc += dq[k][c] * rb[k];
        qb_in[4 * (size_t)i + c] = rb[c] + 0.5 * h * sacc;
    }
    for (int k = 0; k < 3; ++k) {
        const double xb = xb_out[3 * (size_t)i + k];
        xb_in[3 * (size_t)i + k] = xb;
        V[k] = F[k] = vb_out[3 * (size_t)i + k] + h * xb;
        double sacc = 0.0;
        for (int j = 0; j < 4; ++j) sacc += dw[j][k] * rb[j];
        V[3 + k] = F[3 + k] = wb_out[3 * (size_t)i + k] + 0.5 * h * sacc;
    }
}

__global__ void k_adj_lambda(int nc, const int *__restrict__ pa, const int *__restrict__ pb,
                             const int *__restrict__ kin, const double *__restrict__ Ja,
                             const double *__restrict__ Jb, const double *__restrict__ Minv,
                             const double *__restrict__ Vb, double *__restrict__ lb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    double out[3] = {0.0, 0.0, 0.0};
    for (int side = 0; side < 2; ++side) {
        const int b = side == 0 ? pa[c] : pb[c];
        if (b < 0 || kin[b]) continue;
        const double *J = (side == 0 ? Ja : Jb) + 18 * (size_t)c, *M = Minv + 36 * (size_t)b, *x = Vb + 6 * (size_t)b;
        double t[6];
        for (int k = 0; k < 6; ++k) {
            double sacc = 0.0;
            for (int j = 0; j < 6; ++j) sacc += M[k * 6 + j] * x[j];
            t[k] = sacc;
        }
        for (int r = 0; r < 3; ++r) {
            double sacc = 0.0;
            for (int k = 0; k < 6; ++k) sacc += J[r * 6 + k] * t[k];
            out[r] += sacc;
        }
    }
    for (int r = 0; r < 3; ++r) lb[3 * (size_t)c + r] = out[r];
}

// the three planes a face contact's point lies on (box_box's attach bits), or 0
__device__ __forceinline__ int attach_planes(int att)
{
    const int m = (att >> kAttachPlaneShift) & 0x3FF;
    return __popc(m) == 3 ? m : 0;
}

// d bias / d gap of build_scene's normal row
__device__ __forceinline__ double dbias_dgap(double g, double h)
{
    return g > 0.0 ? 1.0 / h : (-g - kSlop > 0.0 ? kBeta / h : 0.0);
}

__device__ __forceinline__ void acc_add(double *acc, double x)
{
    atomicAdd(acc, x);
}

// acc per body: 10 int64 -- xb (3), thb (3), mub (1), pad
__global__ void k_adj_contacts(int nc, const int *__restrict__ pa, const int *__restrict__ pb,
                               const int *__restrict__ kin, const int *__restrict__ attach, const double *__restrict__ p,
                               const double *__restrict__ nrm, const double *__restrict__ gap,
                               const double *__restrict__ x, const double *__restrict__ body_mu,
                               const double *__restrict__ mu_c, const double *__restrict__ bias_b,
                               const double *__restrict__ mu_b, double h, double *__restrict__ acc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    // a face contact's gap moves with its point: k_adj_geom takes it
    const double gb = attach_planes(attach[c]) ? 0.0 : bias_b[3 * (size_t)c] * dbias_dgap(gap[c], h);
    const d3 n = ld3d(nrm, c), pc = ld3d(p, c);
    for (int side = 0; side < 2; ++side) {
        const int b = side == 0 ? pa[c] : pb[c];
        if (b < 0 || kin[b]) continue;
        const double sg = side == 0 ? 1.0 : -1.0;
        const d3 r = dsub(pc, ld3d(x, b));
        const d3 th = dcross(r, n);
        double *A = acc + 8 * (size_t)b;
        if (gb != 0.0) {
            acc_add(A + 0, sg * gb * n.x);
            acc_add(A + 1, sg * gb * n.y);
            acc_add(A + 2, sg * gb * n.z);
            acc_add(A + 3, sg * gb * th.x);
            acc_add(A + 4, sg * gb * th.y);
            acc_add(A + 5, sg * gb * th.z);
        }
        if (body_mu) {
            const int o = side == 0 ? pb[c] : pa[c];
            // mu_c = sqrt(mu_a mu_b): d mu_c / d mu_self = mu_c / (2 mu_self); ground pair: mu_c = mu_a
            const double d = o >= 0 ? mu_c[c] / (2.0 * body_mu[b]) : 1.0;
            acc_add(A + 6, mu_b[c] * d);
        }
    }
}

// derivative of _basis's frame with respect to the normal: given h_k (the adjoints of the rows
// n, t1, t2), the adjoint of n
__device__ __forceinline__ d3 basis_adjoint(d3 n, d3 h0, d3 h1, d3 h2)
{
    const d3 a = fabs(n.x) < 0.9 ? D3(1.0, 0.0, 0.0) : D3(0.0, 1.0, 0.0);
    const double an = ddot(a, n);
    const d3 t = dsub(a, dscale(n, an));
    const double tl = sqrt(ddot(t, t));
    const d3 t1 = dscale(t, 1.0 / tl);
    // t2 = n x t1: d t2 = dn x t1 + n x dt1  ->  adjoints  nb += t1 x h2,  t1b += h2 x n
    d3 nb = dadd(h0, dcross(t1, h2));
    const d3 t1b = dadd(h1, dcross(h2, n));
    // t1 = t / |t|: tb = (t1b - t1 (t1 . t1b)) / |t|;  t = a - (a . n) n: nb += -(a . n) tb - a (n . tb)
    const d3 tb = dscale(dsub(t1b, dscale(t1, ddot(t1, t1b))), 1.0 / tl);
    nb = dsub(nb, dadd(dscale(tb, an), dscale(a, ddot(n, tb))));
    return nb;
}

// The pose dependence of one contact's Jacobian blocks.  Ja rows are (D_k, r_a x D_k), Jb rows
// -(D_k, r_b x D_k), D = (n, t1, t2) from _basis, r_s = p - x_s.  Their adjoints are the NCP's
// (Ja_b, Jb_b: from the contact velocities and velocity changes of every recorded update) plus
// lam (x) Minv Vb from V' = v_free + Minv J^T lambda.  A block adjoint (P_k, Q_k) per row gives
// D_k's adjoint +-(P_k + Q_k x r_s) and r_s's +-sum_k D_k x Q_k.  The point p moves with pa, pb
// or halfway between them (attach: dp = sum_t wgt_t (dx_t + dth_t x r_t)); the normal turns with
// the body it belongs to (dn = dth x n), t1 and t2 follow it through _basis.
__global__ void k_adj_geom(int nc, const int *__restrict__ pa, const int *__restrict__ pb,
                           const int *__restrict__ kin, const int *__restrict__ attach,
                           const double *__restrict__ p, const double *__restrict__ nrm,
                           const double *__restrict__ x, const double *__restrict__ q,
                           const double *__restrict__ gap, const double *__restrict__ bias_b, double h,
                           const double *__restrict__ Ja,
                           const double *__restrict__ Minv, const double *__restrict__ lam,
                           const double *__restrict__ Vb, const double *__restrict__ Ja_b,
                           const double *__restrict__ Jb_b, double *__restrict__ acc)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nc) return;
    const int body[2] = {pa[c], pb[c]};
    const int att = attach[c], ppt = att & 3, pn = (att >> 2) & 3;
    const double *J = Ja + 18 * (size_t)c;
    const d3 D[3] = {D3(J[0], J[1], J[2]), D3(J[6], J[7], J[8]), D3(J[12], J[13], J[14])};
    const d3 n = ld3d(nrm, c), pc = ld3d(p, c);
    const double l[3] = {lam[3 * (size_t)c], lam[3 * (size_t)c + 1], lam[3 * (size_t)c + 2]};
    d3 r[2] = {D3(0, 0, 0), D3(0, 0, 0)}, rb[2] = {D3(0, 0, 0), D3(0, 0, 0)};
    d3 Db[3] = {D3(0, 0, 0), D3(0, 0, 0), D3(0, 0, 0)};
    bool dyn[2];
    for (int s = 0; s < 2; ++s) {
        const int b = body[s];
        dyn[s] = b >= 0 && !kin[b];
        if (b < 0) continue;
        r[s] = dsub(pc, ld3d(x, b));
        const double *Jbar = (s == 0 ? Ja_b : Jb_b) + 18 * (size_t)c;
        double m[6] = {0, 0, 0, 0, 0, 0};
        if (dyn[s]) {
            const double *M = Minv + 36 * (size_t)b, *w = Vb + 6 * (size_t)b;
            for (int k = 0; k < 6; ++k) {
                double sacc = 0.0;
                for (int j = 0; j < 6; ++j) sacc += M[k * 6 + j] * w[j];
                m[k] = sacc;
            }
        }
        const double sg = s == 0 ? 1.0 : -1.0;
        for (int k = 0; k < 3; ++k) {
            const d3 P = D3(Jbar[6 * k] + l[k] * m[0], Jbar[6 * k + 1] + l[k] * m[1], Jbar[6 * k + 2] + l[k] * m[2]);
            const d3 Q = D3(Jbar[6 * k + 3] + l[k] * m[3], Jbar[6 * k + 4] + l[k] * m[4], Jbar[6 * k + 5] + l[k] * m[5]);
            Db[k] = dadd(Db[k], dscale(dadd(P, dcross(Q, r[s])), sg));
            rb[s] = dadd(rb[s], dscale(dcross(D[k], Q), sg));
        }
    }
    d3 xg[2] = {dscale(rb[0], -1.0), dscale(rb[1], -1.0)}, thg[2] = {D3(0, 0, 0), D3(0, 0, 0)};
    d3 pbar = dadd(rb[0], rb[1]);
    const int pm = attach_planes(att);
    bool planes = false;
    if (pm && body[1] >= 0) {
        // A face contact: p lies on three planes, each fixed to the incident (I) or the reference
        // (R) box, so n_k . dp = n_k . (dx_X + dth_X x r_X) for the plane's box X; with the
        // reciprocal basis of the normals, dp's adjoint pbar splits into y_k n_k per plane.  The
        // gap (p - c) . rn (c, rn: the reference face's centre and normal, rn = -n when A is the
        // reference) moves with p and with the reference box.
        const int sR = (att & kAttachRefA) ? 0 : 1, sI = 1 - sR;
        const int raxis = (att >> kAttachAxisShift) & 3, j = (raxis + 1) % 3, k = (raxis + 2) % 3;
        const d3 rn = sR == 0 ? dscale(n, -1.0) : n;
        const double gb = bias_b[3 * (size_t)c] * dbias_dgap(gap[c], h);
        pbar = dadd(pbar, dscale(rn, gb));
        xg[sR] = dsub(xg[sR], dscale(rn, gb));
        thg[sR] = dsub(thg[sR], dscale(dcross(r[sR], rn), gb));
        const dR RI = dquat_R(ld4d(q, body[sI])), RR = dquat_R(ld4d(q, body[sR]));
        d3 nk[3];
        int own[3], m = 0;
        for (int b = 0; b < 10 && m < 3; ++b) {
            if (!((pm >> b) & 1)) continue;
            nk[m] = b < 6 ? RI.col[b >> 1] : RR.col[b < 8 ? j : k];
            own[m] = b < 6 ? sI : sR;
            ++m;
        }
        const d3 c12 = dcross(nk[1], nk[2]), c20 = dcross(nk[2], nk[0]), c01 = dcross(nk[0], nk[1]);
        const double det = ddot(nk[0], c12);
        if (fabs(det) > 1e-9) {
            planes = true;
            const double y[3] = {ddot(pbar, c12) / det, ddot(pbar, c20) / det, ddot(pbar, c01) / det};
            for (int t = 0; t < 3; ++t) {
                const int X = own[t];
                xg[X] = dadd(xg[X], dscale(nk[t], y[t]));
                thg[X] = dadd(thg[X], dscale(dcross(r[X], nk[t]), y[t]));
            }
        }
    }
    if (!planes) {
        if (pm) {  // degenerate planes: the point moves with the incident box, the gap as in k_adj_contacts
            const double gb = bias_b[3 * (size_t)c] * dbias_dgap(gap[c], h);
            for (int s = 0; s < 2; ++s) {
                const double sg = s == 0 ? gb : -gb;
                xg[s] = dadd(xg[s], dscale(n, sg));
                thg[s] = dadd(thg[s], dscale(dcross(r[s], n), sg));
            }
        }
        for (int t = 0; t < 2; ++t) {
            const double wgt = ppt == 2 ? 0.5 : ((ppt == t) ? 1.0 : 0.0);
            if (wgt == 0.0 || body[t] < 0) continue;
            thg[t] = dadd(thg[t], dscale(dcross(r[t], pbar), wgt));
            xg[t] = dadd(xg[t], dscale(pbar, wgt));
        }
    }
    if (pn == 1 || pn == 2) {
        const d3 nb = basis_adjoint(n, Db[0], Db[1], Db[2]);
        const int t = pn - 1;  // 0: pa, 1: pb
        thg[t] = dadd(thg[t], dcross(n, nb));
    }
    for (int s = 0; s < 2; ++s) {
        if (!dyn[s]) continue;
        double *Acc = acc + 8 * (size_t)body[s];
        acc_add(Acc + 0, xg[s].x);
        acc_add(Acc + 1, xg[s].y);
        acc_add(Acc + 2, xg[s].z);
        acc_add(Acc + 3, thg[s].x);
        acc_add(Acc + 4, thg[s].y);
        acc_add(Acc + 5, thg[s].z);
    }
}

// Per body: xb += the contacts' pose adjoints, vb, wb = vfree_b (v_free = [v + g h, w]), mub,
// and the world inertia's turn.  The angular block K = R Ib^-1 R^T of Minv has the adjoint
// Kb = the NCP's (Minv_b's angular block) + Vb_ang (x) tau from V' (tau = K^-1 (w' - w_free)).
// With dK = [dth]x K - K [dth]x: thb += ax(K Kb^T) - ax(Kb^T K), ax(X) = (X_yz - X_zy,
// X_zx - X_xz, X_xy - X_yx).  Then qb += 2 P(q) thb, P = d((w, 0) q)/dw.
__global__ void k_adj_finish(int n, const double *__restrict__ q, const int *__restrict__ kin,
                             const double *__restrict__ vfree_b, double *__restrict__ acc,
                             double *__restrict__ xb, double *__restrict__ qb, double *__restrict__ vb,
                             double *__restrict__ wb, double *__restrict__ mub_body, const double *__restrict__ V6,
                             const double *__restrict__ vfree, const double *__restrict__ Ib,
                             const double *__restrict__ Minv, const double *__restrict__ Vb,
                             const double *__restrict__ Minv_b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *A = acc + 8 * (size_t)i;
    if (kin[i]) {
        for (int k = 0; k < 3; ++k) vb[3 * (size_t)i + k] = wb[3 * (size_t)i + k] = 0.0;
        for (int k = 0; k < 8; ++k) A[k] = 0.0;
        return;
    }
    double th[3];
    for (int k = 0; k < 3; ++k) {
        xb[3 * (size_t)i + k] += A[k];
        th[k] = A[3 + k];
        vb[3 * (size_t)i + k] = vfree_b[6 * (size_t)i + k];
        wb[3 * (size_t)i + k] = vfree_b[6 * (size_t)i + 3 + k];
    }
    if (mub_body) mub_body[i] += A[6];
    const double4 q0 = ld4d(q, i);
    if (V6 && Minv_b) {
        const double *M = Minv + 36 * (size_t)i, *Mb = Minv_b + 36 * (size_t)i;
        double K[3][3], Kb[3][3];
        const d3 y = D3(V6[6 * (size_t)i + 3] - vfree[6 * (size_t)i + 3], V6[6 * (size_t)i + 4] - vfree[6 * (size_t)i + 4],
                        V6[6 * (size_t)i + 5] - vfree[6 * (size_t)i + 5]);
        const dR R = dquat_R(q0);
        const d3 Ibd = ld3d(Ib, i);
        const d3 yb = dRT_apply(R, y);
        const d3 tau = dR_apply(R, D3(Ibd.x * yb.x, Ibd.y * yb.y, Ibd.z * yb.z));
        const double Va[3] = {Vb[6 * (size_t)i + 3], Vb[6 * (size_t)i + 4], Vb[6 * (size_t)i + 5]};
        const double ta[3] = {tau.x, tau.y, tau.z};
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
                K[r][cc] = M[(3 + r) * 6 + 3 + cc];
                Kb[r][cc] = Mb[(3 + r) * 6 + 3 + cc] + Va[r] * ta[cc];
            }
        double X[3][3], Y[3][3];  // K Kb^T, Kb^T K
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
                double sx = 0.0, sy = 0.0;
                for (int k = 0; k < 3; ++k) {
                    sx += K[r][k] * Kb[cc][k];
                    sy += Kb[k][r] * K[k][cc];
                }
                X[r][cc] = sx;
                Y[r][cc] = sy;
            }
        th[0] += (X[1][2] - X[2][1]) - (Y[1][2] - Y[2][1]);
        th[1] += (X[2][0] - X[0][2]) - (Y[2][0] - Y[0][2]);
        th[2] += (X[0][1] - X[1][0]) - (Y[0][1] - Y[1][0]);
    }
    // qb += 2 P(q) thb, P = d((w, 0) q)/dw
    double dq[4][4], dw[4][3];
    qmul_w_partials(q0, D3(0.0, 0.0, 0.0), dq, dw);
    for (int r = 0; r < 4; ++r) qb[4 * (size_t)i + r] += 2.0 * ((dw[r][0] * th[0] + dw[r][1] * th[1]) + dw[r][2] * th[2]);
    for (int k = 0; k < 8; ++k) A[k] = 0.0;
}

}  // namespace world
}  // namespace b2c

using namespace b2c;
using namespace b2c::world;

extern "C" int32_t b2c_world_contacts(b2c_world *wd, b2c_boxes *bx, b2c_header *hdr, b2c_stream stream)
{
    if (!wd || !bx || !hdr || wd->n < 0 || bx->n != wd->n || !wd->x || !wd->q || !wd->half || !wd->xc32 || !wd->x4 ||
        !wd->half4 || !wd->slot_p || !wd->slot_n || !wd->slot_f || !wd->pa || !wd->pb || !wd->fid || !wd->key ||
        !wd->p || !wd->nrm || !wd->gap || !wd->attach || !wd->count) {
        set_error("b2c_world_contacts: bad argument");
        return B2C_EARG;
    }
    cudaStream_t s = stream_of(stream);
    const int n = wd->n, cap = bx->cand_capacity;
    if (n == 0) {
        cudaMemsetAsync(wd->count, 0, sizeof(int32_t), s);
        return check_launch("world_contacts");
    }
    k_mirror<<<blocks_for(n), kThreads, 0, s>>>(n, wd->x, wd->xc32, wd->x4, wd->half, wd->half4);
    b2c_bodies mirror{};
    mirror.n = n;
    mirror.xc = wd->xc32;
    int rc = box_candidates(&mirror, bx, hdr, s);
    if (rc) return rc;
    const int cgrid = std::min(blocks_for(cap, 128), kSMs * 16);
    k_narrow<<<cgrid, 128, 0, s>>>(bx->cand_offset, n, cap, bx->cand_a, bx->cand_b, wd->x4, wd->q, wd->half4,
                                   (double)bx->margin, wd->slot_p, wd->slot_n, wd->slot_f, bx->cont_count);
    if ((rc = check_launch("world_narrow"))) return rc;
    if ((rc = exclusive_scan(bx->cont_count, bx->cont_offset, cap + 1, bx->cand_offset + n, bx->scan_tmp, s)))
        return rc;
    k_emit<<<cgrid, kThreads, 0, s>>>(bx->cand_offset, n, cap, wd->max_contacts, bx->cand_a, bx->cand_b, wd->slot_p,
                                      wd->slot_n, wd->slot_f, bx->cont_count, bx->cont_offset, wd->pa, wd->pb, wd->fid,
                                      reinterpret_cast<long long *>(wd->key), wd->p, wd->nrm, wd->gap, wd->attach,
                                      wd->count);
    return check_launch("world_emit");
}

extern "C" int32_t b2c_world_scene(const b2c_world *wd, int32_t n_contacts, double dt, int32_t gravity, double *Ja,
                                   double *Jb, double *Minv, double *vfree, double *bias, double *mu, int32_t *feature,
                                   b2c_stream stream)
{
    if (!wd || n_contacts < 0 || n_contacts > wd->max_contacts || !(dt > 0.0) || !Minv || !vfree ||
        (n_contacts > 0 && (!Ja || !Jb || !bias || !mu || !feature)) || !wd->mass || !wd->Ib || !wd->kin ||
        !wd->vkin || !wd->v || !wd->w) {
        set_error("b2c_world_scene: bad argument");
        return B2C_EARG;
    }
    cudaStream_t s = stream_of(stream);
    if (wd->n > 0)
        k_bodies<<<blocks_for(wd->n), kThreads, 0, s>>>(wd->n, wd->q, wd->v, wd->w, wd->mass, wd->Ib, wd->kin,
                                                         wd->vkin, dt, gravity, Minv, vfree);
    if (n_contacts > 0)
        k_contacts<<<blocks_for(n_contacts), kThreads, 0, s>>>(n_contacts, wd->pa, wd->pb, wd->fid, wd->p, wd->nrm,
                                                                wd->gap, wd->x, wd->body_mu, wd->mu, dt, Ja, Jb, bias,
                                                                mu, feature);
    return check_launch("world_scene");
}

extern "C" int32_t b2c_world_warm(const b2c_world *wd, int32_t n_contacts, double *lam, b2c_stream stream)
{
    if (!wd || n_contacts < 0 || n_contacts > wd->max_contacts || !wd->warm_keys || !wd->warm_lam || !wd->warm_n ||
        (n_contacts > 0 && !lam)) {
        set_error("b2c_world_warm: bad argument");
        return B2C_EARG;
    }
    if (n_contacts > 0)
        k_warm<false><<<blocks_for(n_contacts), kThreads, 0, stream_of(stream)>>>(
            n_contacts, reinterpret_cast<const long long *>(wd->key), reinterpret_cast<const long long *>(wd->warm_keys),
            wd->warm_lam, wd->warm_n, lam);
    return check_launch("world_warm");
}

extern "C" int32_t b2c_world_warm_adjoint(const b2c_world *wd, int32_t n_contacts, const int64_t *tkeys,
                                          const double *tlam, const int32_t *tn, double *lam_bar, b2c_stream stream)
{
    if (!wd || n_contacts < 0 || n_contacts > wd->max_contacts || !tkeys || !tlam || !tn || (n_contacts > 0 && !lam_bar)) {
        set_error("b2c_world_warm_adjoint: bad argument");
        return B2C_EARG;
    }
    if (n_contacts > 0)
        k_warm<true><<<blocks_for(n_contacts), kThreads, 0, stream_of(stream)>>>(
            n_contacts, reinterpret_cast<const long long *>(wd->key), reinterpret_cast<const long long *>(tkeys), tlam,
            tn, lam_bar);
    return check_launch("world_warm_adjoint");
}

extern "C" int32_t b2c_world_store(b2c_world *wd, int32_t n_contacts, const double *lam, b2c_stream stream)
{
    if (!wd || n_contacts < 0 || n_contacts > wd->max_contacts || !wd->warm_keys || !wd->warm_lam || !wd->warm_n ||
        (n_contacts > 0 && !lam)) {
        set_error("b2c_world_store: bad argument");
        return B2C_EARG;
    }
    k_store<<<blocks_for(std::max(n_contacts, 1)), kThreads, 0, stream_of(stream)>>>(
        n_contacts, reinterpret_cast<const long long *>(wd->key), lam, reinterpret_cast<long long *>(wd->warm_keys),
        wd->warm_lam, wd->warm_n);
    return check_launch("world_store");
}

extern "C" int32_t b2c_world_integrate(b2c_world *wd, const double *v6, double dt, b2c_stream stream)
{
    if (!wd || !v6 || !(dt > 0.0) || !wd->x || !wd->q || !wd->v || !wd->w) {
        set_error("b2c_world_integrate: bad argument");
        return B2C_EARG;
    }
    if (wd->n > 0)
        k_integrate<<<blocks_for(wd->n), kThreads, 0, stream_of(stream)>>>(wd->n, v6, dt, wd->x, wd->q, wd->v, wd->w);
    return check_launch("world_integrate");
}

extern "C" int32_t b2c_world_adj_begin(const b2c_world *wd, const b2c_ncp_scene *sc, const double *V6, double h,
                                       const double *xb_out, const double *qb_out, const double *vb_out,
                                       const double *wb_out, double *xb_in, double *qb_in, double *Vb,
                                       double *vfree_b, double *lam_b, b2c_stream stream)
{
    if (!wd || !sc || sc->dtype != 8 || sc->n_b != wd->n || !V6 || !(h > 0.0) || !xb_out || !qb_out || !vb_out ||
        !wb_out || !xb_in || !qb_in || !Vb || !vfree_b || (sc->n_c > 0 && !lam_b)) {
        set_error("b2c_world_adj_begin: bad argument");
        return B2C_EARG;
    }
    cudaStream_t s = stream_of(stream);
    if (wd->n > 0)
        k_adj_integrate<<<blocks_for(wd->n), kThreads, 0, s>>>(wd->n, wd->q, V6, wd->kin, h, xb_out, qb_out, vb_out,
                                                               wb_out, xb_in, qb_in, Vb, vfree_b);
    if (sc->n_c > 0)
        k_adj_lambda<<<blocks_for(sc->n_c), kThreads, 0, s>>>(sc->n_c, sc->pa, sc->pb, wd->kin,
                                                              (const double *)sc->Ja, (const double *)sc->Jb,
                                                              (const double *)sc->Minv, Vb, lam_b);
    return check_launch("world_adj_begin");
}

extern "C" int32_t b2c_world_adj_end(const b2c_world *wd, const b2c_ncp_scene *sc, const double *lam,
                                     const double *V6, const double *Vb, double h, const double *bias_b,
                                     const double *mu_b, const double *vfree_b, const double *Ja_b, const double *Jb_b,
                                     const double *Minv_b, double *acc, double *xb, double *qb, double *vb,
                                     double *wb, double *mub_body, b2c_stream stream)
{
    if (!wd || !sc || sc->dtype != 8 || sc->n_b != wd->n || !(h > 0.0) || !V6 || !Vb || !vfree_b || !acc || !xb ||
        !qb || !vb || !wb || (sc->n_c > 0 && (!bias_b || !mu_b || !lam || !Ja_b || !Jb_b || !Minv_b))) {
        set_error("b2c_world_adj_end: bad argument");
        return B2C_EARG;
    }
    cudaStream_t s = stream_of(stream);
    double *A = acc;
    if (sc->n_c > 0)
        k_adj_contacts<<<blocks_for(sc->n_c), kThreads, 0, s>>>(sc->n_c, sc->pa, sc->pb, wd->kin, wd->attach, wd->p,
                                                                 wd->nrm,
                                                                 wd->gap, wd->x, wd->body_mu,
                                                                 (const double *)sc->mu, bias_b, mu_b, h, A);
    if (sc->n_c > 0)
        k_adj_geom<<<blocks_for(sc->n_c), kThreads, 0, s>>>(sc->n_c, sc->pa, sc->pb, wd->kin, wd->attach, wd->p,
                                                             wd->nrm, wd->x, wd->q, wd->gap, bias_b, h,
                                                             (const double *)sc->Ja,
                                                             (const double *)sc->Minv, lam, Vb, Ja_b, Jb_b, A);
    if (wd->n > 0)
        k_adj_finish<<<blocks_for(wd->n), kThreads, 0, s>>>(wd->n, wd->q, wd->kin, vfree_b, A, xb, qb, vb, wb,
                                                            mub_body, sc->n_c > 0 ? V6 : nullptr,
                                                            (const double *)sc->v_free, wd->Ib,
                                                            (const double *)sc->Minv, Vb,
                                                            sc->n_c > 0 ? Minv_b : nullptr);
    return check_launch("world_adj_end");
}
