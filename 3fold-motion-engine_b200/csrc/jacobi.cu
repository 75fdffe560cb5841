// Relaxed-Jacobi contact solve with int64 fixed-point accumulation
// (contact_engine_gpu.py:31-169, driven as in RelaxedJacobiContactEngine.step :266-275).
//
// One thread per contact reads the OLD body velocities, computes its impulse change and adds
// the resulting velocity deltas to per-body int64 accumulators (round(delta * 1e10) in
// float64, then an integer atomic).  Integer addition is associative, so the sum -- and the
// result -- is independent of the contact order and of the atomic order: bit-identical run to
// run.  A second kernel per iteration applies v += relax * acc / 1e10 and clears the
// accumulators.  Counts are read from the device header, launches are fixed-size grid-stride
// loops, so the whole solve is capturable into one graph.
#include "b2c_common.cuh"
#include "b2c_grid.cuh"

namespace b2c {

// _acc, contact_engine_gpu.py:31-38
__device__ __forceinline__ void acc3(long long *ax, long long *ay, long long *az, int b, f3 d, float sign, float scale)
{
    const double sc = (double)(sign * scale);
    atomicAdd(reinterpret_cast<unsigned long long *>(ax + b), (unsigned long long)(long long)round((double)d.x * sc));
    atomicAdd(reinterpret_cast<unsigned long long *>(ay + b), (unsigned long long)(long long)round((double)d.y * sc));
    atomicAdd(reinterpret_cast<unsigned long long *>(az + b), (unsigned long long)(long long)round((double)d.z * sc));
}

struct Acc {
    long long *a[6];
};
__host__ __device__ inline Acc acc_of(int64_t *acc, int n)
{
    Acc A;
    for (int k = 0; k < 6; ++k) A.a[k] = reinterpret_cast<long long *>(acc) + (size_t)k * n;
    return A;
}

// k_jac_vel, contact_engine_gpu.py:81-131
__global__ void __launch_bounds__(256) k_jacobi_velocity(const b2c_header *__restrict__ hdr, b2c_contacts c,
                                                        const float *__restrict__ xc, const float *__restrict__ v,
                                                        const float *__restrict__ w,
                                                        const float *__restrict__ invIw,
                                                        const float *__restrict__ invM, float mu, float scale, Acc A)
{
    const int C = hdr->n_contacts;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
        const int bi = c.bi[k], bj = c.bj[k];
        const float4 pA4 = ld4(c.pA, k);
        const f3 nrm = ld3(c.n, k);
        const f3 rA = sub3(xyz(pA4), ld3(xc, bi));
        const float iMA = invM[bi];
        const m3 IA = ldm(invIw, bi);
        const f3 va = add3(ld3(v, bi), cross3(ld3(w, bi), rA));
        f3 vb{0.0f, 0.0f, 0.0f}, rB{0.0f, 0.0f, 0.0f};
        float iMB = 0.0f;
        m3 IB = IA;
        if (bj >= 0) {
            rB = sub3(ld3(c.pB, k), ld3(xc, bj));
            vb = add3(ld3(v, bj), cross3(ld3(w, bj), rB));
            iMB = invM[bj];
            IB = ldm(invIw, bj);
        }
        // slip-direction basis: t1 = slip, t2 = n x t1 (normal-derived t1 when nearly sticking)
        const f3 vrel = sub3(va, vb);
        const float vn = dot3(vrel, nrm);
        const f3 vt{fmaf(-vn, nrm.x, vrel.x), fmaf(-vn, nrm.y, vrel.y), fmaf(-vn, nrm.z, vrel.z)};
        const float mt = len3(vt);
        f3 t1 = div3(vt, mt);
        if (mt <= 5e-3f) {
            f3 aa{1.0f, 0.0f, 0.0f};
            if (fabsf(nrm.x) >= 0.9f) aa = f3{0.0f, 1.0f, 0.0f};
            const float dd = dot3(aa, nrm);
            t1 = normalize3(f3{fmaf(-dd, nrm.x, aa.x), fmaf(-dd, nrm.y, aa.y), fmaf(-dd, nrm.z, aa.z)});
        }
        const f3 t2 = cross3(nrm, t1);
        // normal: accumulated, clamped >= 0
        const f3 rnA = cross3(rA, nrm);
        float meff = iMA + dot3(rnA, matvec(IA, rnA));
        if (bj >= 0) {
            const f3 rnB = cross3(rB, nrm);
            meff = (meff + iMB) + dot3(rnB, matvec(IB, rnB));
        }
        if (meff < 1e-12f) continue;
        float4 imp = ld4(c.imp, k);
        float dj = -vn / meff;
        const float nw = fmaxf(0.0f, imp.x + dj);
        dj = nw - imp.x;
        imp.x = nw;
        const f3 Jn = scale3(nrm, dj);
        acc3(A.a[0], A.a[1], A.a[2], bi, scale3(Jn, iMA), 1.0f, scale);
        acc3(A.a[3], A.a[4], A.a[5], bi, matvec(IA, cross3(rA, Jn)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A.a[0], A.a[1], A.a[2], bj, scale3(Jn, iMB), -1.0f, scale);
            acc3(A.a[3], A.a[4], A.a[5], bj, matvec(IB, cross3(rB, Jn)), -1.0f, scale);
        }
        // friction: own effective mass per tangent, vector clamp to the mu*jn disc
        const f3 rtA1 = cross3(rA, t1);
        float meft1 = iMA + dot3(rtA1, matvec(IA, rtA1));
        const f3 rtA2 = cross3(rA, t2);
        float meft2 = iMA + dot3(rtA2, matvec(IA, rtA2));
        if (bj >= 0) {
            const f3 rtB1 = cross3(rB, t1);
            meft1 = (meft1 + iMB) + dot3(rtB1, matvec(IB, rtB1));
            const f3 rtB2 = cross3(rB, t2);
            meft2 = (meft2 + iMB) + dot3(rtB2, matvec(IB, rtB2));
        }
        const float o1 = imp.y, o2 = imp.z;
        float a1 = o1 - dot3(vrel, t1) / meft1;
        float a2 = o2 - dot3(vrel, t2) / meft2;
        const float mag = sqrtf(fmaf(a1, a1, a2 * a2));
        const float lim = mu * imp.x;
        if (mag > lim && mag > 1e-12f) {
            a1 = a1 * lim / mag;
            a2 = a2 * lim / mag;
        }
        imp.y = a1;
        imp.z = a2;
        st4(c.imp, k, imp);
        // the cross-slip component t2 is damped 0.5x (contact_engine_gpu.py:127-128)
        const float e1 = a1 - o1, e2 = 0.5f * (a2 - o2);
        const f3 Jt{fmaf(e1, t1.x, e2 * t2.x), fmaf(e1, t1.y, e2 * t2.y), fmaf(e1, t1.z, e2 * t2.z)};
        acc3(A.a[0], A.a[1], A.a[2], bi, scale3(Jt, iMA), 1.0f, scale);
        acc3(A.a[3], A.a[4], A.a[5], bi, matvec(IA, cross3(rA, Jt)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A.a[0], A.a[1], A.a[2], bj, scale3(Jt, iMB), -1.0f, scale);
            acc3(A.a[3], A.a[4], A.a[5], bj, matvec(IB, cross3(rB, Jt)), -1.0f, scale);
        }
    }
}

// k_jac_pos, contact_engine_gpu.py:145-169: Baumgarte pseudo-velocity pass
__global__ void __launch_bounds__(256) k_jacobi_position(const b2c_header *__restrict__ hdr, b2c_contacts c,
                                                        const float *__restrict__ xc, const float *__restrict__ pv,
                                                        const float *__restrict__ po,
                                                        const float *__restrict__ invIw,
                                                        const float *__restrict__ invM, float dt, float scale, Acc A)
{
    const int C = hdr->n_contacts;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += gridDim.x * blockDim.x) {
        const int bi = c.bi[k], bj = c.bj[k];
        const float4 pA4 = ld4(c.pA, k);
        const f3 nrm = ld3(c.n, k);
        const f3 rA = sub3(xyz(pA4), ld3(xc, bi));
        const float iMA = invM[bi];
        const m3 IA = ldm(invIw, bi);
        f3 rel = add3(ld3(pv, bi), cross3(ld3(po, bi), rA));
        f3 rB{0.0f, 0.0f, 0.0f};
        float iMB = 0.0f;
        m3 IB = IA;
        if (bj >= 0) {
            rB = sub3(ld3(c.pB, k), ld3(xc, bj));
            rel = sub3(rel, add3(ld3(pv, bj), cross3(ld3(po, bj), rB)));
            iMB = invM[bj];
            IB = ldm(invIw, bj);
        }
        const f3 rnA = cross3(rA, nrm);
        float meff = iMA + dot3(rnA, matvec(IA, rnA));
        if (bj >= 0) {
            const f3 rnB = cross3(rB, nrm);
            meff = (meff + iMB) + dot3(rnB, matvec(IB, rnB));
        }
        if (meff < 1e-12f) continue;
        const float bias = B2C_BETA * fmaxf(pA4.w - B2C_SLOP, 0.0f) / dt;
        float dj = (bias - dot3(rel, nrm)) / meff;
        float jp = c.imp[4 * k + 3];
        const float nw = fmaxf(0.0f, jp + dj);
        dj = nw - jp;
        c.imp[4 * k + 3] = nw;
        const f3 Jn = scale3(nrm, dj);
        acc3(A.a[0], A.a[1], A.a[2], bi, scale3(Jn, iMA), 1.0f, scale);
        acc3(A.a[3], A.a[4], A.a[5], bi, matvec(IA, cross3(rA, Jn)), 1.0f, scale);
        if (bj >= 0) {
            acc3(A.a[0], A.a[1], A.a[2], bj, scale3(Jn, iMB), -1.0f, scale);
            acc3(A.a[3], A.a[4], A.a[5], bj, matvec(IB, cross3(rB, Jn)), -1.0f, scale);
        }
    }
}

// k_apply, contact_engine_gpu.py:133-143: v += relax * float(float64(acc) * float64(1/scale)); acc = 0.
// Skipped in a substep without contacts, as the reference skips the whole solve then.
__global__ void k_jacobi_apply(const b2c_header *__restrict__ hdr, int n, float *__restrict__ v,
                               float *__restrict__ w, float relax, float scale, Acc A)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || hdr->n_contacts == 0) return;
    const float inv = 1.0f / scale;
    float d[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        d[k] = (float)((double)A.a[k][i] * (double)inv);
        A.a[k][i] = 0;
    }
    float4 a = ld4(v, i), b = ld4(w, i);
    a.x = fmaf(relax, d[0], a.x);
    a.y = fmaf(relax, d[1], a.y);
    a.z = fmaf(relax, d[2], a.z);
    b.x = fmaf(relax, d[3], b.x);
    b.y = fmaf(relax, d[4], b.y);
    b.z = fmaf(relax, d[5], b.z);
    st4(v, i, a);
    st4(w, i, b);
}

// contact_engine_gpu.py:266-269: with contacts, zero the impulses and the pseudo-velocities
__global__ void k_jacobi_reset(const b2c_header *__restrict__ hdr, float *__restrict__ imp, int n,
                               float *__restrict__ pv, float *__restrict__ po)
{
    const int C = hdr->n_contacts;
    if (C == 0) return;
    const int stride = gridDim.x * blockDim.x;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < C; k += stride) st4(imp, k, make_float4(0, 0, 0, 0));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        st4(pv, i, make_float4(0, 0, 0, 0));
        st4(po, i, make_float4(0, 0, 0, 0));
    }
}

int jacobi_solve(const b2c_bodies *b, b2c_contacts *c, const b2c_header *hdr, int64_t *acc,
                 const b2c_jacobi_params *p, float dt, cudaStream_t s)
{
    const int nb = b->n;
    const Acc A = acc_of(acc, nb);
    const int cgrid = std::min(blocks_for(c->capacity), kSMs * 8);
    k_jacobi_reset<<<cgrid, kThreads, 0, s>>>(hdr, c->imp, nb, b->pv, b->po);
    for (int it = 0; it < p->vit; ++it) {
        k_jacobi_velocity<<<cgrid, 256, 0, s>>>(hdr, *c, b->xc, b->v, b->w, b->invIw, b->invM, p->mu, B2C_SCALE, A);
        k_jacobi_apply<<<blocks_for(nb), kThreads, 0, s>>>(hdr, nb, b->v, b->w, p->relax, B2C_SCALE, A);
    }
    for (int it = 0; it < p->pit; ++it) {
        k_jacobi_position<<<cgrid, 256, 0, s>>>(hdr, *c, b->xc, b->pv, b->po, b->invIw, b->invM, dt, B2C_SCALE, A);
        k_jacobi_apply<<<blocks_for(nb), kThreads, 0, s>>>(hdr, nb, b->pv, b->po, p->relax, B2C_SCALE, A);
    }
    return check_launch("jacobi_solve");
}

int body_predict_substep(const b2c_bodies *b, float dt, float *vgrav, bool clear_pseudo, cudaStream_t s);
int body_integrate(const b2c_bodies *b, float dt, cudaStream_t s);
int bead_world(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, cudaStream_t s);
int grid_build(const b2c_beads *beads, b2c_grid *g, cudaStream_t s);
int bead_contacts(const b2c_beads *beads, const b2c_grid *g, b2c_contacts *c, b2c_header *hdr, cudaStream_t s);

}  // namespace b2c

extern "C" int32_t b2c_jacobi_solve(const b2c_bodies *b, b2c_contacts *c, const b2c_header *hdr, int64_t *acc,
                                    const b2c_jacobi_params *p, float dt, b2c_stream s)
{
    if (!b || !c || !hdr || !acc || !p || p->vit < 0 || p->pit < 0 || !(dt > 0.0f)) {
        b2c::set_error("b2c_jacobi_solve: bad argument");
        return B2C_EARG;
    }
    return b2c::jacobi_solve(b, c, hdr, acc, p, dt, b2c::stream_of(s));
}

extern "C" int32_t b2c_jacobi_substep(const b2c_bodies *b, const b2c_beads *beads, b2c_grid *g, b2c_contacts *c,
                                      b2c_header *hdr, int64_t *acc, const b2c_jacobi_params *p, float dt,
                                      float *vgrav, b2c_stream s)
{
    if (!b || !beads || !b2c::grid_valid(g) || !c || !hdr || !acc || !p || !vgrav || !(dt > 0.0f)) {
        b2c::set_error("b2c_jacobi_substep: bad argument");
        return B2C_EARG;
    }
    cudaStream_t st = b2c::stream_of(s);
    int rc;
    if ((rc = b2c::body_predict_substep(b, dt, vgrav, false, st))) return rc;
    if ((rc = b2c::bead_world(b, beads, g, st))) return rc;
    if ((rc = b2c::grid_build(beads, g, st))) return rc;
    if ((rc = b2c::bead_contacts(beads, g, c, hdr, st))) return rc;
    if ((rc = b2c::jacobi_solve(b, c, hdr, acc, p, dt, st))) return rc;
    return b2c::body_integrate(b, dt, st);
}
