// Per-body stages of a substep: gravity + world inverse inertia (one kernel), integration.
#include "b2c_common.cuh"

namespace b2c {

// k_grav + k_invIw, contact_engine_gpu.py:40-53.  v += (0, 0, -g) dt for dynamic bodies
// (each component `v + g dt` is one fused multiply-add, as the reference build contracted it);
// invIw = (R IbInv) R^T, zero for kinematic bodies.
// With vgrav set it also keeps the velocity after gravity there (the deferred-force reference
// point, deferred_force.py:33); with pv / po set it clears the position pass's pseudo-velocities
// (deferred_force.py:37-38, 54-55): the copy and the clears a substep starts with, in the same
// launch.
__global__ void k_body_predict(int n, float *__restrict__ v, const float *__restrict__ invM, float dt,
                               const float *__restrict__ q, const float *__restrict__ IbInv,
                               const int *__restrict__ kin, float *__restrict__ invIw, float *__restrict__ vgrav,
                               float *__restrict__ pv, float *__restrict__ po)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = ld4(v, i);
    if (invM[i] > 0.0f) {
        a.x = fmaf(0.0f, dt, a.x);
        a.y = fmaf(0.0f, dt, a.y);
        a.z = fmaf(-B2C_G, dt, a.z);
        st4(v, i, a);
    }
    if (vgrav) st4(vgrav, i, a);
    if (pv) st4(pv, i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    if (po) st4(po, i, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    m3 out;
    if (kin[i] == 1) {
        out = m3{f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 0.0f}, f3{0.0f, 0.0f, 0.0f}};
    } else {
        m3 Rm = quat_to_matrix(ldq(q, i));
        m3 t = matmul(Rm, ldm(IbInv, i));
        out = matmul(t, transpose3(Rm));
    }
    stm(invIw, i, out);
}

// k_integ, contact_engine_gpu.py:171-180
__global__ void k_body_integrate(int n, float *__restrict__ xc, float *__restrict__ q, const float *__restrict__ v,
                                 const float *__restrict__ w, const float *__restrict__ pv,
                                 const float *__restrict__ po, const float *__restrict__ invM, float dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || invM[i] <= 0.0f) return;
    f3 x = ld3(xc, i), s = add3(ld3(v, i), ld3(pv, i));
    st4(xc, i, make_float4(fmaf(s.x, dt, x.x), fmaf(s.y, dt, x.y), fmaf(s.z, dt, x.z), 0.0f));
    f3 ww = add3(ld3(w, i), ld3(po, i));
    qf wq{0.5f * ww.x, 0.5f * ww.y, 0.5f * ww.z, 0.5f * 0.0f};
    qf qi = ldq(q, i);
    qf p = qmul(wq, qi);
    qf qn{fmaf(p.x, dt, qi.x), fmaf(p.y, dt, qi.y), fmaf(p.z, dt, qi.z), fmaf(p.w, dt, qi.w)};
    qn = qnormalize(qn);
    st4(q, i, make_float4(qn.x, qn.y, qn.z, qn.w));
}

int body_predict(const b2c_bodies *b, float dt, cudaStream_t s)
{
    if (b->n <= 0) return B2C_OK;
    k_body_predict<<<blocks_for(b->n), kThreads, 0, s>>>(b->n, b->v, b->invM, dt, b->q, b->IbInv, b->kin, b->invIw,
                                                         nullptr, nullptr, nullptr);
    return check_launch("body_predict");
}

// the first launch of a substep: predict, vgrav = v after gravity, and (clear_pseudo) pv = po = 0
int body_predict_substep(const b2c_bodies *b, float dt, float *vgrav, bool clear_pseudo, cudaStream_t s)
{
    if (b->n <= 0) return B2C_OK;
    k_body_predict<<<blocks_for(b->n), kThreads, 0, s>>>(b->n, b->v, b->invM, dt, b->q, b->IbInv, b->kin, b->invIw,
                                                         vgrav, clear_pseudo ? b->pv : nullptr,
                                                         clear_pseudo ? b->po : nullptr);
    return check_launch("body_predict");
}

int body_integrate(const b2c_bodies *b, float dt, cudaStream_t s)
{
    if (b->n <= 0) return B2C_OK;
    k_body_integrate<<<blocks_for(b->n), kThreads, 0, s>>>(b->n, b->xc, b->q, b->v, b->w, b->pv, b->po, b->invM, dt);
    return check_launch("body_integrate");
}

}  // namespace b2c

static bool bodies_ok(const b2c_bodies *b)
{
    return b && b->n >= 0 && (b->n == 0 || (b->xc && b->q && b->v && b->w && b->pv && b->po && b->invM && b->IbInv &&
                                            b->kin && b->invIw));
}

extern "C" int32_t b2c_body_predict(const b2c_bodies *b, float dt, b2c_stream s)
{
    if (!bodies_ok(b)) {
        b2c::set_error("b2c_body_predict: bad bodies");
        return B2C_EARG;
    }
    return b2c::body_predict(b, dt, b2c::stream_of(s));
}

extern "C" int32_t b2c_body_integrate(const b2c_bodies *b, float dt, b2c_stream s)
{
    if (!bodies_ok(b)) {
        b2c::set_error("b2c_body_integrate: bad bodies");
        return B2C_EARG;
    }
    return b2c::body_integrate(b, dt, b2c::stream_of(s));
}
