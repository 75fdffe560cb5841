// Device float32 math of the contact solve.
//
// The reference's Warp kernels were compiled by nvrtc with floating-point contraction on, so
// their results carry the compiler's fused-multiply-add choices.  This library is compiled
// with -fmad=false: nothing is contracted implicitly, and every multiply-add that the
// reference's build fused is written here as an explicit fmaf().  The pattern (first product
// of a sum fused with the second product as addend; every `x + a*b` of the kernels fused)
// reproduces the reference's golden arrays bit for bit (reports/cross_hardware_l4.npz,
// relaxed-Jacobi stack8 and lattice1000).  Division and sqrt are the IEEE round-to-nearest
// operations (-prec-div=true -prec-sqrt=true), as in the reference build.
//
// Each helper names the Warp builtin it stands for.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define B2C_HD __host__ __device__ __forceinline__

struct f3 {
    float x, y, z;
};
struct m3 {  // row-major rows
    f3 r0, r1, r2;
};
struct qf {  // (x, y, z, w)
    float x, y, z, w;
};

B2C_HD f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
B2C_HD f3 add3(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
B2C_HD f3 sub3(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
B2C_HD f3 scale3(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
B2C_HD f3 div3(f3 a, float s) { return f3{a.x / s, a.y / s, a.z / s}; }  // wp.div(vec3, float)
B2C_HD f3 xyz(float4 a) { return f3{a.x, a.y, a.z}; }
B2C_HD qf qf4(float4 a) { return qf{a.x, a.y, a.z, a.w}; }
B2C_HD float4 f4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// wp.dot(vec3, vec3): a0*b0 + a1*b1 + a2*b2
B2C_HD float dot3(f3 a, f3 b) { return fmaf(a.z, b.z, fmaf(a.x, b.x, a.y * b.y)); }
// wp.cross
B2C_HD f3 cross3(f3 a, f3 b)
{
    return f3{fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x))};
}
// wp.length
B2C_HD float len3(f3 a) { return sqrtf(dot3(a, a)); }
// wp.normalize(vec3)
B2C_HD f3 normalize3(f3 a)
{
    float l = len3(a);
    return l > 0.0f ? div3(a, l) : f3{0.0f, 0.0f, 0.0f};
}
// mat33 * vec3 (sum of scaled columns)
B2C_HD float rowdot(f3 r, f3 b) { return fmaf(r.z, b.z, fmaf(r.x, b.x, r.y * b.y)); }
B2C_HD f3 matvec(const m3 &M, f3 b) { return f3{rowdot(M.r0, b), rowdot(M.r1, b), rowdot(M.r2, b)}; }
// mat33 * mat33 element (sum from zero)
B2C_HD float mmel(float a0, float a1, float a2, float b0, float b1, float b2)
{
    return fmaf(a2, b2, fmaf(a1, b1, fmaf(a0, b0, 0.0f)));
}
B2C_HD m3 matmul(const m3 &A, const m3 &B)
{
    m3 R;
    R.r0 = f3{mmel(A.r0.x, A.r0.y, A.r0.z, B.r0.x, B.r1.x, B.r2.x), mmel(A.r0.x, A.r0.y, A.r0.z, B.r0.y, B.r1.y, B.r2.y),
              mmel(A.r0.x, A.r0.y, A.r0.z, B.r0.z, B.r1.z, B.r2.z)};
    R.r1 = f3{mmel(A.r1.x, A.r1.y, A.r1.z, B.r0.x, B.r1.x, B.r2.x), mmel(A.r1.x, A.r1.y, A.r1.z, B.r0.y, B.r1.y, B.r2.y),
              mmel(A.r1.x, A.r1.y, A.r1.z, B.r0.z, B.r1.z, B.r2.z)};
    R.r2 = f3{mmel(A.r2.x, A.r2.y, A.r2.z, B.r0.x, B.r1.x, B.r2.x), mmel(A.r2.x, A.r2.y, A.r2.z, B.r0.y, B.r1.y, B.r2.y),
              mmel(A.r2.x, A.r2.y, A.r2.z, B.r0.z, B.r1.z, B.r2.z)};
    return R;
}
B2C_HD m3 transpose3(const m3 &A)
{
    return m3{f3{A.r0.x, A.r1.x, A.r2.x}, f3{A.r0.y, A.r1.y, A.r2.y}, f3{A.r0.z, A.r1.z, A.r2.z}};
}
// wp.quat_rotate(q, x) = x (2w^2 - 1) + q.xyz 2 dot(q.xyz, x) + cross(q.xyz, x) w 2
B2C_HD f3 quat_rotate(qf q, f3 x)
{
    float c = fmaf(2.0f * q.w, q.w, -1.0f);
    float d = 2.0f * fmaf(q.z, x.z, fmaf(q.x, x.x, q.y * x.y));
    float cx = fmaf(q.y, x.z, -(q.z * x.y)), cy = fmaf(q.z, x.x, -(q.x * x.z)), cz = fmaf(q.x, x.y, -(q.y * x.x));
    return f3{fmaf(cx * q.w, 2.0f, fmaf(x.x, c, q.x * d)), fmaf(cy * q.w, 2.0f, fmaf(x.y, c, q.y * d)),
              fmaf(cz * q.w, 2.0f, fmaf(x.z, c, q.z * d))};
}
// wp.quat_to_matrix: columns are the rotated unit axes
B2C_HD m3 quat_to_matrix(qf q)
{
    f3 c1 = quat_rotate(q, f3{1.0f, 0.0f, 0.0f});
    f3 c2 = quat_rotate(q, f3{0.0f, 1.0f, 0.0f});
    f3 c3 = quat_rotate(q, f3{0.0f, 0.0f, 1.0f});
    return m3{f3{c1.x, c2.x, c3.x}, f3{c1.y, c2.y, c3.y}, f3{c1.z, c2.z, c3.z}};
}
// quat * quat
B2C_HD qf qmul(qf a, qf b)
{
    qf r;
    r.x = fmaf(-b.y, a.z, fmaf(a.y, b.z, fmaf(a.w, b.x, b.w * a.x)));
    r.y = fmaf(-b.z, a.x, fmaf(a.z, b.x, fmaf(a.w, b.y, b.w * a.y)));
    r.z = fmaf(-b.x, a.y, fmaf(a.x, b.y, fmaf(a.w, b.z, b.w * a.z)));
    r.w = fmaf(-a.z, b.z, fmaf(-a.y, b.y, fmaf(a.w, b.w, -(a.x * b.x))));
    return r;
}
// wp.normalize(quat): multiply by the reciprocal length
B2C_HD qf qnormalize(qf q)
{
    float l = sqrtf(fmaf(q.w, q.w, fmaf(q.z, q.z, fmaf(q.x, q.x, q.y * q.y))));
    if (l > 0.0f) {
        float il = 1.0f / l;
        return qf{q.x * il, q.y * il, q.z * il, q.w * il};
    }
    return qf{0.0f, 0.0f, 0.0f, 1.0f};
}

// reference constants (contact_engine_gpu.py:25-26)
#define B2C_G 9.81f
#define B2C_R 0.05f
#define B2C_2R 0.1f
#define B2C_BETA 0.2f
#define B2C_SLOP 1e-4f
#define B2C_SCALE 1.0e10f
