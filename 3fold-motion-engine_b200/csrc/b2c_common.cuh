// Internal helpers shared by the b2c translation units: status handling, launch shapes,
// 128-bit loads of the SoA records.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "b2c.h"
#include "b2c_math.cuh"

namespace b2c {

// last error message of the calling host thread
void set_error(const char *fmt, ...);

inline int32_t check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return B2C_ECUDA;
    }
    return B2C_OK;
}

inline cudaStream_t stream_of(b2c_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// 148 SMs on a B200; grid-stride kernels that read their count from the device are launched
// on a fixed multiple of the SM count so that the launch never depends on a host read-back.
constexpr int kSMs = 148;
constexpr int kThreads = 256;
inline int blocks_for(long long n, int threads = kThreads)
{
    long long b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 65535LL * 16) b = 65535LL * 16;
    return (int)b;
}

__device__ __forceinline__ float4 ld4(const float *p, int i) { return reinterpret_cast<const float4 *>(p)[i]; }
__device__ __forceinline__ void st4(float *p, int i, float4 v) { reinterpret_cast<float4 *>(p)[i] = v; }
__device__ __forceinline__ f3 ld3(const float *p, int i) { return xyz(ld4(p, i)); }
__device__ __forceinline__ m3 ldm(const float *p, int i)
{
    const float4 *r = reinterpret_cast<const float4 *>(p) + 3 * i;
    return m3{xyz(r[0]), xyz(r[1]), xyz(r[2])};
}
__device__ __forceinline__ void stm(float *p, int i, const m3 &M)
{
    float4 *r = reinterpret_cast<float4 *>(p) + 3 * i;
    r[0] = f4(M.r0, 0.0f);
    r[1] = f4(M.r1, 0.0f);
    r[2] = f4(M.r2, 0.0f);
}
__device__ __forceinline__ qf ldq(const float *p, int i)
{
    float4 a = ld4(p, i);
    return qf{a.x, a.y, a.z, a.w};
}

}  // namespace b2c
