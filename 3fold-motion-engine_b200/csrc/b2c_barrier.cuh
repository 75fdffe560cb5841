// Grid barrier of the persistent kernels (the coloured pair solve and the exact-cone NCP sweep):
// one arrival flag per CTA, no atomics.
//
// Barrier k of a launch (k = 1, 2, ...): every thread of the CTA finishes its writes
// (__syncthreads), then thread 0 stores k into its CTA's flag with release semantics at GPU scope.
// To wait, the CTA's first warp reads every CTA's flag (lane l the flags l, l + 32, ...: a few
// independent loads per lane, one L2 round trip per poll) until all of them have reached k, then
// fences with acquire semantics and releases the CTA with __syncthreads.  Compared with one
// arrival counter, the arrivals do not serialise on one L2 address and the release needs no
// second round trip through a generation word.
//
// The flags restart from zero every launch: the host clears them (cudaMemsetAsync, a graph node
// inside a captured step) before each cooperative launch, so no epoch survives a launch, a
// checkpoint load or a change of grid size.
//
// Every wait is bounded: after timeout_ns of %globaltimer the waiting warp sets err_bit in *err,
// the CTA leaves the barrier with false, and the kernel returns (its other CTAs give up at their
// own next wait).  The host reads the bit and raises; the context stays usable.
#pragma once

#include <cstdint>

namespace b2c {

constexpr int kBarrierFlagBase = 32;   // the flags start on their own 128-byte line
constexpr int kBarrierMaxCTAs = 512;   // flags available; a cooperative grid is capped at this
constexpr int kBarrierWords = kBarrierFlagBase + kBarrierMaxCTAs;

__device__ __forceinline__ unsigned long long barrier_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void flag_store_release(unsigned int *p, unsigned int v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned int flag_load_relaxed(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// arrival at barrier `epoch` (1, 2, ... within a launch); every thread of the CTA calls it
__device__ __forceinline__ void flag_arrive(unsigned int *flags, unsigned int epoch)
{
    __syncthreads();
    if (threadIdx.x == 0) flag_store_release(flags + blockIdx.x, epoch);
}

// wait for every CTA's arrival at barrier `epoch`; every thread of the CTA calls it.  Returns
// false when the wait ran out (or another CTA's had, as *err tells), after setting err_bit.
__device__ __forceinline__ bool flag_wait(const unsigned int *flags, unsigned int epoch, long long timeout_ns,
                                          int *err, int err_bit)
{
    __shared__ int s_flag_ok;
    if (threadIdx.x < 32) {
        const int lane = (int)threadIdx.x, n = (int)gridDim.x;
        const unsigned long long t0 = barrier_ns();
        int ok = 1;
        for (;;) {
            bool mine = true;
            for (int j = lane; j < n; j += 32) mine = mine && (int)(flag_load_relaxed(flags + j) - epoch) >= 0;
            if (__all_sync(0xffffffffu, mine)) break;
            if (__any_sync(0xffffffffu, barrier_ns() - t0 > (unsigned long long)timeout_ns)) {
                if (lane == 0) atomicOr(err, err_bit);
                ok = 0;
                break;
            }
        }
        asm volatile("fence.acq_rel.gpu;\n" ::: "memory");
        if (lane == 0) s_flag_ok = ok && !(*(volatile int *)err & err_bit);
    }
    __syncthreads();
    return s_flag_ok != 0;
}

}  // namespace b2c
