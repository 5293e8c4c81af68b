// Grid-wide barrier of a persistent kernel whose CTAs are all resident (cooperative launch).
//
// bar[0] counts the CTAs that arrived, bar[1] is the generation: the last CTA to arrive resets the
// count and advances the generation, the others poll it with ld.acquire.gpu.  bar[2] is the launch's
// abort word.  Every wait is bounded: a CTA that polls longer than kBarrierPolls times sets bar[2] and
// the caller's error word *err and leaves with false, and a CTA that finds bar[2] set on arrival or
// while waiting leaves at once, so one timed-out wait ends the kernel in every CTA within a few polls
// instead of one bound per remaining barrier.  The launcher zeroes bar[0] and bar[2] before a launch
// (bar[1] may keep any value).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rsg {

constexpr uint32_t kBarrierPolls = 1u << 24;  // ~ seconds of polling with the back-off below

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

struct NoHook {
    __device__ void operator()() const {}
};

// Every thread of every CTA calls it.  `last()` runs in all threads of the last CTA to arrive before
// the others are released (a grid reduction's final sum, say); what it writes is visible to every
// CTA after the barrier.  Returns false in every thread of a CTA that gave up.
template <class LAST = NoHook>
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, unsigned int *err, LAST last = LAST())
{
    __shared__ int state_sh;  // 0 wait, 1 last to arrive, -1 give up
    __shared__ int ok_sh;     // result of the wait
    __shared__ unsigned int gen_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        int state = 0;
        if (ld_acquire(bar + 2) != 0) {
            state = -1;
        } else {
            gen_sh = ld_acquire(bar + 1);
            __threadfence();
            if (atomicAdd(bar, 1u) == gridDim.x - 1) state = 1;
        }
        state_sh = state;
    }
    __syncthreads();
    const int state = state_sh;
    if (state < 0) return false;
    if (state == 1) {
        __threadfence();
        last();
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        }
        __syncthreads();
        return true;
    }
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned int gen = gen_sh;
        uint32_t t = 0;
        while (ld_acquire(bar + 1) == gen) {
            if (++t >= kBarrierPolls) {
                ok = 0;
                atomicExch(bar + 2, 1u);
                if (err) atomicOr(err, 1u);
                break;
            }
            if ((t & 1023u) == 0 && ld_acquire(bar + 2) != 0) {
                ok = 0;
                break;
            }
            if (t > 4096) __nanosleep(64);
        }
        __threadfence();
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

}  // namespace rsg
