// Grid-wide barrier of a persistent kernel whose CTAs are all resident (cooperative launch).
//
// bar[0] counts the CTAs that arrived, bar[1] is the generation: the last CTA to arrive resets the
// count and advances the generation, the others poll it with ld.acquire.gpu.  bar[2] is the launch's
// abort word.  Every wait is bounded: a CTA that polls longer than kBarrierPolls times sets bar[2] and
// the caller's error word *err and leaves with false, and a waiting CTA that finds bar[2] set (checked
// every 1024 polls, off the arrival path) leaves too, so one timed-out wait ends the kernel in every
// CTA within about a thousand polls instead of one bound per remaining barrier.  The launcher zeroes
// bar[0] and bar[2] before a launch (bar[1] may keep any value).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

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
// CTA after the barrier.  Without it the last CTA's thread 0 releases the others at once.  Returns
// false in every thread of a CTA that gave up.
template <class LAST = NoHook>
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, unsigned int *err, LAST last = LAST())
{
    constexpr bool kHook = !std::is_same<LAST, NoHook>::value;
    __shared__ int ok_sh, last_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1, is_last = 0;
        const unsigned int gen = ld_acquire(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            if constexpr (kHook) {
                is_last = 1;  // released after the hook
            } else {
                atomicExch(bar, 0u);
                __threadfence();
                atomicAdd(bar + 1, 1u);
            }
        } else {
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
        }
        __threadfence();
        ok_sh = ok;
        last_sh = is_last;
    }
    __syncthreads();
    if constexpr (kHook) {
        if (last_sh) {
            last();
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicExch(bar, 0u);
                __threadfence();
                atomicAdd(bar + 1, 1u);
            }
        }
    }
    return ok_sh != 0;
}

}  // namespace rsg
