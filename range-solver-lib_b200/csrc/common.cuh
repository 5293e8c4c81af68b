// Shared internals of librsg: context and matrix handles, error plumbing,
// workspace arena, deterministic grid reductions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/rsg.h"

#define RSG_EOD 0xffffffffu

namespace rsg {

constexpr int kBlock = 256;           // threads per block of the streaming kernels
constexpr int kWarpsPerBlock = kBlock / 32;

// Device-resident arena that only grows; slices are 256-byte aligned.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
};

}  // namespace rsg

struct rsg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 0;
    std::string last_error;
    rsg::Arena ws;                    // per-solve workspace
    double *pinned = nullptr;         // small pinned host buffer for readbacks (64 doubles)
    unsigned int *errw = nullptr;     // device word: set when a kernel's bounded wait ran out
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double *persist = nullptr;        // persistent CG loop: phase partials and barrier words (cg_persist.cu)
    int coop_graph = -1;              // a cooperative launch can be captured in a graph: -1 not probed, 0 no, 1 yes
};

struct rsg_csr {
    uint32_t n = 0;
    uint64_t nnz = 0;
    uint32_t *rp = nullptr;           // n+1
    uint32_t *ci = nullptr;           // nnz (+ padding)
    double *val = nullptr;            // nnz (+ padding)
    float *val32 = nullptr;           // FP32 copy for mixed precision
    int16_t *off16 = nullptr;         // col - row when every offset fits in int16
    double norm = 0.0;                // ||A||_F
    uint32_t max_row = 0;             // longest row
    uint32_t max_warp_nnz = 0;        // longest 32-row chunk
    bool has_off16 = false;
    // SELL-32 copy (slice = 32 rows = one warp; element k of lane l at
    // slice_ptr[s] + (k/4)*128 + 4l + k%4, rows padded to a multiple of 4)
    bool use_sell = false;
    uint32_t n_slices = 0;
    uint64_t sell_elems = 0;
    uint32_t *slice_ptr = nullptr;    // n_slices + 1
    uint32_t *slice_len4 = nullptr;   // padded row length / 4 per slice
    double *sval = nullptr;
    float *sval32 = nullptr;
    int16_t *soff = nullptr;          // col - (row & ~31), when every offset fits
    uint32_t *scol = nullptr;         // otherwise uint32 columns
    // launch shapes chosen by the autotuner (0 = the built-in default)
    struct Tune {
        bool valid = false;
        bool from_cache = false;
        int32_t rpw = 0;              // CSR-stream rows per warp chunk (<= the largest that fits)
        int32_t g_dir64 = 0, g_dir32 = 0, g_upd64 = 0, g_upd32 = 0;
        int32_t pdl64 = -1, pdl32 = -1;  // programmatic dependent launch in the CG loop: 1/0, -1 size default
        double it64 = 0, it32 = 0;    // seconds per CG iteration with these shapes
        double it64_default = 0, it32_default = 0;
        uint32_t candidates = 0;
    } tune;
    void *amg = nullptr;              // multilevel preconditioner hierarchy (amg.cu), freed with the matrix
};

namespace rsg {

rsg_status set_error(rsg_context *ctx, rsg_status s, const char *fmt, ...);

#define RSG_CHECK_CUDA(ctx, call)                                                                     \
    do {                                                                                              \
        cudaError_t _e = (call);                                                                      \
        if (_e != cudaSuccess) {                                                                      \
            return ::rsg::set_error((ctx), _e == cudaErrorMemoryAllocation ? RSG_ERR_OUT_OF_MEMORY    \
                                                                           : RSG_ERR_CUDA,            \
                                    "%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(_e)); \
        }                                                                                             \
    } while (0)

#define RSG_TRY(expr)                      \
    do {                                   \
        rsg_status _s = (expr);            \
        if (_s != RSG_OK) return _s;       \
    } while (0)

// Reserve `bytes` from the context arena (grows by reallocation when empty of users).
rsg_status arena_reserve(rsg_context *ctx, size_t bytes);
template <typename T>
T *arena_take(rsg_context *ctx, size_t count)
{
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (ctx->ws.used + bytes > ctx->ws.cap) return nullptr;
    T *p = reinterpret_cast<T *>(ctx->ws.base + ctx->ws.used);
    ctx->ws.used += bytes;
    return p;
}
inline size_t arena_bytes(size_t count, size_t elem) { return (count * elem + 255) & ~size_t(255); }

int grid_for(rsg_context *ctx, const void *kernel, int block, size_t smem, long long work_items);

// ---------------- device helpers ----------------

// Programmatic dependent launch.  A kernel launched with the programmatic stream
// serialization attribute may be scheduled while its predecessor drains; pdl_wait()
// blocks until the predecessor has completed and its writes are visible (it returns at
// once for a normal launch), so it comes before the first access to anything the
// predecessor writes.  pdl_release() lets the successor be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// std::isnormal on the device: finite, non-zero and not subnormal (false for NaN).
__device__ __forceinline__ bool dev_isnormal(double v)
{
    const double a = fabs(v);
    return a >= 2.2250738585072014e-308 && a <= 1.7976931348623157e308;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values per thread; result valid in thread 0.  `sh` holds NV*32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double t = lane < nw ? sh[k * 32 + lane] : 0.0;
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Deterministic grid reduction: every block writes NV partials, the last block
// to finish sums them in block order and returns true (in all its threads).
// `total` (valid in thread 0 of the last block) receives the sums.
template <int NV>
__device__ __forceinline__ bool grid_sum(double (&v)[NV], double *partials, unsigned int *ticket, double *sh,
                                         double (&total)[NV])
{
    block_sum<NV>(v, sh);
    __shared__ bool is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) partials[size_t(blockIdx.x) * NV + k] = v[k];
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += __ldcg(&partials[size_t(b) * NV + k]);
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) total[k] = acc[k];
        *ticket = 0u;
    }
    return true;
}

// Error-free transformations for compensated FP32 sums (Ogita, Rump & Oishi, 2005).
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e)
{
    s = a + b;
    float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
struct Dot2 {
    float s = 0.f, c = 0.f;
    __device__ __forceinline__ void add_prod(float a, float b)
    {
        float p = a * b;
        float pe = fmaf(a, b, -p);
        float t;
        two_sum(s, p, s, t);
        c += t + pe;
    }
    __device__ __forceinline__ double value() const { return double(s) + double(c); }
};

}  // namespace rsg
