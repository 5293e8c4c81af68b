// rsg_true_relres_noalloc: the FP64 true relative residual ||b - A x|| / ||b||
// for callers that cannot allocate device memory.
//
// Some host applications hand all device memory to their own pool allocator
// at start-up, so any cudaMalloc from a library can fail or fragment their
// budget; others run the residual check inside a time-stepping loop where the
// device-wide synchronisation that cudaFree implies is not acceptable.  This
// entry point needs neither: the caller passes the CSR arrays, b, x and a
// 3-double output already in device memory, and the kernel's only scratch (one
// pair of partial sums per 32-row chunk, plus the grid ticket) lives in the
// file-scope array below, which is part of the loaded library image.
//
// Limits and sharing: at most RSG_NOALLOC_MAX_ROWS rows (the array holds
// RSG_NOALLOC_MAX_ROWS / 32 chunk partials, 1 MiB); every GPU that loads the
// library keeps the array until the process exits.  All calls on one device
// share it and it keeps the last call's contents, so the ticket is cleared
// before each launch, and calls whose kernels overlap on the GPU (different
// streams, no ordering between them) race on the array and give wrong
// results: order such calls on one stream.  Every call looks up the array's
// device address (cudaGetSymbolAddress) with the caller's device current, so the
// entry point stays valid across a cudaDeviceReset in the host application; the
// first call on a device also loads the library's device code there if the CUDA
// runtime has not done so yet, so make that first call before any stream capture.
#include <cuda_runtime.h>

#include "../../include/rsg.h"

namespace {

constexpr uint32_t kChunks = RSG_NOALLOC_MAX_ROWS / 32u;
constexpr uint32_t kHeader = 32;  // doubles reserved in front of the partials; word 0 holds the ticket
constexpr int kThreads = 256;

static __device__ __align__(256) double g_noalloc_scratch[kHeader + 2 * size_t(kChunks)];

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One thread per row, one 32-row chunk per warp.  Each warp writes the chunk's
// (sum r^2, sum b^2); the last block to finish adds the chunk partials in chunk
// order, so the result does not depend on the grid or the GPU.
__global__ void __launch_bounds__(kThreads) k_true_relres_noalloc(uint32_t n, const uint32_t *__restrict__ rp,
                                                                  const uint32_t *__restrict__ ci,
                                                                  const double *__restrict__ val,
                                                                  const double *__restrict__ b,
                                                                  const double *__restrict__ x,
                                                                  double *__restrict__ out, double *scratch)
{
    __shared__ double sh[2][kThreads / 32];
    __shared__ bool is_last;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scratch);
    double *part = scratch + kHeader;
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (row < n) {
        double ax = 0.0;
        for (uint32_t j = rp[row]; j < rp[row + 1]; j++) {
            const uint32_t c = ci[j];
            // a column index outside the matrix is not read; it turns the result into NaN
            ax = c < n ? __dadd_rn(ax, __dmul_rn(val[j], x[c])) : __longlong_as_double(0x7ff8000000000000ll);
        }
        const double r = b[row] - ax;
        rr = r * r;
        bb = b[row] * b[row];
    }
    rr = warp_sum(rr);
    bb = warp_sum(bb);
    const uint32_t chunk = row >> 5;
    if ((threadIdx.x & 31) == 0 && chunk * 32u < n) {
        part[2 * size_t(chunk)] = rr;
        part[2 * size_t(chunk) + 1] = bb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const uint32_t n_chunks = (n + 31u) / 32u;
    double s0 = 0.0, s1 = 0.0;
    for (uint32_t c = threadIdx.x; c < n_chunks; c += blockDim.x) {
        s0 += __ldcg(&part[2 * size_t(c)]);
        s1 += __ldcg(&part[2 * size_t(c) + 1]);
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    if ((threadIdx.x & 31) == 0) {
        sh[0][threadIdx.x >> 5] = s0;
        sh[1][threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < kThreads / 32; w++) {
            t0 += sh[0][w];
            t1 += sh[1][w];
        }
        out[0] = sqrt(t0);
        out[1] = sqrt(t1);
        out[2] = t1 > 0.0 ? sqrt(t0 / t1) : sqrt(t0);
        *ticket = 0u;
    }
}

// Device address of the scratch array on the current device.  The lookup is repeated on every call (a host-side
// query that allocates nothing): a cached address would go stale if the host application reset the device
// (cudaDeviceReset), which unloads the library's device code and places the array anew on the next load.
rsg_status scratch_for_current_device(double **ptr)
{
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return RSG_ERR_CUDA;
    *ptr = static_cast<double *>(p);
    return RSG_OK;
}

}  // namespace

extern "C" rsg_status rsg_true_relres_noalloc(uint32_t n_rows, const uint32_t *row_ptr, const uint32_t *col_idx,
                                              const double *values, const double *b, const double *x, double *out3,
                                              void *stream)
{
    if (n_rows == 0 || n_rows > RSG_NOALLOC_MAX_ROWS) return RSG_ERR_INVALID_ARG;
    if (!row_ptr || !col_idx || !values || !b || !x || !out3) return RSG_ERR_INVALID_ARG;
    double *scratch = nullptr;
    rsg_status s = scratch_for_current_device(&scratch);
    if (s != RSG_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(scratch, 0, sizeof(unsigned int), st) != cudaSuccess) return RSG_ERR_CUDA;
    const uint32_t blocks = (n_rows + kThreads - 1) / kThreads;
    k_true_relres_noalloc<<<blocks, kThreads, 0, st>>>(n_rows, row_ptr, col_idx, values, b, x, out3, scratch);
    return cudaGetLastError() == cudaSuccess ? RSG_OK : RSG_ERR_CUDA;
}
