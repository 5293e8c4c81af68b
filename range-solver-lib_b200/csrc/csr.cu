// CSR handles: upload, validation, derived formats, SpMV and preconditioner builds.
//
// Replaces the reference's SparseMatrixCache (src/rmatrixsolver.cpp:14-109):
// the CSR is uploaded once and kept on the GPU behind a handle; a refresh with
// the same pattern only re-sends the values and recomputes ||A||_F.
#include "csr.cuh"

#include <algorithm>
#include <cstdlib>

namespace rsg {

struct AnalyzeOut {
    unsigned int bad;          // bit 0: row pointer, bit 1: column index
    unsigned int nofit16;
    unsigned int max_row;
    unsigned int max_warp_nnz;
    unsigned int ticket;
    unsigned int pad;
    double norm;
};

__global__ void k_csr_analyze(uint32_t n, uint64_t nnz, const uint32_t *__restrict__ rp,
                              const uint32_t *__restrict__ ci, const double *__restrict__ val,
                              float *__restrict__ val32, int16_t *__restrict__ off16, double *partials,
                              AnalyzeOut *out, int values_only)
{
    __shared__ double sh[32];
    double nrm[1] = {0.0};
    unsigned int bad = 0, nofit = 0, max_row = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = rp[i], e = rp[i + 1];
        if (s > e || e > nnz || (i == 0 && s != 0) || (i == n - 1 && e != nnz)) {
            bad |= 1u;
            continue;
        }
        max_row = max(max_row, e - s);
        const int base = int(i & ~31u);
        for (uint32_t j = s; j < e; j++) {
            const double v = val[j];
            nrm[0] += v * v;
            val32[j] = __double2float_rn(v);
            if (!values_only) {
                const uint32_t c = ci[j];
                if (c >= n) bad |= 2u;
                const int o = int(c) - base;
                if (o < -32768 || o > 32767) nofit = 1u;
                else off16[j] = int16_t(o);
            }
        }
        if ((i & 31u) == 0) {
            const uint32_t last = min(i + 32u, n);
            const uint32_t e2 = rp[last];
            if (e2 >= s && e2 <= nnz) atomicMax(&out->max_warp_nnz, e2 - s);
        }
    }
    if (bad) atomicOr(&out->bad, bad);
    if (nofit) atomicOr(&out->nofit16, 1u);
    if (max_row) atomicMax(&out->max_row, max_row);
    double tot[1];
    if (grid_sum<1>(nrm, partials, &out->ticket, sh, tot) && threadIdx.x == 0) out->norm = sqrt(tot[0]);
}

template <typename V, int RPW>
__global__ void __launch_bounds__(kBlock) k_spmv(Csr<V> M, Sell<V> S, int use_sell, const V *__restrict__ x,
                                                 V *__restrict__ y, unsigned int *err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto gx = [&](uint32_t c) { return x[c]; };
    auto epi = [&](uint32_t row, V acc) { y[row] = acc; };
    for_rows_any<V, RPW>(M, S, use_sell != 0, gx, epi, smem_raw, err, true);
}

__global__ void k_jacobi(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                         const double *__restrict__ val, double *__restrict__ d)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double inv = 0.0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
            if (ci[j] == i) {
                const double a = val[j];
                inv = (a == 0.0) ? 0.0 : 1.0 / a;
                break;
            }
        d[i] = inv;
    }
}

// One thread per diagonal block: gather, Gauss-Jordan with partial pivoting, store.
__global__ void k_block_jacobi(uint32_t n, uint32_t w, const uint32_t *__restrict__ rp,
                               const uint32_t *__restrict__ ci, const double *__restrict__ val,
                               double *__restrict__ blocks, unsigned int *singular)
{
    const uint32_t nb = n / w;
    for (uint32_t blk = blockIdx.x * blockDim.x + threadIdx.x; blk < nb; blk += gridDim.x * blockDim.x) {
        double a[kMaxBlock][kMaxBlock], inv[kMaxBlock][kMaxBlock];
        for (uint32_t k = 0; k < w; k++)
            for (uint32_t l = 0; l < w; l++) {
                a[k][l] = 0.0;
                inv[k][l] = (k == l) ? 1.0 : 0.0;
            }
        const uint32_t r0 = blk * w;
        for (uint32_t k = 0; k < w; k++)
            for (uint32_t j = rp[r0 + k]; j < rp[r0 + k + 1]; j++) {
                const uint32_t c = ci[j];
                if (c >= r0 && c < r0 + w) a[k][c - r0] = val[j];
            }
        bool ok = true;
        for (uint32_t c = 0; c < w && ok; c++) {
            uint32_t piv = c;
            for (uint32_t r = c + 1; r < w; r++)
                if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
            if (a[piv][c] == 0.0) {
                ok = false;
                break;
            }
            if (piv != c)
                for (uint32_t k = 0; k < w; k++) {
                    double t = a[piv][k];
                    a[piv][k] = a[c][k];
                    a[c][k] = t;
                    t = inv[piv][k];
                    inv[piv][k] = inv[c][k];
                    inv[c][k] = t;
                }
            const double p = a[c][c];
            for (uint32_t k = 0; k < w; k++) {
                a[c][k] /= p;
                inv[c][k] /= p;
            }
            for (uint32_t r = 0; r < w; r++) {
                if (r == c) continue;
                const double f = a[r][c];
                if (f == 0.0) continue;
                for (uint32_t k = 0; k < w; k++) {
                    a[r][k] -= f * a[c][k];
                    inv[r][k] -= f * inv[c][k];
                }
            }
        }
        if (!ok) atomicOr(singular, 1u);
        for (uint32_t k = 0; k < w; k++)
            for (uint32_t l = 0; l < w; l++) blocks[(size_t(r0) + k) * w + l] = ok ? inv[k][l] : 0.0;
    }
}

template <int RPW>
__global__ void __launch_bounds__(kBlock) k_true_res(Csr<double> M, Sell<double> S, int use_sell, const double *__restrict__ b,
                                                     const double *__restrict__ x, double *partials,
                                                     unsigned int *ticket, double *out, unsigned int *err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    auto gx = [&](uint32_t c) { return x[c]; };
    auto epi = [&](uint32_t row, double ax) {
        const double r = b[row] - ax;
        acc[0] += r * r;
        acc[1] += b[row] * b[row];
    };
    for_rows_any<double, RPW>(M, S, use_sell != 0, gx, epi, smem_raw, err, true);
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        out[0] = sqrt(tot[0]);
        out[1] = sqrt(tot[1]);
        out[2] = tot[1] > 0.0 ? sqrt(tot[0] / tot[1]) : sqrt(tot[0]);
    }
}

__global__ void k_sell_len(uint32_t n, uint32_t n_slices, const uint32_t *__restrict__ rp, uint32_t *len4)
{
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n_slices; s += gridDim.x * blockDim.x) {
        uint32_t m = 0;
        const uint32_t r1 = min(n, s * 32u + 32u);
        for (uint32_t r = s * 32u; r < r1; r++) m = max(m, rp[r + 1] - rp[r]);
        len4[s] = (m + 3u) / 4u;
    }
}

// Scatter CSR entries into the SELL-32 layout (thread per row).
__global__ void k_sell_fill(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                            const double *__restrict__ val, const int16_t *__restrict__ off16,
                            const uint32_t *__restrict__ slice_ptr, double *__restrict__ sval,
                            float *__restrict__ sval32, int16_t *__restrict__ soff, uint32_t *__restrict__ scol,
                            int values_only)
{
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const size_t base = size_t(slice_ptr[r >> 5]) + 4u * (r & 31u);
        const uint32_t s = rp[r], e = rp[r + 1];
        for (uint32_t j = s; j < e; j++) {
            const uint32_t k = j - s;
            const size_t pos = base + size_t(k >> 2) * 128u + (k & 3u);
            sval[pos] = val[j];
            sval32[pos] = __double2float_rn(val[j]);
            if (!values_only) {
                if (soff) soff[pos] = off16[j];
                else scol[pos] = ci[j];
            }
        }
    }
}

// ---------------- host helpers ----------------

static void free_sell(rsg_csr *A)
{
    cudaFree(A->slice_ptr);
    cudaFree(A->slice_len4);
    cudaFree(A->sval);
    cudaFree(A->sval32);
    cudaFree(A->soff);
    cudaFree(A->scol);
    A->slice_ptr = A->slice_len4 = A->scol = nullptr;
    A->sval = nullptr;
    A->sval32 = nullptr;
    A->soff = nullptr;
    A->use_sell = false;
}

static void free_csr(rsg_csr *A)
{
    if (!A) return;
    rsg::amg_release(A->amg);
    free_sell(A);
    cudaFree(A->rp);
    cudaFree(A->ci);
    cudaFree(A->val);
    cudaFree(A->val32);
    cudaFree(A->off16);
    delete A;
}

// Build the SELL-32 copy when its padding costs at most 25% over the CSR (or always when forced).
static rsg_status build_sell(rsg_context *ctx, rsg_csr *A, bool force)
{
    A->n_slices = (A->n + 31u) / 32u;
    if (cudaMalloc(&A->slice_len4, size_t(A->n_slices) * sizeof(uint32_t)) != cudaSuccess)
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "SELL slice lengths");
    const int g = grid_for(ctx, (const void *)k_sell_len, kBlock, 0, A->n_slices);
    k_sell_len<<<g, kBlock, 0, ctx->stream>>>(A->n, A->n_slices, A->rp, A->slice_len4);
    std::vector<uint32_t> len4(A->n_slices);
    std::vector<uint32_t> ptr(size_t(A->n_slices) + 1, 0);
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(len4.data(), A->slice_len4, len4.size() * sizeof(uint32_t),
                                        cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    uint64_t total = 0;
    for (uint32_t s2 = 0; s2 < A->n_slices; s2++) {
        ptr[s2] = uint32_t(total);
        total += uint64_t(len4[s2]) * 128u;
        if (total > 0xfffffff0ull) {
            free_sell(A);
            return RSG_OK;  // too large for 32-bit slice offsets: keep the CSR path
        }
    }
    ptr[A->n_slices] = uint32_t(total);
    if (A->nnz == 0 || (!force && double(total) > 1.25 * double(A->nnz))) {
        free_sell(A);
        return RSG_OK;
    }
    A->sell_elems = total;
    const size_t t = std::max<uint64_t>(total, 1);
    if (cudaMalloc(&A->slice_ptr, ptr.size() * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&A->sval, t * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&A->sval32, t * sizeof(float)) != cudaSuccess ||
        (A->has_off16 ? cudaMalloc(&A->soff, t * sizeof(int16_t)) : cudaMalloc(&A->scol, t * sizeof(uint32_t))) !=
            cudaSuccess) {
        free_sell(A);
        cudaGetLastError();
        return RSG_OK;  // not enough memory for the copy: keep the CSR path
    }
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(A->slice_ptr, ptr.data(), ptr.size() * sizeof(uint32_t),
                                        cudaMemcpyHostToDevice, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(A->sval, 0, t * sizeof(double), ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(A->sval32, 0, t * sizeof(float), ctx->stream));
    if (A->soff) RSG_CHECK_CUDA(ctx, cudaMemsetAsync(A->soff, 0, t * sizeof(int16_t), ctx->stream));
    else RSG_CHECK_CUDA(ctx, cudaMemsetAsync(A->scol, 0, t * sizeof(uint32_t), ctx->stream));
    const int gf = grid_for(ctx, (const void *)k_sell_fill, kBlock, 0, A->n);
    k_sell_fill<<<gf, kBlock, 0, ctx->stream>>>(A->n, A->rp, A->ci, A->val, A->off16, A->slice_ptr, A->sval,
                                               A->sval32, A->soff, A->scol, 0);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    A->use_sell = true;
    return RSG_OK;
}

static rsg_status refill_sell_values(rsg_context *ctx, rsg_csr *A)
{
    if (!A->sval) return RSG_OK;  // refreshed whenever built: the autotuner may switch layouts later
    const int gf = grid_for(ctx, (const void *)k_sell_fill, kBlock, 0, A->n);
    k_sell_fill<<<gf, kBlock, 0, ctx->stream>>>(A->n, A->rp, A->ci, A->val, A->off16, A->slice_ptr, A->sval,
                                               A->sval32, A->soff, A->scol, 1);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

static rsg_status analyze(rsg_context *ctx, rsg_csr *A, bool values_only)
{
    const int grid = grid_for(ctx, (const void *)k_csr_analyze, kBlock, 0, A->n);
    size_t bytes = arena_bytes(sizeof(AnalyzeOut), 1) + arena_bytes(size_t(grid), sizeof(double));
    RSG_TRY(arena_reserve(ctx, bytes));
    auto *out = arena_take<AnalyzeOut>(ctx, 1);
    auto *partials = arena_take<double>(ctx, grid);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(AnalyzeOut), ctx->stream));
    k_csr_analyze<<<grid, kBlock, 0, ctx->stream>>>(A->n, A->nnz, A->rp, A->ci, A->val, A->val32, A->off16, partials,
                                                   out, values_only ? 1 : 0);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    AnalyzeOut h;
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, out, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (!values_only) {
        if (h.bad & 1u) return set_error(ctx, RSG_ERR_INVALID_ARG, "invalid CSR row pointer");
        if (h.bad & 2u) return set_error(ctx, RSG_ERR_INVALID_ARG, "CSR column index out of range");
        A->has_off16 = (h.nofit16 == 0);
        A->max_row = h.max_row;
        A->max_warp_nnz = h.max_warp_nnz;
    }
    A->norm = h.norm;
    return RSG_OK;
}

rsg_status csr_refresh(rsg_context *ctx, rsg_csr *A)
{
    RSG_TRY(analyze(ctx, A, true));
    return refill_sell_values(ctx, A);
}

rsg_status spmv64(rsg_context *ctx, const rsg_csr *A, const double *x, double *y, bool off16)
{
    const Csr<double> M = view<double>(A, off16);
    const size_t smem = A->use_sell ? 0 : tma_smem<double>();
    RSG_RPW_DISPATCH(pick_rpw(A), {
        auto k = k_spmv<double, RPW>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem<double>()));
        const int grid = spmv_grid(ctx, A, (const void *)k, smem, RPW);
        k<<<grid, kBlock, smem, ctx->stream>>>(M, sell_view<double>(A), A->use_sell, x, y, ctx->errw);
    });
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status spmv32(rsg_context *ctx, const rsg_csr *A, const float *x, float *y, bool off16)
{
    const Csr<float> M = view<float>(A, off16);
    const size_t smem = A->use_sell ? 0 : tma_smem<float>();
    RSG_RPW_DISPATCH(pick_rpw(A), {
        auto k = k_spmv<float, RPW>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem<float>()));
        const int grid = spmv_grid(ctx, A, (const void *)k, smem, RPW);
        k<<<grid, kBlock, smem, ctx->stream>>>(M, sell_view<float>(A), A->use_sell, x, y, ctx->errw);
    });
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status jacobi_build(rsg_context *ctx, const rsg_csr *A, double *d)
{
    const int grid = grid_for(ctx, (const void *)k_jacobi, kBlock, 0, A->n);
    k_jacobi<<<grid, kBlock, 0, ctx->stream>>>(A->n, A->rp, A->ci, A->val, d);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

uint32_t block_width(uint32_t n, uint32_t block_size)
{
    uint32_t w = std::max<uint32_t>(1, std::min<uint32_t>(block_size, kMaxBlock));
    while (w > 1 && n % w != 0) w--;
    return w;
}

rsg_status block_jacobi_build(rsg_context *ctx, const rsg_csr *A, uint32_t w, double *blocks, unsigned int *flag)
{
    const int grid = grid_for(ctx, (const void *)k_block_jacobi, 128, 0, A->n / w);
    k_block_jacobi<<<grid, 128, 0, ctx->stream>>>(A->n, w, A->rp, A->ci, A->val, blocks, flag);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status true_residual(rsg_context *ctx, const rsg_csr *A, const double *b, const double *x, double *partials,
                         unsigned int *ticket, double *out3)
{
    const Csr<double> M = view<double>(A, true);
    const size_t smem = A->use_sell ? 0 : tma_smem<double>();
    RSG_RPW_DISPATCH(pick_rpw(A), {
        auto k = k_true_res<RPW>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem<double>()));
        const int grid = spmv_grid(ctx, A, (const void *)k, smem, RPW);
        k<<<grid, kBlock, smem, ctx->stream>>>(M, sell_view<double>(A), A->use_sell, b, x, partials, ticket, out3,
                                               ctx->errw);
    });
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_csr_create(rsg_context *ctx, uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                          int32_t memory, rsg_csr **out)
{
    return csr_create_ex(ctx, n, rp, ci, val, memory, std::getenv("RSG_NO_SELL") ? -1 : 0, out);
}

}  // extern "C"

rsg_status rsg::csr_create_ex(rsg_context *ctx, uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                              int32_t memory, int sell_mode, rsg_csr **out)
{
    if (!ctx || !out || !rp || n == 0) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_create: bad arguments");
    *out = nullptr;
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    uint32_t nnz32 = 0;
    if (memory == RSG_MEM_HOST) {
        if (rp[0] != 0) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_create: row_ptr[0] != 0");
        nnz32 = rp[n];
    } else {
        RSG_CHECK_CUDA(ctx, cudaMemcpy(&nnz32, rp + n, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    if (nnz32 > 0 && (!ci || !val)) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_create: null arrays");
    auto *A = new rsg_csr;
    A->n = n;
    A->nnz = nnz32;
    const size_t padded = (size_t(nnz32) + 8) & ~size_t(7);
    auto fail = [&](rsg_status s) {
        free_csr(A);
        return s;
    };
    if (cudaMalloc(&A->rp, (size_t(n) + 1) * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&A->ci, padded * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&A->val, padded * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&A->val32, padded * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&A->off16, padded * sizeof(int16_t)) != cudaSuccess)
        return fail(set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "csr_create: out of device memory"));
    cudaMemsetAsync(A->ci, 0, padded * sizeof(uint32_t), ctx->stream);
    cudaMemsetAsync(A->val, 0, padded * sizeof(double), ctx->stream);
    cudaMemsetAsync(A->val32, 0, padded * sizeof(float), ctx->stream);
    cudaMemsetAsync(A->off16, 0, padded * sizeof(int16_t), ctx->stream);
    const cudaMemcpyKind kind = memory == RSG_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (cudaMemcpyAsync(A->rp, rp, (size_t(n) + 1) * sizeof(uint32_t), kind, ctx->stream) != cudaSuccess ||
        (nnz32 && cudaMemcpyAsync(A->ci, ci, size_t(nnz32) * sizeof(uint32_t), kind, ctx->stream) != cudaSuccess) ||
        (nnz32 && cudaMemcpyAsync(A->val, val, size_t(nnz32) * sizeof(double), kind, ctx->stream) != cudaSuccess))
        return fail(set_error(ctx, RSG_ERR_CUDA, "csr_create: upload failed"));
    rsg_status s = analyze(ctx, A, false);
    if (s == RSG_OK && sell_mode >= 0) s = build_sell(ctx, A, sell_mode > 0);
    if (s != RSG_OK) return fail(s);
    *out = A;
    return RSG_OK;
}

extern "C" {

rsg_status rsg_csr_update_values(rsg_context *ctx, rsg_csr *A, const double *val, int32_t memory)
{
    if (!ctx || !A || (!val && A->nnz)) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_update_values: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const cudaMemcpyKind kind = memory == RSG_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (A->nnz && val != A->val)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(A->val, val, A->nnz * sizeof(double), kind, ctx->stream));
    return csr_refresh(ctx, A);
}

void rsg_csr_destroy(rsg_context *ctx, rsg_csr *A)
{
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    free_csr(A);
}

rsg_status rsg_csr_info(const rsg_csr *A, uint32_t *n, uint64_t *nnz, double *frob)
{
    if (!A) return RSG_ERR_INVALID_ARG;
    if (n) *n = A->n;
    if (nnz) *nnz = A->nnz;
    if (frob) *frob = A->norm;
    return RSG_OK;
}

rsg_status rsg_csr_device_arrays(const rsg_csr *A, const uint32_t **rp, const uint32_t **ci, const double **val)
{
    if (!A) return RSG_ERR_INVALID_ARG;
    if (rp) *rp = A->rp;
    if (ci) *ci = A->ci;
    if (val) *val = A->val;
    return RSG_OK;
}

rsg_status rsg_csr_copy_to_host(rsg_context *ctx, const rsg_csr *A, uint32_t *rp, uint32_t *ci, double *val)
{
    if (!ctx || !A) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_copy_to_host: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    if (rp)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(rp, A->rp, (size_t(A->n) + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                            ctx->stream));
    if (ci && A->nnz)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ci, A->ci, A->nnz * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (val && A->nnz)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(val, A->val, A->nnz * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return RSG_OK;
}

rsg_status rsg_spmv(rsg_context *ctx, const rsg_csr *A, const double *x, double *y)
{
    if (!ctx || !A || !x || !y) return set_error(ctx, RSG_ERR_INVALID_ARG, "spmv: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    return spmv64(ctx, A, x, y, true);
}

rsg_status rsg_spmv_f32(rsg_context *ctx, const rsg_csr *A, const float *x, float *y)
{
    if (!ctx || !A || !x || !y) return set_error(ctx, RSG_ERR_INVALID_ARG, "spmv_f32: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    return spmv32(ctx, A, x, y, true);
}

rsg_status rsg_jacobi_build(rsg_context *ctx, const rsg_csr *A, double *d)
{
    if (!ctx || !A || !d) return set_error(ctx, RSG_ERR_INVALID_ARG, "jacobi_build: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    return jacobi_build(ctx, A, d);
}

rsg_status rsg_block_jacobi_build(rsg_context *ctx, const rsg_csr *A, uint32_t block_size, double *blocks,
                                  uint32_t *width_out)
{
    if (!ctx || !A || !blocks) return set_error(ctx, RSG_ERR_INVALID_ARG, "block_jacobi_build: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t w = block_width(A->n, block_size);
    if (width_out) *width_out = w;
    RSG_TRY(arena_reserve(ctx, 256));
    auto *flag = arena_take<unsigned int>(ctx, 1);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(flag, 0, sizeof(unsigned int), ctx->stream));
    RSG_TRY(block_jacobi_build(ctx, A, w, blocks, flag));
    unsigned int h = 0;
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, flag, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h) return set_error(ctx, RSG_ERR_SINGULAR, "block_jacobi_build: singular diagonal block");
    return RSG_OK;
}

rsg_status rsg_true_relres(rsg_context *ctx, const rsg_csr *A, const double *b, const double *x, double *relres)
{
    if (!ctx || !A || !b || !x || !relres) return set_error(ctx, RSG_ERR_INVALID_ARG, "true_relres: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_TRY(arena_reserve(ctx, arena_bytes(size_t(kMaxGrid) * 2 + 8, sizeof(double)) + 512));
    auto *partials = arena_take<double>(ctx, size_t(kMaxGrid) * 2);
    auto *ticket = arena_take<unsigned int>(ctx, 1);
    auto *out = arena_take<double>(ctx, 4);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(ticket, 0, sizeof(unsigned int), ctx->stream));
    RSG_TRY(true_residual(ctx, A, b, x, partials, ticket, out));
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->pinned, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *relres = ctx->pinned[2];
    return RSG_OK;
}

}  // extern "C"
