// File formats of the library (no counterpart in the reference, whose model
// restart files belong to range-model-lib):
//   * CSR/RHS dump: a reproducible benchmark input -- the matrix exactly as the
//     solver holds it (row pointers, column indices, FP64 values) and optionally
//     a right-hand side.  Little-endian, 64-byte header:
//       "RSGCSR01" | u32 n | u32 has_b | u64 nnz | u64 reserved[5]
//     then rp[n+1] u32, ci[nnz] u32, val[nnz] f64, b[n] f64 (when has_b).
//   * learned-preconditioner checkpoint: parameters, Adam moments and step.
//       "RSGGNN01" | u32 version (1) | u32 layers | u32 hidden | u32 features |
//       u64 n_params | u64 step | u64 reserved[3]
//     then params, adam_m, adam_v: n_params f32 each.
// And a self-test of failure detection: a kernel waits, with the library's
// bounded mbarrier wait and a short limit, for a completion that never comes,
// flags the context's error word and returns; rsg_synchronize then reports
// RSG_ERR_TIMEOUT and the context stays usable.
#include <cstdio>
#include <cstring>
#include <exception>
#include <vector>

#include "gnn.cuh"
#include "spmv.cuh"

namespace rsg {
namespace {

struct CsrHeader {
    char magic[8];
    uint32_t n, has_b;
    uint64_t nnz;
    uint64_t reserved[5];
};
static_assert(sizeof(CsrHeader) == 64, "CSR dump header is 64 bytes");

struct GnnHeader {
    char magic[8];
    uint32_t version, layers, hidden, features;
    uint64_t n_params, step;
    uint64_t reserved[3];
};
static_assert(sizeof(GnnHeader) == 64, "checkpoint header is 64 bytes");

bool write_all(FILE *f, const void *p, size_t bytes) { return bytes == 0 || std::fwrite(p, 1, bytes, f) == bytes; }
bool read_all(FILE *f, void *p, size_t bytes) { return bytes == 0 || std::fread(p, 1, bytes, f) == bytes; }

// Bytes between the current position and the end of the file (the position is kept).
uint64_t file_bytes_left(FILE *f)
{
    const long here = std::ftell(f);
    if (here < 0 || std::fseek(f, 0, SEEK_END) != 0) return 0;
    const long end = std::ftell(f);
    std::fseek(f, here, SEEK_SET);
    return end > here ? uint64_t(end - here) : 0;
}

// Waits for phase 0 of an mbarrier that expects one arrival which never happens;
// the wait gives up after `limit` polls and flags *err.
__global__ void k_wait_selftest(uint32_t limit, unsigned int *err)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bool ok = false;
        for (uint32_t t = 0; t < limit && !ok; t++) ok = mbar_try_wait(&bar, 0);
        if (!ok) atomicOr(err, 1u);
    }
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_csr_save(rsg_context *ctx, const rsg_csr *A, const double *b_device, const char *path)
{
    if (!ctx || !A || !path) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_save: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    std::vector<uint32_t> rp(size_t(A->n) + 1), ci(A->nnz);
    std::vector<double> val(A->nnz), b(b_device ? A->n : 0);
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaMemcpy(rp.data(), A->rp, rp.size() * 4, cudaMemcpyDeviceToHost));
    RSG_CHECK_CUDA(ctx, cudaMemcpy(ci.data(), A->ci, ci.size() * 4, cudaMemcpyDeviceToHost));
    RSG_CHECK_CUDA(ctx, cudaMemcpy(val.data(), A->val, val.size() * 8, cudaMemcpyDeviceToHost));
    if (b_device) RSG_CHECK_CUDA(ctx, cudaMemcpy(b.data(), b_device, b.size() * 8, cudaMemcpyDeviceToHost));
    CsrHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "RSGCSR01", 8);
    h.n = A->n;
    h.has_b = b_device ? 1u : 0u;
    h.nnz = A->nnz;
    FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_save: cannot open %s", path);
    const bool ok = write_all(f, &h, sizeof(h)) && write_all(f, rp.data(), rp.size() * 4) &&
                    write_all(f, ci.data(), ci.size() * 4) && write_all(f, val.data(), val.size() * 8) &&
                    write_all(f, b.data(), b.size() * 8);
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_save: write to %s failed", path);
    return RSG_OK;
}

rsg_status rsg_csr_load(rsg_context *ctx, const char *path, rsg_csr **A, double *b_device, uint32_t *n_rows,
                        uint64_t *nnz, int32_t *has_b)
{
    if (!ctx || !path || !A) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: cannot open %s", path);
    CsrHeader h;
    if (!read_all(f, &h, sizeof(h)) || std::memcmp(h.magic, "RSGCSR01", 8) != 0) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: %s is not an RSGCSR01 file", path);
    }
    // The header is untrusted: check it against the file's size before sizing any buffer from it.
    const uint64_t payload = file_bytes_left(f);
    const uint64_t want = (uint64_t(h.n) + 1) * 4 + h.nnz * 12 + (h.has_b ? uint64_t(h.n) * 8 : 0);
    if (h.n == 0 || h.nnz > 0xffffffffull || h.has_b > 1 || payload != want) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_INVALID_ARG,
                         "csr_load: %s: header (n %u, nnz %llu, has_b %u) does not match the file's %llu payload bytes",
                         path, h.n, (unsigned long long)h.nnz, h.has_b, (unsigned long long)payload);
    }
    std::vector<uint32_t> rp, ci;
    std::vector<double> val, b;
    bool ok = false;
    try {
        rp.resize(size_t(h.n) + 1);
        ci.resize(h.nnz);
        val.resize(h.nnz);
        b.resize(h.has_b ? h.n : 0);
        ok = read_all(f, rp.data(), rp.size() * 4) && read_all(f, ci.data(), ci.size() * 4) &&
             read_all(f, val.data(), val.size() * 8) && read_all(f, b.data(), b.size() * 8);
    } catch (const std::exception &) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "csr_load: no host memory for %s", path);
    }
    std::fclose(f);
    if (!ok) return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: %s is truncated", path);
    // rsg_csr_create copies rp[n] column indexes and values: they must be the nnz the header sized.
    if (rp[0] != 0 || rp[h.n] != h.nnz)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: %s: row_ptr[0] = %u, row_ptr[n] = %u, nnz = %llu", path,
                         rp[0], rp[h.n], (unsigned long long)h.nnz);
    for (uint32_t i = 0; i < h.n; i++)
        if (rp[i + 1] < rp[i])
            return set_error(ctx, RSG_ERR_INVALID_ARG, "csr_load: %s: row_ptr decreases at row %u", path, i);
    if (n_rows) *n_rows = h.n;
    if (nnz) *nnz = h.nnz;
    if (has_b) *has_b = int32_t(h.has_b);
    RSG_TRY(rsg_csr_create(ctx, h.n, rp.data(), ci.data(), val.data(), RSG_MEM_HOST, A));
    if (b_device && h.has_b) {
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(b_device, b.data(), b.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return RSG_OK;
}

rsg_status rsg_learned_save(rsg_context *ctx, const rsg_learned *G, const char *path)
{
    if (!ctx || !G || !path) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_save: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::vector<float> buf(G->n_params * 3);
    RSG_CHECK_CUDA(ctx, cudaMemcpy(buf.data(), G->params, G->n_params * 4, cudaMemcpyDeviceToHost));
    RSG_CHECK_CUDA(ctx, cudaMemcpy(buf.data() + G->n_params, G->adam_m, G->n_params * 4, cudaMemcpyDeviceToHost));
    RSG_CHECK_CUDA(ctx, cudaMemcpy(buf.data() + 2 * G->n_params, G->adam_v, G->n_params * 4, cudaMemcpyDeviceToHost));
    GnnHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "RSGGNN01", 8);
    h.version = 1;
    h.layers = uint32_t(G->L);
    h.hidden = kGnnHidden;
    h.features = kGnnFeatures;
    h.n_params = G->n_params;
    h.step = G->step;
    FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_save: cannot open %s", path);
    const bool ok = write_all(f, &h, sizeof(h)) && write_all(f, buf.data(), buf.size() * 4);
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_save: write to %s failed", path);
    return RSG_OK;
}

rsg_status rsg_learned_load(rsg_context *ctx, const char *path, rsg_learned **out)
{
    if (!ctx || !path || !out) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_load: bad arguments");
    *out = nullptr;
    FILE *f = std::fopen(path, "rb");
    if (!f) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_load: cannot open %s", path);
    GnnHeader h;
    if (!read_all(f, &h, sizeof(h)) || std::memcmp(h.magic, "RSGGNN01", 8) != 0 || h.version != 1) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_load: %s is not an RSGGNN01 version-1 file", path);
    }
    if (h.hidden != uint32_t(kGnnHidden) || h.features != uint32_t(kGnnFeatures) || h.layers == 0 || h.layers > 32) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "learned_load: %u layers of width %u with %u features", h.layers,
                         h.hidden, h.features);
    }
    // The parameter count follows from the layer count; compare before sizing anything from the header.
    const uint64_t expect = gnn_param_count(int(h.layers));
    const uint64_t payload = file_bytes_left(f);
    if (h.n_params != expect || payload != expect * 3 * 4) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_INVALID_ARG,
                         "learned_load: %s holds %llu parameters in %llu bytes; %u layers need %llu", path,
                         (unsigned long long)h.n_params, (unsigned long long)payload, h.layers,
                         (unsigned long long)expect);
    }
    std::vector<float> buf;
    bool ok = false;
    try {
        buf.resize(expect * 3);
        ok = read_all(f, buf.data(), buf.size() * 4);
    } catch (const std::exception &) {
        std::fclose(f);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned_load: no host memory for %s", path);
    }
    std::fclose(f);
    if (!ok) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_load: %s is truncated", path);
    rsg_learned *G = nullptr;
    RSG_TRY(rsg_learned_create(ctx, h.layers, 0, &G));
    rsg_status s = rsg_learned_set_params(ctx, G, buf.data(), 0);
    if (s == RSG_OK) s = rsg_learned_set_params(ctx, G, buf.data() + expect, 2);
    if (s == RSG_OK) s = rsg_learned_set_params(ctx, G, buf.data() + 2 * expect, 3);
    if (s != RSG_OK) {
        rsg_learned_destroy(ctx, G);
        return s;
    }
    G->step = h.step;
    *out = G;
    return RSG_OK;
}

rsg_status rsg_selftest_wait_timeout(rsg_context *ctx, uint32_t polls)
{
    if (!ctx) return RSG_ERR_INVALID_ARG;
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t limit = polls == 0 ? 1024u : std::min(polls, kWaitLimit);
    k_wait_selftest<<<1, 32, 0, ctx->stream>>>(limit, ctx->errw);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return rsg_synchronize(ctx);
}

}  // extern "C"
