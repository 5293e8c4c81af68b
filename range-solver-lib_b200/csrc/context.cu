// Context lifetime, error strings, workspace arena, launch sizing.
#include "krylov.cuh"

#include <cstring>

namespace rsg {

rsg_status set_error(rsg_context *ctx, rsg_status s, const char *fmt, ...)
{
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return s;
}

rsg_status arena_reserve(rsg_context *ctx, size_t bytes)
{
    ctx->ws.used = 0;
    if (bytes <= ctx->ws.cap) return RSG_OK;
    if (ctx->ws.base) {
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaFree(ctx->ws.base));
        ctx->ws.base = nullptr;
        ctx->ws.cap = 0;
    }
    size_t cap = (bytes + (size_t(1) << 20)) & ~((size_t(1) << 20) - 1);
    RSG_CHECK_CUDA(ctx, cudaMalloc(&ctx->ws.base, cap));
    ctx->ws.cap = cap;
    return RSG_OK;
}

int grid_for(rsg_context *ctx, const void *kernel, int block, size_t smem, long long work_items)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    long long full = (long long)per_sm * ctx->num_sms;
    long long need = (work_items + block - 1) / block;
    if (need < 1) need = 1;
    return int(need < full ? need : full);
}

}  // namespace rsg

extern "C" {

rsg_status rsg_context_create(int device, rsg_context **out)
{
    if (!out) return RSG_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return RSG_ERR_CUDA;
    if (device < 0 || device >= count) return RSG_ERR_INVALID_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return RSG_ERR_CUDA;
    auto *ctx = new rsg_context;
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return RSG_ERR_CUDA;
    }
    ctx->own_stream = true;
    if (cudaMallocHost(&ctx->pinned, 64 * sizeof(double)) != cudaSuccess) {
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return RSG_ERR_CUDA;
    }
    for (auto &e : ctx->ev) cudaEventCreate(&e);
    if (cudaMalloc(&ctx->errw, 256) != cudaSuccess || cudaMemset(ctx->errw, 0, 256) != cudaSuccess) {
        rsg_context_destroy(ctx);
        return RSG_ERR_CUDA;
    }
    *out = ctx;
    return RSG_OK;
}

void rsg_context_destroy(rsg_context *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->ws.base) cudaFree(ctx->ws.base);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->errw) cudaFree(ctx->errw);
    if (ctx->persist) cudaFree(ctx->persist);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *rsg_status_string(rsg_status s)
{
    switch (s) {
    case RSG_OK: return "ok";
    case RSG_NOT_CONVERGED: return "not converged (iteration limit)";
    case RSG_BREAKDOWN: return "breakdown (non-finite or zero residual norm)";
    case RSG_ERR_INVALID_ARG: return "invalid argument";
    case RSG_ERR_CUDA: return "CUDA error";
    case RSG_ERR_OUT_OF_MEMORY: return "out of device memory";
    case RSG_ERR_UNSUPPORTED: return "unsupported";
    case RSG_ERR_SINGULAR: return "singular diagonal block";
    case RSG_ERR_TIMEOUT: return "timeout";
    }
    return "unknown status";
}

const char *rsg_last_error(const rsg_context *ctx) { return ctx ? ctx->last_error.c_str() : ""; }

rsg_status rsg_context_set_stream(rsg_context *ctx, void *cuda_stream)
{
    if (!ctx) return RSG_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->own_stream && ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    if (cuda_stream) {
        ctx->stream = static_cast<cudaStream_t>(cuda_stream);
        ctx->own_stream = false;
    } else {
        RSG_CHECK_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    return RSG_OK;
}

rsg_status rsg_synchronize(rsg_context *ctx)
{
    if (!ctx) return RSG_ERR_INVALID_ARG;
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    unsigned int e = 0;
    RSG_CHECK_CUDA(ctx, cudaMemcpy(&e, ctx->errw, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(ctx->errw, 0, sizeof(e));
        return rsg::set_error(ctx, RSG_ERR_TIMEOUT, "a kernel's bounded wait for its copies ran out");
    }
    return RSG_OK;
}

void rsg_conf_default(rsg_solver_conf *c)
{
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->solver_type = RSG_SOLVER_CG;
    c->n_outer = 1000;
    c->n_inner = 30;
    c->cvg = 1.0e-13;
    c->output_frequency = 0;
    c->output_file = nullptr;
    c->eps = 1.0e-14;
    c->stop_rule = RSG_STOP_REFERENCE;
    c->rtol = 1.0e-10;
    c->precision = RSG_PRECISION_FP64;
    c->scale_equations = 1;
    c->reliable_delta = rsg::kReliableDelta;
    c->flexible = 0;
    c->use_graph = 1;
    c->check_interval = 16;
    c->learned = nullptr;
    c->learned_initial_guess = 0;
}

}  // extern "C"
