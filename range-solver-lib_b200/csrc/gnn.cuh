// Internal interface of the learned (message-passing) preconditioner.
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "csr.cuh"

namespace rsg {
constexpr int kGnnHidden = 64;
constexpr int kGnnFeatures = 8;
constexpr int kGnnGradBlocks = 256;
// Parameters of an L-layer model: W_in (features x hidden) and b_in, per layer W (2 hidden x hidden) and b,
// w_out (hidden) and b_out.
constexpr uint64_t gnn_param_count(int layers)
{
    return uint64_t(kGnnFeatures) * kGnnHidden + kGnnHidden +
           uint64_t(layers) * (2ull * kGnnHidden * kGnnHidden + kGnnHidden) + kGnnHidden + 1;
}
}  // namespace rsg

struct rsg_learned {
    int L = 6;
    size_t n_params = 0;
    uint64_t step = 0;
    float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
    // per-matrix caches and activations (grow-only)
    const rsg_csr *cached = nullptr;
    uint64_t cached_nnz = 0;
    double cached_norm = 0.0;
    uint32_t cap = 0;
    bool train_bufs = false;
    std::vector<float *> h, m;
    float *s = nullptr, *logd = nullptr, *rsum = nullptr, *feat = nullptr, *pre0 = nullptr;
    float *gh = nullptr, *gh2 = nullptr, *gm = nullptr, *dz = nullptr, *blk = nullptr, *scal32 = nullptr;
    double *dbuf = nullptr;
    __nv_bfloat16 *hb[2] = {nullptr, nullptr};  // BF16 activations of the tensor-core inference path
    float *ew = nullptr;                         // edge weights -a_ij s_i s_j (0 on the diagonal), per nonzero
    uint64_t ew_cap = 0;
};

namespace rsg {
void gnn_free_buffers(rsg_learned *G);
rsg_status gnn_prepare(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, bool train);
rsg_status gnn_forward(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, double *z,
                       const double *xyz, bool train, bool tensor_cores);
rsg_status gnn_loss_grad(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, const double *xyz,
                         bool tensor_cores, double *loss);
rsg_status gnn_forward_umma(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, double *z,
                            const double *xyz, const float *rms);
bool gnn_umma_setup(rsg_context *ctx, int *grid);
// Training layers on the tensor cores (tcgen05, BF16 operands, FP32 accumulation; gnn_umma.cu):
// h_out = h + relu([h, m] W + b); the data backward (dz = g [z + b > 0] to dz, g_prev = g + (dz W^T)[:, :H],
// gm = (dz W^T)[:, H:]); the weight gradient as nblk blocks of partial sums (K2*H + H each).
rsg_status gnn_train_dense_umma(rsg_context *ctx, uint32_t n, const float *h, const float *m, const float *W,
                                const float *b, float *hout);
rsg_status gnn_train_bwd_umma(rsg_context *ctx, uint32_t n, const float *hp, const float *m, const float *W,
                              const float *b, const float *g, float *dz, float *gprev, float *gm);
rsg_status gnn_train_wgrad_umma(rsg_context *ctx, uint32_t n, const float *hp, const float *m, const float *dz,
                                float *blk, int nblk);
void rsg_axpy_f32(rsg_context *ctx, size_t n, float a, const float *x, float *y);

struct FcgResult {
    uint32_t iterations, fallbacks, checks;
    int32_t status;
    double rn, bn, seconds;
};
constexpr int kFcgMaxDirs = 16;
uint32_t fcg_dirs(uint32_t n_inner);
size_t fcg_workspace_bytes(uint32_t n, uint32_t m);
rsg_status fcg_run(rsg_context *ctx, const rsg_csr *A, rsg_learned *G, const double *d, const double *b, double *x,
                   double *partials, uint32_t max_it, double rtol, uint32_t m, FcgResult *res);
}  // namespace rsg
