// Internal interface of the CSR module (used by the solvers and assembly).
#pragma once

#include "spmv.cuh"

#include <algorithm>

namespace rsg {

constexpr uint32_t kMaxBlock = 8;   // largest block-Jacobi width handled on the GPU
constexpr int kMaxGrid = 16384;     // upper bound on grid size of reduction kernels

#define RSG_RPW_DISPATCH(rpw, ...)                 \
    switch (rpw) {                                 \
    case 32: {                                     \
        constexpr int RPW = 32;                    \
        __VA_ARGS__;                               \
    } break;                                       \
    case 16: {                                     \
        constexpr int RPW = 16;                    \
        __VA_ARGS__;                               \
    } break;                                       \
    case 8: {                                      \
        constexpr int RPW = 8;                     \
        __VA_ARGS__;                               \
    } break;                                       \
    default: {                                     \
        constexpr int RPW = 4;                     \
        __VA_ARGS__;                               \
    } break;                                       \
    }

// Grid of an SpMV-based kernel: occupancy-sized and persistent (warps stride over
// 32-row slices / chunks).  A sweep over the 1M-row heat matrix on B200 measured
// this at 71% of HBM bandwidth for the FP64 SpMV, ahead of one-slice-per-warp
// grids (whose many block-level reductions stall on barriers), two slices per
// warp, and register-capped variants.
inline int spmv_grid(rsg_context *ctx, const rsg_csr *A, const void *kernel, size_t smem, int rpw)
{
    const long long threads = A->use_sell ? (long long)A->n_slices * 32 : (long long)A->n * 32 / rpw;
    return std::min(grid_for(ctx, kernel, kBlock, smem, threads), kMaxGrid);
}

rsg_status spmv64(rsg_context *ctx, const rsg_csr *A, const double *x, double *y, bool off16);
rsg_status spmv32(rsg_context *ctx, const rsg_csr *A, const float *x, float *y, bool off16);
// rsg_csr_create with an explicit SELL-32 choice: 0 = when padding costs <= 25%, 1 = always, -1 = never.
rsg_status csr_create_ex(rsg_context *ctx, uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                         int32_t memory, int sell_mode, rsg_csr **out);
// Recompute ||A||_F and the FP32 copy after the values were rewritten in place.
rsg_status csr_refresh(rsg_context *ctx, rsg_csr *A);
rsg_status jacobi_build(rsg_context *ctx, const rsg_csr *A, double *d);
// Frees a matrix's multilevel preconditioner hierarchy (amg.cu).
void amg_release(void *hierarchy);
uint32_t block_width(uint32_t n, uint32_t block_size);
rsg_status block_jacobi_build(rsg_context *ctx, const rsg_csr *A, uint32_t w, double *blocks, unsigned int *flag);
// out3 = {||b-Ax||, ||b||, relres}; partials >= 2*grid doubles.
rsg_status true_residual(rsg_context *ctx, const rsg_csr *A, const double *b, const double *x, double *partials,
                         unsigned int *ticket, double *out3);

}  // namespace rsg
