// Internal interface of the Krylov solvers.
#pragma once

#include "csr.cuh"

namespace rsg {

// Device-resident CG state.  Written by the last block of each kernel's grid
// reduction, read by every block of the next kernel.
struct CgState {
    double rho;        // r^T z used by the current alpha
    double rho_new;    // r^T z after the latest update
    double beta;       // direction update factor for the next iteration
    double alpha;
    double pq;
    double rn, xn, bn, an;
    double error, trend;
    double max_r;      // mixed: true residual norm at the last refresh
    double sigma;      // mixed: FP32 vectors hold sigma * (FP64 quantity)
    double cvg, eps, rtol, delta;
    double check_rn;   // block-Jacobi: residual norm computed by the check pass
    uint32_t max_it;
    int32_t stop_rule;
    uint32_t it;
    int32_t done;
    int32_t status;
    int32_t converged;
    int32_t need_check;
    int32_t fold;
    uint32_t n_updates;
    uint32_t body_count;
    uint32_t body_limit;
    int32_t evict_first32;  // L2 policy of the FP32 matrix stream (1 evict_first, 0 evict_last)
    unsigned int ticket[8];  // [7] = bounded-wait error word
    double *history;   // error per iteration (may be null)
    double *trend_hist;
};

struct Precond {
    int kind = 0;                 // 0 none, 1 Jacobi, 2 block Jacobi
    uint32_t w = 1;
    const double *d = nullptr;    // Jacobi inverse diagonal / blocks (n*w)
    const float *d32 = nullptr;   // FP32 copies for the mixed-precision inner solver
};

struct CgArgs {
    const rsg_csr *A;
    Precond P;
    const double *b;              // right-hand side (already equation-scaled)
    double *x;                    // in/out
    double *partials;             // >= 4 * kMaxGrid doubles
    CgState *st;
    // FP64 vectors
    double *r, *z, *p0, *p1, *q;
    // FP32 vectors (mixed)
    float *r32, *z32, *p32a, *p32b, *q32, *y32;
    bool mixed;
    bool use_graph;
    uint32_t check_interval;
};

rsg_status cg_run(rsg_context *ctx, const CgArgs &a, double *seconds);

}  // namespace rsg
