// Internal interface of restarted (flexible) GMRES.
#pragma once

#include "krylov.cuh"

namespace rsg {

constexpr uint32_t kMaxRestart = 128;

struct GmresState {
    double beta;          // ||r|| at the start of the current cycle
    double bn, an, xn;
    double error, trend, cvg, eps, rtol;
    uint32_t m, max_outer;
    uint32_t outer;       // cycles started
    uint32_t outer_logged;
    uint32_t total_inner;
    uint32_t k;           // current inner step
    uint32_t cycle_len;   // Krylov vectors used by the current cycle
    int32_t inner_done;
    int32_t done, status, converged, stop_rule;
    unsigned int ticket[8];
    double *history;
    double *trend_hist;
};

struct GmresArgs {
    const rsg_csr *A;
    Precond P;
    const double *b;
    double *x;
    double *partials;     // >= (m+1) * kMaxGrid doubles
    GmresState *st;
    uint32_t m;
    bool flexible;
    // carved buffers (V, Z, w in FP64, or V32, Z32, w32 in mixed precision)
    double *V, *Z, *w, *ro, *H, *cs, *sn, *g, *y, *hv, *wnorm;
    bool mixed = false;
    float *V32 = nullptr, *Z32 = nullptr, *w32 = nullptr;
    uint32_t st_max_outer;
    rsg_learned *G = nullptr;   // learned (variable) preconditioner: z_k = M(v_k)
    uint32_t *fallbacks = nullptr;  // out: cycles handed over to Jacobi
};

size_t gmres_workspace_bytes(uint32_t n, uint32_t m, bool mixed, uint32_t w);
rsg_status gmres_carve(rsg_context *ctx, GmresArgs &a, uint32_t n, uint32_t m);
rsg_status gmres_run(rsg_context *ctx, const GmresArgs &a, double *seconds);

}  // namespace rsg
