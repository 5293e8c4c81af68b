// Flexible CG with the learned preconditioner and a Jacobi fallback.
//
// The reference's CG (src/rmatrixsolver.cpp:208-355) assumes a fixed
// preconditioner.  With a variable one (the network's output is a non-linear
// function of r) this is truncated flexible CG, FCG(m) (Notay, SIAM J. Sci.
// Comput. 22, 2000): the new direction is A-orthogonalised against the last m
// stored directions,
//     p_k = z_k - sum_j (z_k^T A p_j / p_j^T A p_j) p_j,   j = k-m .. k-1,
//     alpha_k = p_k^T r_k / p_k^T A p_k,
// which for a fixed SPD preconditioner reproduces the reference's recurrences
// (the extra coefficients vanish in exact arithmetic).  m = min(n_inner, 16).
// The learned step is abandoned for Jacobi (the reference's preconditioner)
// as soon as it fails: z not a descent direction (r^T z <= 0), p^T A p <= 0,
// or no new lowest residual norm for kStall iterations.  Stopping: FP64 true
// relative residual, recomputed before stopping.  The loop is host-driven with
// one short synchronisation per iteration: the scalars (coefficients, alpha)
// stay on the device, and the host reads back only ||r||^2 and the failure flags.
#include "gnn.cuh"
#include "krylov.cuh"

namespace rsg {
namespace {

constexpr uint32_t kStall = 25;
constexpr int kDotsNV = kFcgMaxDirs + 1;

struct DirCoef {
    int slot[kFcgMaxDirs];
    int cnt;
};

// device-side scalars of the loop (inside the solver's small scratch block)
struct FcgDev {
    double coef[kFcgMaxDirs];     // z^T A p_j / p_j^T A p_j of the stored directions
    double pq_slot[kFcgMaxDirs + 1];  // p^T A p of the direction held in each slot
    double alpha;
    double rn2;                   // ||r||^2 after the update   } read back together
    double flags;                 // 1: not a descent direction, 2: p^T A p <= 0 }
};

// out[0] = r^T z, out[1 + j] = z^T Q[slot j] (j < cnt)
__global__ void k_fcg_mdots(uint32_t n, const double *__restrict__ r, const double *__restrict__ z,
                            const double *__restrict__ Q, DirCoef dc, double *partials, unsigned int *ticket,
                            FcgDev *dev, int check_descent)
{
    __shared__ double sh[32 * kDotsNV];
    double acc[kDotsNV];
#pragma unroll
    for (int k = 0; k < kDotsNV; k++) acc[k] = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double zi = z[i];
        acc[0] += r[i] * zi;
#pragma unroll
        for (int j = 0; j < kFcgMaxDirs; j++)
            if (j < dc.cnt) acc[1 + j] += zi * Q[size_t(dc.slot[j]) * n + i];
    }
    double tot[kDotsNV];
    if (grid_sum<kDotsNV>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        dev->flags = (check_descent && !(tot[0] > 0.0)) ? 1.0 : 0.0;
        for (int j = 0; j < dc.cnt; j++) dev->coef[j] = tot[1 + j] / dev->pq_slot[dc.slot[j]];
    }
}

__global__ void k_fcg_jacobi(uint32_t n, const double *__restrict__ d, const double *__restrict__ r,
                             double *__restrict__ z)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = d ? d[i] * r[i] : r[i];
}

// p = z - sum_j c_j P[slot j]
__global__ void k_fcg_newdir(uint32_t n, const double *__restrict__ z, const double *__restrict__ P, DirCoef dc,
                             const FcgDev *__restrict__ dev, double *__restrict__ p)
{
    double c[kFcgMaxDirs];
#pragma unroll
    for (int j = 0; j < kFcgMaxDirs; j++) c[j] = j < dc.cnt ? dev->coef[j] : 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = z[i];
#pragma unroll
        for (int j = 0; j < kFcgMaxDirs; j++)
            if (j < dc.cnt) v = fma(-c[j], P[size_t(dc.slot[j]) * n + i], v);
        p[i] = v;
    }
}

// p^T q and p^T r
__global__ void k_fcg_pdots(uint32_t n, const double *__restrict__ p, const double *__restrict__ q,
                            const double *__restrict__ r, double *partials, unsigned int *ticket, FcgDev *dev,
                            int slot)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        acc[0] += p[i] * q[i];
        acc[1] += p[i] * r[i];
    }
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        const double pq = tot[0];
        if (!(pq > 0.0) || !isfinite(pq)) {
            dev->flags = dev->flags + 2.0;
        } else {
            dev->alpha = tot[1] / pq;
            dev->pq_slot[slot] = pq;
        }
    }
}

// x += alpha p, r -= alpha q, ||r||^2 -- skipped when this iteration failed
__global__ void k_fcg_update(uint32_t n, const double *__restrict__ p, const double *__restrict__ q,
                             double *__restrict__ x, double *__restrict__ r, double *partials, unsigned int *ticket,
                             FcgDev *dev)
{
    __shared__ double sh[32];
    if (dev->flags != 0.0) return;
    const double alpha = dev->alpha;
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        acc[0] += ri * ri;
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) dev->rn2 = tot[0];
}

__global__ void k_fcg_resid(uint32_t n, const double *__restrict__ b, const double *__restrict__ ax,
                            double *__restrict__ r, double *partials, unsigned int *ticket, double *out)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ri = b[i] - ax[i];
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += b[i] * b[i];
    }
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

}  // namespace

uint32_t fcg_dirs(uint32_t n_inner) { return std::max<uint32_t>(1, std::min<uint32_t>(n_inner, kFcgMaxDirs)); }

size_t fcg_workspace_bytes(uint32_t n, uint32_t m)
{
    return 2 * arena_bytes(n, sizeof(double)) + 2 * arena_bytes(size_t(m + 1) * n, sizeof(double)) +
           arena_bytes(64, 8) + arena_bytes(sizeof(FcgDev), 1);
}

rsg_status fcg_run(rsg_context *ctx, const rsg_csr *A, rsg_learned *G, const double *d, const double *b, double *x,
                   double *partials, uint32_t max_it, double rtol, uint32_t m, FcgResult *res)
{
    const uint32_t n = A->n;
    cudaStream_t sm = ctx->stream;
    const uint32_t slots = m + 1;  // m stored directions + the one being built
    double *r = arena_take<double>(ctx, n), *z = arena_take<double>(ctx, n);
    double *P = arena_take<double>(ctx, size_t(slots) * n), *Q = arena_take<double>(ctx, size_t(slots) * n);
    double *sc = arena_take<double>(ctx, 64);
    FcgDev *dev = reinterpret_cast<FcgDev *>(arena_take<char>(ctx, sizeof(FcgDev)));
    if (!sc || !dev) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "fcg workspace");
    unsigned int *ticket = reinterpret_cast<unsigned int *>(sc + 32);
    double *out = sc;
    double *h = ctx->pinned;
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(sc, 0, 64 * 8, sm));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(dev, 0, sizeof(FcgDev), sm));
    const int g = std::min(grid_for(ctx, (const void *)k_fcg_update, kBlock, 0, n), kMaxGrid);
    auto fetch = [&](int count) -> rsg_status {
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(h, out, count * sizeof(double), cudaMemcpyDeviceToHost, sm));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
        return RSG_OK;
    };
    if (G) RSG_TRY(gnn_prepare(ctx, G, A, false));
    cudaEventRecord(ctx->ev[0], sm);
    // r = b - A x (Q slot 0 as scratch)
    RSG_TRY(spmv64(ctx, A, x, Q, true));
    k_fcg_resid<<<g, kBlock, 0, sm>>>(n, b, Q, r, partials, ticket, out);
    RSG_TRY(fetch(2));
    const double bn = std::sqrt(h[1]);
    double rn = std::sqrt(h[0]);
    bool learned = G != nullptr;
    double best = rn;
    uint32_t since_best = 0;
    // stored directions, oldest first (their p^T A p stay on the device)
    int ring_slot[kFcgMaxDirs];
    uint32_t cnt = 0, next_slot = 0;
    res->iterations = 0;
    res->fallbacks = 0;
    res->checks = 0;
    res->status = RSG_NOT_CONVERGED;
    auto fall_back = [&]() {
        learned = false;
        res->fallbacks++;
        cnt = 0;
    };
    if (!(rn > rtol * bn)) {
        res->status = RSG_OK;
        max_it = 0;
    }
    for (uint32_t it = 0; it < max_it; it++) {
        DirCoef dc;
        dc.cnt = int(cnt);
        for (uint32_t j = 0; j < cnt; j++) dc.slot[j] = ring_slot[j];
        const int slot = int(next_slot);
        double *p = P + size_t(slot) * n, *q = Q + size_t(slot) * n;
        if (learned) RSG_TRY(gnn_forward(ctx, G, A, r, z, nullptr, false, true));
        else k_fcg_jacobi<<<g, kBlock, 0, sm>>>(n, d, r, z);
        k_fcg_mdots<<<g, kBlock, 0, sm>>>(n, r, z, Q, dc, partials, ticket, dev, learned ? 1 : 0);
        k_fcg_newdir<<<g, kBlock, 0, sm>>>(n, z, P, dc, dev, p);
        RSG_TRY(spmv64(ctx, A, p, q, true));
        k_fcg_pdots<<<g, kBlock, 0, sm>>>(n, p, q, r, partials, ticket, dev, slot);
        k_fcg_update<<<g, kBlock, 0, sm>>>(n, p, q, x, r, partials, ticket, dev);
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(h, &dev->rn2, 2 * sizeof(double), cudaMemcpyDeviceToHost, sm));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
        const int flags = int(h[1]);
        if (flags != 0) {  // the iteration was not applied
            if (learned) {  // not a descent direction, or p^T A p <= 0: hand over to Jacobi
                fall_back();
                continue;
            }
            res->status = RSG_BREAKDOWN;
            break;
        }
        // keep p_k: drop the oldest stored direction when m are held
        if (cnt == m) {
            for (uint32_t j = 1; j < cnt; j++) ring_slot[j - 1] = ring_slot[j];
            cnt--;
        }
        ring_slot[cnt] = slot;
        cnt++;
        // the next free slot is the one no stored direction uses
        for (uint32_t s = 0; s < slots; s++) {
            bool used = false;
            for (uint32_t j = 0; j < cnt; j++) used |= ring_slot[j] == int(s);
            if (!used) {
                next_slot = s;
                break;
            }
        }
        rn = std::sqrt(h[0]);
        res->iterations = it + 1;
        if (!std::isfinite(rn)) {
            res->status = RSG_BREAKDOWN;
            break;
        }
        if (rn < best) {
            best = rn;
            since_best = 0;
        } else if (learned && ++since_best >= kStall) {
            fall_back();
        }
        if (rn <= rtol * bn) {  // recompute the true residual before stopping
            res->checks++;
            double *ax = Q + size_t(next_slot) * n;  // free slot as scratch
            RSG_TRY(spmv64(ctx, A, x, ax, true));
            k_fcg_resid<<<g, kBlock, 0, sm>>>(n, b, ax, r, partials, ticket, out);
            RSG_TRY(fetch(2));
            rn = std::sqrt(h[0]);
            if (rn <= rtol * bn) {
                res->status = RSG_OK;
                break;
            }
            cnt = 0;  // restart the directions on the recomputed residual
        }
    }
    cudaEventRecord(ctx->ev[1], sm);
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    res->seconds = ms * 1e-3;
    res->rn = rn;
    res->bn = bn;
    return RSG_OK;
}

}  // namespace rsg
