// Flexible CG with the learned preconditioner and a Jacobi fallback.
//
// The reference's CG (src/rmatrixsolver.cpp:208-355) assumes a fixed
// preconditioner.  With a variable one (the network's output is a non-linear
// function of r) this is flexible CG with one stored direction (Notay's FCG(1)):
//     p_k = z_k - (z_k^T A p_{k-1} / p_{k-1}^T A p_{k-1}) p_{k-1},
//     alpha_k = p_k^T r_k / p_k^T A p_k,
// which equals the reference's recurrences for a fixed SPD preconditioner.
// The learned step is abandoned for Jacobi (the reference's preconditioner)
// as soon as it fails: z not a descent direction (r^T z <= 0), p^T A p <= 0,
// or no new lowest residual norm for kStall iterations.  Stopping: FP64 true
// relative residual, recomputed before stopping.  The loop is host-driven (one
// short synchronisation per iteration): the network's application is a
// sequence of launches that costs far more than that synchronisation.
#include "gnn.cuh"
#include "krylov.cuh"

namespace rsg {
namespace {

constexpr uint32_t kStall = 10;

// r^T z and z^T q_old (q_old = A p_{k-1})
__global__ void k_fcg_dots(uint32_t n, const double *__restrict__ r, const double *__restrict__ z,
                           const double *__restrict__ q, double *partials, unsigned int *ticket, double *out)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        acc[0] += r[i] * z[i];
        acc[1] += z[i] * q[i];
    }
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

__global__ void k_fcg_jacobi(uint32_t n, const double *__restrict__ d, const double *__restrict__ r,
                             double *__restrict__ z)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        z[i] = d ? d[i] * r[i] : r[i];
}

__global__ void k_fcg_dir(uint32_t n, const double *__restrict__ z, double beta, double *__restrict__ p)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = fma(beta, p[i], z[i]);
}

// p^T q and p^T r
__global__ void k_fcg_pdots(uint32_t n, const double *__restrict__ p, const double *__restrict__ q,
                            const double *__restrict__ r, double *partials, unsigned int *ticket, double *out)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        acc[0] += p[i] * q[i];
        acc[1] += p[i] * r[i];
    }
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        out[0] = tot[0];
        out[1] = tot[1];
    }
}

__global__ void k_fcg_update(uint32_t n, double alpha, const double *__restrict__ p, const double *__restrict__ q,
                             double *__restrict__ x, double *__restrict__ r, double *partials, unsigned int *ticket,
                             double *out)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = fma(alpha, p[i], x[i]);
        const double ri = fma(-alpha, q[i], r[i]);
        r[i] = ri;
        acc[0] += ri * ri;
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) out[0] = tot[0];
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

size_t fcg_workspace_bytes(uint32_t n) { return 4 * arena_bytes(n, sizeof(double)) + arena_bytes(64, 8); }

rsg_status fcg_run(rsg_context *ctx, const rsg_csr *A, rsg_learned *G, const double *d, const double *b, double *x,
                   double *partials, uint32_t max_it, double rtol, FcgResult *res)
{
    const uint32_t n = A->n;
    cudaStream_t sm = ctx->stream;
    double *r = arena_take<double>(ctx, n), *z = arena_take<double>(ctx, n), *p = arena_take<double>(ctx, n),
           *q = arena_take<double>(ctx, n);
    double *sc = arena_take<double>(ctx, 64);
    if (!sc) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "fcg workspace");
    unsigned int *ticket = reinterpret_cast<unsigned int *>(sc + 32);
    double *out = sc;
    double *h = ctx->pinned;
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(sc, 0, 64 * 8, sm));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(p, 0, size_t(n) * 8, sm));
    const int g = std::min(grid_for(ctx, (const void *)k_fcg_update, kBlock, 0, n), kMaxGrid);
    auto fetch = [&](int count) -> rsg_status {
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(h, out, count * sizeof(double), cudaMemcpyDeviceToHost, sm));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
        return RSG_OK;
    };
    if (G) RSG_TRY(gnn_prepare(ctx, G, A, false));
    cudaEventRecord(ctx->ev[0], sm);
    // r = b - A x
    RSG_TRY(spmv64(ctx, A, x, q, true));
    k_fcg_resid<<<g, kBlock, 0, sm>>>(n, b, q, r, partials, ticket, out);
    RSG_TRY(fetch(2));
    const double bn = std::sqrt(h[1]);
    double rn = std::sqrt(h[0]);
    bool learned = G != nullptr;
    double pq_old = 0.0, best = rn;
    uint32_t since_best = 0;
    res->iterations = 0;
    res->fallbacks = 0;
    res->checks = 0;
    res->status = RSG_NOT_CONVERGED;
    bool restart = true;
    auto fall_back = [&]() {
        learned = false;
        res->fallbacks++;
        restart = true;
    };
    if (!(rn > rtol * bn)) {
        res->status = RSG_OK;
        max_it = 0;
    }
    for (uint32_t it = 0; it < max_it; it++) {
        if (learned) RSG_TRY(gnn_forward(ctx, G, A, r, z, nullptr, false, true));
        else k_fcg_jacobi<<<g, kBlock, 0, sm>>>(n, d, r, z);
        k_fcg_dots<<<g, kBlock, 0, sm>>>(n, r, z, q, partials, ticket, out);
        RSG_TRY(fetch(2));
        if (learned && !(h[0] > 0.0)) {  // not a descent direction
            fall_back();
            k_fcg_jacobi<<<g, kBlock, 0, sm>>>(n, d, r, z);
            k_fcg_dots<<<g, kBlock, 0, sm>>>(n, r, z, q, partials, ticket, out);
            RSG_TRY(fetch(2));
        }
        const double beta = restart || !(pq_old > 0.0) ? 0.0 : -h[1] / pq_old;
        restart = false;
        k_fcg_dir<<<g, kBlock, 0, sm>>>(n, z, beta, p);
        RSG_TRY(spmv64(ctx, A, p, q, true));
        k_fcg_pdots<<<g, kBlock, 0, sm>>>(n, p, q, r, partials, ticket, out);
        RSG_TRY(fetch(2));
        const double pq = h[0], pr = h[1];
        if (!(pq > 0.0) || !std::isfinite(pq)) {
            if (learned) {
                fall_back();
                pq_old = 0.0;
                continue;
            }
            res->status = RSG_BREAKDOWN;
            break;
        }
        const double alpha = pr / pq;
        pq_old = pq;
        k_fcg_update<<<g, kBlock, 0, sm>>>(n, alpha, p, q, x, r, partials, ticket, out);
        RSG_TRY(fetch(1));
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
            RSG_TRY(spmv64(ctx, A, x, q, true));
            k_fcg_resid<<<g, kBlock, 0, sm>>>(n, b, q, r, partials, ticket, out);
            RSG_TRY(fetch(2));
            rn = std::sqrt(h[0]);
            if (rn <= rtol * bn) {
                res->status = RSG_OK;
                break;
            }
            restart = true;
            pq_old = 0.0;
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
