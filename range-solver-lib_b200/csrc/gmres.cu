// Restarted GMRES(m) on the GPU, restating RMatrixSolver::solveGMRES
// (src/rmatrixsolver.cpp:357-581):
//   cycle start  true residual ro = b - A x, ||x||, beta = ||ro||, error and
//                stopping rule (:401-427)
//   inner step k v_k = w / h_{k,k-1} (v_0 = ro / beta), z_k = P v_k (:430-446)
//                w = A z_k (:451-455)
//                h_{i,k} = v_i^T w for i <= k, one batched pass (:457-484)
//                w -= sum_i h_{i,k} v_i and ||w|| in one pass (:486-510)
//                Givens rotations on column k, g update, inner exit when
//                |g_{k+1}| < 1e-4 beta (:519-550)
//   cycle end    back substitution (:554-567), x += sum_j z_j y_j (:570-578)
// Z is stored, so a variable preconditioner (flexible GMRES) needs no change.
// Each cycle is one captured CUDA graph; the host polls the device state once
// per cycle.
// Mixed precision: the Arnoldi vectors V, Z, w and the matrix of the inner
// steps are FP32 (dot products accumulated in FP64), while the true residual at
// every restart (FP64 matrix), the Hessenberg matrix, the Givens rotations, the
// least-squares solve and the solution update x += Z y stay FP64 -- restarted
// GMRES as iterative refinement with an FP32 inner cycle.
#include "gmres.cuh"
#include "gnn.cuh"

#include <cmath>

namespace rsg {

template <int RPW>
__global__ void __launch_bounds__(kBlock) k_gm_residual(Csr<double> M, Sell<double> S, int use_sell, const double *__restrict__ b,
                                                        const double *__restrict__ x, double *__restrict__ ro,
                                                        double *__restrict__ H, double *__restrict__ g,
                                                        double *partials, GmresState *st)
{
    pdl_wait();
    pdl_release();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[96];
    if (st->done) return;
    double acc[3] = {0.0, 0.0, 0.0};
    auto gx = [&](uint32_t c) { return x[c]; };
    auto epi = [&](uint32_t row, double ax) {
        const double r = b[row] - ax;
        ro[row] = r;
        acc[0] += x[row] * x[row];
        acc[1] += r * r;
        acc[2] += b[row] * b[row];
    };
    for_rows_any<double, RPW>(M, S, use_sell != 0, gx, epi, smem_raw, &st->ticket[7], true);
    double tot[3];
    if (grid_sum<3>(acc, partials, &st->ticket[0], sh, tot)) {
        const uint32_t m = st->m;
        for (uint32_t i = threadIdx.x; i < (m + 1) * m; i += blockDim.x) H[i] = 0.0;
        for (uint32_t i = threadIdx.x; i <= m; i += blockDim.x) g[i] = 0.0;
        __syncthreads();
        if (threadIdx.x == 0) {
            const double xn = sqrt(tot[0]), beta = sqrt(tot[1]);
            if (st->outer == 0) st->bn = sqrt(tot[2]);
            double norm = st->an * xn + st->bn;
            if (fabs(norm) < st->eps) norm = st->eps;
            const double err = beta / norm;
            st->trend = err - st->error;
            st->error = err;
            st->xn = xn;
            st->beta = beta;
            if (st->history) {
                st->history[st->outer_logged] = err;
                st->trend_hist[st->outer_logged] = st->trend;
            }
            st->outer_logged++;
            bool stop;
            if (st->stop_rule == RSG_STOP_REFERENCE) {
                stop = !dev_isnormal(err) || !dev_isnormal(st->trend) || err < st->cvg || fabs(st->trend) < st->eps * st->eps;
                if (stop) {
                    st->converged = 1;
                    st->status = isfinite(err) ? RSG_OK : RSG_BREAKDOWN;
                }
            } else {
                stop = !(beta > st->rtol * st->bn);
                if (stop) {
                    st->converged = isfinite(beta) ? 1 : 0;
                    st->status = isfinite(beta) ? RSG_OK : RSG_BREAKDOWN;
                }
            }
            if (stop) {
                st->done = 1;
            } else {
                g[0] = beta;
                st->k = 0;
                st->inner_done = 0;
                st->cycle_len = 0;
            }
        }
    }
}

// v_k = src / s (0 if s == 0), z_k = P v_k.  src = ro for k = 0, else w.  T: vector type
// of the Arnoldi vectors (double, or float in mixed precision); D: preconditioner values.
template <int PK, typename T, typename D>
__global__ void __launch_bounds__(kBlock) k_gm_vz(uint32_t n, uint32_t w_, const D *__restrict__ d,
                                                  const double *__restrict__ ro, const T *__restrict__ wv,
                                                  const double *__restrict__ wnorm, T *__restrict__ V,
                                                  T *__restrict__ Z, const GmresState *st, uint32_t k)
{
    pdl_wait();
    pdl_release();
    if (st->done || st->inner_done) return;
    const double s = (k == 0) ? st->beta : wnorm[k];
    T *v = V + size_t(k) * n, *z = Z + size_t(k) * n;
    const uint32_t G = PK == 2 ? w_ : 1, ng = n / G;
    for (uint32_t gi = blockIdx.x * blockDim.x + threadIdx.x; gi < ng; gi += gridDim.x * blockDim.x) {
        T vl[kMaxBlock];
        for (uint32_t j = 0; j < G; j++) {
            const size_t i = size_t(gi) * G + j;
            const double src = (k == 0) ? ro[i] : double(wv[i]);
            vl[j] = T((s == 0.0) ? 0.0 : src / s);
            v[i] = vl[j];
        }
        if (PK == 0) z[gi] = vl[0];
        else if (PK == 1) z[gi] = T(d[gi]) * vl[0];
        else
            for (uint32_t j = 0; j < G; j++) {
                const D *row = d + (size_t(gi) * G + j) * G;
                T acc = T(0);
                for (uint32_t l = 0; l < G; l++) acc += T(row[l]) * vl[l];
                z[size_t(gi) * G + j] = acc;
            }
    }
}

template <int RPW, typename T>
__global__ void __launch_bounds__(kBlock) k_gm_spmv(Csr<T> M, Sell<T> S, int use_sell, const T *__restrict__ Z,
                                                    T *__restrict__ wv, GmresState *st, uint32_t k)
{
    pdl_wait();
    pdl_release();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if (st->done || st->inner_done) return;
    const T *z = Z + size_t(k) * M.n;
    auto gx = [&](uint32_t c) { return z[c]; };
    auto epi = [&](uint32_t row, T v) { wv[row] = v; };
    for_rows_any<T, RPW>(M, S, use_sell != 0, gx, epi, smem_raw, &st->ticket[7], true);
}

// h_i = v_i^T w for i <= k: blockIdx.y = i.  Last block of the 2-D grid stores column k of H.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_gm_dots(uint32_t n, const T *__restrict__ V,
                                                    const T *__restrict__ wv, double *__restrict__ H,
                                                    double *__restrict__ hv, double *partials, GmresState *st,
                                                    uint32_t k)
{
    pdl_wait();
    pdl_release();
    __shared__ double sh[32];
    __shared__ bool is_last;
    if (st->done || st->inner_done) return;
    if (blockIdx.y > k) return;
    const T *v = V + size_t(blockIdx.y) * n;
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc[0] += double(wv[i]) * double(v[i]);
    block_sum<1>(acc, sh);
    const unsigned int nblocks = gridDim.x * (k + 1);
    if (threadIdx.x == 0) {
        partials[size_t(blockIdx.y) * gridDim.x + blockIdx.x] = acc[0];
        __threadfence();
        is_last = (atomicAdd(&st->ticket[1], 1u) == nblocks - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const uint32_t m = st->m;
    for (uint32_t i = 0; i <= k; i++) {
        double s[1] = {0.0};
        for (uint32_t bx = threadIdx.x; bx < gridDim.x; bx += blockDim.x) s[0] += __ldcg(&partials[size_t(i) * gridDim.x + bx]);
        block_sum<1>(s, sh);
        if (threadIdx.x == 0) {
            H[size_t(i) * m + k] = s[0];
            hv[i] = s[0];
        }
    }
    if (threadIdx.x == 0) st->ticket[1] = 0u;
}

// w -= sum_i hv_i v_i; ||w|| -> Givens update of column k (last block).
template <typename T>
__global__ void __launch_bounds__(kBlock) k_gm_correct(uint32_t n, const T *__restrict__ V,
                                                       T *__restrict__ wv, const double *__restrict__ hv_g,
                                                       double *__restrict__ H, double *__restrict__ cs,
                                                       double *__restrict__ sn, double *__restrict__ g,
                                                       double *__restrict__ wnorm, double *partials, GmresState *st,
                                                       uint32_t k)
{
    pdl_wait();
    pdl_release();
    __shared__ double sh[32];
    __shared__ double hv[kMaxRestart + 1];
    if (st->done || st->inner_done) return;
    for (uint32_t i = threadIdx.x; i <= k; i += blockDim.x) hv[i] = hv_g[i];
    __syncthreads();
    double acc[1] = {0.0};
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        double value = double(wv[j]);
        for (uint32_t i = 0; i <= k; i++) value -= hv[i] * double(V[size_t(i) * n + j]);
        const T stored = T(value);
        wv[j] = stored;
        acc[0] += double(stored) * double(stored);
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, &st->ticket[2], sh, tot) && threadIdx.x == 0) {
        const uint32_t m = st->m;
        auto h = [&](uint32_t i, uint32_t j) -> double & { return H[size_t(i) * m + j]; };
        h(k + 1, k) = sqrt(tot[0]);
        // v_{k+1} = w / h_{k+1,k} is formed by the next step's k_gm_vz, after the
        // rotation below has zeroed h_{k+1,k}; keep the norm for it
        wnorm[k + 1] = h(k + 1, k);
        for (uint32_t i = 1; i <= k; i++) {
            const double hsave = h(i - 1, k);
            h(i - 1, k) = cs[i - 1] * hsave + sn[i - 1] * h(i, k);
            h(i, k) = -sn[i - 1] * hsave + cs[i - 1] * h(i, k);
        }
        const double gg = sqrt(h(k, k) * h(k, k) + h(k + 1, k) * h(k + 1, k));
        if (gg == 0.0) {
            cs[k] = sn[k] = 0.0;
        } else {
            cs[k] = h(k, k) / gg;
            sn[k] = h(k + 1, k) / gg;
        }
        h(k, k) = gg;
        h(k + 1, k) = 0.0;
        g[k + 1] = -sn[k] * g[k];
        g[k] = cs[k] * g[k];
        st->total_inner++;
        st->cycle_len = k + 1;
        if (fabs(g[k + 1]) < st->beta * 1.0e-4) st->inner_done = 1;
        st->k = k + 1;
    }
}

__global__ void k_gm_backsub(double *__restrict__ H, double *__restrict__ g, double *__restrict__ y,
                             GmresState *st)
{
    pdl_wait();
    pdl_release();
    if (threadIdx.x != 0 || st->done) return;
    const uint32_t m = st->m, it = st->cycle_len;
    if (it == 0) return;
    auto h = [&](uint32_t i, uint32_t j) -> double & { return H[size_t(i) * m + j]; };
    y[it - 1] = (h(it - 1, it - 1) == 0.0) ? 0.0 : g[it - 1] / h(it - 1, it - 1);
    for (int i = int(it) - 2; i >= 0; i--) {
        for (int j = int(it) - 1; j > i; j--) g[i] -= y[j] * h(i, j);
        y[i] = (h(i, i) == 0.0) ? 0.0 : g[i] / h(i, i);
    }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_gm_update(uint32_t n, const T *__restrict__ Z,
                                                      const double *__restrict__ y_g, double *__restrict__ x,
                                                      GmresState *st)
{
    pdl_wait();
    pdl_release();
    __shared__ double y[kMaxRestart];
    if (st->done) return;
    const uint32_t len = st->cycle_len;
    for (uint32_t j = threadIdx.x; j < len; j += blockDim.x) y[j] = y_g[j];
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double xi = x[i];
        for (uint32_t j = 0; j < len; j++) xi += double(Z[size_t(j) * n + i]) * y[j];
        x[i] = xi;
    }
}

__global__ void k_gm_cycle_end(GmresState *st)
{
    pdl_wait();
    pdl_release();
    if (threadIdx.x != 0) return;
    if (st->done) return;
    st->outer++;
    if (st->outer >= st->max_outer) {
        st->done = 1;
        st->status = RSG_NOT_CONVERGED;
    }
}

size_t gmres_workspace_bytes(uint32_t n, uint32_t m, bool mixed, uint32_t w)
{
    const size_t vn = arena_bytes(n, sizeof(double));
    const size_t vt = mixed ? arena_bytes(size_t(m + 1) * n, sizeof(float)) : arena_bytes(size_t(m + 1) * n, 8);
    return 2 * vt + (mixed ? arena_bytes(n, sizeof(float)) : vn) + vn + arena_bytes(size_t(m + 1) * m, sizeof(double)) +
           6 * arena_bytes(m + 2, sizeof(double)) + (mixed ? arena_bytes(size_t(n) * w, sizeof(float)) : 0);
}

rsg_status gmres_carve(rsg_context *ctx, GmresArgs &a, uint32_t n, uint32_t m)
{
    if (m > kMaxRestart) return set_error(ctx, RSG_ERR_UNSUPPORTED, "GMRES restart length %u > %u", m, kMaxRestart);
    if (a.mixed) {
        a.V32 = arena_take<float>(ctx, size_t(m + 1) * n);
        a.Z32 = arena_take<float>(ctx, size_t(m + 1) * n);
        a.w32 = arena_take<float>(ctx, n);
    } else {
        a.V = arena_take<double>(ctx, size_t(m + 1) * n);
        a.Z = arena_take<double>(ctx, size_t(m + 1) * n);
        a.w = arena_take<double>(ctx, n);
    }
    a.ro = arena_take<double>(ctx, n);
    a.H = arena_take<double>(ctx, size_t(m + 1) * m);
    a.cs = arena_take<double>(ctx, m + 2);
    a.sn = arena_take<double>(ctx, m + 2);
    a.g = arena_take<double>(ctx, m + 2);
    a.y = arena_take<double>(ctx, m + 2);
    a.hv = arena_take<double>(ctx, m + 2);
    a.wnorm = arena_take<double>(ctx, m + 2);
    if (!a.wnorm) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "GMRES workspace");
    return RSG_OK;
}

namespace {

constexpr double kLearnedMinDrop = 0.1;

template <int RPW, int PK>
rsg_status run_typed(rsg_context *ctx, const GmresArgs &a, double *seconds)
{
    const uint32_t n = a.A->n, m = a.m;
    const Csr<double> M = view<double>(a.A, true);
    const size_t s64 = a.A->use_sell ? 0 : tma_smem<double>();
    cudaFuncSetAttribute(k_gm_residual<RPW>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem<double>()));
    cudaFuncSetAttribute(k_gm_spmv<RPW, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(tma_smem<double>()));
    cudaFuncSetAttribute(k_gm_spmv<RPW, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem<float>()));
    const Sell<double> S = sell_view<double>(a.A);
    const Csr<float> M32 = view<float>(a.A, true);
    const Sell<float> S32 = sell_view<float>(a.A);
    const size_t s32 = a.A->use_sell ? 0 : tma_smem<float>();
    const int us = a.A->use_sell;
    const long long ct = (long long)n * 32 / RPW;
    (void)ct;
    const int g_sp = spmv_grid(ctx, a.A, (const void *)k_gm_spmv<RPW, double>, s64, RPW);
    const int g_sp32 = spmv_grid(ctx, a.A, (const void *)k_gm_spmv<RPW, float>, s32, RPW);
    const int g_res = spmv_grid(ctx, a.A, (const void *)k_gm_residual<RPW>, s64, RPW);
    const int g_vec = std::min(grid_for(ctx, (const void *)k_gm_correct<double>, kBlock, 0, n), kMaxGrid);
    const int g_dot =
        std::min(std::min(grid_for(ctx, (const void *)k_gm_dots<double>, kBlock, 0, n), 512), kMaxGrid);

    // One captured graph per cycle; with the learned preconditioner a second graph
    // (Jacobi z_k) is captured as the fallback.
    auto capture = [&](rsg_learned *G, bool pdl, cudaGraph_t *graph, cudaGraphExec_t *exec) -> rsg_status {
        if (G) RSG_TRY(gnn_prepare(ctx, G, a.A, false));  // no allocation inside the capture
        RSG_CHECK_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        cudaStream_t st = ctx->stream;
        launch_k(st, pdl, k_gm_residual<RPW>, g_res, kBlock, s64, M, S, us, a.b, a.x, a.ro, a.H, a.g, a.partials,
                 a.st);
        for (uint32_t k = 0; k < m; k++) {
            if (a.mixed) {  // FP32 Arnoldi step
                launch_k(st, pdl, k_gm_vz<PK, float, float>, g_vec, kBlock, 0, n, a.P.w, a.P.d32, a.ro, a.w32,
                         a.wnorm, a.V32, a.Z32, a.st, k);
                launch_k(st, pdl, k_gm_spmv<RPW, float>, g_sp32, kBlock, s32, M32, S32, us, a.Z32, a.w32, a.st, k);
                launch_k(st, pdl, k_gm_dots<float>, dim3(g_dot, k + 1), kBlock, 0, n, a.V32, a.w32, a.H, a.hv,
                         a.partials, a.st, k);
                launch_k(st, pdl, k_gm_correct<float>, g_vec, kBlock, 0, n, a.V32, a.w32, a.hv, a.H, a.cs, a.sn, a.g,
                         a.wnorm, a.partials, a.st, k);
                continue;
            }
            launch_k(st, pdl, k_gm_vz<PK, double, double>, g_vec, kBlock, 0, n, a.P.w, a.P.d, a.ro, a.w, a.wnorm,
                     a.V, a.Z, a.st, k);
            if (G) {  // flexible GMRES: z_k = M(v_k) from the network (Z is stored, src/rmatrixsolver.cpp:446)
                const rsg_status gs =
                    gnn_forward(ctx, G, a.A, a.V + size_t(k) * n, a.Z + size_t(k) * n, nullptr, false, true);
                if (gs != RSG_OK) {
                    cudaGraph_t dummy = nullptr;
                    cudaStreamEndCapture(ctx->stream, &dummy);
                    if (dummy) cudaGraphDestroy(dummy);
                    return gs;
                }
            }
            launch_k(st, pdl, k_gm_spmv<RPW, double>, g_sp, kBlock, s64, M, S, us, a.Z, a.w, a.st, k);
            launch_k(st, pdl, k_gm_dots<double>, dim3(g_dot, k + 1), kBlock, 0, n, a.V, a.w, a.H, a.hv, a.partials,
                     a.st, k);
            launch_k(st, pdl, k_gm_correct<double>, g_vec, kBlock, 0, n, a.V, a.w, a.hv, a.H, a.cs, a.sn, a.g,
                     a.wnorm, a.partials, a.st, k);
        }
        launch_k(st, pdl, k_gm_backsub, 1, 32, 0, a.H, a.g, a.y, a.st);
        if (a.mixed) launch_k(st, pdl, k_gm_update<float>, g_vec, kBlock, 0, n, a.Z32, a.y, a.x, a.st);
        else launch_k(st, pdl, k_gm_update<double>, g_vec, kBlock, 0, n, a.Z, a.y, a.x, a.st);
        launch_k(st, pdl, k_gm_cycle_end, 1, 32, 0, a.st);
        cudaError_t e = cudaStreamEndCapture(ctx->stream, graph);
        if (e != cudaSuccess) return set_error(ctx, RSG_ERR_CUDA, "GMRES capture: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(exec, *graph, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(*graph);
            *graph = nullptr;
            return set_error(ctx, RSG_ERR_CUDA, "GMRES instantiate: %s", cudaGetErrorString(e));
        }
        return RSG_OK;
    };
    // with programmatic dependent launch when the CG policy picks it for A, else (or if the
    // driver refuses the programmatic edges) plain launches
    auto capture_any = [&](rsg_learned *G, cudaGraph_t *graph, cudaGraphExec_t *exec) -> rsg_status {
        const bool pdl = pdl_for(a.A, a.mixed);
        rsg_status r = capture(G, pdl, graph, exec);
        if (r != RSG_OK && r != RSG_ERR_OUT_OF_MEMORY && pdl) {
            (void)cudaGetLastError();
            r = capture(G, false, graph, exec);
        }
        return r;
    };
    cudaGraph_t graph = nullptr, graph_j = nullptr;
    cudaGraphExec_t exec = nullptr, exec_j = nullptr;
    rsg_status s = capture_any(a.G, &graph, &exec);
    if (s == RSG_OK && a.G) s = capture_any(nullptr, &graph_j, &exec_j);
    if (s != RSG_OK) {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        return s;
    }
    cudaError_t e = cudaSuccess;
    cudaEventRecord(ctx->ev[0], ctx->stream);
    int32_t *done_h = reinterpret_cast<int32_t *>(ctx->pinned);
    double *beta_h = ctx->pinned + 1;
    bool learned = a.G != nullptr;
    double beta_prev = 0.0;
    if (a.fallbacks) *a.fallbacks = 0;
    // k_gm_cycle_end marks the state done after max_outer cycles; the host bound is a backstop
    const uint64_t max_cycles = uint64_t(a.st_max_outer) + 2;
    for (uint64_t cycle = 0; cycle < max_cycles; cycle++) {
        e = cudaGraphLaunch(learned ? exec : (exec_j ? exec_j : exec), ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(done_h, &a.st->done, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess && a.G)
            e = cudaMemcpyAsync(beta_h, &a.st->beta, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) {
            s = set_error(ctx, RSG_ERR_CUDA, "GMRES cycle: %s", cudaGetErrorString(e));
            break;
        }
        if (*done_h) break;
        // beta of this cycle is the residual left by the previous one: a learned cycle
        // that removed less than kLearnedMinDrop of it hands over to Jacobi for good
        if (learned && cycle > 0 && !(*beta_h < (1.0 - kLearnedMinDrop) * beta_prev)) {
            learned = false;
            if (a.fallbacks) (*a.fallbacks)++;
        }
        beta_prev = *beta_h;
    }
    cudaEventRecord(ctx->ev[1], ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    *seconds = ms * 1e-3;
    if (exec_j) cudaGraphExecDestroy(exec_j);
    if (graph_j) cudaGraphDestroy(graph_j);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    return s;
}

}  // namespace

rsg_status gmres_run(rsg_context *ctx, const GmresArgs &a, double *seconds)
{
    const int rpw = pick_rpw(a.A);
    switch (a.P.kind) {
    case 0: RSG_RPW_DISPATCH(rpw, return (run_typed<RPW, 0>(ctx, a, seconds)));
    case 1: RSG_RPW_DISPATCH(rpw, return (run_typed<RPW, 1>(ctx, a, seconds)));
    default: RSG_RPW_DISPATCH(rpw, return (run_typed<RPW, 2>(ctx, a, seconds)));
    }
    return RSG_ERR_UNSUPPORTED;
}

}  // namespace rsg
