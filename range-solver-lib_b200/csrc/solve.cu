// rsg_solve: the GPU replacement of RMatrixSolver::solve (src/rmatrixsolver.cpp:158-201).
//
// Steps, in the reference's order: build the preconditioner
// (RMatrixPreconditioner ctor, src/rmatrixpreconditioner.cpp:16-35), take
// ||A||_F from the matrix handle (computed at upload, :37-51), scale b and x by
// 1e9 ||A||_F / ||b|| (:164-184), run CG or GMRES, undo the scaling (:198).
// Afterwards the FP64 true relative residual of the returned x is recomputed
// on the GPU and reported, and the per-iteration errors are printed / written
// in RIterationInfo's formats (src/riterationinfo.cpp:111-193) when asked.
#include <cstdlib>

#include "amg.cuh"
#include "gmres.cuh"
#include "gnn.cuh"
#include "krylov.cuh"

#include <chrono>
#include <cstring>

namespace rsg {

__global__ void k_norm2(uint32_t n, const double *__restrict__ v, double *partials, unsigned int *ticket,
                        double *out)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc[0] += v[i] * v[i];
    double tot[1];
    if (grid_sum<1>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) *out = sqrt(tot[0]);
}

__global__ void k_scale(uint32_t n, const double *__restrict__ src, double *__restrict__ dst, double s)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[i] * s;
}

__global__ void k_to_f32(size_t n, const double *__restrict__ src, float *__restrict__ dst)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dst[i] = float(src[i]);
}

static void write_log(const rsg_solver_conf &c, const char *title, uint32_t iters, const double *err,
                      const double *trend, bool converged)
{
    if (c.output_frequency > 0) {
        std::printf("-------------------------------------------------------------------------------\n");
        std::printf("%s\n", title);
        std::printf("-------------------------------------------------------------------------------\n");
        std::printf(">    Iteration     |   Residual   |    Trend     |                             \n");
        std::printf("-------------------------------------------------------------------------------\n");
    }
    FILE *f = nullptr;
    bool first = false;
    if (c.output_file && c.output_file[0]) {
        FILE *probe = std::fopen(c.output_file, "r");
        first = (probe == nullptr);
        if (probe) std::fclose(probe);
        f = std::fopen(c.output_file, "a");
        if (f && first) std::fprintf(f, "Iteration number|Solver residual|Solver convergence\n");
    }
    for (uint32_t it = 0; it < iters; it++) {
        const bool last = (it + 1 == iters) && converged;
        if (c.output_frequency == 0) break;
        if (!last && it % c.output_frequency != 0) continue;
        std::printf("> %6u of %-6u |% 12e |% 12e |\n", it + 1, c.n_outer, err[it], trend[it]);
        if (f) std::fprintf(f, "%u|%.7e|%.7e\n", it + 1, err[it], trend[it]);
    }
    if (c.output_frequency > 0)
        std::printf("-------------------------------------------------------------------------------\n");
    if (f) std::fclose(f);
}

}  // namespace rsg

using namespace rsg;

extern "C" rsg_status rsg_solve(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf_in, int32_t prec_type,
                                uint32_t block_size, const double *b, double *x, int32_t memory, rsg_stats *stats)
{
    if (!ctx || !A || !conf_in || !b || !x) return set_error(ctx, RSG_ERR_INVALID_ARG, "solve: null argument");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const auto t_start = std::chrono::steady_clock::now();
    rsg_solver_conf c = *conf_in;
    rsg_stats st_out;
    std::memset(&st_out, 0, sizeof(st_out));
    if (c.solver_type != RSG_SOLVER_CG && c.solver_type != RSG_SOLVER_GMRES)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "Unknown matrix solver type '%d'", c.solver_type);
    if (prec_type < RSG_PREC_NONE || prec_type > RSG_PREC_AMG)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "Invalid matrix preconditioner type '%d'", prec_type);
    if (prec_type == RSG_PREC_AMG && (c.solver_type != RSG_SOLVER_CG || c.precision != RSG_PRECISION_MIXED))
        return set_error(ctx, RSG_ERR_UNSUPPORTED,
                         "the multilevel preconditioner runs in the mixed-precision CG (solver CG, precision MIXED)");
    rsg_learned *G = static_cast<rsg_learned *>(const_cast<void *>(c.learned));
    if ((prec_type == RSG_PREC_LEARNED || c.learned_initial_guess) && !G)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "learned preconditioner requested without conf.learned");
    if (prec_type == RSG_PREC_LEARNED && c.solver_type == RSG_SOLVER_CG && c.stop_rule != RSG_STOP_TRUE_RELRES)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "flexible CG with the learned preconditioner needs TRUE_RELRES");
    if (prec_type == RSG_PREC_LEARNED && c.precision != RSG_PRECISION_FP64)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "the learned preconditioner runs with FP64 Krylov vectors");
    const bool learned = prec_type == RSG_PREC_LEARNED;
    if (learned) c.flexible = 1;
    if (c.autotune && !A->tune.valid) RSG_TRY(autotune_run(ctx, A, std::getenv("RSG_TUNE_CACHE")));
    if (c.precision == RSG_PRECISION_AUTO && (c.solver_type != RSG_SOLVER_CG || prec_type == RSG_PREC_AMG || learned))
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "precision AUTO is for CG with NONE, JACOBI or BLOCK_JACOBI");
    if ((c.precision == RSG_PRECISION_MIXED || c.precision == RSG_PRECISION_AUTO) && c.stop_rule != RSG_STOP_TRUE_RELRES)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "mixed precision requires stop_rule TRUE_RELRES");
    if (c.precision < RSG_PRECISION_FP64 || c.precision > RSG_PRECISION_AUTO)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "Invalid precision '%d'", c.precision);
    const uint32_t n = A->n;
    const bool mixed = c.precision == RSG_PRECISION_MIXED || c.precision == RSG_PRECISION_AUTO;
    const bool gmres = c.solver_type == RSG_SOLVER_GMRES;
    const uint32_t w = prec_type == RSG_PREC_BLOCK_JACOBI ? block_width(n, block_size) : 1;
    const uint32_t max_it = std::max<uint32_t>(c.n_outer, 1);
    const uint32_t m = std::max<uint32_t>(c.n_inner, 1);
    const bool want_hist = c.output_frequency > 0 || (c.output_file && c.output_file[0]);
    const uint32_t hist_len = gmres ? max_it + 1 : max_it;

    // ---- workspace ----
    const size_t vn = arena_bytes(n, sizeof(double)), vf = arena_bytes(n, sizeof(float));
    size_t bytes = 0;
    bytes += 2 * vn;                                   // b_dev, x_dev
    bytes += vn;                                       // y = scaled b
    bytes += arena_bytes(size_t(n) * w, sizeof(double));
    bytes += arena_bytes(size_t(4) * kMaxGrid * 32, sizeof(double));  // partials (GMRES multi-dot needs m+1 each)
    bytes += arena_bytes(1, sizeof(CgState)) + arena_bytes(1, sizeof(GmresState));
    bytes += arena_bytes(64, sizeof(double));
    if (want_hist) bytes += 2 * arena_bytes(hist_len, sizeof(double));
    if (learned && !gmres) {
        bytes += fcg_workspace_bytes(n, fcg_dirs(c.n_inner));
    } else if (!gmres) {
        bytes += 5 * vn;                               // r z p0 p1 q
        if (mixed) bytes += 6 * vf + arena_bytes(size_t(n) * w, sizeof(float));
    } else {
        bytes += gmres_workspace_bytes(n, m, mixed, w);
    }
    RSG_TRY(arena_reserve(ctx, bytes));
    double *b_dev = memory == RSG_MEM_HOST ? arena_take<double>(ctx, n) : const_cast<double *>(b);
    double *x_dev = memory == RSG_MEM_HOST ? arena_take<double>(ctx, n) : x;
    double *y = arena_take<double>(ctx, n);
    double *d = arena_take<double>(ctx, size_t(n) * w);
    double *partials = arena_take<double>(ctx, size_t(4) * kMaxGrid * 32);
    CgState *cst = arena_take<CgState>(ctx, 1);
    GmresState *gst = arena_take<GmresState>(ctx, 1);
    double *scal = arena_take<double>(ctx, 64);
    double *hist = want_hist ? arena_take<double>(ctx, hist_len) : nullptr;
    double *thist = want_hist ? arena_take<double>(ctx, hist_len) : nullptr;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scal + 32);

    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(scal, 0, 64 * sizeof(double), ctx->stream));
    if (memory == RSG_MEM_HOST) {
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(b_dev, b, size_t(n) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(x_dev, x, size_t(n) * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    }

    // ---- preconditioner ----
    Precond P;
    P.kind = learned ? RSG_PREC_JACOBI : (prec_type == RSG_PREC_AMG ? 3 : prec_type);
    P.w = w;
    if (prec_type == RSG_PREC_AMG) {
        RSG_TRY(amg_setup(ctx, A, c.persistent > 0));  // rebuilt from the current values on every solve
    } else if (prec_type == RSG_PREC_JACOBI || learned) {
        RSG_TRY(jacobi_build(ctx, A, d));
    } else if (prec_type == RSG_PREC_BLOCK_JACOBI) {
        unsigned int *flag = ticket + 8;
        RSG_TRY(block_jacobi_build(ctx, A, w, d, flag));
        unsigned int hflag = 0;
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&hflag, flag, sizeof(hflag), cudaMemcpyDeviceToHost, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (hflag) return set_error(ctx, RSG_ERR_SINGULAR, "block Jacobi: singular diagonal block");
    }
    P.d = d;

    // ---- equation scaling ----
    {
        const int g = std::min(grid_for(ctx, (const void *)k_norm2, kBlock, 0, n), kMaxGrid);
        k_norm2<<<g, kBlock, 0, ctx->stream>>>(n, b_dev, partials, ticket, scal);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->pinned, scal, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    const double bn = ctx->pinned[0], an = A->norm;
    double scale = 1.0;
    if (c.scale_equations && bn != 0.0 && an != 0.0) scale = 1.0e9 / std::abs(bn / an);
    st_out.norm_a = an;
    st_out.norm_b = bn;
    st_out.equation_scale = scale;
    const int gv = std::min(grid_for(ctx, (const void *)k_scale, kBlock, 0, n), kMaxGrid);
    k_scale<<<gv, kBlock, 0, ctx->stream>>>(n, b_dev, y, scale);
    if (scale != 1.0) k_scale<<<gv, kBlock, 0, ctx->stream>>>(n, x_dev, x_dev, scale);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());

    if (c.learned_initial_guess) {
        // x0 = M(b): the network's estimate of A^{-1} b (M is positively homogeneous,
        // so the equation scaling carries over)
        RSG_TRY(gnn_forward(ctx, G, A, y, x_dev, nullptr, false, true));
    }

    double solve_seconds = 0.0;
    rsg_status solve_status = RSG_OK;
    if (learned && !gmres) {
        FcgResult fr;
        RSG_TRY(fcg_run(ctx, A, G, d, y, x_dev, partials, max_it, c.rtol, fcg_dirs(c.n_inner), &fr));
        st_out.iterations = fr.iterations;
        st_out.outer = fr.checks;
        st_out.fallbacks = fr.fallbacks;
        st_out.converged = fr.status == RSG_OK;
        st_out.error = fr.bn > 0.0 ? fr.rn / fr.bn : fr.rn;
        solve_seconds = fr.seconds;
        solve_status = rsg_status(fr.status);
    } else if (!gmres) {
        CgArgs a = {};
        a.A = A;
        a.b = y;
        a.x = x_dev;
        a.partials = partials;
        a.st = cst;
        a.r = arena_take<double>(ctx, n);
        a.z = arena_take<double>(ctx, n);
        a.p0 = arena_take<double>(ctx, n);
        a.p1 = arena_take<double>(ctx, n);
        a.q = arena_take<double>(ctx, n);
        a.mixed = mixed;
        a.use_graph = c.use_graph != 0;
        a.persistent = c.persistent;
        a.check_interval = std::max<uint32_t>(2, c.check_interval);
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.p0, 0, size_t(n) * sizeof(double), ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.p1, 0, size_t(n) * sizeof(double), ctx->stream));
        if (mixed) {
            a.r32 = arena_take<float>(ctx, n);
            a.z32 = arena_take<float>(ctx, n);
            a.p32a = arena_take<float>(ctx, n);
            a.p32b = arena_take<float>(ctx, n);
            a.q32 = arena_take<float>(ctx, n);
            a.y32 = arena_take<float>(ctx, n);
            float *d32 = arena_take<float>(ctx, size_t(n) * w);
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.p32a, 0, size_t(n) * sizeof(float), ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.p32b, 0, size_t(n) * sizeof(float), ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.y32, 0, size_t(n) * sizeof(float), ctx->stream));
            if (prec_type == RSG_PREC_JACOBI || prec_type == RSG_PREC_BLOCK_JACOBI)
                k_to_f32<<<gv, kBlock, 0, ctx->stream>>>(size_t(n) * w, d, d32);
            P.d32 = d32;
        }
        a.P = P;
        a.amg = prec_type == RSG_PREC_AMG ? amg_of(A) : nullptr;
        a.amg_sweeps = c.amg_sweeps == 2 ? 2 : 1;
        if (a.amg) {
            a.P.d32 = amg_finest_weights(a.amg);  // omega / a_ii: the V-cycle's first smoothing step
            a.amg_x0 = amg_finest_x0(a.amg);
        }
        CgState h;
        std::memset(&h, 0, sizeof(h));
        h.an = an;
        h.cvg = c.cvg;
        h.eps = c.eps;
        h.rtol = c.rtol;
        h.delta = c.reliable_delta > 0.0 && c.reliable_delta < 1.0 ? c.reliable_delta : kReliableDelta;
        h.sigma = 1.0;
        h.max_it = max_it;
        h.stop_rule = c.stop_rule;
        h.body_limit = max_it / 2 + 16;
        h.history = hist;
        h.trend_hist = thist;
        h.evict_first32 = c.l2_resident_f32 ? 0 : 1;
        h.auto_switch = c.precision == RSG_PRECISION_AUTO ? 1 : 0;
        const CgState h_init = h;
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(cst, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
        RSG_TRY(cg_run(ctx, a, &solve_seconds));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, cst, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        uint32_t logged = h.it, outer = h.n_updates;
        if (h.switched) {
            // precision AUTO: the FP32 recurrence drifted -- continue in FP64 from the folded x with the
            // iterations left (fresh directions; the history continues where it stopped)
            const uint32_t used = h.it;
            CgArgs a64 = a;
            a64.mixed = false;
            CgState h2 = h_init;
            h2.auto_switch = 0;
            h2.max_it = max_it > used ? max_it - used : 1;
            h2.body_limit = h2.max_it / 2 + 16;
            h2.history = hist ? hist + used : nullptr;
            h2.trend_hist = thist ? thist + used : nullptr;
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a64.p0, 0, size_t(n) * sizeof(double), ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a64.p1, 0, size_t(n) * sizeof(double), ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(cst, &h2, sizeof(h2), cudaMemcpyHostToDevice, ctx->stream));
            double s2 = 0.0;
            RSG_TRY(cg_run(ctx, a64, &s2));
            solve_seconds += s2;
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, cst, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            st_out.fp64_iterations = h.it;
            logged = used + h.it;
            outer += h.n_updates;
        }
        st_out.iterations = logged;
        st_out.outer = outer;
        st_out.error = h.error;
        st_out.trend = h.trend;
        st_out.converged = h.converged;
        solve_status = h.ticket[7] ? RSG_ERR_TIMEOUT : rsg_status(h.status);
        if (want_hist) {
            h.it = logged;
            std::vector<double> e(h.it), t(h.it);
            cudaMemcpy(e.data(), hist, h.it * sizeof(double), cudaMemcpyDeviceToHost);
            cudaMemcpy(t.data(), thist, h.it * sizeof(double), cudaMemcpyDeviceToHost);
            write_log(c, "Conjugate Gradient", h.it, e.data(), t.data(), h.converged != 0);
        }
    } else {
        GmresArgs a = {};
        a.A = A;
        a.P = P;
        a.b = y;
        a.x = x_dev;
        a.partials = partials;
        a.st = gst;
        a.m = m;
        a.flexible = c.flexible != 0;
        a.G = learned ? G : nullptr;
        a.mixed = mixed;
        uint32_t gm_fallbacks = 0;
        a.fallbacks = &gm_fallbacks;
        a.st_max_outer = max_it;
        RSG_TRY(gmres_carve(ctx, a, n, m));
        if (mixed && prec_type != RSG_PREC_NONE) {  // FP32 copy of the preconditioner for the inner steps
            float *d32 = arena_take<float>(ctx, size_t(n) * w);
            if (!d32) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "GMRES workspace");
            k_to_f32<<<gv, kBlock, 0, ctx->stream>>>(size_t(n) * w, d, d32);
            a.P.d32 = d32;
        }
        GmresState h;
        std::memset(&h, 0, sizeof(h));
        h.an = an;
        h.cvg = c.cvg;
        h.eps = c.eps;
        h.rtol = c.rtol;
        h.max_outer = max_it;
        h.m = m;
        h.stop_rule = c.stop_rule;
        h.history = hist;
        h.trend_hist = thist;
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(gst, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
        RSG_TRY(gmres_run(ctx, a, &solve_seconds));
        st_out.fallbacks = gm_fallbacks;
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, gst, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        st_out.iterations = h.total_inner;
        st_out.outer = h.outer;
        st_out.error = h.error;
        st_out.trend = h.trend;
        st_out.converged = h.converged;
        solve_status = h.ticket[7] ? RSG_ERR_TIMEOUT : rsg_status(h.status);
        if (want_hist) {
            std::vector<double> e(h.outer_logged), t(h.outer_logged);
            cudaMemcpy(e.data(), hist, h.outer_logged * sizeof(double), cudaMemcpyDeviceToHost);
            cudaMemcpy(t.data(), thist, h.outer_logged * sizeof(double), cudaMemcpyDeviceToHost);
            write_log(c, "Generalized Minimal Residual", h.outer_logged, e.data(), t.data(), h.converged != 0);
        }
    }

    // ---- unscale, true residual, download ----
    if (scale != 1.0) k_scale<<<gv, kBlock, 0, ctx->stream>>>(n, x_dev, x_dev, 1.0 / scale);
    {
        unsigned int *t2 = ticket + 4;
        RSG_TRY(true_residual(ctx, A, b_dev, x_dev, partials, t2, scal + 8));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->pinned, scal + 8, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                            ctx->stream));
    }
    if (memory == RSG_MEM_HOST)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(x, x_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    st_out.true_relres = ctx->pinned[2];
    st_out.seconds_solve = solve_seconds;
    st_out.seconds_setup =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count() - solve_seconds;
    st_out.status = solve_status;
    if (stats) *stats = st_out;
    if (solve_status == RSG_ERR_TIMEOUT)
        return set_error(ctx, RSG_ERR_TIMEOUT, "solve loop hit its hard limit or a bounded copy wait ran out");
    return solve_status;
}
