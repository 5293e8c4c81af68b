// Autotuner of the CG loop's launch shapes.
//
// The reference has nothing to tune (its loops are OpenMP over rows,
// src/rmatrixsolver.cpp:233-354).  Here the solve's time per iteration depends
// on the matrix layout (SELL-32, or the CSR stream with some rows per warp
// chunk) and on the grid sizes of the two kernels of each iteration (the fused
// direction + SpMV kernel and the update kernel).  The tuner runs short,
// fixed-length solves of A itself through rsg_solve for each candidate -- the
// same graph-driven loop as a real solve, so L2 traffic between the kernels is
// what a solve sees -- and keeps the fastest shapes in A.  The built-in
// defaults are always a candidate, so tuning never selects shapes that were
// measured slower than them.  Last, per precision, the loop is timed with
// programmatic dependent launch switched the other way from its size default.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "krylov.cuh"

namespace rsg {
namespace {

constexpr uint32_t kTuneIters = 64;  // iterations of each timed solve
constexpr int kTuneReps = 3;         // timed solves per candidate (median)

__global__ void k_fill(uint32_t n, double v, double *__restrict__ x)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = v;
}

// candidate grids: 0 (the built-in default), multiples of the SM count, one block per 256 items
std::vector<int> grid_candidates(const rsg_context *ctx, long long items)
{
    std::vector<int> g;
    for (int k : {1, 2, 3, 4, 6, 8}) g.push_back(k * ctx->num_sms);
    g.push_back(int(std::min<long long>(std::max<long long>((items + kBlock - 1) / kBlock, 1), kMaxGrid)));
    std::sort(g.begin(), g.end());
    g.erase(std::unique(g.begin(), g.end()), g.end());
    return g;
}

std::string tune_key(const rsg_context *ctx, const rsg_csr *A)
{
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    std::string name(prop.name);
    for (char &c : name)
        if (c == ' ') c = '_';
    char buf[256];
    std::snprintf(buf, sizeof(buf), "rsg-tune-v2 %s sms=%d n=%u nnz=%llu maxrow=%u sell=%d", name.c_str(),
                  ctx->num_sms, A->n, (unsigned long long)A->nnz, A->max_row, A->sval ? 1 : 0);
    return buf;
}

bool tune_load(const char *path, const std::string &key, rsg_csr *A)
{
    FILE *f = std::fopen(path, "r");
    if (!f) return false;
    char line[512];
    bool found = false;
    rsg_csr::Tune t;
    int use_sell = 0;
    while (std::fgets(line, sizeof(line), f)) {
        const char *sep = std::strstr(line, " : ");
        if (!sep || std::string(line, size_t(sep - line)) != key) continue;
        rsg_csr::Tune c;
        int us = 0;
        double i64 = 0, i32 = 0;
        if (std::sscanf(sep + 3, "sell=%d rpw=%d dir64=%d dir32=%d upd64=%d upd32=%d pdl64=%d pdl32=%d it_us=%lf,%lf",
                        &us, &c.rpw, &c.g_dir64, &c.g_dir32, &c.g_upd64, &c.g_upd32, &c.pdl64, &c.pdl32, &i64,
                        &i32) == 10) {
            c.it64 = i64 * 1e-6;
            c.it32 = i32 * 1e-6;
            t = c;
            use_sell = us;
            found = true;  // the last matching line wins
        }
    }
    std::fclose(f);
    if (!found || (use_sell && !A->sval)) return false;
    A->use_sell = use_sell != 0;
    A->tune = t;
    A->tune.valid = true;
    A->tune.from_cache = true;
    return true;
}

void tune_store(const char *path, const std::string &key, const rsg_csr *A)
{
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    const rsg_csr::Tune &t = A->tune;
    std::fprintf(f, "%s : sell=%d rpw=%d dir64=%d dir32=%d upd64=%d upd32=%d pdl64=%d pdl32=%d it_us=%.3f,%.3f\n",
                 key.c_str(), A->use_sell ? 1 : 0, t.rpw, t.g_dir64, t.g_dir32, t.g_upd64, t.g_upd32, t.pdl64,
                 t.pdl32, t.it64 * 1e6, t.it32 * 1e6);
    std::fclose(f);
}

struct Bench {
    rsg_context *ctx;
    rsg_csr *A;
    double *b, *x;
    uint32_t count = 0;
    // median seconds per iteration of kTuneReps fixed-length Jacobi-PCG solves with A's current shapes
    rsg_status per_iteration(int32_t precision, double *out)
    {
        rsg_solver_conf c;
        rsg_conf_default(&c);
        c.n_outer = kTuneIters;
        c.stop_rule = RSG_STOP_TRUE_RELRES;
        c.rtol = 0.0;  // never met: every solve runs kTuneIters iterations
        c.precision = precision;
        c.autotune = 0;
        double t[kTuneReps];
        for (int r = 0; r < kTuneReps; r++) {
            RSG_CHECK_CUDA(ctx, cudaMemsetAsync(x, 0, size_t(A->n) * sizeof(double), ctx->stream));
            rsg_stats st;
            const rsg_status s = rsg_solve(ctx, A, &c, RSG_PREC_JACOBI, 1, b, x, RSG_MEM_DEVICE, &st);
            if (s < 0) return s;
            t[r] = st.seconds_solve / double(std::max<uint32_t>(st.iterations, 1));
            count++;
        }
        std::sort(t, t + kTuneReps);
        *out = t[kTuneReps / 2];
        return RSG_OK;
    }
};

}  // namespace

rsg_status autotune_run(rsg_context *ctx, rsg_csr *A, const char *cache_path)
{
    const std::string key = tune_key(ctx, A);
    if (cache_path && cache_path[0] && tune_load(cache_path, key, A)) return RSG_OK;
    const uint32_t n = A->n;
    Bench B{ctx, A, nullptr, nullptr};
    if (cudaMalloc(&B.b, size_t(n) * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&B.x, size_t(n) * sizeof(double)) != cudaSuccess) {
        cudaFree(B.b);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "autotune: right-hand side");
    }
    k_fill<<<std::min(grid_for(ctx, (const void *)k_fill, kBlock, 0, n), kMaxGrid), kBlock, 0, ctx->stream>>>(
        n, 1.0, B.b);

    struct Layout {
        bool sell;
        int rpw;
    };
    std::vector<Layout> layouts;
    if (A->sval) layouts.push_back({true, 0});
    for (int r = natural_rpw(A); r >= 4 && layouts.size() < 3; r /= 2) layouts.push_back({false, r});
    const bool sell_default = A->sval != nullptr;

    rsg_status s = RSG_OK;
    rsg_csr::Tune best;
    bool best_sell = sell_default;
    double best_score = 1e300, def64 = 0, def32 = 0;
    for (const Layout &L : layouts) {
        A->use_sell = L.sell;
        A->tune = rsg_csr::Tune();
        A->tune.valid = true;
        A->tune.rpw = L.sell ? 0 : L.rpw;
        const long long dir_items = L.sell ? (long long)A->n_slices * 32 : (long long)n * 32 / pick_rpw(A);
        rsg_csr::Tune t = A->tune;
        // coordinate descent per precision: direction-kernel grid first, then the update grid
        for (int32_t prec : {RSG_PRECISION_FP64, RSG_PRECISION_MIXED}) {
            int32_t &gd = prec == RSG_PRECISION_FP64 ? A->tune.g_dir64 : A->tune.g_dir32;
            int32_t &gu = prec == RSG_PRECISION_FP64 ? A->tune.g_upd64 : A->tune.g_upd32;
            gd = 0;
            gu = 0;
            double tbest = 0;
            if ((s = B.per_iteration(prec, &tbest)) != RSG_OK) break;
            if (&L == &layouts[0]) (prec == RSG_PRECISION_FP64 ? def64 : def32) = tbest;
            int bd = 0, bu = 0;
            for (int g : grid_candidates(ctx, dir_items)) {
                gd = g;
                double tt = 0;
                if ((s = B.per_iteration(prec, &tt)) != RSG_OK) break;
                if (tt < tbest) {
                    tbest = tt;
                    bd = g;
                }
            }
            if (s != RSG_OK) break;
            gd = bd;
            for (int g : grid_candidates(ctx, (long long)n / 4)) {
                gu = g;
                double tt = 0;
                if ((s = B.per_iteration(prec, &tt)) != RSG_OK) break;
                if (tt < tbest) {
                    tbest = tt;
                    bu = g;
                }
            }
            if (s != RSG_OK) break;
            gu = bu;
            // programmatic dependent launch: the other setting than the size default
            int32_t &pd = prec == RSG_PRECISION_FP64 ? A->tune.pdl64 : A->tune.pdl32;
            pd = pdl_default(A) ? 0 : 1;
            double tp = 0;
            if ((s = B.per_iteration(prec, &tp)) != RSG_OK) break;
            if (tp < tbest) tbest = tp;
            else pd = -1;
            (prec == RSG_PRECISION_FP64 ? t.pdl64 : t.pdl32) = pd;
            (prec == RSG_PRECISION_FP64 ? t.g_dir64 : t.g_dir32) = bd;
            (prec == RSG_PRECISION_FP64 ? t.g_upd64 : t.g_upd32) = bu;
            (prec == RSG_PRECISION_FP64 ? t.it64 : t.it32) = tbest;
        }
        if (s != RSG_OK) break;
        if (t.it64 + t.it32 < best_score) {
            best_score = t.it64 + t.it32;
            best = t;
            best_sell = L.sell;
        }
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(B.b);
    cudaFree(B.x);
    if (s != RSG_OK) {  // leave A with its built-in shapes
        A->use_sell = sell_default;
        A->tune = rsg_csr::Tune();
        return s;
    }
    A->use_sell = best_sell;
    best.valid = true;
    best.candidates = B.count;
    best.it64_default = def64;
    best.it32_default = def32;
    A->tune = best;
    if (cache_path && cache_path[0]) tune_store(cache_path, key, A);
    return RSG_OK;
}

}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_tune_get(const rsg_csr *A, rsg_tune_info *out)
{
    if (!A || !out) return RSG_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    const rsg_csr::Tune &t = A->tune;
    out->tuned = t.valid ? 1 : 0;
    out->from_cache = t.from_cache ? 1 : 0;
    out->format = A->use_sell ? 1 : 0;
    out->rows_per_warp = A->use_sell ? 32u : uint32_t(pick_rpw(A));
    out->grid_dir_fp64 = uint32_t(t.g_dir64);
    out->grid_dir_fp32 = uint32_t(t.g_dir32);
    out->grid_update_fp64 = uint32_t(t.g_upd64);
    out->grid_update_fp32 = uint32_t(t.g_upd32);
    out->seconds_iter_fp64 = t.it64;
    out->seconds_iter_fp32 = t.it32;
    out->seconds_iter_fp64_default = t.it64_default;
    out->seconds_iter_fp32_default = t.it32_default;
    out->candidates = t.candidates;
    out->pdl_fp64 = pdl_for(A, false) ? 1 : 0;
    out->pdl_fp32 = pdl_for(A, true) ? 1 : 0;
    return RSG_OK;
}

rsg_status rsg_autotune(rsg_context *ctx, rsg_csr *A, const char *cache_path, rsg_tune_info *out)
{
    if (!ctx || !A) return set_error(ctx, RSG_ERR_INVALID_ARG, "autotune: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_TRY(autotune_run(ctx, A, cache_path));
    return out ? rsg_tune_get(A, out) : RSG_OK;
}

}  // extern "C"
