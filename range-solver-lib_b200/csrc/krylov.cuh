// Internal interface of the Krylov solvers.
#pragma once

#include "csr.cuh"

#include <utility>

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
    int32_t auto_switch;    // RSG_PRECISION_AUTO: a drifted refresh ends the mixed loop (switched = 1)
    int32_t switched;
    unsigned int ticket[8];  // [7] = bounded-wait error word
    double *history;   // error per iteration (may be null)
    double *trend_hist;
};

struct AmgHierarchy;

struct Precond {
    int kind = 0;                 // 0 none, 1 Jacobi, 2 block Jacobi, 3 multilevel (amg.cu)
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
    const AmgHierarchy *amg;      // kind 3: the matrix's hierarchy
    int amg_sweeps;               // kind 3: smoothing sweeps per side of the V-cycle (1 or 2)
    float *amg_x0;                // kind 3: omega D^-1 r, written by the update / check kernels (P.d32 = omega / a_ii)
    int persistent = 0;           // the loop as one cooperative kernel: 1 when possible, 0 small systems, -1 never
};

rsg_status autotune_run(rsg_context *ctx, rsg_csr *A, const char *cache_path);
// Programmatic dependent launch in the CG loop: the size default (n <= kPdlDefaultRows)
// and the effective choice for A (autotuned value, else the default).
constexpr uint32_t kPdlDefaultRows = 262144;
inline bool pdl_default(const rsg_csr *A) { return A->n <= kPdlDefaultRows; }
bool pdl_for(const rsg_csr *A, bool mixed);

// Launch of a loop kernel; pdl adds the programmatic stream serialization attribute
// (captured into a graph as a programmatic edge), so the kernel's blocks are scheduled
// while its predecessor drains and wait in pdl_wait().
template <typename... P, typename... A>
void launch_k(cudaStream_t stream, bool pdl, void (*k)(P...), dim3 grid, int block, size_t smem, A &&...args)
{
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at.val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cfg.attrs = &at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
}

rsg_status cg_run(rsg_context *ctx, const CgArgs &a, double *seconds);
// The CG loop as one persistent cooperative kernel (cg_persist.cu), bit for bit the graph loop's
// results with the same grids; *ran = false when it could not be launched (nothing was).
rsg_status cg_persist_run(rsg_context *ctx, const CgArgs &a, int g_dir, int g_upd, int g_chk, bool *ran);
// Rows up to which the loop runs persistent by default (conf.persistent = 0): measured per CG
// iteration, graph loop -> persistent, FP64 / mixed: 8k rows 17.3 -> 12.2 / 17.1 -> 11.3 us;
// 65k rows 18.4 -> 14.1 / 18.4 -> 12.4 us; 266k rows 29.0 -> 36.9 / 24.5 -> 24.4 us.
constexpr uint32_t kPersistRows = 131072;

// ---------------- state transitions (thread 0 of the last block) ----------------

__device__ __forceinline__ void finalize_update64(CgState *st, double rz, double rr, double xx)
{
    st->rho_new = rz;
    st->beta = rz / st->rho;
    const double rn = sqrt(rr), xn = sqrt(xx);
    st->rn = rn;
    st->xn = xn;
    double norm = st->an * xn + st->bn;
    if (fabs(norm) < st->eps) norm = st->eps;
    const double err = rn / norm;
    st->trend = err - st->error;
    st->error = err;
    const uint32_t it = ++st->it;
    if (st->history) {
        st->history[it - 1] = err;
        st->trend_hist[it - 1] = st->trend;
    }
    if (st->stop_rule == RSG_STOP_REFERENCE) {
        // RIterationInfo::hasConverged, src/riterationinfo.cpp:90-109
        const bool conv = !dev_isnormal(err) || !dev_isnormal(st->trend) || err < st->cvg ||
                          fabs(st->trend) < st->eps * st->eps;
        if (conv) {
            st->done = 1;
            st->converged = 1;
            st->status = isfinite(err) ? RSG_OK : RSG_BREAKDOWN;
        } else if (it >= st->max_it) {
            st->done = 1;
            st->status = RSG_NOT_CONVERGED;
        }
    } else {
        if (!isfinite(rn)) {
            st->done = 1;
            st->status = RSG_BREAKDOWN;
        } else if (rn <= st->rtol * st->bn) {
            st->need_check = 1;
        } else if (it >= st->max_it) {
            st->done = 1;
            st->status = RSG_NOT_CONVERGED;
        }
    }
}

__device__ __forceinline__ void finalize_check64(CgState *st, double rz, double rn)
{
    st->n_updates++;
    st->rn = rn;
    if (!isfinite(rn)) {
        st->done = 1;
        st->status = RSG_BREAKDOWN;
    } else if (rn <= st->rtol * st->bn) {
        st->done = 1;
        st->converged = 1;
        st->status = RSG_OK;
    } else {
        // the recurrence drifted from the true residual: restart the direction
        // (p = z) so that a tolerance below the attainable accuracy stagnates
        // instead of diverging
        st->rho_new = rz;
        st->beta = 0.0;
        st->need_check = 0;
        if (st->it >= st->max_it) {
            st->done = 1;
            st->status = RSG_NOT_CONVERGED;
        }
    }
}

__device__ __forceinline__ void finalize_update_mixed(CgState *st, double rz, double rr)
{
    st->rho_new = rz;
    st->beta = rz / st->rho;
    const double rn = sqrt(rr) / st->sigma;
    st->rn = rn;
    const uint32_t it = ++st->it;
    const double rel = st->bn > 0.0 ? rn / st->bn : rn;
    st->trend = rel - st->error;
    st->error = rel;
    if (st->history) {
        st->history[it - 1] = rel;
        st->trend_hist[it - 1] = st->trend;
    }
    if (!isfinite(rn) || rn <= st->rtol * st->bn || rn <= st->delta * st->max_r) st->need_check = 1;
    else if (it >= st->max_it) {
        st->done = 1;
        st->status = RSG_NOT_CONVERGED;
    }
}

// Residual replacement keeps the search direction while the FP32 recurrence tracked the
// true residual.  When the true residual comes back more than kRestartGap times larger
// than the recurrence claimed, the recurrence has drifted too far for the old direction
// to stay conjugate to the new residual (stiff systems in FP32: on the 64x32x32
// elasticity beam with a 1e-3 refresh factor the claimed 9.7e-4 was really 1.3e-2, and
// the continued recurrence then stalled near 1e-2), so the direction restarts from z.
// Measured on that beam with a 1e-2 factor: 4138 iterations with a gap of 2, 2587 with
// 1.25; heat and magnetostatic solves are unchanged between the two.
constexpr double kRestartGap = 1.25;

// RSG_PRECISION_AUTO switches to FP64 when a refresh finds the true residual more than kSwitchGap
// times the FP32 recurrence's claim.  Measured: 13x on the elasticity beam at its first refresh
// (after ~400 iterations), within 1.25x on the heat systems.  Refreshing early instead (every 10x
// reduction) does not reveal it: the drift per decade stays below 1.25x on the beam too -- what
// costs mixed precision its iterations there is the FP32-rounded matrix, which shows only after a
// few decades.
constexpr double kSwitchGap = 2.0;

// Default refresh factor of the mixed-precision CG (rsg_solver_conf.reliable_delta):
// 1e-3 measured equal or better than 1e-2 on heat (40^3 to 100^3, several seeds) and on
// the elasticity beam (2412 against 2587 iterations), 2% more iterations on 40^3
// magnetostatics.
constexpr double kReliableDelta = 1.0e-3;

__device__ __forceinline__ void finalize_check_mixed(CgState *st, double rz, double rn)
{
    const double claimed = st->rn;  // the recurrence's residual norm that triggered this check
    st->n_updates++;
    st->fold = 1;
    st->rn = rn;
    if (!isfinite(rn)) {
        st->done = 1;
        st->status = RSG_BREAKDOWN;
    } else if (rn <= st->rtol * st->bn) {
        st->done = 1;
        st->converged = 1;
        st->status = RSG_OK;
    } else if (st->auto_switch && rn > kSwitchGap * claimed) {
        st->switched = 1;  // the caller continues in FP64 from the folded x
        st->done = 1;
        st->status = RSG_OK;
    } else {
        st->max_r = rn;
        st->rho_new = rz;
        st->beta = rn > kRestartGap * claimed ? 0.0 : rz / st->rho;
        st->need_check = 0;
        if (st->it >= st->max_it) {
            st->done = 1;
            st->status = RSG_NOT_CONVERGED;
        }
    }
}

__device__ __forceinline__ double clamp_pq(double pq, double eps)
{
    // src/rmatrixsolver.cpp:304-315; with eps = 0 (no clamp) only an exact zero is guarded
    if (pq > 0.0) return fmax(pq, eps);
    if (pq < 0.0) return fmin(pq, -eps);
    return eps > 0.0 ? eps : 1e-300;
}



}  // namespace rsg
