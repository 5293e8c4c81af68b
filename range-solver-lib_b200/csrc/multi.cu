// Several right-hand sides of one matrix solved together (FP64 Jacobi-PCG).
//
// The reference solves one right-hand side per RMatrixSolver::solve call
// (src/rmatrixsolver.cpp:158-201); callers with many load cases, or
// REigenValueSolver's repeated solves with one matrix
// (src/reigenvaluesolver.cpp:119-392), stream the matrix once per iteration
// per right-hand side.  Here the k vectors of every Krylov quantity are stored
// interleaved (row i holds the K values of its k columns contiguously, K = k
// rounded up to 2, 4, 8 or 16), so one pass over the matrix serves all
// columns: each stored element is loaded once and multiplied into K
// accumulators, and a gathered column fetches K contiguous values.  Every
// column runs the reference's CG recurrences (src/rmatrixsolver.cpp:233-354)
// with its own scalars, stops on its FP64 true relative residual (recomputed
// before stopping, as RSG_STOP_TRUE_RELRES does for one column) and is frozen
// once done; the loop is one CUDA graph `while` node that runs until every
// column is done.  Row sums use separate multiply and add in CSR order, as the
// reference's multiplyRow (src/rmatrixsolver.cpp:111-119).
#include "krylov.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace rsg {
namespace {

constexpr int kMaxRhs = 16;

struct MrCol {
    double rho, alpha, beta, bn, rn, pq, relres;
    uint32_t it, checks;
    int32_t done, converged, need_check, status;
};

struct MrState {
    uint32_t k, max_it, body_count, body_limit;
    int32_t all_done, any_check, timeout, pad;
    double rtol;
    unsigned int ticket[8];
    MrCol col[kMaxRhs];
};

struct MView {
    const uint32_t *rp, *ci;
    const double *val;
    // SELL-32 copy when the matrix has one: element e of row r (lane r%32 of slice r/32)
    // at slice_ptr[r/32] + (e/4)*128 + 4*(r%32) + e%4, so a warp's loads stay coalesced
    const uint32_t *slice_ptr;
    const double *sval;
    const int16_t *soff;
    const uint32_t *scol;
    int use_sell;
    uint32_t n;
};

// Thread mapping: column pairs.  A row's K interleaved values are K/2 double2;
// LPR = K/2 lanes share a row, lane li of the group owns columns 2li and 2li+1.
// A warp covers 32/LPR rows at a time; consecutive lanes read consecutive 16-byte
// pieces of a row, so every gathered neighbour row is one contiguous 8K-byte read.
template <int K>
struct Map {
    static constexpr int LPR = K / 2;
    static constexpr int RPW = 32 / LPR;
};

__device__ __forceinline__ double2 ld2(const double *__restrict__ base, size_t idx)
{
    return __ldg(reinterpret_cast<const double2 *>(base) + idx);
}

// acc = sum over the row's entries (CSR order) of a_rc * g(c); g returns this
// lane's column pair of the gathered row c.  All 32 lanes must call it.
template <int K, class G>
__device__ __forceinline__ double2 row_product(const MView &M, uint32_t row, bool valid, G &g)
{
    constexpr int LPR = Map<K>::LPR;
    const int lane = threadIdx.x & 31, li = lane % LPR, g0 = lane - li;
    uint32_t jb = 0, je = 0;
    if (valid) {
        jb = __ldg(&M.rp[row]);
        je = __ldg(&M.rp[row + 1]);
    }
    const uint32_t trips = __reduce_max_sync(0xffffffffu, (je - jb + LPR - 1) / LPR);
    double2 acc = make_double2(0.0, 0.0);
    for (uint32_t t = 0; t < trips; t++) {
        const uint32_t e = jb + t * LPR + uint32_t(li);
        uint32_t c_mine = 0;
        double v_mine = 0.0;
        if (e < je) {
            if (M.use_sell) {
                const uint32_t k = e - jb, row0 = row & ~31u;
                const size_t pos = size_t(__ldg(&M.slice_ptr[row >> 5])) + size_t(k >> 2) * 128u +
                                   4u * (row & 31u) + (k & 3u);
                c_mine = M.soff ? uint32_t(int(row0) + __ldg(&M.soff[pos])) : __ldg(&M.scol[pos]);
                v_mine = __ldg(&M.sval[pos]);
            } else {
                c_mine = __ldg(&M.ci[e]);
                v_mine = __ldg(&M.val[e]);
            }
        }
#pragma unroll
        for (int u = 0; u < LPR; u++) {
            const uint32_t c = __shfl_sync(0xffffffffu, c_mine, g0 + u);
            const double v = __shfl_sync(0xffffffffu, v_mine, g0 + u);
            if (jb + t * LPR + uint32_t(u) < je) {
                const double2 x = g(c);
                acc.x = __dadd_rn(acc.x, __dmul_rn(v, x.x));
                acc.y = __dadd_rn(acc.y, __dmul_rn(v, x.y));
            }
        }
    }
    return acc;
}

// Column sums over the grid: each lane holds NQ quantities for its column pair.
// Returns true in the last block to finish; tot[q*K + j] then holds the totals
// (valid in every thread of that block).  Fixed order: lanes, warps, blocks.
template <int K, int NQ>
__device__ __forceinline__ bool grid_cols_sum(double2 (&v)[NQ], double *partials, unsigned int *ticket, double *sh,
                                              double *tot)
{
    constexpr int LPR = Map<K>::LPR, NV = NQ * K;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++)
        for (int o = LPR; o < 32; o <<= 1) {
            v[q].x += __shfl_xor_sync(0xffffffffu, v[q].x, o);
            v[q].y += __shfl_xor_sync(0xffffffffu, v[q].y, o);
        }
    if (lane < LPR)
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            sh[warp * NV + q * K + 2 * lane] = v[q].x;
            sh[warp * NV + q * K + 2 * lane + 1] = v[q].y;
        }
    __syncthreads();
    __shared__ bool is_last;
    for (int t = threadIdx.x; t < NV; t += blockDim.x) {
        double a = 0.0;
        for (int w = 0; w < nw; w++) a += sh[w * NV + t];
        partials[size_t(blockIdx.x) * NV + t] = a;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    for (int t = threadIdx.x; t < NV; t += blockDim.x) {
        double a = 0.0;
        for (unsigned int b = 0; b < gridDim.x; b++) a += __ldcg(&partials[size_t(b) * NV + t]);
        tot[t] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// interleave: out[i*K + j] = src[j*ld + i] for j < k, 0 for the padding columns
__global__ void k_mr_pack(uint32_t n, uint32_t k, uint32_t K, const double *__restrict__ src, size_t ld,
                          double *__restrict__ out)
{
    const size_t total = size_t(n) * K;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const uint32_t i = uint32_t(e / K), j = uint32_t(e % K);
        out[e] = j < k ? src[size_t(j) * ld + i] : 0.0;
    }
}

__global__ void k_mr_unpack(uint32_t n, uint32_t k, uint32_t K, const double *__restrict__ in, size_t ld,
                            double *__restrict__ dst)
{
    const size_t total = size_t(n) * k;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const uint32_t j = uint32_t(e / n), i = uint32_t(e % n);
        dst[size_t(j) * ld + i] = in[size_t(i) * K + j];
    }
}

__device__ void refresh_all_done(MrState *st)
{
    int all = 1, chk = 0;
    for (uint32_t j = 0; j < st->k; j++) {
        all &= st->col[j].done;
        chk |= st->col[j].need_check;
    }
    st->all_done = all;
    st->any_check = chk;
}

// rows visited by this warp-group pass: grid-stride over groups of RPW rows
#define MR_FOR_ROWS(K, n, row, valid)                                                                          \
    const int lane_ = threadIdx.x & 31;                                                                        \
    const uint32_t warps_ = gridDim.x * (blockDim.x >> 5);                                                     \
    const uint32_t groups_ = ((n) + Map<K>::RPW - 1) / Map<K>::RPW;                                            \
    for (uint32_t grp_ = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); grp_ < groups_; grp_ += warps_) { \
        const uint32_t row = grp_ * Map<K>::RPW + uint32_t(lane_ / Map<K>::LPR);                               \
        const bool valid = row < (n);

// r = b - A x, z = D r; per column ||b||^2, ||r||^2, r^T z
template <int K>
__global__ void __launch_bounds__(kBlock) k_mr_init(MView M, const double *__restrict__ d, const double *__restrict__ b,
                                                    const double *__restrict__ x, double *__restrict__ r,
                                                    double *__restrict__ z, double *partials, MrState *st)
{
    __shared__ double sh[8 * 3 * K];
    __shared__ double tot[3 * K];
    const int li = (threadIdx.x & 31) % Map<K>::LPR;
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    auto gx = [&](uint32_t c) { return ld2(x, size_t(c) * (K / 2) + li); };
    MR_FOR_ROWS(K, M.n, row, valid)
        const double2 ax = row_product<K>(M, row, valid, gx);
        if (valid) {
            const size_t idx = size_t(row) * (K / 2) + li;
            const double2 bv = ld2(b, idx);
            const double di = d ? d[row] : 1.0;
            const double2 rv = make_double2(bv.x - ax.x, bv.y - ax.y);
            const double2 zv = make_double2(di * rv.x, di * rv.y);
            reinterpret_cast<double2 *>(r)[idx] = rv;
            reinterpret_cast<double2 *>(z)[idx] = zv;
            acc[0].x += bv.x * bv.x;
            acc[0].y += bv.y * bv.y;
            acc[1].x += rv.x * rv.x;
            acc[1].y += rv.y * rv.y;
            acc[2].x += rv.x * zv.x;
            acc[2].y += rv.y * zv.y;
        }
    }
    if (grid_cols_sum<K, 3>(acc, partials, &st->ticket[0], sh, tot) && threadIdx.x == 0) {
        for (uint32_t j = 0; j < st->k; j++) {
            MrCol &c = st->col[j];
            c.bn = sqrt(tot[j]);
            c.rn = sqrt(tot[K + j]);
            c.rho = tot[2 * K + j];
            c.beta = 0.0;
            c.alpha = 0.0;
            c.it = 0;
            c.checks = 0;
            c.need_check = 0;
            c.converged = 0;
            c.status = RSG_NOT_CONVERGED;
            c.done = 0;
            if (!(c.rn > st->rtol * c.bn)) {  // already solved (includes b = 0, x = 0)
                c.done = 1;
                c.converged = 1;
                c.status = RSG_OK;
            } else if (!(c.rho > 0.0) || !isfinite(c.rho)) {
                c.done = 1;
                c.status = RSG_BREAKDOWN;
            }
        }
        refresh_all_done(st);
    }
}

// p = z + beta p_old (own row, and gathered on the fly), q = A p; per column p^T q -> alpha
template <int K>
__global__ void __launch_bounds__(kBlock) k_mr_dir(MView M, const double *__restrict__ z,
                                                   const double *__restrict__ po, double *__restrict__ pn,
                                                   double *__restrict__ q, double *partials, MrState *st)
{
    __shared__ double sh[8 * K];
    __shared__ double tot[K];
    if (st->all_done) return;
    const int li = (threadIdx.x & 31) % Map<K>::LPR;
    const double bx = 2 * li < int(st->k) ? st->col[2 * li].beta : 0.0;
    const double by = 2 * li + 1 < int(st->k) ? st->col[2 * li + 1].beta : 0.0;
    auto gp = [&](uint32_t c) {
        const size_t idx = size_t(c) * (K / 2) + li;
        const double2 zv = ld2(z, idx), pv = ld2(po, idx);
        return make_double2(fma(bx, pv.x, zv.x), fma(by, pv.y, zv.y));
    };
    double2 acc[1] = {make_double2(0, 0)};
    MR_FOR_ROWS(K, M.n, row, valid)
        const double2 qv = row_product<K>(M, row, valid, gp);
        if (valid) {
            const size_t idx = size_t(row) * (K / 2) + li;
            const double2 pv = gp(row);
            reinterpret_cast<double2 *>(pn)[idx] = pv;
            reinterpret_cast<double2 *>(q)[idx] = qv;
            acc[0].x += pv.x * qv.x;
            acc[0].y += pv.y * qv.y;
        }
    }
    if (grid_cols_sum<K, 1>(acc, partials, &st->ticket[1], sh, tot) && threadIdx.x == 0) {
        for (uint32_t j = 0; j < st->k; j++) {
            MrCol &c = st->col[j];
            if (c.done) {
                c.alpha = 0.0;
                continue;
            }
            c.pq = tot[j];
            if (!(c.pq > 0.0) || !isfinite(c.pq)) {
                c.alpha = 0.0;
                c.done = 1;
                c.status = RSG_BREAKDOWN;
            } else {
                c.alpha = c.rho / c.pq;
            }
        }
        refresh_all_done(st);
    }
}

// x += alpha p, r -= alpha q, z = D r for the active columns; r^T z, ||r||^2 -> beta, stop tests.
// Streaming: one thread per 16-byte column pair of a row.
template <int K>
__global__ void __launch_bounds__(kBlock) k_mr_update(uint32_t n, const double *__restrict__ d,
                                                      const double *__restrict__ p, const double *__restrict__ q,
                                                      double *__restrict__ x, double *__restrict__ r,
                                                      double *__restrict__ z, double *partials, MrState *st)
{
    __shared__ double sh[8 * 2 * K];
    __shared__ double tot[2 * K];
    const int li = (threadIdx.x & 31) % Map<K>::LPR;
    const int j0 = 2 * li, j1 = 2 * li + 1;
    const bool a0 = j0 < int(st->k) && !st->col[j0].done, a1 = j1 < int(st->k) && !st->col[j1].done;
    const double al0 = a0 ? st->col[j0].alpha : 0.0, al1 = a1 ? st->col[j1].alpha : 0.0;
    double2 acc[2] = {make_double2(0, 0), make_double2(0, 0)};
    const size_t total = size_t(n) * (K / 2);
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const double2 pv = ld2(p, e), qv = ld2(q, e);
        double2 xv = reinterpret_cast<const double2 *>(x)[e];
        double2 rv = reinterpret_cast<const double2 *>(r)[e];
        double2 zv = reinterpret_cast<const double2 *>(z)[e];
        const double di = d ? d[e / (K / 2)] : 1.0;
        if (a0) {
            xv.x = fma(al0, pv.x, xv.x);
            rv.x = fma(-al0, qv.x, rv.x);
            zv.x = di * rv.x;
        }
        if (a1) {
            xv.y = fma(al1, pv.y, xv.y);
            rv.y = fma(-al1, qv.y, rv.y);
            zv.y = di * rv.y;
        }
        reinterpret_cast<double2 *>(x)[e] = xv;
        reinterpret_cast<double2 *>(r)[e] = rv;
        reinterpret_cast<double2 *>(z)[e] = zv;
        acc[0].x += rv.x * zv.x;
        acc[0].y += rv.y * zv.y;
        acc[1].x += rv.x * rv.x;
        acc[1].y += rv.y * rv.y;
    }
    if (grid_cols_sum<K, 2>(acc, partials, &st->ticket[2], sh, tot) && threadIdx.x == 0) {
        for (uint32_t j = 0; j < st->k; j++) {
            MrCol &c = st->col[j];
            if (c.done) continue;
            c.it++;
            const double rho_new = tot[j];
            c.rn = sqrt(tot[K + j]);
            if (!isfinite(c.rn) || !isfinite(rho_new)) {
                c.done = 1;
                c.status = RSG_BREAKDOWN;
                continue;
            }
            c.beta = rho_new / c.rho;
            c.rho = rho_new;
            if (c.rn <= st->rtol * c.bn) c.need_check = 1;
            else if (c.it >= st->max_it) c.done = 1;  // status stays NOT_CONVERGED
        }
        refresh_all_done(st);
    }
}

// For the columns whose recurrence residual met rtol: the FP64 true residual
// r = b - A x decides; a column that fails continues from it with a restarted direction.
template <int K>
__global__ void __launch_bounds__(kBlock) k_mr_check(MView M, const double *__restrict__ d,
                                                     const double *__restrict__ b, const double *__restrict__ x,
                                                     double *__restrict__ r, double *__restrict__ z, double *partials,
                                                     MrState *st)
{
    __shared__ double sh[8 * 2 * K];
    __shared__ double tot[2 * K];
    if (!st->any_check) return;
    const int li = (threadIdx.x & 31) % Map<K>::LPR;
    const bool c0 = 2 * li < int(st->k) && st->col[2 * li].need_check;
    const bool c1 = 2 * li + 1 < int(st->k) && st->col[2 * li + 1].need_check;
    auto gx = [&](uint32_t c) { return ld2(x, size_t(c) * (K / 2) + li); };
    double2 acc[2] = {make_double2(0, 0), make_double2(0, 0)};
    MR_FOR_ROWS(K, M.n, row, valid)
        const double2 ax = row_product<K>(M, row, valid, gx);
        if (valid) {
            const size_t idx = size_t(row) * (K / 2) + li;
            const double2 bv = ld2(b, idx);
            double2 rv = reinterpret_cast<const double2 *>(r)[idx];
            double2 zv = reinterpret_cast<const double2 *>(z)[idx];
            const double di = d ? d[row] : 1.0;
            if (c0) {
                rv.x = bv.x - ax.x;
                zv.x = di * rv.x;
            }
            if (c1) {
                rv.y = bv.y - ax.y;
                zv.y = di * rv.y;
            }
            reinterpret_cast<double2 *>(r)[idx] = rv;
            reinterpret_cast<double2 *>(z)[idx] = zv;
            acc[0].x += rv.x * zv.x;
            acc[0].y += rv.y * zv.y;
            acc[1].x += rv.x * rv.x;
            acc[1].y += rv.y * rv.y;
        }
    }
    if (grid_cols_sum<K, 2>(acc, partials, &st->ticket[3], sh, tot) && threadIdx.x == 0) {
        for (uint32_t j = 0; j < st->k; j++) {
            MrCol &c = st->col[j];
            if (!c.need_check) continue;
            c.need_check = 0;
            c.checks++;
            c.rn = sqrt(tot[K + j]);
            if (c.rn <= st->rtol * c.bn) {
                c.done = 1;
                c.converged = 1;
                c.status = RSG_OK;
            } else if (c.it >= st->max_it) {
                c.done = 1;
            } else {
                c.rho = tot[j];
                c.beta = 0.0;  // restart the direction from the true residual
                if (!(c.rho > 0.0)) {
                    c.done = 1;
                    c.status = RSG_BREAKDOWN;
                }
            }
        }
        refresh_all_done(st);
    }
}

// per column ||b - A x|| / ||b|| of the final x
template <int K>
__global__ void __launch_bounds__(kBlock) k_mr_true(MView M, const double *__restrict__ b,
                                                    const double *__restrict__ x, double *partials, MrState *st)
{
    __shared__ double sh[8 * 2 * K];
    __shared__ double tot[2 * K];
    const int li = (threadIdx.x & 31) % Map<K>::LPR;
    auto gx = [&](uint32_t c) { return ld2(x, size_t(c) * (K / 2) + li); };
    double2 acc[2] = {make_double2(0, 0), make_double2(0, 0)};
    MR_FOR_ROWS(K, M.n, row, valid)
        const double2 ax = row_product<K>(M, row, valid, gx);
        if (valid) {
            const double2 bv = ld2(b, size_t(row) * (K / 2) + li);
            const double tx = bv.x - ax.x, ty = bv.y - ax.y;
            acc[0].x += tx * tx;
            acc[0].y += ty * ty;
            acc[1].x += bv.x * bv.x;
            acc[1].y += bv.y * bv.y;
        }
    }
    if (grid_cols_sum<K, 2>(acc, partials, &st->ticket[4], sh, tot) && threadIdx.x == 0) {
        for (uint32_t j = 0; j < st->k; j++) {
            const double bn = sqrt(tot[K + j]), rn = sqrt(tot[j]);
            st->col[j].relres = bn > 0.0 ? rn / bn : rn;
        }
    }
}

__global__ void k_mr_tail(MrState *st, cudaGraphConditionalHandle h, int use_cond)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint32_t bc = ++st->body_count;
    if (!st->all_done && bc >= st->body_limit) {
        st->all_done = 1;
        st->timeout = 1;
    }
    if (use_cond) cudaGraphSetConditional(h, st->all_done ? 0u : 1u);
}

struct MrArgs {
    MView M;
    const double *d, *b;
    double *x, *r, *z, *p[2], *q, *partials;
    MrState *st;
    int g;
};

template <int K>
void mr_body(rsg_context *ctx, const MrArgs &a, cudaGraphConditionalHandle h, int use_cond)
{
    for (int half = 0; half < 2; half++) {
        const double *po = a.p[half];
        double *pn = a.p[half ^ 1];
        k_mr_dir<K><<<a.g, kBlock, 0, ctx->stream>>>(a.M, a.z, po, pn, a.q, a.partials, a.st);
        k_mr_update<K><<<a.g, kBlock, 0, ctx->stream>>>(a.M.n, a.d, pn, a.q, a.x, a.r, a.z, a.partials, a.st);
        k_mr_check<K><<<a.g, kBlock, 0, ctx->stream>>>(a.M, a.d, a.b, a.x, a.r, a.z, a.partials, a.st);
    }
    k_mr_tail<<<1, 32, 0, ctx->stream>>>(a.st, h, use_cond);
}

template <int K>
rsg_status mr_run(rsg_context *ctx, MrArgs &a, bool use_graph, double *seconds)
{
    const int g = std::min(grid_for(ctx, (const void *)k_mr_dir<K>, kBlock, 0, (long long)a.M.n * (K / 2)), kMaxGrid);
    // SELL-32 keeps the loads of 1-2 lanes per row coalesced; with 4-8 lanes per row the
    // CSR arrays (a row's entries contiguous) measured faster
    if (K >= 8) a.M.use_sell = 0;
    a.g = g;
    cudaEventRecord(ctx->ev[0], ctx->stream);
    k_mr_init<K><<<g, kBlock, 0, ctx->stream>>>(a.M, a.d, a.b, a.x, a.r, a.z, a.partials, a.st);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    rsg_status s = RSG_OK;
    if (use_graph) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphConditionalHandle h;
        RSG_CHECK_CUDA(ctx, cudaGraphCreate(&graph, 0));
        do {
            if (cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
                s = set_error(ctx, RSG_ERR_CUDA, "multi-RHS: conditional handle");
                break;
            }
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            if (cudaGraphAddNode(&node, graph, nullptr, 0, &cp) != cudaSuccess) {
                s = set_error(ctx, RSG_ERR_CUDA, "multi-RHS: while node");
                break;
            }
            if (cudaStreamBeginCaptureToGraph(ctx->stream, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                s = set_error(ctx, RSG_ERR_CUDA, "multi-RHS: capture");
                break;
            }
            mr_body<K>(ctx, a, h, 1);
            cudaGraph_t captured = nullptr;
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &captured);
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (e == cudaSuccess) e = cudaGraphLaunch(exec, ctx->stream);
            if (e != cudaSuccess) s = set_error(ctx, RSG_ERR_CUDA, "multi-RHS graph: %s", cudaGetErrorString(e));
        } while (0);
        if (s == RSG_OK) {
            cudaError_t e = cudaStreamSynchronize(ctx->stream);
            if (e != cudaSuccess) s = set_error(ctx, RSG_ERR_CUDA, "multi-RHS solve: %s", cudaGetErrorString(e));
        }
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (s != RSG_OK) return s;
    } else {
        int32_t *done_h = reinterpret_cast<int32_t *>(ctx->pinned);
        for (uint64_t b = 0;; b++) {
            for (int k = 0; k < 8; k++) mr_body<K>(ctx, a, 0, 0);
            RSG_CHECK_CUDA(ctx, cudaGetLastError());
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(done_h, &a.st->all_done, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                                ctx->stream));
            RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            if (*done_h) break;
        }
    }
    k_mr_true<K><<<g, kBlock, 0, ctx->stream>>>(a.M, a.b, a.x, a.partials, a.st);
    RSG_CHECK_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    *seconds = ms * 1e-3;
    return RSG_OK;
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" rsg_status rsg_solve_multi(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf, int32_t prec_type,
                                      uint32_t k, const double *B, double *X, int32_t memory, rsg_stats *per_rhs,
                                      rsg_stats *summary)
{
    if (!ctx || !A || !conf || !B || !X) return set_error(ctx, RSG_ERR_INVALID_ARG, "solve_multi: null argument");
    if (k < 1 || k > uint32_t(kMaxRhs))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "solve_multi: %u right-hand sides (1..%d)", k, kMaxRhs);
    if (memory != RSG_MEM_HOST && memory != RSG_MEM_DEVICE)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "solve_multi: bad memory kind %d", memory);
    if (conf->stop_rule != RSG_STOP_TRUE_RELRES)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "solve_multi: needs stop_rule TRUE_RELRES");
    if (conf->precision != RSG_PRECISION_FP64 || conf->solver_type != RSG_SOLVER_CG)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "solve_multi: FP64 CG only");
    if (prec_type != RSG_PREC_NONE && prec_type != RSG_PREC_JACOBI)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "solve_multi: preconditioner %d (NONE or JACOBI)", prec_type);
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t n = A->n;
    const uint32_t K = k <= 2 ? 2 : k <= 4 ? 4 : k <= 8 ? 8 : 16;
    const size_t vk = arena_bytes(size_t(n) * K, sizeof(double));
    size_t bytes = 7 * vk + arena_bytes(n, sizeof(double)) + arena_bytes(size_t(kMaxGrid) * 3 * K, sizeof(double)) +
                   arena_bytes(1, sizeof(MrState)) + 4096;
    if (memory == RSG_MEM_HOST) bytes += 2 * arena_bytes(size_t(n) * k, sizeof(double));
    RSG_TRY(arena_reserve(ctx, bytes));
    MrArgs a;
    double *bi = arena_take<double>(ctx, size_t(n) * K);
    a.x = arena_take<double>(ctx, size_t(n) * K);
    a.r = arena_take<double>(ctx, size_t(n) * K);
    a.z = arena_take<double>(ctx, size_t(n) * K);
    a.p[0] = arena_take<double>(ctx, size_t(n) * K);
    a.p[1] = arena_take<double>(ctx, size_t(n) * K);
    a.q = arena_take<double>(ctx, size_t(n) * K);
    double *d = arena_take<double>(ctx, n);
    a.partials = arena_take<double>(ctx, size_t(kMaxGrid) * 3 * K);
    a.st = arena_take<MrState>(ctx, 1);
    const double *Bsrc = B;
    double *Xdst = X, *Xsrc = X;
    if (memory == RSG_MEM_HOST) {
        double *bs = arena_take<double>(ctx, size_t(n) * k), *xs = arena_take<double>(ctx, size_t(n) * k);
        if (!xs) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "solve_multi workspace");
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(bs, B, size_t(n) * k * 8, cudaMemcpyHostToDevice, ctx->stream));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(xs, X, size_t(n) * k * 8, cudaMemcpyHostToDevice, ctx->stream));
        Bsrc = bs;
        Xsrc = Xdst = xs;
    }
    if (!a.st) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "solve_multi workspace");
    a.b = bi;
    a.d = prec_type == RSG_PREC_JACOBI ? d : nullptr;
    if (a.d) RSG_TRY(jacobi_build(ctx, A, d));
    const int gp = std::min(grid_for(ctx, (const void *)k_mr_pack, kBlock, 0, (long long)n * K), kMaxGrid);
    k_mr_pack<<<gp, kBlock, 0, ctx->stream>>>(n, k, K, Bsrc, n, bi);
    k_mr_pack<<<gp, kBlock, 0, ctx->stream>>>(n, k, K, Xsrc, n, a.x);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.p[0], 0, size_t(n) * K * 8, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(a.partials, 0, 8, ctx->stream));
    MrState h;
    std::memset(&h, 0, sizeof(h));
    h.k = k;
    h.max_it = std::max<uint32_t>(conf->n_outer, 1);
    h.body_limit = h.max_it / 2 + 16;
    h.rtol = conf->rtol;
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(a.st, &h, sizeof(h), cudaMemcpyHostToDevice, ctx->stream));
    a.M.rp = A->rp;
    a.M.ci = A->ci;
    a.M.val = A->val;
    a.M.slice_ptr = A->slice_ptr;
    a.M.sval = A->sval;
    a.M.soff = A->soff;
    a.M.scol = A->scol;
    a.M.use_sell = A->use_sell && A->sval ? 1 : 0;
    a.M.n = n;
    double seconds = 0.0;
    rsg_status s = RSG_OK;
    switch (K) {
    case 2: s = mr_run<2>(ctx, a, conf->use_graph != 0, &seconds); break;
    case 4: s = mr_run<4>(ctx, a, conf->use_graph != 0, &seconds); break;
    case 8: s = mr_run<8>(ctx, a, conf->use_graph != 0, &seconds); break;
    default: s = mr_run<16>(ctx, a, conf->use_graph != 0, &seconds); break;
    }
    if (s != RSG_OK) return s;
    const int gu = std::min(grid_for(ctx, (const void *)k_mr_unpack, kBlock, 0, (long long)n * k), kMaxGrid);
    k_mr_unpack<<<gu, kBlock, 0, ctx->stream>>>(n, k, K, a.x, n, Xdst);
    if (memory == RSG_MEM_HOST)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(X, Xdst, size_t(n) * k * 8, cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&h, a.st, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    rsg_stats sum;
    std::memset(&sum, 0, sizeof(sum));
    sum.converged = 1;
    sum.status = RSG_OK;
    sum.seconds_solve = seconds;
    sum.norm_a = A->norm;
    for (uint32_t j = 0; j < k; j++) {
        const MrCol &c = h.col[j];
        rsg_stats st;
        std::memset(&st, 0, sizeof(st));
        st.iterations = c.it;
        st.outer = c.checks;
        st.error = c.bn > 0.0 ? c.rn / c.bn : c.rn;
        st.true_relres = c.relres;
        st.equation_scale = 1.0;
        st.norm_a = A->norm;
        st.norm_b = c.bn;
        st.seconds_solve = seconds;
        st.converged = c.converged;
        st.status = h.timeout ? RSG_ERR_TIMEOUT : c.status;
        if (per_rhs) per_rhs[j] = st;
        sum.iterations = std::max(sum.iterations, st.iterations);
        sum.true_relres = std::max(sum.true_relres, st.true_relres);
        sum.converged &= st.converged;
        if (st.status != RSG_OK && (sum.status == RSG_OK || st.status < 0)) sum.status = st.status;
    }
    if (summary) *summary = sum;
    if (h.timeout) return set_error(ctx, RSG_ERR_TIMEOUT, "solve_multi: loop hit its hard limit");
    return sum.status < 0 ? rsg_status(sum.status) : (sum.converged ? RSG_OK : RSG_NOT_CONVERGED);
}
