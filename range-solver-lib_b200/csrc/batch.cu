// Batched solves of many independent systems of uneven size in one device-driven loop.
//
// The reference solves one system per RMatrixSolver::solve call
// (src/rmatrixsolver.cpp:158-201); callers such as a transient or multi-load-case
// run, or many small meshes, then pay one solve's launch and synchronisation
// costs per system.  Here the systems are packed block-diagonally into one
// matrix, each padded to a multiple of 32 rows with identity rows, so that
// every 32-row SELL slice belongs to exactly one system.  Each system keeps its
// own CG state (the same CgState and transitions as the single-system solver:
// stop on FP64 true relative residual, FP64 or mixed precision with reliable
// updates).  Per iteration the same three phases as the single-system solver
// (direction + SpMV, update, residual check) run over the slices of a list of
// systems: the active systems for the first two, and for the check only the
// systems whose update asked for one (a refresh or a convergence claim) -- the
// check is an FP64 SpMV, and spread over all active systems' slices its few
// listed systems would leave most warps idle and a few working through long
// runs of slices.  Each slice writes its partial sums; one block per listed
// system then adds them in slice order and advances the system's state, and the
// last of those blocks after an update builds the check list.  The loop is one
// CUDA graph `while` node; the tail kernel rebuilds the active list and keeps
// the loop running while any system is active.
#include "krylov.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

struct rsg_batch {
    uint32_t n_sys = 0;
    uint32_t user_rows = 0, pad_rows = 0;
    rsg_csr *A = nullptr;                  // padded block-diagonal matrix
    std::vector<uint32_t> user_begin, pad_begin;
    uint32_t *d_slice_sys = nullptr;       // system of each slice
    uint32_t *d_sys_slice = nullptr;       // first slice of each system (n_sys + 1)
    uint32_t *d_user2pad = nullptr;        // padded row of each user row
    // grid of the slice kernels picked by rsg_batch_autotune (0 = the built-in default)
    int32_t g64 = 0, g32 = 0;
    double it64 = 0, it32 = 0, it64_default = 0, it32_default = 0;
    uint32_t tune_candidates = 0;
    bool tuned = false;
};

namespace rsg {
namespace {

struct BatchCtl {
    uint32_t body_count;
    uint32_t body_limit;
    int32_t timeout;
    int32_t pad;
    uint32_t arrive;  // blocks of the update reduction that have finished (reset by the last)
};

struct BView {
    const uint32_t *slice_sys;
    const uint32_t *sys_slice;
    uint32_t n_slices, n_sys;
};

// Systems a kernel visits: ids and the exclusive prefix of their slice counts.
struct Active {
    uint32_t n_sys;      // number of listed systems
    uint32_t n_slices;   // their slices in total
    uint32_t *sys;       // [capacity]
    uint32_t *prefix;    // [capacity + 1]
};

// Block-wide (blockDim.x == kBlock): lists in order the systems in_sys[0..n_in) (0..n_in when in_sys
// is null) that keep(system) accepts, with the exclusive prefix of their slice counts.  Every
// thread calls it; keep must give the same answer on both of its calls.
template <class KEEP>
__device__ __forceinline__ void build_list(uint32_t n_in, const uint32_t *in_sys, const uint32_t *sys_slice,
                                           Active *out, KEEP keep)
{
    __shared__ uint32_t cnt_sys[kBlock], cnt_sl[kBlock];
    const uint32_t t = threadIdx.x, per = (n_in + blockDim.x - 1) / blockDim.x;
    const uint32_t i0 = min(n_in, t * per), i1 = min(n_in, i0 + per);
    uint32_t ns = 0, nsl = 0;
    for (uint32_t i = i0; i < i1; i++) {
        const uint32_t sys = in_sys ? in_sys[i] : i;
        if (keep(sys)) {
            ns++;
            nsl += sys_slice[sys + 1] - sys_slice[sys];
        }
    }
    cnt_sys[t] = ns;
    cnt_sl[t] = nsl;
    __syncthreads();
    if (t == 0) {  // exclusive scan (blockDim entries)
        uint32_t a = 0, b = 0;
        for (uint32_t k = 0; k < blockDim.x; k++) {
            const uint32_t x = cnt_sys[k], y = cnt_sl[k];
            cnt_sys[k] = a;
            cnt_sl[k] = b;
            a += x;
            b += y;
        }
        out->n_sys = a;
        out->n_slices = b;
        out->prefix[a] = b;
    }
    __syncthreads();
    uint32_t o = cnt_sys[t], pre = cnt_sl[t];
    for (uint32_t i = i0; i < i1; i++) {
        const uint32_t sys = in_sys ? in_sys[i] : i;
        if (keep(sys)) {
            out->sys[o] = sys;
            out->prefix[o] = pre;
            pre += sys_slice[sys + 1] - sys_slice[sys];
            o++;
        }
    }
    __syncthreads();
}

// SELL row product of this lane's row in slice s.
template <typename V, class GX>
__device__ __forceinline__ V sell_row(const Sell<V> &M, uint32_t s, int lane, GX &gx)
{
    const uint32_t row0 = s * 32u, row = row0 + lane;
    const uint32_t len = row < M.n ? __ldg(&M.rp[row + 1]) - __ldg(&M.rp[row]) : 0u;
    const uint32_t g4 = __ldg(&M.slice_len4[s]);
    const size_t base = size_t(__ldg(&M.slice_ptr[s])) + 4u * lane;
    V acc = V(0);
#pragma unroll 4
    for (uint32_t g = 0; g < g4; g++) {
        const size_t e = base + size_t(g) * 128u;
        V v[4];
        ld4(M.val + e, v);
        uint32_t c[4];
        if (M.off) {
            const short4 o = __ldcs(reinterpret_cast<const short4 *>(M.off + e));
            c[0] = uint32_t(int(row0) + o.x);
            c[1] = uint32_t(int(row0) + o.y);
            c[2] = uint32_t(int(row0) + o.z);
            c[3] = uint32_t(int(row0) + o.w);
        } else {
            const uint4 o = __ldcs(reinterpret_cast<const uint4 *>(M.col + e));
            c[0] = o.x;
            c[1] = o.y;
            c[2] = o.z;
            c[3] = o.w;
        }
#pragma unroll
        for (int t = 0; t < 4; t++)
            if (4u * g + t < len) acc = row_acc(acc, v[t], V(gx(c[t])));
    }
    return acc;
}

// Warp loop over a contiguous block of the listed systems' slices (so warps share
// the active work evenly).  Systems that `skip(st)` rejects are jumped over as a
// whole.  For every visited slice, `body(s, st, v)` fills this lane's
// contributions; the warp sums them and lane 0 stores the slice's partials.
// No atomics: the per-system totals are formed by bk_reduce.
template <int NV, class SKIP, class BODY>
__device__ __forceinline__ void batch_loop(const BView &B, const Active *L, CgState *S, double *part, SKIP skip,
                                           BODY body)
{
    const int lane = threadIdx.x & 31;
    const uint32_t W = gridDim.x * (blockDim.x >> 5);
    const uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t total = L->n_slices, n_list = L->n_sys;
    const uint32_t per = (total + W - 1) / W;
    const uint32_t a_begin = min(total, w * per), a_end = min(total, a_begin + per);
    if (a_begin >= a_end) return;
    uint32_t lo = 0, hi = n_list;  // last k with prefix[k] <= a_begin
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (L->prefix[mid] <= a_begin) lo = mid;
        else hi = mid;
    }
    uint32_t k = lo;
    uint32_t a = a_begin;
    while (a < a_end) {
        const uint32_t sys = L->sys[k], k_end = L->prefix[k + 1];
        CgState *st = &S[sys];
        if (skip(st)) {
            a = k_end;
            k++;
            continue;
        }
        const uint32_t base = B.sys_slice[sys] - L->prefix[k];
        const uint32_t stop = min(a_end, k_end);
        for (; a < stop; a++) {
            const uint32_t s = base + a;
            double v[NV];
            body(s, st, v);
#pragma unroll
            for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
            if (lane == 0)
#pragma unroll
                for (int q = 0; q < NV; q++) part[size_t(s) * NV + q] = v[q];
        }
        k++;
    }
}

// One block per listed system: adds the system's slice partials in a fixed order
// and applies the state transition KIND (the same transitions as the
// single-system solver).
enum RedKind { RED_INIT_RES = 0, RED_INIT_Z, RED_DIR64, RED_DIR32, RED_UPD64, RED_UPD32, RED_CHK64, RED_CHK32, RED_TRUE };

template <int NV, int KIND>
__device__ __forceinline__ void finalize(CgState *st, const double (&acc)[NV], double *relres, uint32_t sys)
{
    if constexpr (KIND == RED_INIT_RES) {
        st->rn = sqrt(acc[0]);
        st->bn = sqrt(acc[1]);
        st->max_r = st->rn;
        st->sigma = st->bn > 0.0 ? 1.0 / st->bn : 1.0;
        if (!(st->rn > st->rtol * st->bn)) {
            st->done = 1;
            st->converged = 1;
            st->status = isfinite(st->rn) ? RSG_OK : RSG_BREAKDOWN;
        }
    } else if constexpr (KIND == RED_INIT_Z) {
        st->rho = st->rho_new = acc[0];
        st->beta = 0.0;
    } else if constexpr (KIND == RED_DIR64 || KIND == RED_DIR32) {
        double pq = acc[0];
        if constexpr (KIND == RED_DIR32) {
            if (pq == 0.0) pq = 1e-300;
        } else {
            pq = clamp_pq(pq, st->eps);
        }
        st->pq = pq;
        st->rho = st->rho_new;
        st->alpha = st->rho / pq;
        st->fold = 0;
    } else if constexpr (KIND == RED_UPD64) {
        finalize_update64(st, acc[0], acc[1], acc[2]);
    } else if constexpr (KIND == RED_UPD32) {
        finalize_update_mixed(st, acc[0], acc[1]);
    } else if constexpr (KIND == RED_CHK64) {
        finalize_check64(st, acc[0], sqrt(acc[1]));
    } else if constexpr (KIND == RED_CHK32) {
        finalize_check_mixed(st, acc[0], sqrt(acc[1]));
    } else {
        relres[sys] = acc[1] > 0.0 ? sqrt(acc[0] / acc[1]) : sqrt(acc[0]);
    }
}

template <int NV, int KIND>
__global__ void __launch_bounds__(kBlock) bk_reduce(BView B, const Active *L, CgState *S, const double *part,
                                                    double *relres, Active *L_chk = nullptr, uint32_t *arrive = nullptr)
{
    __shared__ double sh[NV * 32];
    __shared__ uint32_t last_sh;
    if (blockIdx.x < L->n_sys) {
        const uint32_t sys = L->sys[blockIdx.x];
        CgState *st = &S[sys];
        const bool skip = (KIND == RED_INIT_RES || KIND == RED_TRUE) ? false
                          : (KIND == RED_CHK64 || KIND == RED_CHK32) ? (st->done || !st->need_check)
                                                                     : st->done != 0;
        if (!skip) {
            const uint32_t b0 = B.sys_slice[sys], b1 = B.sys_slice[sys + 1];
            double acc[NV];
#pragma unroll
            for (int q = 0; q < NV; q++) acc[q] = 0.0;
            for (uint32_t s = b0 + threadIdx.x; s < b1; s += blockDim.x)
#pragma unroll
                for (int q = 0; q < NV; q++) acc[q] += part[size_t(s) * NV + q];
            block_sum<NV>(acc, sh);
            if (threadIdx.x == 0) finalize<NV, KIND>(st, acc, relres, sys);
        }
    }
    if (!L_chk) return;
    // after an update: the last block to finish lists the systems that asked for a check
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last_sh = atomicAdd(arrive, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_sh) return;
    __threadfence();
    build_list(L->n_sys, L->sys, B.sys_slice, L_chk,
               [&](uint32_t i) { return __ldcg(&S[i].done) == 0 && __ldcg(&S[i].need_check) != 0; });
    if (threadIdx.x == 0) *arrive = 0;
}

#define BATCH_ROWS_LOOP                                                                                      \
    const int lane = threadIdx.x & 31;                                                                      \
    const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);                                             \
    for (uint32_t s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < B.n_slices; s += warps_total)

__global__ void __launch_bounds__(kBlock) bk_init_res(Sell<double> M, BView B, const Active *L, const double *__restrict__ b,
                                                      const double *__restrict__ x, double *__restrict__ r,
                                                      double *part, CgState *S)
{
    const int lane = threadIdx.x & 31;
    auto gx = [&](uint32_t c) { return x[c]; };
    batch_loop<2>(
        B, L, S, part, [](const CgState *) { return false; },
        [&](uint32_t s, CgState *, double(&v)[2]) {
            const double ax = sell_row<double>(M, s, lane, gx);
            const uint32_t row = s * 32u + lane;
            v[0] = v[1] = 0.0;
            if (row < M.n) {
                const double ri = b[row] - ax;
                r[row] = ri;
                v[0] = ri * ri;
                v[1] = b[row] * b[row];
            }
        });
}

template <bool MIXED>
__global__ void __launch_bounds__(kBlock) bk_init_z(BView B, const Active *L, uint32_t n, const double *__restrict__ d,
                                                    const float *__restrict__ d32, const double *__restrict__ r,
                                                    double *__restrict__ z, float *__restrict__ r32,
                                                    float *__restrict__ z32, double *part, CgState *S)
{
    const int lane = threadIdx.x & 31;
    batch_loop<1>(
        B, L, S, part, [](const CgState *st) { return st->done != 0; },
        [&](uint32_t s, CgState *st, double(&v)[1]) {
            const uint32_t row = s * 32u + lane;
            v[0] = 0.0;
            if (row < n) {
                if (MIXED) {
                    const float rf = float(r[row] * st->sigma);
                    const float zf = d32 ? d32[row] * rf : rf;
                    r32[row] = rf;
                    z32[row] = zf;
                    v[0] = double(rf) * double(zf);
                } else {
                    const double zi = d ? d[row] * r[row] : r[row];
                    z[row] = zi;
                    v[0] = r[row] * zi;
                }
            }
        });
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) bk_dir(Sell<V> M, BView B, const Active *L, const V *__restrict__ z,
                                                 const V *__restrict__ p_old, V *__restrict__ p_new,
                                                 V *__restrict__ q, double *__restrict__ x, float *__restrict__ y,
                                                 double *part, CgState *S)
{
    const int lane = threadIdx.x & 31;
    batch_loop<1>(
        B, L, S, part, [](const CgState *st) { return st->done != 0; },
        [&](uint32_t s, CgState *st, double(&v)[1]) {
            const V beta = V(st->beta);
            auto gx = [&](uint32_t c) { return MIXED ? V(fmaf(float(beta), float(p_old[c]), float(z[c])))
                                                     : V(fma(double(beta), double(p_old[c]), double(z[c]))); };
            const V ax = sell_row<V>(M, s, lane, gx);
            const uint32_t row = s * 32u + lane;
            v[0] = 0.0;
            if (row < M.n) {
                const V p = gx(row);
                p_new[row] = p;
                q[row] = ax;
                v[0] = double(p) * double(ax);
                if (MIXED && st->fold) {
                    x[row] = fma(double(y[row]), 1.0 / st->sigma, x[row]);
                    y[row] = 0.f;
                }
            }
        });
}

template <typename V, bool MIXED>
__global__ void __launch_bounds__(kBlock) bk_update(BView B, const Active *L, uint32_t n, const V *__restrict__ d,
                                                    const V *__restrict__ p, const V *__restrict__ q,
                                                    V *__restrict__ xy, V *__restrict__ r, V *__restrict__ z,
                                                    double *part, CgState *S)
{
    const int lane = threadIdx.x & 31;
    batch_loop<3>(
        B, L, S, part, [](const CgState *st) { return st->done != 0; },
        [&](uint32_t s, CgState *st, double(&v)[3]) {
            const V alpha = V(st->alpha);
            const uint32_t row = s * 32u + lane;
            v[0] = v[1] = v[2] = 0.0;
            if (row < n) {
                const V xi = MIXED ? V(fmaf(float(alpha), float(p[row]), float(xy[row])))
                                   : V(fma(double(alpha), double(p[row]), double(xy[row])));
                const V ri = MIXED ? V(fmaf(-float(alpha), float(q[row]), float(r[row])))
                                   : V(fma(-double(alpha), double(q[row]), double(r[row])));
                const V zi = d ? d[row] * ri : ri;
                xy[row] = xi;
                r[row] = ri;
                z[row] = zi;
                v[0] = double(ri) * double(zi);
                v[1] = double(ri) * double(ri);
                v[2] = double(xi) * double(xi);
            }
        });
}

template <bool MIXED>
__global__ void __launch_bounds__(kBlock) bk_check(Sell<double> M, BView B, const Active *L, const double *__restrict__ d,
                                                   const float *__restrict__ d32, const double *__restrict__ b,
                                                   const double *__restrict__ x, const float *__restrict__ y,
                                                   double *__restrict__ r, double *__restrict__ z,
                                                   float *__restrict__ r32, float *__restrict__ z32, double *part,
                                                   CgState *S)
{
    const int lane = threadIdx.x & 31;
    batch_loop<2>(
        B, L, S, part, [](const CgState *st) { return st->done != 0 || st->need_check == 0; },
        [&](uint32_t s, CgState *st, double(&v)[2]) {
            const double sigma = st->sigma, inv_sigma = 1.0 / sigma;
            auto gx = [&](uint32_t c) { return MIXED ? fma(double(y[c]), inv_sigma, x[c]) : x[c]; };
            const double ax = sell_row<double>(M, s, lane, gx);
            const uint32_t row = s * 32u + lane;
            v[0] = v[1] = 0.0;
            if (row < M.n) {
                const double ri = b[row] - ax;
                v[1] = ri * ri;
                if (MIXED) {
                    const float rf = float(ri * sigma);
                    const float zf = d32 ? d32[row] * rf : rf;
                    r32[row] = rf;
                    z32[row] = zf;
                    v[0] = double(rf) * double(zf);
                } else {
                    const double zi = d ? d[row] * ri : ri;
                    r[row] = ri;
                    z[row] = zi;
                    v[0] = ri * zi;
                }
            }
        });
}

__global__ void bk_fold(BView B, uint32_t n, double *__restrict__ x, float *__restrict__ y, const CgState *S)
{
    BATCH_ROWS_LOOP
    {
        const uint32_t row = s * 32u + lane;
        if (row < n) {
            x[row] = fma(double(y[row]), 1.0 / S[B.slice_sys[s]].sigma, x[row]);
            y[row] = 0.f;
        }
    }
}

__global__ void bk_true_res(Sell<double> M, BView B, const Active *L, const double *__restrict__ b, const double *__restrict__ x,
                            double *part, CgState *S, double *relres)
{
    const int lane = threadIdx.x & 31;
    auto gx = [&](uint32_t c) { return x[c]; };
    batch_loop<2>(
        B, L, S, part, [](const CgState *) { return false; },
        [&](uint32_t s, CgState *, double(&v)[2]) {
            const double ax = sell_row<double>(M, s, lane, gx);
            const uint32_t row = s * 32u + lane;
            v[0] = v[1] = 0.0;
            if (row < M.n) {
                const double ri = b[row] - ax;
                v[0] = ri * ri;
                v[1] = b[row] * b[row];
            }
        });
}

// Loop control: rebuilds the list of active systems, keeps the graph's while node
// running while any system is active, enforces the hard limit.
__global__ void __launch_bounds__(kBlock) bk_tail(const CgState *S, const uint32_t *sys_slice, uint32_t n_sys,
                                                  Active *L, BatchCtl *ctl, cudaGraphConditionalHandle h,
                                                  int use_cond)
{
    build_list(n_sys, nullptr, sys_slice, L, [&](uint32_t i) { return S[i].done == 0; });
    if (threadIdx.x == 0) {
        const uint32_t bc = ++ctl->body_count;
        int keep = L->n_sys > 0;
        if (keep && bc >= ctl->body_limit) {
            ctl->timeout = 1;
            keep = 0;
        }
        if (use_cond) cudaGraphSetConditional(h, keep ? 1u : 0u);
        ctl->pad = keep;
    }
}

__global__ void bk_to_f32(uint32_t n, const double *__restrict__ src, float *__restrict__ dst)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = float(src[i]);
}

__global__ void bk_scatter(uint32_t n_user, const uint32_t *__restrict__ map, const double *__restrict__ src,
                           double *__restrict__ dst)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_user; i += gridDim.x * blockDim.x)
        dst[map[i]] = src[i];
}
__global__ void bk_gather(uint32_t n_user, const uint32_t *__restrict__ map, const double *__restrict__ src,
                          double *__restrict__ dst)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_user; i += gridDim.x * blockDim.x)
        dst[i] = src[map[i]];
}

}  // namespace
}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_batch_create(rsg_context *ctx, uint32_t n_sys, const uint32_t *sys_row_begin, const uint32_t *row_ptr,
                            const uint32_t *col_idx, const double *values, rsg_batch **out)
{
    if (!ctx || !out || !sys_row_begin || !row_ptr || n_sys == 0)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_create: bad arguments");
    *out = nullptr;
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    if (sys_row_begin[0] != 0) return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_create: systems must start at row 0");
    auto *B = new rsg_batch;
    B->n_sys = n_sys;
    B->user_begin.assign(sys_row_begin, sys_row_begin + n_sys + 1);
    B->pad_begin.assign(size_t(n_sys) + 1, 0);
    uint64_t pad_total = 0;
    for (uint32_t s = 0; s < n_sys; s++) {
        if (B->user_begin[s + 1] < B->user_begin[s] || B->user_begin[s + 1] == B->user_begin[s]) {
            delete B;
            return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_create: empty or decreasing system %u", s);
        }
        B->pad_begin[s] = uint32_t(pad_total);
        pad_total += (uint64_t(B->user_begin[s + 1] - B->user_begin[s]) + 31u) & ~uint64_t(31);
        if (pad_total > 0xffffff00ull) {
            delete B;
            return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_create: more than 2^32 rows after padding");
        }
    }
    B->pad_begin[n_sys] = uint32_t(pad_total);
    B->user_rows = B->user_begin[n_sys];
    B->pad_rows = uint32_t(pad_total);
    if (row_ptr[0] != 0) {
        delete B;
        return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_create: row_ptr[0] != 0");
    }
    // padded block-diagonal CSR; identity rows fill each system to a multiple of 32
    std::vector<uint32_t> rp(size_t(pad_total) + 1, 0), ci, map(B->user_rows);
    std::vector<double> val;
    ci.reserve(row_ptr[B->user_rows] + (pad_total - B->user_rows));
    val.reserve(ci.capacity());
    std::vector<uint32_t> slice_sys(pad_total / 32), sys_slice(size_t(n_sys) + 1);
    uint32_t prow = 0;
    for (uint32_t s = 0; s < n_sys; s++) {
        const uint32_t u0 = B->user_begin[s], u1 = B->user_begin[s + 1], p0 = B->pad_begin[s], p1 = B->pad_begin[s + 1];
        sys_slice[s] = p0 / 32;
        for (uint32_t q = p0 / 32; q < p1 / 32; q++) slice_sys[q] = s;
        for (uint32_t i = u0; i < u1; i++) {
            map[i] = p0 + (i - u0);
            for (uint32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++) {
                const uint32_t c = col_idx[j];
                if (c < u0 || c >= u1) {
                    delete B;
                    return set_error(ctx, RSG_ERR_INVALID_ARG,
                                     "batch_create: row %u has column %u outside its system %u", i, c, s);
                }
                ci.push_back(p0 + (c - u0));
                val.push_back(values[j]);
            }
            rp[++prow] = uint32_t(ci.size());
        }
        for (uint32_t i = p0 + (u1 - u0); i < p1; i++) {
            ci.push_back(i);
            val.push_back(1.0);
            rp[++prow] = uint32_t(ci.size());
        }
    }
    sys_slice[n_sys] = uint32_t(pad_total / 32);
    rsg_status st = csr_create_ex(ctx, B->pad_rows, rp.data(), ci.data(), val.data(), RSG_MEM_HOST, 1, &B->A);
    if (st != RSG_OK) {
        delete B;
        return st;
    }
    if (!B->A->use_sell) {
        rsg_csr_destroy(ctx, B->A);
        delete B;
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "batch_create: rows too uneven for the SELL-32 layout");
    }
    auto up = [&](uint32_t **d, const std::vector<uint32_t> &h) -> bool {
        return cudaMalloc(d, std::max<size_t>(h.size(), 1) * sizeof(uint32_t)) == cudaSuccess &&
               cudaMemcpy(*d, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice) == cudaSuccess;
    };
    if (!up(&B->d_slice_sys, slice_sys) || !up(&B->d_sys_slice, sys_slice) || !up(&B->d_user2pad, map)) {
        rsg_batch_destroy(ctx, B);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "batch_create: maps");
    }
    *out = B;
    return RSG_OK;
}

void rsg_batch_destroy(rsg_context *ctx, rsg_batch *B)
{
    if (!B) return;
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    if (B->A) rsg_csr_destroy(ctx, B->A);
    cudaFree(B->d_slice_sys);
    cudaFree(B->d_sys_slice);
    cudaFree(B->d_user2pad);
    delete B;
}

rsg_status rsg_batch_info(const rsg_batch *B, uint32_t *n_sys, uint32_t *rows, uint32_t *padded_rows, uint64_t *nnz)
{
    if (!B) return RSG_ERR_INVALID_ARG;
    if (n_sys) *n_sys = B->n_sys;
    if (rows) *rows = B->user_rows;
    if (padded_rows) *padded_rows = B->pad_rows;
    if (nnz) *nnz = B->A->nnz;
    return RSG_OK;
}

rsg_status rsg_batch_solve(rsg_context *ctx, rsg_batch *B, const rsg_solver_conf *conf, int32_t prec_type,
                           const double *b, double *x, int32_t memory, rsg_stats *per_system, rsg_stats *summary)
{
    if (!ctx || !B || !conf || !b || !x) return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_solve: null argument");
    if (conf->solver_type != RSG_SOLVER_CG)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "batch_solve: CG only");
    if (conf->stop_rule != RSG_STOP_TRUE_RELRES)
        return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_solve: stop_rule must be TRUE_RELRES");
    if (prec_type != RSG_PREC_NONE && prec_type != RSG_PREC_JACOBI)
        return set_error(ctx, RSG_ERR_UNSUPPORTED, "batch_solve: preconditioner must be NONE or JACOBI");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const bool mixed = conf->precision == RSG_PRECISION_MIXED;
    const uint32_t n = B->pad_rows, ns = B->n_sys, nsl = n / 32;
    const uint32_t max_it = std::max<uint32_t>(conf->n_outer, 1);
    const size_t vn = arena_bytes(n, sizeof(double)), vf = arena_bytes(n, sizeof(float));
    size_t bytes = 8 * vn + arena_bytes(size_t(nsl) * 3, sizeof(double)) + arena_bytes(ns, sizeof(CgState)) +
                   3 * arena_bytes(1, sizeof(Active)) + 6 * arena_bytes(size_t(ns) + 1, sizeof(uint32_t)) +
                   arena_bytes(ns, sizeof(double)) + arena_bytes(1, sizeof(BatchCtl)) + 2 * arena_bytes(B->user_rows, 8);
    if (mixed) bytes += 7 * vf;
    RSG_TRY(arena_reserve(ctx, bytes));
    double *bp = arena_take<double>(ctx, n), *xp = arena_take<double>(ctx, n), *r = arena_take<double>(ctx, n),
           *z = arena_take<double>(ctx, n), *p0 = arena_take<double>(ctx, n), *p1 = arena_take<double>(ctx, n),
           *q = arena_take<double>(ctx, n), *d = arena_take<double>(ctx, n);
    double *part = arena_take<double>(ctx, size_t(nsl) * 3);
    CgState *S = arena_take<CgState>(ctx, ns);
    double *relres = arena_take<double>(ctx, ns);
    BatchCtl *ctl = arena_take<BatchCtl>(ctx, 1);
    Active *L_all = arena_take<Active>(ctx, 1), *L_act = arena_take<Active>(ctx, 1);
    uint32_t *la_sys = arena_take<uint32_t>(ctx, size_t(ns) + 1), *la_pre = arena_take<uint32_t>(ctx, size_t(ns) + 1);
    uint32_t *lb_sys = arena_take<uint32_t>(ctx, size_t(ns) + 1), *lb_pre = arena_take<uint32_t>(ctx, size_t(ns) + 1);
    Active *L_chk = arena_take<Active>(ctx, 1);  // systems that asked for a check (built by the update reduction)
    uint32_t *lc_sys = arena_take<uint32_t>(ctx, size_t(ns) + 1), *lc_pre = arena_take<uint32_t>(ctx, size_t(ns) + 1);
    double *bu = memory == RSG_MEM_HOST ? arena_take<double>(ctx, B->user_rows) : const_cast<double *>(b);
    double *xu = memory == RSG_MEM_HOST ? arena_take<double>(ctx, B->user_rows) : x;
    float *r32 = nullptr, *z32 = nullptr, *pa = nullptr, *pb = nullptr, *q32 = nullptr, *y32 = nullptr, *d32 = nullptr;
    if (mixed) {
        r32 = arena_take<float>(ctx, n);
        z32 = arena_take<float>(ctx, n);
        pa = arena_take<float>(ctx, n);
        pb = arena_take<float>(ctx, n);
        q32 = arena_take<float>(ctx, n);
        y32 = arena_take<float>(ctx, n);
        d32 = arena_take<float>(ctx, n);
    }
    cudaStream_t sm = ctx->stream;
    const auto t0 = std::chrono::steady_clock::now();
    if (memory == RSG_MEM_HOST) {
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(bu, b, size_t(B->user_rows) * 8, cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(xu, x, size_t(B->user_rows) * 8, cudaMemcpyHostToDevice, sm));
    }
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(bp, 0, size_t(n) * 8, sm));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(xp, 0, size_t(n) * 8, sm));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(p0, 0, size_t(n) * 8, sm));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(p1, 0, size_t(n) * 8, sm));
    if (mixed) {
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(pa, 0, size_t(n) * 4, sm));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(pb, 0, size_t(n) * 4, sm));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(y32, 0, size_t(n) * 4, sm));
    }
    const int gu = std::min(grid_for(ctx, (const void *)bk_scatter, kBlock, 0, B->user_rows), kMaxGrid);
    bk_scatter<<<gu, kBlock, 0, sm>>>(B->user_rows, B->d_user2pad, bu, bp);
    bk_scatter<<<gu, kBlock, 0, sm>>>(B->user_rows, B->d_user2pad, xu, xp);
    const bool jac = prec_type == RSG_PREC_JACOBI;
    if (jac) {
        RSG_TRY(jacobi_build(ctx, B->A, d));
        if (mixed) {
            const int gv = std::min(grid_for(ctx, (const void *)bk_to_f32, kBlock, 0, n), kMaxGrid);
            bk_to_f32<<<gv, kBlock, 0, sm>>>(n, d, d32);
        }
    }
    // per-system state
    {
        CgState h;
        std::memset(&h, 0, sizeof(h));
        // no equation scaling here (each system keeps its own magnitude), so the
        // reference's p^T A p clamp, calibrated for scaled equations, is off
        h.eps = 0.0;
        h.cvg = conf->cvg;
        h.rtol = conf->rtol;
        h.delta = conf->reliable_delta > 0.0 && conf->reliable_delta < 1.0 ? conf->reliable_delta : kReliableDelta;
        h.sigma = 1.0;
        h.max_it = max_it;
        h.stop_rule = RSG_STOP_TRUE_RELRES;
        std::vector<CgState> hs(ns, h);
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(S, hs.data(), ns * sizeof(CgState), cudaMemcpyHostToDevice, sm));
        BatchCtl c = {0, max_it / 2 + 16, 0, 1, 0};
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(ctl, &c, sizeof(c), cudaMemcpyHostToDevice, sm));
        // both lists start with every system
        std::vector<uint32_t> ids(ns), pre(size_t(ns) + 1);
        for (uint32_t i = 0; i < ns; i++) {
            ids[i] = i;
            pre[i] = B->pad_begin[i] / 32;
        }
        pre[ns] = nsl;
        Active la = {ns, nsl, la_sys, la_pre}, lb = {ns, nsl, lb_sys, lb_pre}, lc = {0, 0, lc_sys, lc_pre};
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(la_sys, ids.data(), ns * 4, cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(la_pre, pre.data(), (size_t(ns) + 1) * 4, cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(lb_sys, ids.data(), ns * 4, cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(lb_pre, pre.data(), (size_t(ns) + 1) * 4, cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(L_all, &la, sizeof(Active), cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(L_act, &lb, sizeof(Active), cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(L_chk, &lc, sizeof(Active), cudaMemcpyHostToDevice, sm));
        RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
    }
    const BView V{B->d_slice_sys, B->d_sys_slice, nsl, ns};
    const Sell<double> M64 = sell_view<double>(B->A);
    const Sell<float> M32 = sell_view<float>(B->A);
    const int g_tuned = B->tuned ? (mixed ? B->g32 : B->g64) : 0;
    const int g = g_tuned > 0
                      ? g_tuned
                      : std::min(grid_for(ctx, (const void *)bk_dir<double, false>, kBlock, 0, (long long)nsl * 32),
                                 kMaxGrid);
    cudaEventRecord(ctx->ev[0], sm);
    const int gr = int(ns);  // reduce kernels: one block per listed system
    bk_init_res<<<g, kBlock, 0, sm>>>(M64, V, L_all, bp, xp, r, part, S);
    bk_reduce<2, RED_INIT_RES><<<gr, kBlock, 0, sm>>>(V, L_all, S, part, nullptr);
    if (mixed) {
        bk_init_z<true><<<g, kBlock, 0, sm>>>(V, L_all, n, jac ? d : nullptr, jac ? d32 : nullptr, r, z, r32, z32, part, S);
    } else {
        bk_init_z<false><<<g, kBlock, 0, sm>>>(V, L_all, n, jac ? d : nullptr, nullptr, r, z, r32, z32, part, S);
    }
    bk_reduce<1, RED_INIT_Z><<<gr, kBlock, 0, sm>>>(V, L_all, S, part, nullptr);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());

    auto body = [&](cudaGraphConditionalHandle h, int use_cond) {
        for (int half = 0; half < 2; half++) {
            if (!mixed) {
                double *po = half ? p1 : p0, *pn = half ? p0 : p1;
                bk_dir<double, false><<<g, kBlock, 0, sm>>>(M64, V, L_act, z, po, pn, q, xp, nullptr, part, S);
                bk_reduce<1, RED_DIR64><<<gr, kBlock, 0, sm>>>(V, L_act, S, part, nullptr);
                bk_update<double, false><<<g, kBlock, 0, sm>>>(V, L_act, n, jac ? d : nullptr, pn, q, xp, r, z, part, S);
                bk_reduce<3, RED_UPD64><<<gr, kBlock, 0, sm>>>(V, L_act, S, part, nullptr, L_chk, &ctl->arrive);
                bk_check<false><<<g, kBlock, 0, sm>>>(M64, V, L_chk, jac ? d : nullptr, nullptr, bp, xp, nullptr, r, z,
                                                     nullptr, nullptr, part, S);
                bk_reduce<2, RED_CHK64><<<gr, kBlock, 0, sm>>>(V, L_chk, S, part, nullptr);
            } else {
                float *po = half ? pb : pa, *pn = half ? pa : pb;
                bk_dir<float, true><<<g, kBlock, 0, sm>>>(M32, V, L_act, z32, po, pn, q32, xp, y32, part, S);
                bk_reduce<1, RED_DIR32><<<gr, kBlock, 0, sm>>>(V, L_act, S, part, nullptr);
                bk_update<float, true><<<g, kBlock, 0, sm>>>(V, L_act, n, jac ? d32 : nullptr, pn, q32, y32, r32, z32, part,
                                                            S);
                bk_reduce<3, RED_UPD32><<<gr, kBlock, 0, sm>>>(V, L_act, S, part, nullptr, L_chk, &ctl->arrive);
                bk_check<true><<<g, kBlock, 0, sm>>>(M64, V, L_chk, nullptr, jac ? d32 : nullptr, bp, xp, y32, r, z, r32,
                                                    z32, part, S);
                bk_reduce<2, RED_CHK32><<<gr, kBlock, 0, sm>>>(V, L_chk, S, part, nullptr);
            }
        }
        bk_tail<<<1, kBlock, 0, sm>>>(S, B->d_sys_slice, ns, L_act, ctl, h, use_cond);
    };

    rsg_status status = RSG_OK;
    if (conf->use_graph) {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        RSG_CHECK_CUDA(ctx, cudaGraphCreate(&graph, 0));
        do {
            cudaGraphConditionalHandle h;
            if (cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
                status = set_error(ctx, RSG_ERR_CUDA, "batch: conditional handle");
                break;
            }
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            if (cudaGraphAddNode(&node, graph, nullptr, 0, &cp) != cudaSuccess ||
                cudaStreamBeginCaptureToGraph(sm, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                              cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
                status = set_error(ctx, RSG_ERR_CUDA, "batch: graph capture");
                break;
            }
            body(h, 1);
            cudaGraph_t captured;
            if (cudaStreamEndCapture(sm, &captured) != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess ||
                cudaGraphLaunch(exec, sm) != cudaSuccess) {
                status = set_error(ctx, RSG_ERR_CUDA, "batch: graph launch");
                break;
            }
        } while (0);
        cudaError_t e = cudaStreamSynchronize(sm);
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(graph);
        if (status != RSG_OK) return status;
        if (e != cudaSuccess) return set_error(ctx, RSG_ERR_CUDA, "batch solve: %s", cudaGetErrorString(e));
    } else {
        const uint32_t polls = std::max<uint32_t>(1, conf->check_interval / 2);
        int32_t *keep = reinterpret_cast<int32_t *>(ctx->pinned);
        for (;;) {
            for (uint32_t k = 0; k < polls; k++) body(0, 0);
            RSG_CHECK_CUDA(ctx, cudaGetLastError());
            RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(keep, &ctl->pad, sizeof(int32_t), cudaMemcpyDeviceToHost, sm));
            RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
            if (!*keep) break;
        }
    }
    if (mixed) bk_fold<<<g, kBlock, 0, sm>>>(V, n, xp, y32, S);
    bk_true_res<<<g, kBlock, 0, sm>>>(M64, V, L_all, bp, xp, part, S, relres);
    bk_reduce<2, RED_TRUE><<<gr, kBlock, 0, sm>>>(V, L_all, S, part, relres);
    cudaEventRecord(ctx->ev[1], sm);
    bk_gather<<<gu, kBlock, 0, sm>>>(B->user_rows, B->d_user2pad, xp, xu);
    if (memory == RSG_MEM_HOST)
        RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(x, xu, size_t(B->user_rows) * 8, cudaMemcpyDeviceToHost, sm));
    std::vector<CgState> hs(ns);
    std::vector<double> rr(ns);
    BatchCtl hc;
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(hs.data(), S, ns * sizeof(CgState), cudaMemcpyDeviceToHost, sm));
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(rr.data(), relres, ns * sizeof(double), cudaMemcpyDeviceToHost, sm));
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, sm));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    rsg_stats sum;
    std::memset(&sum, 0, sizeof(sum));
    sum.converged = 1;
    rsg_status worst = RSG_OK;
    for (uint32_t s = 0; s < ns; s++) {
        rsg_stats st;
        std::memset(&st, 0, sizeof(st));
        st.iterations = hs[s].it;
        st.outer = hs[s].n_updates;
        st.error = hs[s].error;
        st.true_relres = rr[s];
        st.norm_b = hs[s].bn;
        st.converged = hs[s].converged;
        st.status = hs[s].ticket[7] ? RSG_ERR_TIMEOUT : hs[s].status;
        if (hs[s].done == 0) st.status = RSG_NOT_CONVERGED;
        if (per_system) per_system[s] = st;
        sum.iterations = std::max(sum.iterations, st.iterations);
        sum.outer += st.outer;
        sum.true_relres = std::max(sum.true_relres, st.true_relres);
        sum.converged &= st.converged;
        if (st.status != RSG_OK && (worst == RSG_OK || st.status < 0)) worst = rsg_status(st.status);
    }
    if (hc.timeout) worst = RSG_ERR_TIMEOUT;
    sum.status = worst;
    sum.seconds_solve = ms * 1e-3;
    sum.seconds_setup =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - sum.seconds_solve;
    if (summary) *summary = sum;
    if (worst == RSG_ERR_TIMEOUT) return set_error(ctx, RSG_ERR_TIMEOUT, "batch solve hit its hard limit");
    return worst;
}


// Batch autotuner (no reference counterpart): the grid of the slice kernels (direction,
// update, check) is chosen per precision by timing short fixed-length batch solves
// (every system runs kTuneIters iterations: rtol 0 is never met) for the built-in
// default and multiples of the SM count; three solves per candidate, median.
rsg_status rsg_batch_autotune(rsg_context *ctx, rsg_batch *B, rsg_tune_info *out)
{
    if (!ctx || !B) return set_error(ctx, RSG_ERR_INVALID_ARG, "batch_autotune: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    constexpr uint32_t kTuneIters = 32;
    constexpr int kReps = 3;
    const size_t nu = B->user_rows;
    double *b = nullptr, *x = nullptr;
    if (cudaMalloc(&b, nu * sizeof(double)) != cudaSuccess || cudaMalloc(&x, nu * sizeof(double)) != cudaSuccess) {
        cudaFree(b);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "batch_autotune: vectors");
    }
    std::vector<double> ones(nu, 1.0);
    rsg_status s = RSG_OK;
    if (cudaMemcpy(b, ones.data(), nu * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        s = set_error(ctx, RSG_ERR_CUDA, "batch_autotune: upload");
    rsg_solver_conf c;
    rsg_conf_default(&c);
    c.n_outer = kTuneIters;
    c.stop_rule = RSG_STOP_TRUE_RELRES;
    c.rtol = 0.0;
    const uint32_t nsl = B->A->n_slices;
    std::vector<int> cand = {0};
    for (int k : {1, 2, 3, 4, 6, 8}) cand.push_back(k * ctx->num_sms);
    cand.push_back(int(std::min<long long>(((long long)nsl * 32 + kBlock - 1) / kBlock, (long long)kMaxGrid)));
    B->tuned = true;
    uint32_t count = 0;
    for (int32_t prec : {RSG_PRECISION_FP64, RSG_PRECISION_MIXED}) {
        if (s != RSG_OK) break;
        c.precision = prec;
        int32_t &gsel = prec == RSG_PRECISION_FP64 ? B->g64 : B->g32;
        double best = 1e300, def = 0;
        int bestg = 0;
        for (int gc : cand) {
            gsel = gc;
            double t[kReps];
            for (int r = 0; r < kReps && s == RSG_OK; r++) {
                if (cudaMemsetAsync(x, 0, nu * sizeof(double), ctx->stream) != cudaSuccess) {
                    s = set_error(ctx, RSG_ERR_CUDA, "batch_autotune: memset");
                    break;
                }
                rsg_stats sum;
                const rsg_status rs = rsg_batch_solve(ctx, B, &c, RSG_PREC_JACOBI, b, x, RSG_MEM_DEVICE, nullptr, &sum);
                if (rs < 0) {
                    s = rs;
                    break;
                }
                t[r] = sum.seconds_solve / double(std::max<uint32_t>(sum.iterations, 1));
                count++;
            }
            if (s != RSG_OK) break;
            std::sort(t, t + kReps);
            const double tm = t[kReps / 2];
            if (gc == 0) def = tm;
            if (tm < best) {
                best = tm;
                bestg = gc;
            }
        }
        gsel = bestg;
        (prec == RSG_PRECISION_FP64 ? B->it64 : B->it32) = best;
        (prec == RSG_PRECISION_FP64 ? B->it64_default : B->it32_default) = def;
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(b);
    cudaFree(x);
    if (s != RSG_OK) {
        B->tuned = false;
        B->g64 = B->g32 = 0;
        return s;
    }
    B->tune_candidates = count;
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->tuned = 1;
        out->format = 1;
        out->rows_per_warp = 32;
        out->grid_dir_fp64 = out->grid_update_fp64 = uint32_t(B->g64);
        out->grid_dir_fp32 = out->grid_update_fp32 = uint32_t(B->g32);
        out->seconds_iter_fp64 = B->it64;
        out->seconds_iter_fp32 = B->it32;
        out->seconds_iter_fp64_default = B->it64_default;
        out->seconds_iter_fp32_default = B->it32_default;
        out->candidates = count;
    }
    return RSG_OK;
}

}  // extern "C"
