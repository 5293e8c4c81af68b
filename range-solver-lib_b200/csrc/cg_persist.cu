// The CG loop of a small system as one persistent cooperative kernel.
//
// Below a few hundred thousand rows a CG iteration of the graph-driven loop (cg.cu: direction + SpMV,
// update, check, one launch each) costs its launch latencies, not its bytes: ~19 us per iteration at
// 64k rows against ~5 us of traffic.  Here one cooperative launch runs the whole loop -- the
// reference's recurrences of solveCG (src/rmatrixsolver.cpp:258-331) as in cg.cu -- with a grid
// barrier between the phases instead of a kernel boundary.
//
// Same results bit for bit as the graph loop: every phase runs the graph loop's grid as virtual
// blocks (vb = blockIdx.x, blockIdx.x + gridDim.x, ...), each with the row assignment, per-thread
// accumulation order and block reduction of the kernel it replaces, and writes that kernel's
// per-block partial sums; after the barrier every CTA adds the partials exactly as the graph
// kernels' last block does and applies the same state transition (krylov.cuh) to its own copy of
// the CG state in shared memory, so all CTAs take the same decisions without another barrier.
// CTA 0 keeps the convergence history and writes the state back at the end.  Vectors written
// inside the kernel are read with ld.global.cg (L2), never through the non-coherent path.
//
// Barrier waits are bounded: a CTA that waits longer than kBarrierPolls polls flags the context's
// error word, marks the state RSG_ERR_TIMEOUT and leaves; the others then time out as well.
#include "grid_sync.cuh"
#include "krylov.cuh"

#include <algorithm>

namespace rsg {
namespace {

struct PersistArgs {
    Sell<double> S64;
    Sell<float> S32;
    uint32_t n;
    const double *b, *d;
    const float *d32;
    double *x, *r, *z, *p0, *p1, *q;
    float *r32, *z32, *p32a, *p32b, *q32, *y32;
    double *part_dir, *part_upd, *part_chk;  // per-virtual-block partials of the three phases
    CgState *st;
    unsigned int *bar;                       // [0] arrivals, [1] generation, [2] abort (grid_sync.cuh)
    uint32_t g_dir, g_upd, g_chk;           // the graph loop's grids (virtual)
    unsigned int *err;
};

// The graph kernels' last-block sum of G per-block partials (NV each): strided over the threads,
// then the block reduction -- the same order as grid_sum (common.cuh).  Valid in thread 0.
template <int NV>
__device__ __forceinline__ void final_sum(const double *partials, uint32_t G, double *sh, double (&total)[NV])
{
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) acc[k] = 0.0;
    for (unsigned int b = threadIdx.x; b < G; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; k++) acc[k] += __ldcg(&partials[size_t(b) * NV + k]);
    block_sum<NV>(acc, sh);
#pragma unroll
    for (int k = 0; k < NV; k++) total[k] = acc[k];
}

// Block partials of virtual block vb (block_sum, then thread 0 stores them).
template <int NV>
__device__ __forceinline__ void store_partials(double (&v)[NV], double *sh, double *partials, uint32_t vb)
{
    block_sum<NV>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; k++) partials[size_t(vb) * NV + k] = v[k];
}

// ---- FP64 phases (k_cg_dir, k_cg_update, k_cg_check of cg.cu, PK 0 none / 1 Jacobi) ----

__device__ __forceinline__ void dir64(const PersistArgs &a, const CgState &s, const double *p_old, double *p_new,
                                      double *sh)
{
    const double beta = s.beta;
    const double *z = a.z;
    for (uint32_t vb = blockIdx.x; vb < a.g_dir; vb += gridDim.x) {
        double acc[1] = {0.0};
        auto gx = [&](uint32_t c) { return fma(beta, __ldcg(p_old + c), __ldcg(z + c)); };
        auto epi = [&](uint32_t row, double v) {
            const double p = fma(beta, __ldcg(p_old + row), __ldcg(z + row));
            p_new[row] = p;
            a.q[row] = v;
            acc[0] += p * v;
        };
        for_rows_sell_v<double>(a.S64, gx, epi, vb, a.g_dir);
        store_partials<1>(acc, sh, a.part_dir, vb);
    }
}

template <int PK>
__device__ __forceinline__ void update64(const PersistArgs &a, const CgState &s, const double *p, double *sh)
{
    const double alpha = s.alpha;
    const uint32_t n = a.n;
    double *x = a.x, *r = a.r, *z = a.z;
    const double *q = a.q, *d = a.d;
    for (uint32_t vb = blockIdx.x; vb < a.g_upd; vb += gridDim.x) {
        double acc[3] = {0.0, 0.0, 0.0};
        const uint32_t tid = vb * blockDim.x + threadIdx.x, stride = a.g_upd * blockDim.x;
        auto row2 = [&](double2 pv, double2 qv, double2 xv, double2 rv, double2 dv, uint32_t i2) {
            double2 xo, ro, zo;
            xo.x = fma(alpha, pv.x, xv.x);
            xo.y = fma(alpha, pv.y, xv.y);
            ro.x = fma(-alpha, qv.x, rv.x);
            ro.y = fma(-alpha, qv.y, rv.y);
            zo.x = PK == 1 ? dv.x * ro.x : ro.x;
            zo.y = PK == 1 ? dv.y * ro.y : ro.y;
            reinterpret_cast<double2 *>(x)[i2] = xo;
            reinterpret_cast<double2 *>(r)[i2] = ro;
            reinterpret_cast<double2 *>(z)[i2] = zo;
            acc[0] += ro.x * zo.x + ro.y * zo.y;
            acc[1] += ro.x * ro.x + ro.y * ro.y;
            acc[2] += xo.x * xo.x + xo.y * xo.y;
        };
        const uint32_t npair = n / 2;
        for (uint32_t i2 = tid; i2 < npair; i2 += stride) {
            const double2 pv = __ldcg(reinterpret_cast<const double2 *>(p) + i2);
            const double2 qv = __ldcg(reinterpret_cast<const double2 *>(q) + i2);
            const double2 xv = __ldcg(reinterpret_cast<const double2 *>(x) + i2);
            const double2 rv = __ldcg(reinterpret_cast<const double2 *>(r) + i2);
            const double2 dv = PK == 1 ? __ldcg(reinterpret_cast<const double2 *>(d) + i2) : make_double2(1.0, 1.0);
            row2(pv, qv, xv, rv, dv, i2);
        }
        if ((n & 1u) && tid == 0) {
            const uint32_t i = n - 1;
            const double xi = fma(alpha, __ldcg(p + i), __ldcg(x + i));
            const double ri = fma(-alpha, __ldcg(q + i), __ldcg(r + i));
            const double zi = PK == 1 ? __ldcg(d + i) * ri : ri;
            x[i] = xi;
            r[i] = ri;
            z[i] = zi;
            acc[0] += ri * zi;
            acc[1] += ri * ri;
            acc[2] += xi * xi;
        }
        store_partials<3>(acc, sh, a.part_upd, vb);
    }
}

template <int PK>
__device__ __forceinline__ void check64(const PersistArgs &a, double *sh)
{
    const double *x = a.x, *b = a.b, *d = a.d;
    for (uint32_t vb = blockIdx.x; vb < a.g_chk; vb += gridDim.x) {
        double acc[2] = {0.0, 0.0};
        auto gx = [&](uint32_t c) { return __ldcg(x + c); };
        auto epi = [&](uint32_t row, double ax) {
            const double ri = b[row] - ax;
            a.r[row] = ri;
            acc[1] += ri * ri;
            if (PK == 0) {
                a.z[row] = ri;
                acc[0] += ri * ri;
            } else {
                const double zi = d[row] * ri;
                a.z[row] = zi;
                acc[0] += ri * zi;
            }
        };
        for_rows_sell_v<double>(a.S64, gx, epi, vb, a.g_chk);
        store_partials<2>(acc, sh, a.part_chk, vb);
    }
}

// ---- mixed-precision phases (k_mx_dir, k_mx_update, k_mx_check of cg.cu, PK 0 / 1) ----

__device__ __forceinline__ void dir32(const PersistArgs &a, const CgState &s, const float *p_old, float *p_new,
                                      double *sh)
{
    const float beta = float(s.beta);
    const int fold = s.fold;
    const double inv_sigma = 1.0 / s.sigma;
    const float *z = a.z32;
    double *x = a.x;
    float *y = a.y32;
    for (uint32_t vb = blockIdx.x; vb < a.g_dir; vb += gridDim.x) {
        Dot2 pq;
        auto gx = [&](uint32_t c) { return fmaf(beta, __ldcg(p_old + c), __ldcg(z + c)); };
        auto epi = [&](uint32_t row, float v) {
            const float p = fmaf(beta, __ldcg(p_old + row), __ldcg(z + row));
            p_new[row] = p;
            a.q32[row] = v;
            pq.add_prod(p, v);
            if (fold) {
                x[row] = fma(double(__ldcg(y + row)), inv_sigma, __ldcg(x + row));
                y[row] = 0.f;
            }
        };
        for_rows_sell_v<float>(a.S32, gx, epi, vb, a.g_dir);
        double acc[1] = {pq.value()};
        store_partials<1>(acc, sh, a.part_dir, vb);
    }
}

template <int PK>
__device__ __forceinline__ void update32(const PersistArgs &a, const CgState &s, const float *p, double *sh)
{
    const float alpha = float(s.alpha);
    const uint32_t n = a.n;
    const float *q = a.q32, *d = a.d32;
    float *y = a.y32, *r = a.r32, *z = a.z32;
    for (uint32_t vb = blockIdx.x; vb < a.g_upd; vb += gridDim.x) {
        Dot2 rz, rr;
        const uint32_t tid = vb * blockDim.x + threadIdx.x, stride = a.g_upd * blockDim.x;
        const uint32_t nq = n / 4;
        for (uint32_t i4 = tid; i4 < nq; i4 += stride) {
            const float4 pv = __ldcg(reinterpret_cast<const float4 *>(p) + i4);
            const float4 qv = __ldcg(reinterpret_cast<const float4 *>(q) + i4);
            float4 yv = __ldcg(reinterpret_cast<const float4 *>(y) + i4);
            float4 rv = __ldcg(reinterpret_cast<const float4 *>(r) + i4);
            const float4 dv = PK == 1 ? __ldcg(reinterpret_cast<const float4 *>(d) + i4) : make_float4(1.f, 1.f, 1.f, 1.f);
            float4 zv;
            yv.x = fmaf(alpha, pv.x, yv.x);
            yv.y = fmaf(alpha, pv.y, yv.y);
            yv.z = fmaf(alpha, pv.z, yv.z);
            yv.w = fmaf(alpha, pv.w, yv.w);
            rv.x = fmaf(-alpha, qv.x, rv.x);
            rv.y = fmaf(-alpha, qv.y, rv.y);
            rv.z = fmaf(-alpha, qv.z, rv.z);
            rv.w = fmaf(-alpha, qv.w, rv.w);
            zv.x = PK == 1 ? dv.x * rv.x : rv.x;
            zv.y = PK == 1 ? dv.y * rv.y : rv.y;
            zv.z = PK == 1 ? dv.z * rv.z : rv.z;
            zv.w = PK == 1 ? dv.w * rv.w : rv.w;
            reinterpret_cast<float4 *>(y)[i4] = yv;
            reinterpret_cast<float4 *>(r)[i4] = rv;
            reinterpret_cast<float4 *>(z)[i4] = zv;
            rz.add_prod(rv.x, zv.x);
            rz.add_prod(rv.y, zv.y);
            rz.add_prod(rv.z, zv.z);
            rz.add_prod(rv.w, zv.w);
            rr.add_prod(rv.x, rv.x);
            rr.add_prod(rv.y, rv.y);
            rr.add_prod(rv.z, rv.z);
            rr.add_prod(rv.w, rv.w);
        }
        for (uint32_t i = nq * 4 + tid; i < n; i += stride) {
            y[i] = fmaf(alpha, __ldcg(p + i), __ldcg(y + i));
            const float ri = fmaf(-alpha, __ldcg(q + i), __ldcg(r + i));
            const float zi = PK == 1 ? __ldcg(d + i) * ri : ri;
            r[i] = ri;
            z[i] = zi;
            rz.add_prod(ri, zi);
            rr.add_prod(ri, ri);
        }
        double acc[2] = {rz.value(), rr.value()};
        store_partials<2>(acc, sh, a.part_upd, vb);
    }
}

template <int PK>
__device__ __forceinline__ void check32(const PersistArgs &a, const CgState &s, double *sh)
{
    const double sigma = s.sigma, inv_sigma = 1.0 / sigma;
    const double *x = a.x, *b = a.b;
    const float *y = a.y32, *d = a.d32;
    for (uint32_t vb = blockIdx.x; vb < a.g_chk; vb += gridDim.x) {
        Dot2 rz;
        double rr[1] = {0.0};
        auto gx = [&](uint32_t c) { return fma(double(__ldcg(y + c)), inv_sigma, __ldcg(x + c)); };
        auto epi = [&](uint32_t row, double ax) {
            const double ri = b[row] - ax;
            rr[0] += ri * ri;
            const float rf = float(ri * sigma);
            a.r32[row] = rf;
            if (PK == 0) {
                a.z32[row] = rf;
                rz.add_prod(rf, rf);
            } else {
                const float zf = d[row] * rf;
                a.z32[row] = zf;
                rz.add_prod(rf, zf);
            }
        };
        for_rows_sell_v<double>(a.S64, gx, epi, vb, a.g_chk);
        double acc[2] = {rz.value(), rr[0]};
        store_partials<2>(acc, sh, a.part_chk, vb);
    }
}

// ---- the loop ----
// Two iterations make one body of the graph loop (its tail kernel counts bodies against
// body_limit); the loop below keeps that count, so the state ends exactly as the graph's does.
template <bool MIXED, int PK>
__global__ void __launch_bounds__(kBlock) k_cg_persist(PersistArgs a)
{
    __shared__ CgState s;
    __shared__ double sh[96];
    if (threadIdx.x == 0) {
        s = *a.st;
        if (blockIdx.x != 0) {  // CTA 0 alone records the convergence history
            s.history = nullptr;
            s.trend_hist = nullptr;
        }
    }
    __syncthreads();
    int half = 0;
    bool ok = true;
    while (!s.done) {
        // direction + SpMV, then alpha (k_cg_dir / k_mx_dir)
        if (MIXED) dir32(a, s, half ? a.p32b : a.p32a, half ? a.p32a : a.p32b, sh);
        else dir64(a, s, half ? a.p1 : a.p0, half ? a.p0 : a.p1, sh);
        if (!(ok = grid_barrier(a.bar, a.err))) break;
        {
            double tot[1];
            final_sum<1>(a.part_dir, a.g_dir, sh, tot);
            if (threadIdx.x == 0) {
                if (MIXED) {
                    double dd = tot[0];
                    if (dd == 0.0 || !isfinite(dd)) dd = (dd == 0.0) ? 1e-300 : dd;
                    s.pq = dd;
                    s.rho = s.rho_new;
                    s.alpha = s.rho / dd;
                    s.fold = 0;
                } else {
                    const double pq = clamp_pq(tot[0], s.eps);
                    s.pq = pq;
                    s.rho = s.rho_new;
                    s.alpha = s.rho / pq;
                }
            }
            __syncthreads();
        }
        // update, then beta and the stopping rule (k_cg_update / k_mx_update)
        if (MIXED) update32<PK>(a, s, half ? a.p32a : a.p32b, sh);
        else update64<PK>(a, s, half ? a.p0 : a.p1, sh);
        if (!(ok = grid_barrier(a.bar, a.err))) break;
        if (MIXED) {
            double tot[2];
            final_sum<2>(a.part_upd, a.g_upd, sh, tot);
            if (threadIdx.x == 0) finalize_update_mixed(&s, tot[0], tot[1]);
        } else {
            double tot[3];
            final_sum<3>(a.part_upd, a.g_upd, sh, tot);
            if (threadIdx.x == 0) finalize_update64(&s, tot[0], tot[1], tot[2]);
        }
        __syncthreads();
        // true-residual check when the recurrence asks for one (k_cg_check / k_mx_check)
        if (!s.done && s.need_check) {
            if (MIXED) check32<PK>(a, s, sh);
            else check64<PK>(a, sh);
            if (!(ok = grid_barrier(a.bar, a.err))) break;
            double tot[2];
            final_sum<2>(a.part_chk, a.g_chk, sh, tot);
            if (threadIdx.x == 0) {
                if (MIXED) finalize_check_mixed(&s, tot[0], sqrt(tot[1]));
                else finalize_check64(&s, tot[0], sqrt(tot[1]));
            }
            __syncthreads();
        }
        half ^= 1;
        if (half == 0) {  // the graph's tail after each body
            if (threadIdx.x == 0) {
                const uint32_t bc = ++s.body_count;
                if (!s.done && bc >= s.body_limit) {
                    s.done = 1;
                    s.status = RSG_ERR_TIMEOUT;
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        if (!ok) {
            s.done = 1;
            s.status = RSG_ERR_TIMEOUT;
        } else if (half == 1) {
            ++s.body_count;  // the graph's tail of the body in which the loop ended
        }
        if (blockIdx.x == 0) *a.st = s;
    }
}

}  // namespace

// Runs the loop of cg.cu's run_typed as one cooperative launch; *ran = false (and nothing launched)
// when the device cannot make every CTA resident, and the caller takes the graph loop.
rsg_status cg_persist_run(rsg_context *ctx, const CgArgs &a, int g_dir, int g_upd, int g_chk, bool *ran)
{
    *ran = false;
    const int pk = a.P.kind;
    if (pk != 0 && pk != 1) return RSG_OK;
    const void *k = a.mixed ? (pk ? (const void *)k_cg_persist<true, 1> : (const void *)k_cg_persist<true, 0>)
                            : (pk ? (const void *)k_cg_persist<false, 1> : (const void *)k_cg_persist<false, 0>);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kBlock, 0) != cudaSuccess || per_sm < 1) {
        (void)cudaGetLastError();
        return RSG_OK;
    }
    if (std::max(g_dir, std::max(g_upd, g_chk)) > kMaxGrid) return RSG_OK;
    // every resident CTA, but no more than the largest virtual grid (measured at 65k rows: 1 CTA per SM
    // 14.4 -> 18.5 us per FP64 iteration; 2 or 5 per SM alike; at 266k rows 5 per SM beats 2)
    const int grid = std::max(1, std::min(per_sm * ctx->num_sms, std::max(g_dir, std::max(g_upd, g_chk))));
    if (!ctx->persist) {
        if (cudaMalloc(&ctx->persist, size_t(6) * kMaxGrid * sizeof(double) + 256) != cudaSuccess) {
            ctx->persist = nullptr;
            (void)cudaGetLastError();
            return RSG_OK;
        }
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->persist, 0, size_t(6) * kMaxGrid * sizeof(double) + 256, ctx->stream));
    }
    double *part = ctx->persist;
    unsigned int *bar = reinterpret_cast<unsigned int *>(part + size_t(6) * kMaxGrid);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(bar, 0, 3 * sizeof(unsigned int), ctx->stream));  // no arrivals, no abort
    PersistArgs pa;
    pa.S64 = sell_view<double>(a.A);
    pa.S32 = sell_view<float>(a.A);
    pa.n = a.A->n;
    pa.b = a.b;
    pa.d = a.P.d;
    pa.d32 = a.P.d32;
    pa.x = a.x;
    pa.r = a.r;
    pa.z = a.z;
    pa.p0 = a.p0;
    pa.p1 = a.p1;
    pa.q = a.q;
    pa.r32 = a.r32;
    pa.z32 = a.z32;
    pa.p32a = a.p32a;
    pa.p32b = a.p32b;
    pa.q32 = a.q32;
    pa.y32 = a.y32;
    pa.part_dir = part;
    pa.part_upd = part + kMaxGrid;
    pa.part_chk = part + size_t(4) * kMaxGrid;
    pa.st = a.st;
    pa.bar = bar;
    pa.g_dir = uint32_t(g_dir);
    pa.g_upd = uint32_t(g_upd);
    pa.g_chk = uint32_t(g_chk);
    pa.err = ctx->errw;
    void *args[] = {&pa};
    const cudaError_t e = cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kBlock), args, 0, ctx->stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return RSG_OK;
    }
    *ran = true;
    return RSG_OK;
}

}  // namespace rsg
