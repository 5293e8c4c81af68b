// CSR SpMV core shared by every solver kernel.
//
// The reference's row product (multiplyRow, src/rmatrixsolver.cpp:111-119) is
// a scalar loop per row.  Here one warp owns a chunk of RPW consecutive rows:
//   1. stream phase: the chunk's nonzeros [rp[row0], rp[row0+RPW]) are one
//      contiguous range; the 32 lanes read it with 16-byte vector loads of
//      values and column indexes (fully coalesced, no per-row divergence),
//      multiply by the gathered x and park the products in shared memory;
//   2. row phase: FP32 -- 32/RPW lanes per row sum that row's products; FP64 --
//      one lane per row adds them serially in CSR column order (the
//      reference's multiplyRow arithmetic); the sum goes to the caller's epilogue.
// Chunks whose nonzeros exceed kCap fall back to warp-per-row.
//
// The x operand is a functor so callers fuse vector updates into the gather
// (e.g. CG's p = z + beta p_old computed on the fly), and the epilogue fuses the
// row's output with dot-product partials.  Column indexes are either uint32 or
// 16-bit offsets from the row's 32-row block base (col - (row & ~31)), which
// cuts index traffic in half for banded matrices such as structured meshes.
#pragma once

#include "common.cuh"

#include <type_traits>

namespace rsg {

constexpr uint32_t kCap = 512;  // products per warp held in shared memory

template <typename V>
struct Csr {
    const uint32_t *rp;
    const uint32_t *ci;
    const int16_t *off;   // non-null -> 16-bit offsets are used
    const V *val;
    uint32_t n;
};

// Streaming loads of the matrix: read-only path, not allocated in L1 (the
// matrix is used once per product; L1 is kept for the x gathers).
__device__ __forceinline__ double2 ld_stream(const double2 *p)
{
    double2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ float4 ld_stream(const float4 *p)
{
    float4 v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}
__device__ __forceinline__ uint2 ld_stream(const uint2 *p)
{
    uint2 v;
    asm("ld.global.nc.L1::no_allocate.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
    return v;
}
__device__ __forceinline__ uint4 ld_stream(const uint4 *p)
{
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t *p)
{
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

template <typename V>
struct VecLoad;
template <>
struct VecLoad<double> {
    static constexpr int W = 2;
    __device__ __forceinline__ static void vals(const double *p, double (&v)[2])
    {
        double2 t = ld_stream(reinterpret_cast<const double2 *>(p));
        v[0] = t.x;
        v[1] = t.y;
    }
    __device__ __forceinline__ static void cols(const uint32_t *p, uint32_t (&c)[2])
    {
        uint2 t = ld_stream(reinterpret_cast<const uint2 *>(p));
        c[0] = t.x;
        c[1] = t.y;
    }
    __device__ __forceinline__ static void offs(const int16_t *p, int (&c)[2])
    {
        uint32_t t = ld_stream(reinterpret_cast<const uint32_t *>(p));
        c[0] = int(int16_t(t & 0xffffu));
        c[1] = int(int16_t(t >> 16));
    }
};
template <>
struct VecLoad<float> {
    static constexpr int W = 4;
    __device__ __forceinline__ static void vals(const float *p, float (&v)[4])
    {
        float4 t = ld_stream(reinterpret_cast<const float4 *>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
    __device__ __forceinline__ static void cols(const uint32_t *p, uint32_t (&c)[4])
    {
        uint4 t = ld_stream(reinterpret_cast<const uint4 *>(p));
        c[0] = t.x;
        c[1] = t.y;
        c[2] = t.z;
        c[3] = t.w;
    }
    __device__ __forceinline__ static void offs(const int16_t *p, int (&c)[4])
    {
        uint2 t = ld_stream(reinterpret_cast<const uint2 *>(p));
        c[0] = int(int16_t(t.x & 0xffffu));
        c[1] = int(int16_t(t.x >> 16));
        c[2] = int(int16_t(t.y & 0xffffu));
        c[3] = int(int16_t(t.y >> 16));
    }
};

// Row product for one row by a whole warp (rows too long to stage).  FP32 (inner
// solver only): lanes take strided elements and a shuffle tree adds them.  FP64:
// lane 0 sums the row serially in CSR column order with separate multiply and
// add, the reference's multiplyRow arithmetic (src/rmatrixsolver.cpp:111-119),
// so every FP64 path gives the same bits as the SELL-32 path.
template <typename V, typename A, class GX>
__device__ __forceinline__ A warp_row(const Csr<V> &M, uint32_t row, GX &gx, int lane)
{
    const uint32_t s = M.rp[row], e = M.rp[row + 1];
    const int base = int(row & ~31u);
    A acc = A(0);
    if constexpr (std::is_same<A, double>::value) {
        if (lane == 0)
            for (uint32_t j = s; j < e; j++) {
                const uint32_t c = M.off ? uint32_t(base + int(M.off[j])) : M.ci[j];
                acc = __dadd_rn(acc, __dmul_rn(double(M.val[j]), double(gx(c))));
            }
        return __shfl_sync(0xffffffffu, acc, 0);
    } else {
        for (uint32_t j = s + lane; j < e; j += 32) {
            const uint32_t c = M.off ? uint32_t(base + int(M.off[j])) : M.ci[j];
            acc += A(M.val[j]) * A(gx(c));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        return acc;
    }
}

// ---------------------------------------------------------------------------
// TMA-staged pipeline.  Each warp streams its row chunks through NS shared-
// memory stages: one lane issues bulk copies (cp.async.bulk, the TMA unit) of
// the chunk's values and column indexes and arms the stage's mbarrier with the
// byte count; the warp computes the previous chunk meanwhile.  Products are
// formed in place in the stage, summed per row, and the stage is re-armed
// with the chunk NS positions ahead.  The matrix stream therefore never
// occupies registers, and every warp keeps one chunk in flight while it
// computes another.  Waits are bounded: past kWaitLimit polls the kernel
// records an error, drains its own copies (again bounded) and stops taking
// chunks, so a stuck copy cannot hang the GPU.
// ---------------------------------------------------------------------------
constexpr int kStages = 2;
constexpr uint32_t kStageElems = kCap + 16;  // chunk nonzeros plus alignment slack
constexpr uint32_t kWaitLimit = 1u << 20;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arm(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// bounded wait; returns false (and flags *err) when the limit is reached
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, unsigned int *err)
{
    for (uint32_t t = 0; t < kWaitLimit; t++)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, 1u);
    return false;
}

template <typename V>
struct Stage {
    // index slots are sized for uint32 columns; 16-bit offsets use the first half
    static constexpr uint32_t kValBytes = kStageElems * sizeof(V);
    static constexpr uint32_t kIdxBytes = kStageElems * sizeof(uint32_t);
    static constexpr uint32_t kBytes = kValBytes + kIdxBytes;
    // per warp: kStages stages + kStages mbarriers (16-byte padded)
    static constexpr uint32_t kWarpBytes = kStages * kBytes + 16 * kStages;
};

// Product rounded on its own (never contracted into a later add).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return a * b; }

template <typename V>
constexpr size_t tma_smem() { return size_t(kWarpsPerBlock) * Stage<V>::kWarpBytes; }

// Grid-stride over row chunks with the TMA pipeline.  Every thread of the block
// calls it; returns normally even on a wait timeout (the caller's grid
// reduction still runs).  `evict_first` selects the L2 policy of the stream.
template <typename V, int RPW, class GX, class EPI>
__device__ __forceinline__ void for_rows_tma(const Csr<V> &M, GX &gx, EPI &epi, unsigned char *smem,
                                             unsigned int *err, bool evict_first)
{
    using S = Stage<V>;
    constexpr int L = 32 / RPW;
    const bool off = M.off != nullptr;
    const uint32_t isz = off ? 2u : 4u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char *wbase = smem + size_t(warp) * S::kWarpBytes;
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbase + kStages * S::kBytes);
    const uint32_t n_chunks = (M.n + RPW - 1) / RPW;
    const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
    const uint32_t first = blockIdx.x * (blockDim.x >> 5) + warp;
    const unsigned char *idx_g = off ? reinterpret_cast<const unsigned char *>(M.off)
                                     : reinterpret_cast<const unsigned char *>(M.ci);
    const uint64_t pol = evict_first ? policy_evict_first() : policy_evict_last();

    if (lane == 0) {
        for (int s = 0; s < kStages; s++) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncwarp();

    // issue chunk c into stage s (lane 0); returns whether a copy is in flight
    auto issue = [&](uint32_t c, int s) -> bool {
        if (c >= n_chunks) return false;
        const uint32_t row0 = c * RPW;
        const uint32_t nrows = min(uint32_t(RPW), M.n - row0);
        const uint32_t start = __ldg(&M.rp[row0]), end = __ldg(&M.rp[row0 + nrows]);
        if (end - start > kCap) return false;  // long rows: handled without staging
        const uint32_t a0 = start & ~7u, a1 = (end + 7u) & ~7u;
        if (a1 == a0) return false;
        if (lane == 0) {
            unsigned char *st = wbase + s * S::kBytes;
            const uint32_t vb = (a1 - a0) * sizeof(V), ib = (a1 - a0) * isz;
            mbar_arm(&bar[s], vb + ib);
            bulk_load(st, M.val + a0, vb, &bar[s], pol);
            bulk_load(st + S::kValBytes, idx_g + size_t(a0) * isz, ib, &bar[s], pol);
        }
        return true;
    };

    bool inflight[kStages];
    uint32_t phase[kStages];
#pragma unroll
    for (int s = 0; s < kStages; s++) {
        phase[s] = 0;
        inflight[s] = issue(first + s * warps_total, s);
    }
    bool failed = false;
    int s = 0;
    for (uint32_t c = first; c < n_chunks; c += warps_total) {
        const uint32_t row0 = c * RPW;
        const uint32_t nrows = min(uint32_t(RPW), M.n - row0);
        const uint32_t end = __ldg(&M.rp[row0 + nrows]);
        const uint32_t my_rp = (lane < int(nrows)) ? __ldg(&M.rp[row0 + lane]) : end;
        const uint32_t start = __shfl_sync(0xffffffffu, my_rp, 0);
        const int base = int(row0 & ~31u);
        if (inflight[s]) {
            if (!mbar_wait(&bar[s], phase[s], err)) {
                failed = true;
                break;
            }
            phase[s] ^= 1u;
            inflight[s] = false;
            unsigned char *st = wbase + s * S::kBytes;
            V *sv = reinterpret_cast<V *>(st);
            const int16_t *so = reinterpret_cast<const int16_t *>(st + S::kValBytes);
            const uint32_t *sc = reinterpret_cast<const uint32_t *>(st + S::kValBytes);
            const uint32_t a0 = start & ~7u;
            if (off) {
#pragma unroll 4
                for (uint32_t j = start + lane; j < end; j += 32) {
                    const uint32_t k = j - a0;
                    sv[k] = mul_rn(sv[k], V(gx(uint32_t(base + int(so[k])))));
                }
            } else {
#pragma unroll 4
                for (uint32_t j = start + lane; j < end; j += 32) {
                    const uint32_t k = j - a0;
                    sv[k] = mul_rn(sv[k], V(gx(sc[k])));
                }
            }
            __syncwarp();
            const int r = lane / L, sub = lane % L;
            const uint32_t rs = __shfl_sync(0xffffffffu, my_rp, r) - a0;
            const uint32_t nx = __shfl_sync(0xffffffffu, my_rp, min(r + 1, 31));
            const uint32_t re = ((r + 1 < int(nrows)) ? nx : end) - a0;
            V acc = V(0);
            if constexpr (std::is_same<V, double>::value) {
                // FP64: one lane per row adds the row's rounded products serially in CSR column order
                // (multiplyRow, src/rmatrixsolver.cpp:111-119); the products were rounded on their own above.
                if (sub == 0 && r < int(nrows))
                    for (uint32_t k = rs; k < re; k++) acc = __dadd_rn(acc, sv[k]);
            } else {
                if (r < int(nrows))
                    for (uint32_t k = rs + sub; k < re; k += L) acc += sv[k];
#pragma unroll
                for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            }
            if (sub == 0 && r < int(nrows)) epi(row0 + r, acc);
            __syncwarp();
            fence_async_shared();  // generic writes to the stage precede the next async copy into it
            __syncwarp();
        } else if (end - start > 0) {
            // long rows (or a chunk that was not staged): whole warp per row from global memory
            for (uint32_t rr = 0; rr < nrows; rr++) {
                V acc = warp_row<V, V>(M, row0 + rr, gx, lane);
                if (lane == 0) epi(row0 + rr, acc);
            }
        } else {
            if (lane < int(nrows)) epi(row0 + lane, V(0));
        }
        inflight[s] = issue(c + kStages * warps_total, s);
        s = (s + 1 == kStages) ? 0 : s + 1;
    }
    if (failed) {
        // drain every copy this warp still has in flight before the shared memory is released
#pragma unroll
        for (int t = 0; t < kStages; t++)
            if (inflight[t]) mbar_wait(&bar[t], phase[t], nullptr);
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// SELL-32 path (preferred when padding is small).  One warp per 32-row slice,
// one thread per row; every lane reads 4 consecutive elements of its row per
// 16-byte load (two for FP64 values), so a warp load instruction moves 512 B
// (FP32) / 1 KB (FP64) of contiguous matrix data, and all of a row's loads are
// independent.  Each row is summed by one thread in CSR column order with no
// fused multiply-add, which is the reference's multiplyRow arithmetic
// (src/rmatrixsolver.cpp:111-119) step for step.
// ---------------------------------------------------------------------------
template <typename V>
struct Sell {
    const uint32_t *rp;
    const uint32_t *slice_ptr;
    const uint32_t *slice_len4;
    const V *val;
    const int16_t *off;
    const uint32_t *col;
    uint32_t n, n_slices;
};

// FP64: separate multiply and add (no contraction), as the reference's loop;
// FP32 (inner solver only): fused multiply-add.
__device__ __forceinline__ double row_acc(double acc, double v, double x) { return __dadd_rn(acc, __dmul_rn(v, x)); }
__device__ __forceinline__ float row_acc(float acc, float v, float x) { return fmaf(v, x, acc); }

__device__ __forceinline__ void ld4(const double *p, double (&v)[4])
{
    const double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    v[0] = a.x;
    v[1] = a.y;
    v[2] = b.x;
    v[3] = b.y;
}
__device__ __forceinline__ void ld4(const float *p, float (&v)[4])
{
    const float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
}

// The rows of virtual block vb of a grid of vgrid blocks (a persistent kernel runs several virtual
// blocks per CTA with the same row assignment, and so the same sums, as a grid of vgrid blocks).
template <typename V, class GX, class EPI>
__device__ __forceinline__ void for_rows_sell_v(const Sell<V> &M, GX &gx, EPI &epi, uint32_t vb, uint32_t vgrid)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warps_total = vgrid * (blockDim.x >> 5);
    for (uint32_t s = vb * (blockDim.x >> 5) + (threadIdx.x >> 5); s < M.n_slices; s += warps_total) {
        const uint32_t row0 = s * 32u, row = row0 + lane;
        const bool valid = row < M.n;
        const uint32_t len = valid ? __ldg(&M.rp[row + 1]) - __ldg(&M.rp[row]) : 0u;
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
        if (valid) epi(row, acc);
    }
}

template <typename V, class GX, class EPI>
__device__ __forceinline__ void for_rows_sell(const Sell<V> &M, GX &gx, EPI &epi)
{
    for_rows_sell_v<V>(M, gx, epi, blockIdx.x, gridDim.x);
}

template <typename V>
inline Sell<V> sell_view(const rsg_csr *A);
template <>
inline Sell<double> sell_view<double>(const rsg_csr *A)
{
    return Sell<double>{A->rp, A->slice_ptr, A->slice_len4, A->sval, A->soff, A->scol, A->n, A->n_slices};
}
template <>
inline Sell<float> sell_view<float>(const rsg_csr *A)
{
    return Sell<float>{A->rp, A->slice_ptr, A->slice_len4, A->sval32, A->soff, A->scol, A->n, A->n_slices};
}

// Runs the SELL path when the matrix has it, else the TMA-staged CSR stream.
template <typename V, int RPW, class GX, class EPI>
__device__ __forceinline__ void for_rows_any(const Csr<V> &M, const Sell<V> &S, bool use_sell, GX &gx, EPI &epi,
                                             unsigned char *smem, unsigned int *err, bool evict_first)
{
    if (use_sell) for_rows_sell<V>(S, gx, epi);
    else for_rows_tma<V, RPW>(M, gx, epi, smem, err, evict_first);
}

template <typename V>
inline Csr<V> view(const rsg_csr *A, bool use_off16);
template <>
inline Csr<double> view<double>(const rsg_csr *A, bool use_off16)
{
    return Csr<double>{A->rp, A->ci, use_off16 && A->has_off16 ? A->off16 : nullptr, A->val, A->n};
}
template <>
inline Csr<float> view<float>(const rsg_csr *A, bool use_off16)
{
    return Csr<float>{A->rp, A->ci, use_off16 && A->has_off16 ? A->off16 : nullptr, A->val32, A->n};
}

// Rows per warp chosen from the longest 32-row chunk: smaller chunks keep the
// stream phase inside kCap for wider stencils (elasticity: up to 81 per row).
// Largest rows-per-warp chunk of the CSR stream whose products fit the staging buffer.
inline int natural_rpw(const rsg_csr *A)
{
    if (A->max_warp_nnz <= kCap) return 32;
    if (A->max_warp_nnz <= 2 * kCap) return 16;
    if (A->max_warp_nnz <= 4 * kCap) return 8;
    return 4;
}
// The autotuner may pick a smaller chunk (always valid: fewer rows, fewer products).
inline int pick_rpw(const rsg_csr *A)
{
    const int nat = natural_rpw(A);
    return A->tune.rpw > 0 && A->tune.rpw < nat ? A->tune.rpw : nat;
}

template <typename A>
constexpr size_t prod_smem() { return size_t(kWarpsPerBlock) * kCap * sizeof(A); }

}  // namespace rsg
