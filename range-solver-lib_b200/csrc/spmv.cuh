// CSR SpMV core shared by every solver kernel.
//
// The reference's row product (multiplyRow, src/rmatrixsolver.cpp:111-119) is
// a scalar loop per row.  Here one warp owns a chunk of RPW consecutive rows:
//   1. stream phase: the chunk's nonzeros [rp[row0], rp[row0+RPW]) are one
//      contiguous range; the 32 lanes read it with 16-byte vector loads of
//      values and column indexes (fully coalesced, no per-row divergence),
//      multiply by the gathered x and park the products in shared memory;
//   2. row phase: 32/RPW lanes per row sum that row's products and hand the
//      result to the caller's epilogue.
// Chunks whose nonzeros exceed kCap fall back to warp-per-row.
//
// The x operand is a functor so callers fuse vector updates into the gather
// (e.g. CG's p = z + beta p_old computed on the fly), and the epilogue fuses the
// row's output with dot-product partials.  Column indexes are either uint32 or
// 16-bit offsets from the row's 32-row block base (col - (row & ~31)), which
// cuts index traffic in half for banded matrices such as structured meshes.
#pragma once

#include "common.cuh"

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

template <typename V>
struct VecLoad;
template <>
struct VecLoad<double> {
    static constexpr int W = 2;
    __device__ __forceinline__ static void vals(const double *p, double (&v)[2])
    {
        double2 t = __ldg(reinterpret_cast<const double2 *>(p));
        v[0] = t.x;
        v[1] = t.y;
    }
    __device__ __forceinline__ static void cols(const uint32_t *p, uint32_t (&c)[2])
    {
        uint2 t = __ldg(reinterpret_cast<const uint2 *>(p));
        c[0] = t.x;
        c[1] = t.y;
    }
    __device__ __forceinline__ static void offs(const int16_t *p, int (&c)[2])
    {
        short2 t = __ldg(reinterpret_cast<const short2 *>(p));
        c[0] = t.x;
        c[1] = t.y;
    }
};
template <>
struct VecLoad<float> {
    static constexpr int W = 4;
    __device__ __forceinline__ static void vals(const float *p, float (&v)[4])
    {
        float4 t = __ldg(reinterpret_cast<const float4 *>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
    __device__ __forceinline__ static void cols(const uint32_t *p, uint32_t (&c)[4])
    {
        uint4 t = __ldg(reinterpret_cast<const uint4 *>(p));
        c[0] = t.x;
        c[1] = t.y;
        c[2] = t.z;
        c[3] = t.w;
    }
    __device__ __forceinline__ static void offs(const int16_t *p, int (&c)[4])
    {
        short4 t = __ldg(reinterpret_cast<const short4 *>(p));
        c[0] = t.x;
        c[1] = t.y;
        c[2] = t.z;
        c[3] = t.w;
    }
};

// Row product for one row by a whole warp (long rows).
template <typename V, typename A, class GX>
__device__ __forceinline__ A warp_row(const Csr<V> &M, uint32_t row, GX &gx, int lane)
{
    const uint32_t s = M.rp[row], e = M.rp[row + 1];
    const int base = int(row & ~31u);
    A acc = A(0);
    for (uint32_t j = s + lane; j < e; j += 32) {
        uint32_t c = M.off ? uint32_t(base + int(M.off[j])) : M.ci[j];
        acc += A(M.val[j]) * A(gx(c));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// Process rows [row0, row0 + RPW) of M with one warp.  `prod` is this warp's
// kCap-element shared buffer.  Accumulation type A (double for FP64, float for FP32).
template <typename V, typename A, int RPW, class GX, class EPI>
__device__ __forceinline__ void warp_chunk(const Csr<V> &M, uint32_t row0, GX &gx, EPI &epi, A *prod, int lane)
{
    static_assert(32 % RPW == 0, "RPW must divide 32");
    constexpr int L = 32 / RPW;  // lanes per row in the row phase
    constexpr int W = VecLoad<V>::W;
    const uint32_t nrows = min(uint32_t(RPW), M.n - row0);
    // lane i < nrows holds rp[row0 + i]; every lane also reads the chunk end
    const uint32_t end = __ldg(&M.rp[row0 + nrows]);
    const uint32_t my_rp = (lane < int(nrows)) ? __ldg(&M.rp[row0 + lane]) : end;
    const uint32_t start = __shfl_sync(0xffffffffu, my_rp, 0);
    const int base = int(row0 & ~31u);

    if (end - start <= kCap) {
        const uint32_t g = start & ~uint32_t(W - 1);
        for (uint32_t j0 = g + uint32_t(lane) * W; j0 < end; j0 += 32u * W) {
            V v[W];
            VecLoad<V>::vals(M.val + j0, v);
            uint32_t c[W];
            if (M.off) {
                int o[W];
                VecLoad<V>::offs(M.off + j0, o);
#pragma unroll
                for (int k = 0; k < W; k++) c[k] = uint32_t(base + o[k]);
            } else {
                VecLoad<V>::cols(M.ci + j0, c);
            }
#pragma unroll
            for (int k = 0; k < W; k++) {
                uint32_t j = j0 + k;
                if (j >= start && j < end) prod[j - start] = A(v[k]) * A(gx(c[k]));
            }
        }
        __syncwarp();
        const int r = lane / L, sub = lane % L;
        const uint32_t rs = __shfl_sync(0xffffffffu, my_rp, r) - start;
        const uint32_t nx = __shfl_sync(0xffffffffu, my_rp, min(r + 1, 31));
        const uint32_t re = ((r + 1 < int(nrows)) ? nx : end) - start;
        A acc = A(0);
        if (r < int(nrows))
            for (uint32_t k = rs + sub; k < re; k += L) acc += prod[k];
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (sub == 0 && r < int(nrows)) epi(row0 + r, acc);
        __syncwarp();
    } else {
        for (uint32_t r = 0; r < nrows; r++) {
            A acc = warp_row<V, A>(M, row0 + r, gx, lane);
            if (lane == 0) epi(row0 + r, acc);
        }
    }
}

// Grid-stride driver over all row chunks.  Every thread of the block must call it.
template <typename V, typename A, int RPW, class GX, class EPI>
__device__ __forceinline__ void for_rows(const Csr<V> &M, GX &gx, EPI &epi, A *smem_prod)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    A *prod = smem_prod + size_t(warp) * kCap;
    const uint32_t n_chunks = (M.n + RPW - 1) / RPW;
    const uint32_t warps_total = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + warp; c < n_chunks; c += warps_total)
        warp_chunk<V, A, RPW>(M, c * RPW, gx, epi, prod, lane);
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
inline int pick_rpw(const rsg_csr *A)
{
    if (A->max_warp_nnz <= kCap) return 32;
    if (A->max_warp_nnz <= 2 * kCap) return 16;
    if (A->max_warp_nnz <= 4 * kCap) return 8;
    return 4;
}

template <typename A>
constexpr size_t prod_smem() { return size_t(kWarpsPerBlock) * kCap * sizeof(A); }

}  // namespace rsg
