// Inference path of the learned preconditioner on the 5th-generation tensor
// cores: one fused kernel per message-passing layer,
//     h_out = h + relu([h, G h] W_l + b_l),   G_ij = -a_ij s_i s_j (i != j),
// with h stored as BF16 (128 B per row).  A CTA owns a tile of 128 rows:
//   1. its 8 warps gather m = G h for the tile (8 lanes per row, 16-byte loads
//      of the neighbours' BF16 rows, FP32 accumulation) and write [h | m] into
//      shared memory in the canonical K-major layout (8x16-byte core matrices);
//   2. one thread issues 8 tcgen05.mma (M=128, N=64, K=16 each, BF16 in, FP32
//      accumulate) into a 64-column TMEM accumulator and commits to an mbarrier;
//   3. all warps read the accumulator back with tcgen05.ld and apply bias, ReLU
//      and the residual connection; the last layer also applies the output
//      layer and writes z = M(r) in FP64.
// W_l^T lives in shared memory as BF16 for the CTA's lifetime (persistent CTAs).
// Waits on the mbarrier are bounded: past kWaitLimit polls the kernel flags the
// context's error word, waits (bounded) for its MMAs, frees its TMEM and returns.
#include "gnn.cuh"
#include "spmv.cuh"

namespace rsg {
namespace {

constexpr int H = kGnnHidden;   // 64
constexpr int F = kGnnFeatures; // 8
constexpr int K2 = 2 * H;       // 128
constexpr int kTileRows = 128;
constexpr int kThreads = 256;
constexpr uint32_t kTmemCols = 64;
constexpr uint32_t kATileBytes = kTileRows * K2 * 2;  // 32 KB
constexpr uint32_t kBTileBytes = H * K2 * 2;          // 16 KB
constexpr uint32_t kLBO = 128;                        // K-adjacent core matrices
constexpr uint32_t kSBO = (K2 / 8) * 128;             // 8-row groups: 16 core matrices of 128 B
constexpr uint32_t kOffB = kATileBytes;
constexpr uint32_t kOffBias = kOffB + kBTileBytes;
constexpr uint32_t kOffWout = kOffBias + H * 4;
constexpr uint32_t kOffPart = kOffWout + H * 4;
constexpr uint32_t kOffBar = kOffPart + kTileRows * 4;
constexpr uint32_t kOffTmem = kOffBar + 16;
constexpr uint32_t kLayerSmem = kOffTmem + 16;

// Instruction descriptor of tcgen05.mma kind::f16: FP32 accumulator (bits 4-5 = 1),
// A and B BF16 (bits 7-9 and 10-12 = 1), both K-major, N>>3 at bits 17-22, M>>4 at 24-28.
constexpr uint32_t kIdesc =
    (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(H >> 3) << 17) | (uint32_t(kTileRows >> 4) << 24);

// byte offset of BF16 element (row, k) in a K-major tile without swizzle
__device__ __forceinline__ uint32_t tile_off(uint32_t row, uint32_t k)
{
    return (row >> 3) * kSBO + (k >> 3) * kLBO + (row & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: start address, LBO, SBO (all >> 4), version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
    return uint64_t((saddr & 0x3FFFFu) >> 4) | (uint64_t(kLBO >> 4) << 16) | (uint64_t(kSBO >> 4) << 32) |
           (uint64_t(1) << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
}

__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8])
{
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int t = 0; t < 4; t++) {
        f[2 * t] = __uint_as_float(w[t] << 16);
        f[2 * t + 1] = __uint_as_float(w[t] & 0xffff0000u);
    }
}

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// features and input layer, BF16 output: h0 = relu(f W_in + b_in)
__global__ void k_gnn_input_bf16(uint32_t n, const double *__restrict__ r, const float *__restrict__ s,
                                 const float *__restrict__ logd, const float *__restrict__ rsum,
                                 const float *__restrict__ mean_logd, const float *__restrict__ rms,
                                 const double *__restrict__ xyz, const float *__restrict__ P,
                                 __nv_bfloat16 *__restrict__ h0)
{
    __shared__ float w[F * H + H];
    for (int k = threadIdx.x; k < F * H + H; k += blockDim.x) w[k] = P[k];
    __syncthreads();
    const float inv = 1.0f / *rms, ml = *mean_logd;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float f[F];
        f[0] = float(r[i] * double(s[i])) * inv;
        f[1] = logd[i] - ml;
        f[2] = rsum[i];
        f[3] = xyz ? float(xyz[3 * size_t(i)]) : 0.f;
        f[4] = xyz ? float(xyz[3 * size_t(i) + 1]) : 0.f;
        f[5] = xyz ? float(xyz[3 * size_t(i) + 2]) : 0.f;
        f[6] = 1.f;
        f[7] = 0.f;
        uint4 *dst = reinterpret_cast<uint4 *>(h0 + size_t(i) * H);
#pragma unroll 1
        for (int c8 = 0; c8 < H / 8; c8++) {
            float o[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int c = c8 * 8 + t;
                float z = w[F * H + c];
#pragma unroll
                for (int k = 0; k < F; k++) z = fmaf(f[k], w[k * H + c], z);
                o[t] = fmaxf(z, 0.f);
            }
            dst[c8] = make_uint4(pack2(o[0], o[1]), pack2(o[2], o[3]), pack2(o[4], o[5]), pack2(o[6], o[7]));
        }
    }
}

template <bool LAST>
__global__ void __launch_bounds__(kThreads) k_gnn_layer_umma(
    uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci, const float *__restrict__ ew,
    const float *__restrict__ s, const __nv_bfloat16 *__restrict__ h, const float *__restrict__ W,
    const float *__restrict__ bias, const float *__restrict__ pout, const float *__restrict__ rms,
    __nv_bfloat16 *__restrict__ h_out, double *__restrict__ z, unsigned int *err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *At = sm;
    unsigned char *Bt = sm + kOffB;
    float *bs = reinterpret_cast<float *>(sm + kOffBias);
    float *wo = reinterpret_cast<float *>(sm + kOffWout);
    float *part = reinterpret_cast<float *>(sm + kOffPart);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kOffBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kOffTmem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // B = W^T (N = 64 output columns x K = 128), BF16, K-major
    for (int e = tid; e < K2 * H; e += kThreads) {
        const int k = e / H, c = e % H;
        *reinterpret_cast<__nv_bfloat16 *>(Bt + tile_off(c, k)) = __float2bfloat16_rn(W[e]);
    }
    if (tid < H) {
        bs[tid] = bias[tid];
        wo[tid] = LAST ? pout[tid] : 0.f;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const float b_out = LAST ? pout[H] : 0.f;
    const float sc = LAST ? *rms : 0.f;
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const int q = lane >> 3, kc = lane & 7;  // gather: 4 rows per warp pass, 8 lanes x 16 B per row
    const int quarter = warp & 3, half = warp >> 2;
    uint32_t phase = 0;
    bool in_flight = false, failed = false;

    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t r0 = tile * kTileRows;
        // 1. gather m = G h and stage [h | m] (BF16) in the A tile.  The 8 lanes of a row
        //    fetch 8 of its (column, weight) pairs at once and then 8 neighbour rows
        //    back to back, so each lane keeps 8 independent 16-byte loads in flight.
#pragma unroll 1
        for (int pass = 0; pass < 4; pass++) {
            const uint32_t trow = uint32_t(warp * 16 + pass * 4 + q);
            const uint32_t row = r0 + trow;
            float acc[8];
#pragma unroll
            for (int t = 0; t < 8; t++) acc[t] = 0.f;
            uint4 hown = make_uint4(0u, 0u, 0u, 0u);
            uint32_t jb = 0, je = 0;
            if (row < n) {
                hown = *reinterpret_cast<const uint4 *>(h + size_t(row) * H + kc * 8);
                jb = rp[row];
                je = rp[row + 1];
            }
            const uint32_t trips = __reduce_max_sync(0xffffffffu, (je - jb + 7) / 8);
            const uint32_t rown = row < n ? row : 0u;
            for (uint32_t it = 0; it < trips; it++) {
                const uint32_t jj = jb + it * 8 + uint32_t(kc);
                uint32_t c_mine = rown;
                float w_mine = 0.f;
                if (jj < je) {  // the diagonal's weight is 0
                    c_mine = ci[jj];
                    w_mine = ew[jj];
                }
                uint4 hv[8];
                float wt[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const uint32_t ct = __shfl_sync(0xffffffffu, c_mine, (lane & ~7) + t);
                    wt[t] = __shfl_sync(0xffffffffu, w_mine, (lane & ~7) + t);
                    hv[t] = *reinterpret_cast<const uint4 *>(h + size_t(ct) * H + kc * 8);
                }
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    float f[8];
                    unpack8(hv[t], f);
#pragma unroll
                    for (int u = 0; u < 8; u++) acc[u] = fmaf(wt[t], f[u], acc[u]);
                }
            }
            *reinterpret_cast<uint4 *>(At + tile_off(trow, kc * 8)) = hown;
            *reinterpret_cast<uint4 *>(At + tile_off(trow, H + kc * 8)) =
                make_uint4(pack2(acc[0], acc[1]), pack2(acc[2], acc[3]), pack2(acc[4], acc[5]),
                           pack2(acc[6], acc[7]));
        }
        fence_async_shared();  // generic-proxy smem writes -> visible to the tensor core
        __syncthreads();
        // 2. one thread issues the MMAs: D[128 x 64] = A[128 x 128] B^T
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(At), b0 = smem_u32(Bt);
#pragma unroll
            for (int ks = 0; ks < K2 / 16; ks++)
                umma_bf16(tmem, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO), ks > 0 ? 1u : 0u);
            umma_commit(bar);
        }
        in_flight = true;
        const bool ok = mbar_wait(bar, phase, err);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        in_flight = false;
        phase ^= 1u;
        tc_fence_after();
        // 3. epilogue: warp (quarter, half) reads TMEM lanes 32*quarter.., columns 32*half..
        const uint32_t trow = uint32_t(quarter * 32 + lane), row = r0 + trow;
        uint32_t v[32];
        tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(half * 32), v);
        float o[32];
        float dot = 0.f;
#pragma unroll
        for (int c8 = 0; c8 < 4; c8++) {
            const int cb = half * 32 + c8 * 8;
            float hp[8];
            unpack8(*reinterpret_cast<const uint4 *>(At + tile_off(trow, cb)), hp);
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int c = cb + t;
                const float val_o = hp[t] + fmaxf(__uint_as_float(v[c8 * 8 + t]) + bs[c], 0.f);
                o[c8 * 8 + t] = val_o;
                dot = fmaf(val_o, wo[c], dot);
            }
        }
        if constexpr (!LAST) {
            if (row < n) {
                uint4 *dst = reinterpret_cast<uint4 *>(h_out + size_t(row) * H + half * 32);
#pragma unroll
                for (int c8 = 0; c8 < 4; c8++)
                    dst[c8] = make_uint4(pack2(o[c8 * 8], o[c8 * 8 + 1]), pack2(o[c8 * 8 + 2], o[c8 * 8 + 3]),
                                         pack2(o[c8 * 8 + 4], o[c8 * 8 + 5]), pack2(o[c8 * 8 + 6], o[c8 * 8 + 7]));
            }
        } else {
            if (half == 1) part[trow] = dot;
            __syncthreads();
            if (half == 0 && row < n) z[row] = double(dot + part[trow] + b_out) * double(sc) * double(s[row]);
        }
        tc_fence_before();
        __syncthreads();  // A tile, TMEM and part[] free for the next tile
    }
    if (failed && in_flight && tid == 0) mbar_wait(bar, phase, nullptr);  // let the MMAs drain (bounded)
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

__host__ __device__ inline size_t off_layer(int l) { return size_t(F) * H + H + size_t(l) * (size_t(K2) * H + H); }

}  // namespace

bool gnn_umma_setup(rsg_context *ctx, int *grid)
{
    static bool attr = false;
    if (!attr) {
        for (const void *f : {(const void *)k_gnn_layer_umma<false>, (const void *)k_gnn_layer_umma<true>}) {
            if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kLayerSmem)) != cudaSuccess ||
                cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
                return false;
        }
        attr = true;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gnn_layer_umma<false>, kThreads, kLayerSmem) !=
            cudaSuccess ||
        per_sm < 1)
        return false;
    // Four CTAs fit an SM by shared memory and registers; CTAs beyond the resident
    // ones wait for a slot, so a larger grid never over-commits the 512 TMEM columns
    // (each resident CTA holds kTmemCols of them).
    per_sm = std::min(std::max(per_sm, 4), int(512 / kTmemCols));
    *grid = per_sm * ctx->num_sms;
    return true;
}

// z = M(r) through the BF16 tensor-core layers; h buffers hb[0], hb[1] (n x 64 BF16 each).
rsg_status gnn_forward_umma(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, double *z,
                            const double *xyz, const float *rms)
{
    const uint32_t n = A->n;
    cudaStream_t sm = ctx->stream;
    int gl = 0;
    if (!gnn_umma_setup(ctx, &gl)) return set_error(ctx, RSG_ERR_CUDA, "learned: tensor-core layer set-up");
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    gl = int(std::min<uint32_t>(uint32_t(gl), std::max<uint32_t>(tiles, 1)));
    const int gi = std::min(grid_for(ctx, (const void *)k_gnn_input_bf16, kBlock, 0, n), kMaxGrid);
    k_gnn_input_bf16<<<gi, kBlock, 0, sm>>>(n, r, G->s, G->logd, G->rsum, G->scal32, rms, xyz, G->params, G->hb[0]);
    for (int l = 0; l < G->L; l++) {
        const float *W = G->params + off_layer(l), *b = W + size_t(K2) * H;
        const float *pout = G->params + off_layer(G->L);
        const __nv_bfloat16 *hin = G->hb[l & 1];
        __nv_bfloat16 *hout = G->hb[(l + 1) & 1];
        if (l + 1 < G->L)
            k_gnn_layer_umma<false><<<gl, kThreads, kLayerSmem, sm>>>(n, A->rp, A->ci, G->ew, G->s, hin, W, b, pout,
                                                                     rms, hout, z, ctx->errw);
        else
            k_gnn_layer_umma<true><<<gl, kThreads, kLayerSmem, sm>>>(n, A->rp, A->ci, G->ew, G->s, hin, W, b, pout,
                                                                    rms, hout, z, ctx->errw);
    }
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

// ---------------------------------------------------------------------------------------------
// Training on the 5th-generation tensor cores (BF16 operands, FP32 accumulation in TMEM).
//   forward:  h_out = h + relu([h, m] W + b)                 (M=128 rows, N=64, K=128)
//   backward: z = [h_prev, m] W (recomputed), dz = g [z + b > 0],
//             [g_prev - g | g_m] = dz W^T                    (M=128 rows, N=128, K=64)
//   weights:  dW = [h_prev, m]^T dz over a contiguous row range per CTA, accumulated in TMEM across
//             its 128-row tiles                               (M=128 features, N=64, K=128 rows)
// The activations stay FP32 in global memory; each tile is rounded to BF16 when it is staged.
namespace {

constexpr uint32_t kSBO64 = (H / 8) * 128;  // K = 64 tiles: 8 core matrices per 8-row group
constexpr uint32_t kTile64Bytes = kTileRows * H * 2;  // 16 KB

__device__ __forceinline__ uint32_t tile_off_s(uint32_t row, uint32_t k, uint32_t sbo)
{
    return (row >> 3) * sbo + (k >> 3) * kLBO + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t smem_desc_s(uint32_t saddr, uint32_t sbo)
{
    return uint64_t((saddr & 0x3FFFFu) >> 4) | (uint64_t(kLBO >> 4) << 16) | (uint64_t(sbo >> 4) << 32) |
           (uint64_t(1) << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N and M as given
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16_id(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                             uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t tmem, uint32_t cols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols) : "memory");
}

// Stages rows r0 .. r0+127 of X = [a | b] (two n x 64 FP32 arrays) as a BF16 K-major A tile
// (M = 128 rows, K = 128); rows past n are zero.
__device__ __forceinline__ void stage_rows_ab(unsigned char *At, uint32_t r0, uint32_t n, const float *a,
                                              const float *b)
{
    for (uint32_t e = threadIdx.x; e < kTileRows * (K2 / 8); e += blockDim.x) {
        const uint32_t trow = e / (K2 / 8), k8 = e % (K2 / 8), row = r0 + trow;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (row < n) {
            const float *src = k8 < H / 8 ? a + size_t(row) * H + k8 * 8 : b + size_t(row) * H + (k8 - H / 8) * 8;
            const float4 x0 = *reinterpret_cast<const float4 *>(src);
            const float4 x1 = *reinterpret_cast<const float4 *>(src + 4);
            v = make_uint4(pack2(x0.x, x0.y), pack2(x0.z, x0.w), pack2(x1.x, x1.y), pack2(x1.z, x1.w));
        }
        *reinterpret_cast<uint4 *>(At + tile_off(trow, k8 * 8)) = v;
    }
}

// B = W^T (N = 64 output columns x K = 128), BF16, K-major (W: K2 x H row-major)
__device__ __forceinline__ void stage_wt(unsigned char *Bt, const float *W)
{
    for (int e = threadIdx.x; e < K2 * H; e += blockDim.x) {
        const int k = e / H, c = e % H;
        *reinterpret_cast<__nv_bfloat16 *>(Bt + tile_off(c, k)) = __float2bfloat16_rn(W[e]);
    }
}

// forward: h_out = h + relu([h, m] W + b) for 128-row tiles (FP32 in and out)
constexpr uint32_t kFwdOffB = kATileBytes;
constexpr uint32_t kFwdOffBias = kFwdOffB + kBTileBytes;
constexpr uint32_t kFwdOffBar = kFwdOffBias + H * 4;
constexpr uint32_t kFwdOffTmem = kFwdOffBar + 16;
constexpr uint32_t kFwdSmem = kFwdOffTmem + 16;

__global__ void __launch_bounds__(kThreads) k_gnn_dense_umma(uint32_t n, const float *__restrict__ h,
                                                              const float *__restrict__ m,
                                                              const float *__restrict__ W,
                                                              const float *__restrict__ bias,
                                                              float *__restrict__ h_out, unsigned int *err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *At = sm, *Bt = sm + kFwdOffB;
    float *bs = reinterpret_cast<float *>(sm + kFwdOffBias);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kFwdOffBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kFwdOffTmem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    stage_wt(Bt, W);
    if (tid < H) bs[tid] = bias[tid];
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tslot, kTmemCols);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const int quarter = warp & 3, half = warp >> 2;
    uint32_t phase = 0;
    bool in_flight = false, failed = false;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t r0 = tile * kTileRows;
        stage_rows_ab(At, r0, n, h, m);
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(At), b0 = smem_u32(Bt);
#pragma unroll
            for (int ks = 0; ks < K2 / 16; ks++)
                umma_bf16(tmem, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO), ks > 0 ? 1u : 0u);
            umma_commit(bar);
        }
        in_flight = true;
        const bool ok = mbar_wait(bar, phase, err);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        in_flight = false;
        phase ^= 1u;
        tc_fence_after();
        const uint32_t row = r0 + uint32_t(quarter * 32 + lane);
        uint32_t v[32];
        tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(half * 32), v);
        if (row < n) {
#pragma unroll
            for (int c4 = 0; c4 < 8; c4++) {
                const int c = half * 32 + c4 * 4;
                const float4 hv = *reinterpret_cast<const float4 *>(h + size_t(row) * H + c);
                float4 o;
                o.x = hv.x + fmaxf(__uint_as_float(v[c4 * 4]) + bs[c], 0.f);
                o.y = hv.y + fmaxf(__uint_as_float(v[c4 * 4 + 1]) + bs[c + 1], 0.f);
                o.z = hv.z + fmaxf(__uint_as_float(v[c4 * 4 + 2]) + bs[c + 2], 0.f);
                o.w = hv.w + fmaxf(__uint_as_float(v[c4 * 4 + 3]) + bs[c + 3], 0.f);
                *reinterpret_cast<float4 *>(h_out + size_t(row) * H + c) = o;
            }
        }
        tc_fence_before();
        __syncthreads();  // the A tile and TMEM are free for the next tile
    }
    if (failed && in_flight && tid == 0) mbar_wait(bar, phase, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, kTmemCols);
    }
}

// backward (data): per 128-row tile, D1 = [h_prev, m] W^T-tile product (z without bias, TMEM
// columns 0..63); dz = g [z + b > 0] (FP32 to dz_out, BF16 into A2); D2 = dz W^T (TMEM columns
// 64..191): g_prev = g + D2[:, :64], gm = D2[:, 64:].
constexpr uint32_t kBwdTmemCols = 256;
constexpr uint32_t kBwOffB1 = kATileBytes;                  // W^T: N = 64 x K = 128
constexpr uint32_t kBwOffA2 = kBwOffB1 + kBTileBytes;       // dz: M = 128 x K = 64
constexpr uint32_t kBwOffB2 = kBwOffA2 + kTile64Bytes;      // W: N = 128 x K = 64
constexpr uint32_t kBwOffBias = kBwOffB2 + K2 * H * 2;
constexpr uint32_t kBwOffBar = kBwOffBias + H * 4;
constexpr uint32_t kBwOffTmem = kBwOffBar + 16;
constexpr uint32_t kBwdUmmaSmem = kBwOffTmem + 16;

__global__ void __launch_bounds__(kThreads) k_gnn_bwd_umma(uint32_t n, const float *__restrict__ hp,
                                                            const float *__restrict__ m, const float *__restrict__ W,
                                                            const float *__restrict__ bias,
                                                            const float *__restrict__ g, float *__restrict__ dz_out,
                                                            float *__restrict__ gprev, float *__restrict__ gm,
                                                            unsigned int *err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *A1 = sm, *B1 = sm + kBwOffB1, *A2 = sm + kBwOffA2, *B2 = sm + kBwOffB2;
    float *bs = reinterpret_cast<float *>(sm + kBwOffBias);
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kBwOffBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kBwOffTmem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    stage_wt(B1, W);
    for (int e = tid; e < K2 * H; e += kThreads) {  // B2 = W (N = K2 input features x K = H outputs)
        const int kin = e / H, c = e % H;
        *reinterpret_cast<__nv_bfloat16 *>(B2 + tile_off_s(kin, c, kSBO64)) = __float2bfloat16_rn(W[e]);
    }
    if (tid < H) bs[tid] = bias[tid];
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tslot, kBwdTmemCols);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot, tmem2 = tmem + H;
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const int quarter = warp & 3, half = warp >> 2;
    constexpr uint32_t kId2 = idesc_bf16(kTileRows, K2);
    uint32_t phase = 0;
    bool in_flight = false, failed = false;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t r0 = tile * kTileRows;
        const uint32_t trow = uint32_t(quarter * 32 + lane), row = r0 + trow;
        stage_rows_ab(A1, r0, n, hp, m);
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(A1), b0 = smem_u32(B1);
#pragma unroll
            for (int ks = 0; ks < K2 / 16; ks++)
                umma_bf16(tmem, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO), ks > 0 ? 1u : 0u);
            umma_commit(bar);
        }
        in_flight = true;
        bool ok = mbar_wait(bar, phase, err);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        in_flight = false;
        phase ^= 1u;
        tc_fence_after();
        {  // dz = g [z + b > 0]
            uint32_t v[32];
            tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(half * 32), v);
#pragma unroll
            for (int c8 = 0; c8 < 4; c8++) {
                const int cb = half * 32 + c8 * 8;
                float d[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    const int c = cb + t;
                    d[t] = (row < n && __uint_as_float(v[c8 * 8 + t]) + bs[c] > 0.f) ? g[size_t(row) * H + c] : 0.f;
                }
                if (row < n) {
                    float4 *dst = reinterpret_cast<float4 *>(dz_out + size_t(row) * H + cb);
                    dst[0] = make_float4(d[0], d[1], d[2], d[3]);
                    dst[1] = make_float4(d[4], d[5], d[6], d[7]);
                }
                *reinterpret_cast<uint4 *>(A2 + tile_off_s(trow, uint32_t(cb), kSBO64)) =
                    make_uint4(pack2(d[0], d[1]), pack2(d[2], d[3]), pack2(d[4], d[5]), pack2(d[6], d[7]));
            }
        }
        fence_async_shared();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(A2), b0 = smem_u32(B2);
#pragma unroll
            for (int ks = 0; ks < H / 16; ks++)
                umma_bf16_id(tmem2, smem_desc_s(a0 + ks * 2 * kLBO, kSBO64), smem_desc_s(b0 + ks * 2 * kLBO, kSBO64),
                             kId2, ks > 0 ? 1u : 0u);
            umma_commit(bar);
        }
        in_flight = true;
        ok = mbar_wait(bar, phase, err);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        in_flight = false;
        phase ^= 1u;
        tc_fence_after();
#pragma unroll
        for (int part = 0; part < 2; part++) {  // warp half covers D2 columns 64 half .. +64
            const int cb = half * 64 + part * 32;
            uint32_t v[32];
            tmem_ld32(tmem2 + (uint32_t(quarter * 32) << 16) + uint32_t(cb), v);
            if (row < n) {
#pragma unroll
                for (int c4 = 0; c4 < 8; c4++) {
                    const int c = cb + c4 * 4;
                    float4 o = make_float4(__uint_as_float(v[c4 * 4]), __uint_as_float(v[c4 * 4 + 1]),
                                           __uint_as_float(v[c4 * 4 + 2]), __uint_as_float(v[c4 * 4 + 3]));
                    if (c < H) {
                        const float4 gv = *reinterpret_cast<const float4 *>(g + size_t(row) * H + c);
                        o.x += gv.x;
                        o.y += gv.y;
                        o.z += gv.z;
                        o.w += gv.w;
                        *reinterpret_cast<float4 *>(gprev + size_t(row) * H + c) = o;
                    } else {
                        *reinterpret_cast<float4 *>(gm + size_t(row) * H + (c - H)) = o;
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();  // A1, A2 and TMEM free for the next tile
    }
    if (failed && in_flight && tid == 0) mbar_wait(bar, phase, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, kBwdTmemCols);
    }
}

// weight gradient: dW = X^T dz (X = [h_prev, m]) and db = column sums of dz over a contiguous row
// range per CTA, its 128-row tiles accumulated in one TMEM accumulator (M = 128 features,
// N = 64 columns, K = 128 rows per tile); db in FP32 on CUDA cores, rows in order.  Output: one
// block of K2*H + H partial sums per CTA (summed in CTA order by k_gnn_sum_blocks).
constexpr uint32_t kWgOffB = kATileBytes;  // dz^T: N = 64 x K = 128 rows
constexpr uint32_t kWgOffBar = kWgOffB + kBTileBytes;
constexpr uint32_t kWgOffTmem = kWgOffBar + 16;
constexpr uint32_t kWgUmmaSmem = kWgOffTmem + 16;

__global__ void __launch_bounds__(kThreads) k_gnn_wgrad_umma(uint32_t n, const float *__restrict__ hp,
                                                              const float *__restrict__ m, const float *__restrict__ dz,
                                                              float *__restrict__ blk, unsigned int *err)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *At = sm, *Bt = sm + kWgOffB;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + kWgOffBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + kWgOffTmem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t rows_per = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(n, blockIdx.x * rows_per), r1 = min(n, r0 + rows_per);
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tslot, kTmemCols);
    fence_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    float db = 0.f;  // threads 0..63: column tid of db
    uint32_t phase = 0;
    bool in_flight = false, failed = false, any = false;
    for (uint32_t t0 = r0; t0 < r1; t0 += kTileRows) {
        const uint32_t cnt = min(uint32_t(kTileRows), r1 - t0);
        // A = X^T (row = feature k2, k = tile row), B = dz^T (row = column c, k = tile row)
        for (uint32_t e = tid; e < kTileRows * (K2 / 8); e += kThreads) {
            const uint32_t rr = e / (K2 / 8), k8 = e % (K2 / 8);
            float x[8];
            if (rr < cnt) {
                const float *src = k8 < H / 8 ? hp + size_t(t0 + rr) * H + k8 * 8 : m + size_t(t0 + rr) * H + (k8 - H / 8) * 8;
                const float4 x0 = *reinterpret_cast<const float4 *>(src), x1 = *reinterpret_cast<const float4 *>(src + 4);
                x[0] = x0.x; x[1] = x0.y; x[2] = x0.z; x[3] = x0.w; x[4] = x1.x; x[5] = x1.y; x[6] = x1.z; x[7] = x1.w;
            } else {
#pragma unroll
                for (int t = 0; t < 8; t++) x[t] = 0.f;
            }
#pragma unroll
            for (int t = 0; t < 8; t++)
                *reinterpret_cast<__nv_bfloat16 *>(At + tile_off(k8 * 8 + t, rr)) = __float2bfloat16_rn(x[t]);
        }
        for (uint32_t e = tid; e < kTileRows * (H / 8); e += kThreads) {
            const uint32_t rr = e / (H / 8), c8 = e % (H / 8);
            float d[8];
            if (rr < cnt) {
                const float4 d0 = *reinterpret_cast<const float4 *>(dz + size_t(t0 + rr) * H + c8 * 8);
                const float4 d1 = *reinterpret_cast<const float4 *>(dz + size_t(t0 + rr) * H + c8 * 8 + 4);
                d[0] = d0.x; d[1] = d0.y; d[2] = d0.z; d[3] = d0.w; d[4] = d1.x; d[5] = d1.y; d[6] = d1.z; d[7] = d1.w;
            } else {
#pragma unroll
                for (int t = 0; t < 8; t++) d[t] = 0.f;
            }
#pragma unroll
            for (int t = 0; t < 8; t++)
                *reinterpret_cast<__nv_bfloat16 *>(Bt + tile_off(c8 * 8 + t, rr)) = __float2bfloat16_rn(d[t]);
        }
        if (tid < H)
            for (uint32_t rr = 0; rr < cnt; rr++) db += dz[size_t(t0 + rr) * H + tid];
        fence_async_shared();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(At), b0 = smem_u32(Bt);
#pragma unroll
            for (int ks = 0; ks < kTileRows / 16; ks++)
                umma_bf16(tmem, smem_desc(a0 + ks * 2 * kLBO), smem_desc(b0 + ks * 2 * kLBO),
                          (any || ks > 0) ? 1u : 0u);
            umma_commit(bar);
        }
        any = true;
        in_flight = true;
        const bool ok = mbar_wait(bar, phase, err);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        in_flight = false;
        phase ^= 1u;
        tc_fence_before();
        __syncthreads();  // the tiles are free for the next rows
    }
    float *out = blk + size_t(blockIdx.x) * (K2 * H + H);
    if (!failed) {
        tc_fence_after();
        const int quarter = warp & 3, half = warp >> 2;
        const uint32_t k2 = uint32_t(quarter * 32 + lane);
        uint32_t v[32];
        if (any) tmem_ld32(tmem + (uint32_t(quarter * 32) << 16) + uint32_t(half * 32), v);
#pragma unroll
        for (int j = 0; j < 32; j++) out[size_t(k2) * H + half * 32 + j] = any ? __uint_as_float(v[j]) : 0.f;
        if (tid < H) out[K2 * H + tid] = db;
    }
    if (failed && in_flight && tid == 0) mbar_wait(bar, phase, nullptr);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_free(tmem, kTmemCols);
    }
}

}  // namespace

// Host wrappers of the training kernels (grids: persistent over tiles for the forward and the
// data backward, gnn grad blocks for the weight gradient).
static bool train_umma_attr(rsg_context *ctx)
{
    static bool done = false;
    if (done) return true;
    const std::pair<const void *, uint32_t> ks[] = {{(const void *)k_gnn_dense_umma, kFwdSmem},
                                                    {(const void *)k_gnn_bwd_umma, kBwdUmmaSmem},
                                                    {(const void *)k_gnn_wgrad_umma, kWgUmmaSmem}};
    for (const auto &k : ks)
        if (cudaFuncSetAttribute(k.first, cudaFuncAttributeMaxDynamicSharedMemorySize, int(k.second)) != cudaSuccess)
            return false;
    done = true;
    return true;
}

rsg_status gnn_train_dense_umma(rsg_context *ctx, uint32_t n, const float *h, const float *m, const float *W,
                                const float *b, float *hout)
{
    if (!train_umma_attr(ctx)) return set_error(ctx, RSG_ERR_CUDA, "learned: tensor-core training set-up");
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const int g = int(std::max<uint32_t>(1, std::min<uint32_t>(tiles, uint32_t(ctx->num_sms) * 4)));
    k_gnn_dense_umma<<<g, kThreads, kFwdSmem, ctx->stream>>>(n, h, m, W, b, hout, ctx->errw);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status gnn_train_bwd_umma(rsg_context *ctx, uint32_t n, const float *hp, const float *m, const float *W,
                              const float *b, const float *g, float *dz, float *gprev, float *gm)
{
    if (!train_umma_attr(ctx)) return set_error(ctx, RSG_ERR_CUDA, "learned: tensor-core training set-up");
    const uint32_t tiles = (n + kTileRows - 1) / kTileRows;
    const int gr = int(std::max<uint32_t>(1, std::min<uint32_t>(tiles, uint32_t(ctx->num_sms) * 2)));
    k_gnn_bwd_umma<<<gr, kThreads, kBwdUmmaSmem, ctx->stream>>>(n, hp, m, W, b, g, dz, gprev, gm, ctx->errw);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status gnn_train_wgrad_umma(rsg_context *ctx, uint32_t n, const float *hp, const float *m, const float *dz,
                                float *blk, int nblk)
{
    if (!train_umma_attr(ctx)) return set_error(ctx, RSG_ERR_CUDA, "learned: tensor-core training set-up");
    k_gnn_wgrad_umma<<<nblk, kThreads, kWgUmmaSmem, ctx->stream>>>(n, hp, m, dz, blk, ctx->errw);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

}  // namespace rsg
