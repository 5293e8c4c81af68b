// Learned preconditioner: a message-passing network over the matrix graph.
//
// No counterpart in the reference (its preconditioners are Jacobi and block
// Jacobi, src/rmatrixpreconditioner.cpp).  M(r) approximates A^{-1} r:
//   node features f_i = [u_i, log(a_ii) - mean log a, sum_j a_ij / a_ii, x_i, y_i, z_i, 1, 0]
//     with u = D^{-1/2} r / rms(D^{-1/2} r)
//   edge weights   w_ij = -a_ij / sqrt(a_ii a_jj)  (j != i; the normalised off-diagonals)
//   h0 = relu(f W_in + b_in)                                  (8 -> H)
//   layer l: m = W h, h <- h + relu([h, m] W_l + b_l)         (2H -> H, tensor cores)
//   y = h w_out + b_out;  M(r)_i = y_i rms(D^{-1/2} r) / sqrt(a_ii)
// so M is positively homogeneous (M(c r) = c M(r)).  Training minimises
// ||r - A M(r)||^2 / ||r||^2 over residuals r of plain solver trajectories,
// with hand-written backward kernels and Adam.  The dense layers run on the
// tensor cores (mma.sync m16n8k16, BF16 inputs, FP32 accumulation); an FP32
// CUDA-core path computes the same layer exactly for gradient checks.
#include "gnn.cuh"

#include <cmath>
#include <cstring>
#include <random>
#include <vector>

namespace rsg {
namespace {

constexpr int H = kGnnHidden;      // 64
constexpr int F = kGnnFeatures;    // 8
constexpr int K2 = 2 * H;          // 128

// parameter offsets in the flat FP32 vector
__host__ __device__ inline size_t off_win() { return 0; }
__host__ __device__ inline size_t off_bin() { return size_t(F) * H; }
__host__ __device__ inline size_t off_layer(int l) { return size_t(F) * H + H + size_t(l) * (size_t(K2) * H + H); }
__host__ __device__ inline size_t off_wout(int L) { return off_layer(L); }
__host__ __device__ inline size_t off_bout(int L) { return off_layer(L) + H; }

// ---------------- per-matrix features ----------------

__global__ void k_gnn_prep(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                           const double *__restrict__ val, float *__restrict__ s, float *__restrict__ logd,
                           float *__restrict__ rsum, double *partials, unsigned int *ticket, float *mean_logd)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0, sum = 0.0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            sum += val[j];
            if (ci[j] == i) d = val[j];
        }
        const double dd = d > 0.0 ? d : 1.0;
        s[i] = float(1.0 / sqrt(dd));
        logd[i] = float(log(dd));
        rsum[i] = float(sum / dd);
        acc[0] += log(dd);
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) *mean_logd = float(tot[0] / double(n));
}

// normalised edge weights of the message passing, one per stored nonzero
__global__ void k_gnn_edges(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                            const double *__restrict__ val, const float *__restrict__ s, float *__restrict__ ew)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float si = s[i];
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            const uint32_t c = ci[j];
            ew[j] = c == i ? 0.f : -float(val[j]) * si * s[c];
        }
    }
}

// ||D^{-1/2} r||^2 -> rms
__global__ void k_gnn_rms(uint32_t n, const double *__restrict__ r, const float *__restrict__ s, double *partials,
                          unsigned int *ticket, float *rms)
{
    __shared__ double sh[32];
    double acc[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double u = r[i] * double(s[i]);
        acc[0] += u * u;
    }
    double tot[1];
    if (grid_sum<1>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        const double v = sqrt(tot[0] / double(n));
        *rms = float(v > 0.0 ? v : 1.0);
    }
}

// features and input layer: pre0 = f W_in + b_in, h0 = relu(pre0)
__global__ void k_gnn_input(uint32_t n, const double *__restrict__ r, const float *__restrict__ s,
                            const float *__restrict__ logd, const float *__restrict__ rsum,
                            const float *__restrict__ mean_logd, const float *__restrict__ rms,
                            const double *__restrict__ xyz, const float *__restrict__ P, float *__restrict__ feat,
                            float *__restrict__ pre0, float *__restrict__ h0)
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
        if (feat)
            for (int k = 0; k < F; k++) feat[size_t(i) * F + k] = f[k];
        for (int c = 0; c < H; c++) {
            float z = w[F * H + c];
            for (int k = 0; k < F; k++) z = fmaf(f[k], w[k * H + c], z);
            if (pre0) pre0[size_t(i) * H + c] = z;
            h0[size_t(i) * H + c] = fmaxf(z, 0.f);
        }
    }
}

// m = W h with W_ij = -a_ij s_i s_j (j != i), from the per-nonzero edge weights
// (0 on the diagonal): warp per row, 2 features per lane.
__global__ void k_gnn_spmm(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                           const float *__restrict__ ew, const float *__restrict__ h, float *__restrict__ m)
{
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        float2 acc = make_float2(0.f, 0.f);
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            const float wgt = ew[j];
            const float2 hv = reinterpret_cast<const float2 *>(h + size_t(ci[j]) * H)[lane];
            acc.x = fmaf(wgt, hv.x, acc.x);
            acc.y = fmaf(wgt, hv.y, acc.y);
        }
        reinterpret_cast<float2 *>(m + size_t(i) * H)[lane] = acc;
    }
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Dense layer on tensor cores: z = [h, m] W + b, h_out = h + relu(z).
// Block = 4 warps, 16 rows per warp; W^T held in shared memory as BF16.
constexpr int kTcWarps = 4;
constexpr int kXs = K2 + 8;  // padded row stride (bf16 elements) of the X and W^T tiles
__global__ void __launch_bounds__(32 * kTcWarps) k_gnn_dense_tc(uint32_t n, const float *__restrict__ h,
                                                                const float *__restrict__ m,
                                                                const float *__restrict__ W,
                                                                const float *__restrict__ bias,
                                                                float *__restrict__ h_out)
{
    __shared__ __align__(16) __nv_bfloat16 wt[H * kXs];            // W^T: [n][k]
    __shared__ __align__(16) __nv_bfloat16 xs[kTcWarps][16 * kXs];  // X tile per warp: [row][k]
    __shared__ float bs[H];
    for (int e = threadIdx.x; e < K2 * H; e += blockDim.x) {
        const int k = e / H, c = e % H;
        wt[c * kXs + k] = __float2bfloat16_rn(W[e]);
    }
    for (int c = threadIdx.x; c < H; c += blockDim.x) bs[c] = bias[c];
    __syncthreads();
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    __nv_bfloat16 *x = xs[wi];
    const uint32_t tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * kTcWarps + wi; tile < tiles; tile += gridDim.x * kTcWarps) {
        const uint32_t r0 = tile * 16;
        // stage X = [h | m] for 16 rows (zero past n)
        for (int e = lane; e < 16 * H; e += 32) {
            const int rr = e / H, c = e % H;
            const uint32_t row = r0 + rr;
            const bool ok = row < n;
            x[rr * kXs + c] = __float2bfloat16_rn(ok ? h[size_t(row) * H + c] : 0.f);
            x[rr * kXs + H + c] = __float2bfloat16_rn(ok ? m[size_t(row) * H + c] : 0.f);
        }
        __syncwarp();
        float acc[H / 8][4];
#pragma unroll
        for (int nt = 0; nt < H / 8; nt++)
#pragma unroll
            for (int q = 0; q < 4; q++) acc[nt][q] = 0.f;
#pragma unroll
        for (int ks = 0; ks < K2 / 16; ks++) {
            const int k0 = ks * 16 + t * 2;
            uint32_t a[4];
            a[0] = *reinterpret_cast<const uint32_t *>(&x[g * kXs + k0]);
            a[1] = *reinterpret_cast<const uint32_t *>(&x[(g + 8) * kXs + k0]);
            a[2] = *reinterpret_cast<const uint32_t *>(&x[g * kXs + k0 + 8]);
            a[3] = *reinterpret_cast<const uint32_t *>(&x[(g + 8) * kXs + k0 + 8]);
#pragma unroll
            for (int nt = 0; nt < H / 8; nt++) {
                uint32_t b[2];
                b[0] = *reinterpret_cast<const uint32_t *>(&wt[(nt * 8 + g) * kXs + k0]);
                b[1] = *reinterpret_cast<const uint32_t *>(&wt[(nt * 8 + g) * kXs + k0 + 8]);
                mma_bf16(acc[nt], a, b);
            }
        }
#pragma unroll
        for (int nt = 0; nt < H / 8; nt++) {
            const int c = nt * 8 + t * 2;
#pragma unroll
            for (int half = 0; half < 2; half++) {
                const uint32_t row = r0 + g + half * 8;
                if (row >= n) continue;
                const float z0 = acc[nt][half * 2] + bs[c], z1 = acc[nt][half * 2 + 1] + bs[c + 1];
                const float2 hv = *reinterpret_cast<const float2 *>(&h[size_t(row) * H + c]);
                *reinterpret_cast<float2 *>(&h_out[size_t(row) * H + c]) =
                    make_float2(hv.x + fmaxf(z0, 0.f), hv.y + fmaxf(z1, 0.f));
            }
        }
        __syncwarp();
    }
}

// The same layer in FP32 on CUDA cores (thread per output entry).
__global__ void k_gnn_dense_f32(uint32_t n, const float *__restrict__ h, const float *__restrict__ m,
                                const float *__restrict__ W, const float *__restrict__ bias, float *__restrict__ h_out)
{
    const size_t total = size_t(n) * H;
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < total; e += size_t(gridDim.x) * blockDim.x) {
        const size_t row = e / H;
        const int c = int(e % H);
        float z = bias[c];
        for (int k = 0; k < H; k++) z = fmaf(h[row * H + k], W[size_t(k) * H + c], z);
        for (int k = 0; k < H; k++) z = fmaf(m[row * H + k], W[size_t(H + k) * H + c], z);
        h_out[e] = h[e] + fmaxf(z, 0.f);
    }
}

// y = h w_out + b_out;  z = y * rms * s  (double output)
__global__ void k_gnn_output(uint32_t n, const float *__restrict__ h, const float *__restrict__ P, int L,
                             const float *__restrict__ s, const float *__restrict__ rms, double *__restrict__ z,
                             float *__restrict__ y_out)
{
    const float *w = P + off_wout(L);
    const float b = P[off_bout(L)], sc = *rms;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float y = b;
        for (int k = 0; k < H; k++) y = fmaf(h[size_t(i) * H + k], w[k], y);
        if (y_out) y_out[i] = y;
        z[i] = double(y) * double(sc) * double(s[i]);
    }
}

// ---------------- backward ----------------

// gy_i = dL/dz_i * rms * s_i ; gh_L = gy w_out ; partial dw_out, db_out per block
__global__ void k_gnn_output_bwd(uint32_t n, const double *__restrict__ gz, const float *__restrict__ h,
                                 const float *__restrict__ P, int L, const float *__restrict__ s,
                                 const float *__restrict__ rms, float *__restrict__ gh, float *__restrict__ blk)
{
    __shared__ float acc[H + 1];
    for (int k = threadIdx.x; k < H + 1; k += blockDim.x) acc[k] = 0.f;
    __syncthreads();
    const float *w = P + off_wout(L);
    const float sc = *rms;
    float la[H + 1];
    for (int k = 0; k < H + 1; k++) la[k] = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gy = float(gz[i] * double(sc) * double(s[i]));
        for (int k = 0; k < H; k++) {
            gh[size_t(i) * H + k] = gy * w[k];
            la[k] = fmaf(gy, h[size_t(i) * H + k], la[k]);
        }
        la[H] += gy;
    }
    // block reduction in fixed order: warp shuffles, then warps in order
    const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
    __shared__ float wsum[8][H + 1];
    for (int k = 0; k < H + 1; k++) {
        float v = la[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) wsum[wi][k] = v;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < H + 1; k += blockDim.x) {
        float v = 0.f;
        for (int w2 = 0; w2 < int(blockDim.x >> 5); w2++) v += wsum[w2][k];
        blk[size_t(blockIdx.x) * (H + 1) + k] = v;
    }
}

// Layer backward, part 1, for tiles of 64 rows with W and W^T in shared memory and
// register tiles (4 rows x 4 columns of z, 4 rows x 8 features of gx per thread):
// recompute z = [h_prev, m] W + b (FP32, k in order), dz = g * [z > 0], gx = dz W^T
// (c in order) -> g_prev = g + gx[:H], gm = gx[H:].  Every output is accumulated in the
// order of a sequential loop over its row.  The weight gradient is k_gnn_layer_wgrad.
constexpr int kBwdRows = 64;
constexpr int kXsStride = K2 + 4;
constexpr int kDsStride = H + 4;
constexpr size_t kBwdSmem =
    sizeof(float) * (size_t(K2) * H + size_t(H) * K2 + size_t(kBwdRows) * kXsStride + size_t(kBwdRows) * kDsStride + H);

__global__ void __launch_bounds__(256) k_gnn_layer_bwd(uint32_t n, const float *__restrict__ hp,
                                                       const float *__restrict__ m, const float *__restrict__ W,
                                                       const float *__restrict__ bias, const float *__restrict__ g,
                                                       float *__restrict__ dz_out, float *__restrict__ gprev,
                                                       float *__restrict__ gm)
{
    extern __shared__ __align__(16) float sb[];
    float *Ws = sb;                               // [K2][H]
    float *WT = Ws + K2 * H;                      // [H][K2]
    float *Xs = WT + H * K2;                      // [kBwdRows][kXsStride]
    float *Ds = Xs + kBwdRows * kXsStride;        // [kBwdRows][kDsStride]
    float *bs = Ds + kBwdRows * kDsStride;        // [H]
    const int tid = threadIdx.x;
    for (int e = tid; e < K2 * H; e += blockDim.x) {
        const float w = W[e];
        Ws[e] = w;
        WT[(e % H) * K2 + e / H] = w;
    }
    for (int c = tid; c < H; c += blockDim.x) bs[c] = bias[c];
    // phase A: rows 4*ra .. +3, columns 4*ca .. +3 (16 x 16 threads)
    const int ra = tid >> 4, ca = tid & 15;
    // phase B: rows 4*rb .. +3, features 8*kb .. +7 (16 x 16 threads)
    const int rb = tid >> 4, kb = tid & 15;
    const uint32_t tiles = (n + kBwdRows - 1) / kBwdRows;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t r0 = tile * kBwdRows;
        __syncthreads();
        for (int e = tid; e < kBwdRows * K2; e += blockDim.x) {
            const int rr = e / K2, k = e % K2;
            const uint32_t row = r0 + rr;
            Xs[rr * kXsStride + k] = row < n ? (k < H ? hp[size_t(row) * H + k] : m[size_t(row) * H + k - H]) : 0.f;
        }
        __syncthreads();
        {
            float z[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) z[i][j] = bs[4 * ca + j];
            for (int k = 0; k < K2; k++) {
                const float4 w = *reinterpret_cast<const float4 *>(&Ws[k * H + 4 * ca]);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float x = Xs[(4 * ra + i) * kXsStride + k];
                    z[i][0] = fmaf(x, w.x, z[i][0]);
                    z[i][1] = fmaf(x, w.y, z[i][1]);
                    z[i][2] = fmaf(x, w.z, z[i][2]);
                    z[i][3] = fmaf(x, w.w, z[i][3]);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t row = r0 + 4 * ra + i;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int c = 4 * ca + j;
                    const float d = (row < n && z[i][j] > 0.f) ? g[size_t(row) * H + c] : 0.f;
                    Ds[(4 * ra + i) * kDsStride + c] = d;
                    if (row < n) dz_out[size_t(row) * H + c] = d;
                }
            }
        }
        __syncthreads();
        {
            float gx[4][8];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) gx[i][j] = 0.f;
            for (int c = 0; c < H; c++) {
                const float4 w0 = *reinterpret_cast<const float4 *>(&WT[c * K2 + 8 * kb]);
                const float4 w1 = *reinterpret_cast<const float4 *>(&WT[c * K2 + 8 * kb + 4]);
                const float w[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const float d = Ds[(4 * rb + i) * kDsStride + c];
#pragma unroll
                    for (int j = 0; j < 8; j++) gx[i][j] = fmaf(d, w[j], gx[i][j]);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t row = r0 + 4 * rb + i;
                if (row >= n) continue;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int k = 8 * kb + j;
                    if (k < H) gprev[size_t(row) * H + k] = g[size_t(row) * H + k] + gx[i][j];
                    else gm[size_t(row) * H + (k - H)] = gx[i][j];
                }
            }
        }
    }
}

// dW = X^T dz and db = sum dz over a contiguous row range per block (rows in order),
// X = [h_prev, m]: register tiles of 4 features x 8 columns per thread, rows staged in
// shared memory 32 at a time.
constexpr int kWgRows = 32;
__global__ void __launch_bounds__(256) k_gnn_layer_wgrad(uint32_t n, const float *__restrict__ hp,
                                                         const float *__restrict__ m, const float *__restrict__ dz,
                                                         float *__restrict__ blk)
{
    __shared__ float Xs[kWgRows][K2 + 4];
    __shared__ float Ds[kWgRows][H + 4];
    const uint32_t rows_per = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(n, blockIdx.x * rows_per), r1 = min(n, r0 + rows_per);
    const int tid = threadIdx.x, kb = tid >> 3, cb = tid & 7;  // features 4kb..4kb+3, columns 8cb..8cb+7
    float acc[4][8];
    float accb[8];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
#pragma unroll
    for (int j = 0; j < 8; j++) accb[j] = 0.f;
    for (uint32_t t0 = r0; t0 < r1; t0 += kWgRows) {
        const uint32_t cnt = min(uint32_t(kWgRows), r1 - t0);
        __syncthreads();
        for (int e = tid; e < kWgRows * K2; e += blockDim.x) {
            const int rr = e / K2, k = e % K2;
            const uint32_t row = t0 + rr;
            Xs[rr][k] = uint32_t(rr) < cnt ? (k < H ? hp[size_t(row) * H + k] : m[size_t(row) * H + k - H]) : 0.f;
        }
        for (int e = tid; e < kWgRows * H; e += blockDim.x) {
            const int rr = e / H, c = e % H;
            Ds[rr][c] = uint32_t(rr) < cnt ? dz[size_t(t0 + rr) * H + c] : 0.f;
        }
        __syncthreads();
        for (uint32_t rr = 0; rr < cnt; rr++) {
            float x[4], d[8];
#pragma unroll
            for (int i = 0; i < 4; i++) x[i] = Xs[rr][4 * kb + i];
#pragma unroll
            for (int j = 0; j < 8; j++) d[j] = Ds[rr][8 * cb + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = fmaf(x[i], d[j], acc[i][j]);
            if (kb == 0)
#pragma unroll
                for (int j = 0; j < 8; j++) accb[j] += d[j];
        }
    }
    const int total = K2 * H + H;
    float *out = blk + size_t(blockIdx.x) * total;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) out[(4 * kb + i) * H + 8 * cb + j] = acc[i][j];
    if (kb == 0)
#pragma unroll
        for (int j = 0; j < 8; j++) out[K2 * H + 8 * cb + j] = accb[j];
}

// input layer: dpre = gh0 * [pre0 > 0]; dW_in = f^T dpre, db_in = sum dpre over a
// contiguous row range per block (rows in order); thread = (feature k, column pair).
__global__ void __launch_bounds__(256) k_gnn_input_wgrad(uint32_t n, const float *__restrict__ feat,
                                                         const float *__restrict__ pre0,
                                                         const float *__restrict__ gh0, float *__restrict__ blk)
{
    __shared__ float Fs[32][F];
    __shared__ float Ps[32][H + 2];
    const uint32_t rows_per = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t r0 = min(n, blockIdx.x * rows_per), r1 = min(n, r0 + rows_per);
    const int tid = threadIdx.x, k = tid >> 5, c0 = 2 * (tid & 31);
    float a0 = 0.f, a1 = 0.f, b0 = 0.f, b1 = 0.f;
    for (uint32_t t0 = r0; t0 < r1; t0 += 32) {
        const uint32_t cnt = min(32u, r1 - t0);
        __syncthreads();
        for (int e = tid; e < 32 * F; e += blockDim.x)
            Fs[e / F][e % F] = uint32_t(e / F) < cnt ? feat[size_t(t0 + e / F) * F + e % F] : 0.f;
        for (int e = tid; e < 32 * H; e += blockDim.x) {
            const int rr = e / H, c = e % H;
            float dp = 0.f;
            if (uint32_t(rr) < cnt) {
                const size_t idx = size_t(t0 + rr) * H + c;
                dp = pre0[idx] > 0.f ? gh0[idx] : 0.f;
            }
            Ps[rr][c] = dp;
        }
        __syncthreads();
        for (uint32_t rr = 0; rr < cnt; rr++) {
            const float f = Fs[rr][k];
            const float d0 = Ps[rr][c0], d1 = Ps[rr][c0 + 1];
            a0 = fmaf(f, d0, a0);
            a1 = fmaf(f, d1, a1);
            if (k == 0) {
                b0 += d0;
                b1 += d1;
            }
        }
    }
    float *out = blk + size_t(blockIdx.x) * (F * H + H);
    out[k * H + c0] = a0;
    out[k * H + c0 + 1] = a1;
    if (k == 0) {
        out[F * H + c0] = b0;
        out[F * H + c0 + 1] = b1;
    }
}

// sum per-block partials (fixed order) into grad[off .. off+count)
__global__ void k_gnn_sum_blocks(const float *__restrict__ blk, int nblk, int count, float *__restrict__ grad)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        float v = 0.f;
#pragma unroll 16
        for (int b = 0; b < nblk; b++) v += blk[size_t(b) * count + e];
        grad[e] = v;
    }
}

__global__ void k_gnn_adam(size_t count, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                           float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// loss pieces: e = r - A z (given az), L = ||e||^2/||r||^2
__global__ void k_gnn_resid(uint32_t n, const double *__restrict__ r, const double *__restrict__ az,
                            double *__restrict__ e, double *partials, unsigned int *ticket, double *out)
{
    __shared__ double sh[64];
    double acc[2] = {0.0, 0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double ei = r[i] - az[i];
        e[i] = ei;
        acc[0] += ei * ei;
        acc[1] += r[i] * r[i];
    }
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) {
        out[0] = tot[0] / (tot[1] > 0.0 ? tot[1] : 1.0);
        out[1] = tot[1];
    }
}

__global__ void k_gnn_scale(uint32_t n, const double *__restrict__ src, const double *__restrict__ rr, double c,
                            double *__restrict__ dst)
{
    const double f = c / (rr[1] > 0.0 ? rr[1] : 1.0);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = f * src[i];
}

template <typename T>
T *dev_alloc(size_t count)
{
    T *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    return p;
}

__global__ void k_axpy_f32(size_t n, float a, const float *__restrict__ x, float *__restrict__ y)
{
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        y[i] = fmaf(a, x[i], y[i]);
}

}  // namespace

void rsg_axpy_f32(rsg_context *ctx, size_t n, float a, const float *x, float *y)
{
    const int g = std::min(grid_for(ctx, (const void *)k_axpy_f32, kBlock, 0, (long long)n), kMaxGrid);
    k_axpy_f32<<<g, kBlock, 0, ctx->stream>>>(n, a, x, y);
}

void gnn_free_buffers(rsg_learned *G)
{
    for (float *p : G->h) cudaFree(p);
    for (float *p : G->m) cudaFree(p);
    G->h.clear();
    G->m.clear();
    float **bufs[] = {&G->s, &G->logd, &G->rsum, &G->feat, &G->pre0, &G->gh, &G->gh2, &G->gm, &G->dz, &G->blk,
                      &G->scal32};
    for (float **b : bufs) {
        cudaFree(*b);
        *b = nullptr;
    }
    cudaFree(G->dbuf);
    G->dbuf = nullptr;
    cudaFree(G->ew);
    G->ew = nullptr;
    G->ew_cap = 0;
    for (auto &b : G->hb) {
        cudaFree(b);
        b = nullptr;
    }
    G->cap = 0;
    G->cached = nullptr;
}

// (Re)build the per-matrix caches and activation buffers for n rows.
rsg_status gnn_prepare(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, bool train)
{
    const uint32_t n = A->n;
    const bool realloc = n > G->cap || (train && !G->train_bufs);
    if (realloc) {
        gnn_free_buffers(G);
        G->cap = n;
        G->train_bufs = train;
        const int nh = train ? G->L + 1 : 2;
        const int nm = train ? G->L : 1;
        for (int i = 0; i < nh; i++) G->h.push_back(dev_alloc<float>(size_t(n) * H));
        for (int i = 0; i < nm; i++) G->m.push_back(dev_alloc<float>(size_t(n) * H));
        G->s = dev_alloc<float>(n);
        G->logd = dev_alloc<float>(n);
        G->rsum = dev_alloc<float>(n);
        G->scal32 = dev_alloc<float>(64);
        G->dbuf = dev_alloc<double>(size_t(4) * n + size_t(4) * kMaxGrid + 64);
        for (auto &b : G->hb) b = dev_alloc<__nv_bfloat16>(size_t(n) * H);
        if (train) {
            G->feat = dev_alloc<float>(size_t(n) * F);
            G->pre0 = dev_alloc<float>(size_t(n) * H);
            G->gh = dev_alloc<float>(size_t(n) * H);
            G->gh2 = dev_alloc<float>(size_t(n) * H);
            G->gm = dev_alloc<float>(size_t(n) * H);
            G->dz = dev_alloc<float>(size_t(n) * H);
            G->blk = dev_alloc<float>(size_t(kGnnGradBlocks) * (K2 * H + H));
        }
        for (float *p : G->h)
            if (!p) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned: activations");
        for (float *p : G->m)
            if (!p) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned: activations");
        if (!G->s || !G->logd || !G->rsum || !G->dbuf || !G->scal32 || !G->hb[0] || !G->hb[1] ||
            (train && (!G->feat || !G->pre0 || !G->gh || !G->gh2 || !G->gm || !G->dz || !G->blk)))
            return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned: buffers");
    }
    int umma_grid = 0;
    if (!gnn_umma_setup(ctx, &umma_grid)) return set_error(ctx, RSG_ERR_CUDA, "learned: tensor-core layer set-up");
    if (A->nnz > G->ew_cap) {
        cudaFree(G->ew);
        G->ew = dev_alloc<float>(A->nnz);
        G->ew_cap = G->ew ? A->nnz : 0;
        if (!G->ew) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned: edge weights");
        G->cached = nullptr;
    }
    if (G->cached != A || realloc || G->cached_nnz != A->nnz || G->cached_norm != A->norm) {
        double *partials = G->dbuf + size_t(4) * n;
        unsigned int *ticket = reinterpret_cast<unsigned int *>(partials + size_t(4) * kMaxGrid);
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(ticket, 0, 64, ctx->stream));
        const int g = std::min(grid_for(ctx, (const void *)k_gnn_prep, kBlock, 0, n), kMaxGrid);
        k_gnn_prep<<<g, kBlock, 0, ctx->stream>>>(n, A->rp, A->ci, A->val, G->s, G->logd, G->rsum, partials, ticket,
                                                  G->scal32);
        k_gnn_edges<<<g, kBlock, 0, ctx->stream>>>(n, A->rp, A->ci, A->val, G->s, G->ew);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        G->cached = A;
        G->cached_nnz = A->nnz;
        G->cached_norm = A->norm;
    }
    return RSG_OK;
}

// Forward pass: z = M(r).  train -> keep every activation for the backward pass.
rsg_status gnn_forward(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, double *z,
                       const double *xyz, bool train, bool tensor_cores)
{
    RSG_TRY(gnn_prepare(ctx, G, A, train));
    const uint32_t n = A->n;
    cudaStream_t sm = ctx->stream;
    double *partials = G->dbuf + size_t(4) * n;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(partials + size_t(4) * kMaxGrid) + 4;
    float *rms = G->scal32 + 1;
    const int gv = std::min(grid_for(ctx, (const void *)k_gnn_rms, kBlock, 0, n), kMaxGrid);
    k_gnn_rms<<<gv, kBlock, 0, sm>>>(n, r, G->s, partials, ticket, rms);
    if (!train && tensor_cores) return gnn_forward_umma(ctx, G, A, r, z, xyz, rms);
    const int gi = std::min(grid_for(ctx, (const void *)k_gnn_input, kBlock, 0, n), kMaxGrid);
    float *h0 = G->h[0];
    k_gnn_input<<<gi, kBlock, 0, sm>>>(n, r, G->s, G->logd, G->rsum, G->scal32, rms, xyz, G->params,
                                       train ? G->feat : nullptr, train ? G->pre0 : nullptr, h0);
    const int gs = std::min(grid_for(ctx, (const void *)k_gnn_spmm, kBlock, 0, (long long)n * 32), kMaxGrid);
    const int gt = std::min(int((n + 16 * kTcWarps - 1) / (16 * kTcWarps)), kMaxGrid);
    const int gf = std::min(grid_for(ctx, (const void *)k_gnn_dense_f32, kBlock, 0, (long long)n * H), kMaxGrid);
    for (int l = 0; l < G->L; l++) {
        const float *hin = train ? G->h[l] : G->h[l & 1];
        float *hout = train ? G->h[l + 1] : G->h[(l + 1) & 1];
        float *m = train ? G->m[l] : G->m[0];
        const float *W = G->params + off_layer(l), *b = W + size_t(K2) * H;
        k_gnn_spmm<<<gs, kBlock, 0, sm>>>(n, A->rp, A->ci, G->ew, hin, m);
        if (tensor_cores && train) RSG_TRY(gnn_train_dense_umma(ctx, n, hin, m, W, b, hout));
        else if (tensor_cores) k_gnn_dense_tc<<<gt, 32 * kTcWarps, 0, sm>>>(n, hin, m, W, b, hout);
        else k_gnn_dense_f32<<<gf, kBlock, 0, sm>>>(n, hin, m, W, b, hout);
    }
    const float *hl = train ? G->h[G->L] : G->h[G->L & 1];
    k_gnn_output<<<gi, kBlock, 0, sm>>>(n, hl, G->params, G->L, G->s, rms, z, nullptr);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

// Loss L = ||r - A M(r)||^2 / ||r||^2 and its gradient into G->grad (device).
rsg_status gnn_loss_grad(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, const double *xyz,
                         bool tensor_cores, double *loss)
{
    const uint32_t n = A->n;
    cudaStream_t sm = ctx->stream;
    RSG_TRY(gnn_prepare(ctx, G, A, true));
    double *z = G->dbuf, *az = G->dbuf + n, *e = G->dbuf + 2 * size_t(n), *gz = G->dbuf + 3 * size_t(n);
    RSG_TRY(gnn_forward(ctx, G, A, r, z, xyz, true, tensor_cores));
    RSG_TRY(spmv64(ctx, A, z, az, true));
    double *partials = G->dbuf + size_t(4) * n;
    unsigned int *ticket = reinterpret_cast<unsigned int *>(partials + size_t(4) * kMaxGrid) + 8;
    double *out = reinterpret_cast<double *>(ticket + 8);
    const int gv = std::min(grid_for(ctx, (const void *)k_gnn_resid, kBlock, 0, n), kMaxGrid);
    k_gnn_resid<<<gv, kBlock, 0, sm>>>(n, r, az, e, partials, ticket, out);
    // dL/dz = -2 A e / ||r||^2 (A symmetric)
    RSG_TRY(spmv64(ctx, A, e, gz, true));
    k_gnn_scale<<<gv, kBlock, 0, sm>>>(n, gz, out, -2.0, gz);
    const int L = G->L;
    const int nb = kGnnGradBlocks;
    float *rms = G->scal32 + 1;
    // output layer
    const int gi = std::min(grid_for(ctx, (const void *)k_gnn_output_bwd, kBlock, 0, n), kGnnGradBlocks);
    k_gnn_output_bwd<<<gi, kBlock, 0, sm>>>(n, gz, G->h[L], G->params, L, G->s, rms, G->gh, G->blk);
    k_gnn_sum_blocks<<<1, 128, 0, sm>>>(G->blk, gi, H + 1, G->grad + off_wout(L));
    const int gs = std::min(grid_for(ctx, (const void *)k_gnn_spmm, kBlock, 0, (long long)n * 32), kMaxGrid);
    static bool bwd_attr = false;
    if (!bwd_attr) {
        RSG_CHECK_CUDA(ctx, cudaFuncSetAttribute(k_gnn_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 int(kBwdSmem)));
        bwd_attr = true;
    }
    const int gb = std::min(grid_for(ctx, (const void *)k_gnn_layer_bwd, 256, kBwdSmem,
                                     (long long)(n + kBwdRows - 1) / kBwdRows * 256), kMaxGrid);
    float *g = G->gh, *g2 = G->gh2;
    for (int l = L - 1; l >= 0; l--) {
        const float *W = G->params + off_layer(l), *b = W + size_t(K2) * H;
        if (tensor_cores) {
            RSG_TRY(gnn_train_bwd_umma(ctx, n, G->h[l], G->m[l], W, b, g, G->dz, g2, G->gm));
            RSG_TRY(gnn_train_wgrad_umma(ctx, n, G->h[l], G->m[l], G->dz, G->blk, nb));
        } else {
            k_gnn_layer_bwd<<<gb, 256, kBwdSmem, sm>>>(n, G->h[l], G->m[l], W, b, g, G->dz, g2, G->gm);
            k_gnn_layer_wgrad<<<nb, kBlock, 0, sm>>>(n, G->h[l], G->m[l], G->dz, G->blk);
        }
        k_gnn_sum_blocks<<<32, kBlock, 0, sm>>>(G->blk, nb, K2 * H + H, G->grad + off_layer(l));
        // g_prev += W^T-graph gm (the graph weights are symmetric): reuse the SpMM into gm, then add
        k_gnn_spmm<<<gs, kBlock, 0, sm>>>(n, A->rp, A->ci, G->ew, G->gm, G->dz);
        // g_prev = g2 + dz
        auto *a = g2;
        const size_t cnt = size_t(n) * H;
        rsg_axpy_f32(ctx, cnt, 1.0f, G->dz, a);
        std::swap(g, g2);
    }
    k_gnn_input_wgrad<<<nb, kBlock, 0, sm>>>(n, G->feat, G->pre0, g, G->blk);
    k_gnn_sum_blocks<<<4, kBlock, 0, sm>>>(G->blk, nb, F * H + H, G->grad + off_win());
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    double h_out[2];
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(h_out, out, sizeof(h_out), cudaMemcpyDeviceToHost, sm));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(sm));
    if (loss) *loss = h_out[0];
    return RSG_OK;
}

}  // namespace rsg

using namespace rsg;

extern "C" {

rsg_status rsg_learned_create(rsg_context *ctx, uint32_t layers, uint64_t seed, rsg_learned **out)
{
    if (!ctx || !out || layers == 0 || layers > 32) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_create");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    auto *G = new rsg_learned;
    G->L = int(layers);
    G->n_params = off_bout(G->L) + 1;
    G->params = dev_alloc<float>(G->n_params);
    G->grad = dev_alloc<float>(G->n_params);
    G->adam_m = dev_alloc<float>(G->n_params);
    G->adam_v = dev_alloc<float>(G->n_params);
    if (!G->params || !G->grad || !G->adam_m || !G->adam_v) {
        rsg_learned_destroy(ctx, G);
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "learned_create");
    }
    // Glorot-uniform weights, zero biases; small output layer so M starts close to 0
    std::vector<float> p(G->n_params, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t off, int fan_in, int fan_out, float gain) {
        const float a = gain * std::sqrt(6.f / float(fan_in + fan_out));
        std::uniform_real_distribution<float> u(-a, a);
        for (size_t i = 0; i < size_t(fan_in) * fan_out; i++) p[off + i] = u(rng);
    };
    fill(off_win(), F, H, 1.f);
    for (int l = 0; l < G->L; l++) fill(off_layer(l), K2, H, 0.5f);
    fill(off_wout(G->L), H, 1, 0.1f);
    cudaMemcpy(G->params, p.data(), p.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(G->grad, 0, p.size() * sizeof(float));
    cudaMemset(G->adam_m, 0, p.size() * sizeof(float));
    cudaMemset(G->adam_v, 0, p.size() * sizeof(float));
    *out = G;
    return RSG_OK;
}

void rsg_learned_destroy(rsg_context *ctx, rsg_learned *G)
{
    if (!G) return;
    if (ctx) {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
    }
    gnn_free_buffers(G);
    cudaFree(G->params);
    cudaFree(G->grad);
    cudaFree(G->adam_m);
    cudaFree(G->adam_v);
    delete G;
}

rsg_status rsg_learned_info(const rsg_learned *G, uint32_t *layers, uint32_t *hidden, uint64_t *n_params,
                            uint64_t *step)
{
    if (!G) return RSG_ERR_INVALID_ARG;
    if (layers) *layers = uint32_t(G->L);
    if (hidden) *hidden = H;
    if (n_params) *n_params = G->n_params;
    if (step) *step = G->step;
    return RSG_OK;
}

rsg_status rsg_learned_get_params(rsg_context *ctx, const rsg_learned *G, float *host, int32_t which)
{
    if (!ctx || !G || !host) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_get_params");
    const float *src = which == 0 ? G->params : which == 1 ? G->grad : which == 2 ? G->adam_m : G->adam_v;
    RSG_CHECK_CUDA(ctx, cudaMemcpy(host, src, G->n_params * sizeof(float), cudaMemcpyDeviceToHost));
    return RSG_OK;
}

rsg_status rsg_learned_set_params(rsg_context *ctx, rsg_learned *G, const float *host, int32_t which)
{
    if (!ctx || !G || !host) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_set_params");
    float *dst = which == 0 ? G->params : which == 1 ? G->grad : which == 2 ? G->adam_m : G->adam_v;
    RSG_CHECK_CUDA(ctx, cudaMemcpy(dst, host, G->n_params * sizeof(float), cudaMemcpyHostToDevice));
    return RSG_OK;
}

rsg_status rsg_learned_set_step(rsg_learned *G, uint64_t step)
{
    if (!G) return RSG_ERR_INVALID_ARG;
    G->step = step;
    return RSG_OK;
}

rsg_status rsg_learned_apply(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r, double *z,
                             const double *xyz, int32_t tensor_cores)
{
    if (!ctx || !G || !A || !r || !z) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_apply");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    return gnn_forward(ctx, G, A, r, z, xyz, false, tensor_cores != 0);
}

rsg_status rsg_learned_loss_grad(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r,
                                 const double *xyz, int32_t tensor_cores, double *loss)
{
    if (!ctx || !G || !A || !r) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_loss_grad");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    return gnn_loss_grad(ctx, G, A, r, xyz, tensor_cores != 0, loss);
}

rsg_status rsg_learned_train_step(rsg_context *ctx, rsg_learned *G, const rsg_csr *A, const double *r,
                                  const double *xyz, float lr, double *loss)
{
    if (!ctx || !G || !A || !r) return set_error(ctx, RSG_ERR_INVALID_ARG, "learned_train_step");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_TRY(gnn_loss_grad(ctx, G, A, r, xyz, true, loss));
    G->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(G->step)), c2 = 1.f - std::pow(b2, float(G->step));
    k_gnn_adam<<<64, kBlock, 0, ctx->stream>>>(G->n_params, G->params, G->grad, G->adam_m, G->adam_v, lr, b1, b2,
                                              1e-8f, c1, c2);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

}  // extern "C"
