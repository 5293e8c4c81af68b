// Multilevel aggregation preconditioner (RSG_PREC_AMG): hierarchy set-up and V-cycle on the GPU.
//
// No counterpart in the reference (its preconditioners are NONE / JACOBI / BLOCK_JACOBI,
// src/rmatrixpreconditioner.cpp); it serves the same slot, P.compute(r, z) in solveCG
// (src/rmatrixsolver.cpp:258), as a fixed symmetric positive definite operator.
//
// Set-up, per level, all on the GPU and deterministic (integer work, and floating-point sums in
// a fixed order):
//   1. strength: j is a strong neighbour of i when |a_ij| >= theta sqrt(|a_ii a_jj|);
//   2. roots: a distance-2 independent set of the strength graph by synchronous rounds over the
//      tuples (state, hash(i), i) -- an undecided node whose tuple is the largest within distance 2
//      becomes a root, one that sees a root within distance 2 drops out;
//   3. aggregates: every root opens one (numbered in root index order); a node with a strong root
//      neighbour joins the one with the largest key, then a node with a strong neighbour that has
//      joined takes that neighbour's aggregate (largest key again); anything left is a singleton;
//   4. Galerkin product with the piecewise-constant prolongation: coarse entry (I, J) is the sum of
//      a_ij over i in I, j in J, added in the order of the fine rows of I (ascending) and of the
//      entries within each row -- one CTA per coarse row stages the entries, sorts them by
//      (J, position) and adds each run serially;
//   5. until the level has at most kAmgCoarsest rows, whose dense inverse (in-place Gauss-Jordan,
//      FP64, no pivoting: the Galerkin matrices of an SPD matrix are SPD) is kept in FP32.
// The host reads back a handful of counters per level (set sizes), nothing else.
//
// V-cycle (FP32), per level with right-hand side b, diagonal weights dw = omega / a_ii:
//   pre-smoothing from x = 0 (one or two damped-Jacobi sweeps), residual, restriction (sum over the
//   aggregate, in ascending row order), the coarse level, prolongation scaled by s, post-smoothing
//   with the same sweeps.  Every sweep is one pass over the level's matrix with the smoother fused
//   into the gather; the finest level reads the matrix's FP32 SELL-32 (or CSR-stream) copy, the
//   coarse levels their CSR with 4 lanes per row.  Levels 1..kAmgKLevels are solved by two
//   flexible-CG steps each (K-cycle); the last smoothed level and the dense coarse solve run as one
//   single-CTA kernel.  Each step is its own kernel, launched with programmatic dependent launch; on
//   request (conf.persistent > 0) the levels of at most kCoarsePersistRows rows run instead as one
//   persistent cooperative kernel per visit, with the same bits (measured slower on B200).
#include "amg.cuh"
#include "grid_sync.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

namespace rsg {

// ---------------------------------------------------------------- keys ----------------------

// 32-bit integer hash (the "lowbias32" finalizer published by C. Wellons).
__host__ __device__ __forceinline__ uint32_t amg_hash(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
// 62-bit priority of node i: 30 hash bits above the index (unique).
__host__ __device__ __forceinline__ uint64_t amg_key(uint32_t i) { return (uint64_t(amg_hash(i) >> 2) << 32) | i; }
constexpr uint64_t kStateShift = 62;
__device__ __forceinline__ uint32_t tup_state(uint64_t t) { return uint32_t(t >> kStateShift); }
__device__ __forceinline__ uint32_t tup_index(uint64_t t) { return uint32_t(t & 0xffffffffu); }

namespace {

// ---------------------------------------------------------------- scan ----------------------

constexpr int kScanThreads = 256;
constexpr int kScanTile = 1024;  // 4 elements per thread

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *sh, uint32_t &total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    __syncthreads();
    if (lane == 31) sh[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) sh[32 + lane] = w;
    }
    __syncthreads();
    total = sh[32 + nw - 1];
    const uint32_t warp_off = warp ? sh[32 + warp - 1] : 0u;
    return warp_off + inc - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t *__restrict__ in, uint32_t n,
                                                             uint32_t *__restrict__ sums)
{
    __shared__ uint32_t sh[64];
    const size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * 4;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_exclusive_scan(s, sh, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t *sums, uint32_t nb)
{
    __shared__ uint32_t sh[64];
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < nb; c0 += kScanThreads) {
        const uint32_t i = c0 + threadIdx.x;
        const uint32_t v = i < nb ? sums[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive_scan(v, sh, total);
        if (i < nb) sums[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
}

// out[i] = sum of in[0..i); out[n] = the total (out holds n + 1 entries).
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const uint32_t *__restrict__ in, uint32_t n,
                                                             const uint32_t *__restrict__ sums,
                                                             uint32_t *__restrict__ out)
{
    __shared__ uint32_t sh[64];
    const size_t base = size_t(blockIdx.x) * kScanTile + size_t(threadIdx.x) * 4;
    uint32_t v[4], s = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t run = sums[blockIdx.x] + block_exclusive_scan(s, sh, total);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
        if (base + k + 1 == n) out[n] = run;
    }
}

// Launch accounting: every kernel launch of this file is counted (rsg_amg_info reports the set-up's
// launches); a dry run of the cycle skips its launches and only counts them.
thread_local uint32_t t_launches = 0;
thread_local bool t_dry = false;
inline void count_launch() { ++t_launches; }
template <class... P, class... A>
void amg_launch(cudaStream_t stream, bool pdl, void (*k)(P...), dim3 grid, int block, size_t smem, A &&...args)
{
    ++t_launches;
    if (!t_dry) launch_k(stream, pdl, k, grid, block, smem, std::forward<A>(args)...);
}

// Exclusive scan of in[0..n) into out[0..n]; the total lands in *total_dev (device word).
rsg_status scan_u32(rsg_context *ctx, AmgHierarchy *H, const uint32_t *in, uint32_t n, uint32_t *out)
{
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (n == 0) {
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(out, 0, sizeof(uint32_t), ctx->stream));
        return RSG_OK;
    }
    if (!H->scan_blocks.ensure(nb)) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: scan workspace");
    count_launch();
    k_scan_tiles<<<nb, kScanThreads, 0, ctx->stream>>>(in, n, H->scan_blocks.p);
    count_launch();
    k_scan_sums<<<1, kScanThreads, 0, ctx->stream>>>(H->scan_blocks.p, nb);
    count_launch();
    k_scan_apply<<<nb, kScanThreads, 0, ctx->stream>>>(in, n, H->scan_blocks.p, out);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

// ---------------------------------------------------------------- set-up kernels ------------

inline int grid_rows(uint64_t rows, int per_block = kBlock) { return int(std::min<uint64_t>((rows + per_block - 1) / per_block, 65535ull * 16)); }

__global__ void k_amg_diag(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                           const double *__restrict__ val, double *__restrict__ diag, float *__restrict__ dw)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
            if (ci[j] == i) d = val[j];
        diag[i] = d;
        dw[i] = d != 0.0 ? float(double(kAmgOmega) / d) : 0.f;
    }
}

// Passes with heavy per-entry work (the FP64 strength test, the coarse-row copy) give each row
// kRowLanes lanes, entries strided by kRowLanes.  (The light passes -- diagonal, independent-set
// rounds, joins -- stay one thread per row: with 8 lanes they measured 2-5x slower, the grid of
// short blocks costing more than the shorter serial loops save.)
constexpr int kRowLanes = 8;

// f(i, valid, lane) for every row i, kRowLanes lanes each; warps run whole rounds.
template <class F>
__device__ __forceinline__ void for_row_groups(uint32_t n, F &&f)
{
    const uint32_t lane = threadIdx.x & (kRowLanes - 1);
    const uint32_t stride = (gridDim.x * blockDim.x) / kRowLanes;
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32 / kRowLanes); base < n; base += stride) {
        const uint32_t i = base + (threadIdx.x & 31) / kRowLanes;
        f(i, i < n, lane);
    }
}

inline int grid_groups(uint64_t rows) { return grid_rows(rows * kRowLanes); }

__global__ void k_amg_strength(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                               const double *__restrict__ val, const double *__restrict__ diag, double theta,
                               uint8_t *__restrict__ smask)
{
    for_row_groups(n, [&](uint32_t i, bool ok, uint32_t lane) {
        if (!ok) return;
        const double di = diag[i];
        for (uint32_t j = rp[i] + lane; j < rp[i + 1]; j += kRowLanes) {
            const uint32_t c = ci[j];
            bool st = false;
            if (c != i && c < n) st = fabs(val[j]) >= theta * sqrt(fabs(di * diag[c])) && val[j] != 0.0;
            smask[j] = st ? 1 : 0;
        }
    });
}

__global__ void k_amg_mis_init(uint32_t n, uint64_t *__restrict__ T)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        T[i] = (uint64_t(1) << kStateShift) | amg_key(i);
}

__device__ __forceinline__ uint64_t strong_max(uint32_t i, const uint32_t *__restrict__ rp,
                                               const uint32_t *__restrict__ ci, const uint8_t *__restrict__ smask,
                                               const uint64_t *__restrict__ in)
{
    uint64_t m = in[i];
    for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
        if (smask[j]) m = max(m, in[ci[j]]);
    return m;
}

// The decision of an undecided node i from M2_i (the largest tuple within distance 2): a root when
// it is the node's own tuple, out when it belongs to a root, else still undecided (returns true).
__device__ __forceinline__ bool mis_decide(uint32_t i, uint64_t t, uint64_t m2, uint64_t *__restrict__ T)
{
    if (m2 == t) T[i] = (uint64_t(2) << kStateShift) | amg_key(i);
    else if (tup_state(m2) == 2) T[i] = amg_key(i);
    else return true;
    return false;
}

// out_i = max(in_i, max over strong neighbours j of in_j), for the nodes the second pass will read:
// in round 0 all of them, later only those stamped need_i = round by the previous round (the nodes
// still undecided and their strong neighbours), so late rounds skip most of the graph.  Rounds are
// launched in batches; once a round has left no node undecided (*prev == 0) the later rounds return
// at once.
__global__ void k_amg_nbmax(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                            const uint8_t *__restrict__ smask, const uint64_t *__restrict__ in,
                            uint64_t *__restrict__ out, const uint32_t *__restrict__ need, uint32_t round,
                            const unsigned int *prev)
{
    if (prev && *prev == 0) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (round == 0 || need[i] == round) out[i] = strong_max(i, rp, ci, smask, in);
}

// Second half of a synchronous round, fused with the decision: for every node still undecided,
// M2_i = max(M1_i, max over strong neighbours j of M1_j) (decided nodes need no M2).  A node left
// undecided stamps itself and its strong neighbours need = round + 1.  *count (zeroed beforehand)
// receives the number of nodes still undecided; nothing is done once the previous round left none
// (*prev == 0).
__global__ void k_amg_mis_round2(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                                 const uint8_t *__restrict__ smask, const uint64_t *__restrict__ M1,
                                 uint64_t *__restrict__ T, uint32_t *__restrict__ need, uint32_t round,
                                 const unsigned int *prev, unsigned int *count)
{
    if (prev && *prev == 0) return;
    unsigned int left = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t t = T[i];
        if (tup_state(t) != 1) continue;
        if (mis_decide(i, t, strong_max(i, rp, ci, smask, M1), T)) {
            left++;
            need[i] = round + 1;
            for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
                if (smask[j]) need[ci[j]] = round + 1;
        }
    }
    left = __reduce_add_sync(0xffffffffu, left);
    if ((threadIdx.x & 31) == 0 && left) atomicAdd(count, left);
}

// All rounds of a small level in one CTA (the passes separated by barriers): out[0] = the rounds
// run, out[1] = the nodes still undecided after them (0 unless kMaxRounds ran out).
constexpr uint32_t kMisCtaRows = 4096;
constexpr int kMisCtaThreads = 1024;
constexpr uint32_t kMisMaxRounds = 128;
__global__ void __launch_bounds__(kMisCtaThreads) k_amg_mis_cta(uint32_t n, const uint32_t *__restrict__ rp,
                                                                const uint32_t *__restrict__ ci,
                                                                const uint8_t *__restrict__ smask,
                                                                uint64_t *__restrict__ T, uint64_t *__restrict__ M1,
                                                                unsigned int *out)
{
    __shared__ unsigned int left;
    uint32_t r = 0;
    unsigned int l = n;
    while (r < kMisMaxRounds && l > 0) {
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) M1[i] = strong_max(i, rp, ci, smask, T);
        if (threadIdx.x == 0) left = 0;
        __syncthreads();
        unsigned int mine = 0;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint64_t t = T[i];
            if (tup_state(t) != 1) continue;
            if (mis_decide(i, t, strong_max(i, rp, ci, smask, M1), T)) mine++;
        }
        mine = __reduce_add_sync(0xffffffffu, mine);
        if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&left, mine);
        __syncthreads();
        l = left;
        r++;
        __syncthreads();  // every thread has read left before the next round resets it
    }
    if (threadIdx.x == 0) {
        out[0] = r;
        out[1] = l;
    }
}

__global__ void k_amg_root_flags(uint32_t n, const uint64_t *__restrict__ T, uint32_t *__restrict__ flag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = tup_state(T[i]) == 2 ? 1u : 0u;
}

// Roots take their number; others join the strong root neighbour with the largest tuple.
__global__ void k_amg_join1(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                            const uint8_t *__restrict__ smask, const uint64_t *__restrict__ T,
                            const uint32_t *__restrict__ root_rank, uint32_t *__restrict__ agg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (tup_state(T[i]) == 2) {
            agg[i] = root_rank[i];
            continue;
        }
        uint64_t best = 0;
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
            if (!smask[j]) continue;
            const uint64_t t = T[ci[j]];
            if (tup_state(t) == 2) best = max(best, t);
        }
        agg[i] = best ? root_rank[tup_index(best)] : kAmgUnset;
    }
}

// A node left out joins the aggregate of its strong neighbour with the largest key among those
// that joined in the first pass; flags[1] counts nodes still without an aggregate.
__global__ void k_amg_join2(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                            const uint8_t *__restrict__ smask, const uint32_t *__restrict__ agg_in,
                            uint32_t *__restrict__ agg_out, unsigned int *flags)
{
    unsigned int left = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t a = agg_in[i];
        if (a == kAmgUnset) {
            uint64_t best = 0;
            uint32_t pick = kAmgUnset;
            for (uint32_t j = rp[i]; j < rp[i + 1]; j++) {
                if (!smask[j]) continue;
                const uint32_t c = ci[j];
                if (agg_in[c] == kAmgUnset) continue;
                const uint64_t k = amg_key(c) + 1;
                if (k > best) {
                    best = k;
                    pick = agg_in[c];
                }
            }
            a = pick;
            if (a == kAmgUnset) left++;
        }
        agg_out[i] = a;
    }
    left = __reduce_add_sync(0xffffffffu, left);
    if ((threadIdx.x & 31) == 0 && left) atomicAdd(&flags[1], left);
}

__global__ void k_amg_unset_flags(uint32_t n, const uint32_t *__restrict__ agg, uint32_t *__restrict__ flag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flag[i] = agg[i] == kAmgUnset ? 1u : 0u;
}

__global__ void k_amg_singletons(uint32_t n, uint32_t first, const uint32_t *__restrict__ rank,
                                 uint32_t *__restrict__ agg)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (agg[i] == kAmgUnset) agg[i] = first + rank[i];
}

__global__ void k_amg_count(uint32_t n, const uint32_t *__restrict__ agg, uint32_t *__restrict__ cnt)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicAdd(&cnt[agg[i]], 1u);
}

__global__ void k_amg_fill(uint32_t n, const uint32_t *__restrict__ agg, const uint32_t *__restrict__ ptr,
                           uint32_t *__restrict__ cursor, uint32_t *__restrict__ rows)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t a = agg[i];
        rows[ptr[a] + atomicAdd(&cursor[a], 1u)] = i;
    }
}

// Sort each aggregate's rows ascending (insertion sort: aggregates are small) and record the
// number of fine entries the aggregate's rows hold (flags[2] = the largest; flags[3] = the largest
// aggregate).
__global__ void k_amg_sort_agg(uint32_t nc, const uint32_t *__restrict__ ptr, uint32_t *__restrict__ rows,
                               const uint32_t *__restrict__ rp, uint32_t *__restrict__ entries, unsigned int *flags)
{
    for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < nc; a += gridDim.x * blockDim.x) {
        const uint32_t b = ptr[a], e = ptr[a + 1];
        uint32_t tot = 0;
        for (uint32_t k = b + 1; k < e; k++) {
            const uint32_t v = rows[k];
            uint32_t m = k;
            while (m > b && rows[m - 1] > v) {
                rows[m] = rows[m - 1];
                m--;
            }
            rows[m] = v;
        }
        for (uint32_t k = b; k < e; k++) tot += rp[rows[k] + 1] - rp[rows[k]];
        entries[a] = tot;
        atomicMax(&flags[2], tot);
        atomicMax(&flags[3], e - b);
    }
}

// Galerkin coarse row I (one CTA): stage the entries of the aggregate's fine rows as keys
// (J << 32 | position) with J the aggregate of the column, sort, add each run of equal J serially
// in position order, and write the row's distinct (J, sum) pairs compacted at eoff[I].
constexpr int kGalThreads = 128;
__global__ void __launch_bounds__(kGalThreads) k_amg_galerkin(uint32_t nc, const uint32_t *__restrict__ ptr,
                                                              const uint32_t *__restrict__ rows,
                                                              const uint32_t *__restrict__ rp,
                                                              const uint32_t *__restrict__ ci,
                                                              const double *__restrict__ val,
                                                              const uint32_t *__restrict__ agg,
                                                              const uint32_t *__restrict__ eoff,
                                                              uint32_t *__restrict__ tcol, double *__restrict__ tval,
                                                              uint32_t *__restrict__ count)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t sh_scan[64];
    const uint32_t I = blockIdx.x;
    if (I >= nc) return;
    const uint32_t b = ptr[I], e = ptr[I + 1];
    const uint32_t E = eoff[I + 1] - eoff[I];
    uint32_t P = 32;
    while (P < E) P <<= 1;
    uint64_t *key = reinterpret_cast<uint64_t *>(smem);
    double *sval = reinterpret_cast<double *>(key + P);
    uint32_t *rstart = reinterpret_cast<uint32_t *>(sval + P);  // staging offset of each fine row
    // staging offsets of the aggregate's rows (serial prefix: aggregates are short)
    if (threadIdx.x == 0) {
        uint32_t o = 0;
        for (uint32_t k = b; k < e; k++) {
            rstart[k - b] = o;
            o += rp[rows[k] + 1] - rp[rows[k]];
        }
        rstart[e - b] = o;
    }
    __syncthreads();
    const uint32_t nr = e - b;
    for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) {
        if (t < E) {
            uint32_t lo = 0, hi = nr;  // the row holding staging slot t: rstart[lo] <= t < rstart[lo+1]
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (rstart[mid] <= t) lo = mid;
                else hi = mid;
            }
            const uint32_t i = rows[b + lo];
            const uint32_t j = rp[i] + (t - rstart[lo]);
            key[t] = (uint64_t(agg[ci[j]]) << 32) | t;
            sval[t] = val[j];
        } else {
            key[t] = ~uint64_t(0);
        }
    }
    __syncthreads();
    // bitonic sort of the keys
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) {
                const uint32_t u = t ^ j;
                if (u > t) {
                    const bool up = (t & k) == 0;
                    const uint64_t a = key[t], c = key[u];
                    if ((a > c) == up) {
                        key[t] = c;
                        key[u] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    // heads of runs of equal J, ranked in order
    uint32_t base_rank = 0;
    for (uint32_t t0 = 0; t0 < E; t0 += blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        const bool head = t < E && (t == 0 || (key[t] >> 32) != (key[t - 1] >> 32));
        uint32_t total;
        const uint32_t rank = base_rank + block_exclusive_scan(head ? 1u : 0u, sh_scan, total);
        if (head) {
            const uint32_t J = uint32_t(key[t] >> 32);
            double s = 0.0;
            for (uint32_t k = t; k < E && uint32_t(key[k] >> 32) == J; k++) s += sval[uint32_t(key[k] & 0xffffffffu)];
            tcol[size_t(eoff[I]) + rank] = J;
            tval[size_t(eoff[I]) + rank] = s;
        }
        base_rank += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) count[I] = base_rank;
}

// The same coarse rows with one warp per row and no sort: the warp walks the aggregate's entries in
// staging order (fine rows ascending, entries in CSR order) as one flattened sequence, 32 entries at
// a time across row boundaries (the indexes, columns and values of kGalAhead chunks loaded before
// the first is used), keeps one accumulator per distinct J in shared memory (slots in order of first
// occurrence, found through an open-addressing hash table), and adds each chunk's values into the
// accumulators serially in lane order -- so every sum is taken in staging order, as in the sorting
// kernel above.  The row's (J, sum) pairs are then written in ascending J.  A row with more than
// kGalUnique distinct columns sets flags[5] (the caller then runs the sorting kernel).
constexpr int kGalWarps = 4;
constexpr int kGalUnique = 128;
constexpr uint32_t kGalHashBits = 8;
constexpr uint32_t kGalHash = 1u << kGalHashBits;  // hash slots per warp: load factor <= 1/2, so a probe ends
constexpr uint32_t kGalEmpty = 0xffffffffu;
constexpr int kGalAhead = 4;
__device__ __forceinline__ uint32_t gal_hash(uint32_t J) { return (J * 2654435761u) >> (32 - kGalHashBits); }
__global__ void __launch_bounds__(32 * kGalWarps) k_amg_galerkin_warp(
    uint32_t nc, const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ rows, const uint32_t *__restrict__ rp,
    const uint32_t *__restrict__ ci, const double *__restrict__ val, const uint32_t *__restrict__ agg,
    const uint32_t *__restrict__ eoff, uint32_t *__restrict__ tcol, double *__restrict__ tval,
    uint32_t *__restrict__ count, unsigned int *flags)
{
    static_assert(kGalHash >= 2u * kGalUnique && kGalHash <= 256u, "hash table size");
    __shared__ uint32_t hkey[kGalWarps][kGalHash];
    __shared__ uint8_t hslot[kGalWarps][kGalHash];
    __shared__ uint8_t hpos[kGalWarps][kGalUnique];
    __shared__ uint32_t ucol[kGalWarps][kGalUnique];
    __shared__ double uacc[kGalWarps][kGalUnique];
    __shared__ double cval[kGalWarps][32];
    __shared__ uint32_t rpre[kGalWarps][33], rbeg[kGalWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t *hk = hkey[w], *uc = ucol[w], *pre = rpre[w], *beg = rbeg[w];
    uint8_t *hs = hslot[w], *hp = hpos[w];
    double *ua = uacc[w];
    for (uint32_t t = lane; t < kGalHash; t += 32) hk[t] = kGalEmpty;
    __syncwarp();
    for (uint32_t I = blockIdx.x * kGalWarps + w; I < nc; I += gridDim.x * kGalWarps) {
        uint32_t U = 0;
        bool overflow = false;
        const uint32_t k0 = ptr[I], k1 = ptr[I + 1];
        for (uint32_t kb = k0; kb < k1 && !overflow; kb += 32) {
            // this batch of up to 32 rows: starts and exclusive prefix of lengths
            const uint32_t nr = min(32u, k1 - kb);
            uint32_t len = 0, start = 0;
            if (uint32_t(lane) < nr) {
                const uint32_t i = rows[kb + lane];
                start = rp[i];
                len = rp[i + 1] - start;
            }
            uint32_t inc = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
            beg[lane] = start;
            pre[lane] = inc - len;
            if (lane == 31) pre[32] = total;
            __syncwarp();
            for (uint32_t fa = 0; fa < total && !overflow; fa += 32 * kGalAhead) {
                uint32_t jj[kGalAhead], Jr[kGalAhead];
                double vr[kGalAhead];
#pragma unroll
                for (int t = 0; t < kGalAhead; t++) {
                    const uint32_t f = fa + 32u * t + uint32_t(lane);
                    uint32_t lo = 0, hi = nr;  // pre[lo] <= f < pre[hi]
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (pre[mid] <= f) lo = mid;
                        else hi = mid;
                    }
                    jj[t] = f < total ? beg[lo] + (f - pre[lo]) : kAmgUnset;
                }
#pragma unroll
                for (int t = 0; t < kGalAhead; t++) {
                    Jr[t] = jj[t] != kAmgUnset ? ci[jj[t]] : 0u;
                    vr[t] = jj[t] != kAmgUnset ? val[jj[t]] : 0.0;
                }
#pragma unroll
                for (int t = 0; t < kGalAhead; t++) Jr[t] = jj[t] != kAmgUnset ? agg[Jr[t]] : kAmgUnset;
#pragma unroll
                for (int t = 0; t < kGalAhead; t++) {
                    if (fa + 32u * t >= total || overflow) break;  // warp-uniform
                    const bool valid = jj[t] != kAmgUnset;
                    const uint32_t J = Jr[t];
                    uint32_t slot = kAmgUnset;
                    if (valid)
                        for (uint32_t h = gal_hash(J);; h = (h + 1) & (kGalHash - 1)) {
                            const uint32_t k = hk[h];
                            if (k == J) {
                                slot = hs[h];
                                break;
                            }
                            if (k == kGalEmpty) break;
                        }
                    __syncwarp();  // every lookup done before this chunk's inserts
                    // new columns take slots in order of first occurrence (lane order)
                    const bool fresh = valid && slot == kAmgUnset;
                    const unsigned int same = __match_any_sync(0xffffffffu, fresh ? J : kAmgUnset);
                    const int leader = __ffs(same) - 1;
                    const bool is_leader = fresh && leader == lane;
                    const unsigned int leaders = __ballot_sync(0xffffffffu, is_leader);
                    if (U + __popc(leaders) > uint32_t(kGalUnique)) {
                        overflow = true;
                        break;
                    }
                    if (is_leader) {
                        const uint32_t sl = U + __popc(leaders & ((1u << lane) - 1u));
                        uint32_t h = gal_hash(J);
                        while (atomicCAS(&hk[h], kGalEmpty, J) != kGalEmpty) h = (h + 1) & (kGalHash - 1);
                        hs[h] = uint8_t(sl);
                        hp[sl] = uint8_t(h);
                        uc[sl] = J;
                        ua[sl] = 0.0;
                        slot = sl;
                    }
                    const uint32_t from_leader = __shfl_sync(0xffffffffu, slot, fresh ? leader : lane);
                    if (fresh) slot = from_leader;
                    U += __popc(leaders);
                    cval[w][lane] = vr[t];
                    __syncwarp();
                    // the lowest lane of each group of equal slots adds the group's values in lane order
                    const unsigned int grp = __match_any_sync(0xffffffffu, slot);
                    if (valid && (__ffs(grp) - 1) == lane) {
                        double acc = ua[slot];
                        for (unsigned int m = grp; m; m &= m - 1) acc += cval[w][__ffs(m) - 1];
                        ua[slot] = acc;
                    }
                    __syncwarp();
                }
            }
        }
        if (!overflow) {
            // ascending J: each pair's rank among the row's distinct columns
            for (uint32_t t = lane; t < U; t += 32) {
                const uint32_t J = uc[t];
                uint32_t rank = 0;
                for (uint32_t u = 0; u < U; u++) rank += uc[u] < J ? 1u : 0u;
                tcol[size_t(eoff[I]) + rank] = J;
                tval[size_t(eoff[I]) + rank] = ua[t];
            }
        }
        __syncwarp();
        // empty the hash table for the next row (the slots in use are listed in hp)
        for (uint32_t t = lane; t < U; t += 32) hk[hp[t]] = kGalEmpty;
        if (lane == 0) {
            count[I] = overflow ? 0u : U;
            if (overflow) atomicOr(&flags[5], 1u);
        }
        __syncwarp();
    }
}

__global__ void k_amg_compact(uint32_t nc, const uint32_t *__restrict__ eoff, const uint32_t *__restrict__ count,
                              const uint32_t *__restrict__ rp_c, const uint32_t *__restrict__ tcol,
                              const double *__restrict__ tval, uint32_t *__restrict__ ci_c, double *__restrict__ val_c,
                              float *__restrict__ val32_c)
{
    for_row_groups(nc, [&](uint32_t I, bool ok, uint32_t lane) {
        if (!ok) return;
        const uint32_t src = eoff[I], dst = rp_c[I];
        for (uint32_t k = lane; k < count[I]; k += kRowLanes) {
            const double v = tval[src + k];
            ci_c[dst + k] = tcol[src + k];
            val_c[dst + k] = v;
            val32_c[dst + k] = float(v);
        }
    });
}

// Dense inverse of the coarsest level (n <= kAmgCoarsest) by in-place Gauss-Jordan elimination in
// shared memory (FP64, no pivoting: the matrix is SPD).  A pivot that is not positive leaves its
// row and column at zero (the coarse correction then ignores that direction).
__global__ void k_amg_dense_inverse(uint32_t n, const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                                    const double *__restrict__ val, float *__restrict__ inv)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double *a = reinterpret_cast<double *>(smem);
    __shared__ double pinv;
    __shared__ int skip;
    for (uint32_t t = threadIdx.x; t < n * n; t += blockDim.x) a[t] = 0.0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        for (uint32_t j = rp[i]; j < rp[i + 1]; j++)
            if (ci[j] < n) a[i * n + ci[j]] = val[j];
    __syncthreads();
    for (uint32_t k = 0; k < n; k++) {
        if (threadIdx.x == 0) {
            const double p = a[k * n + k];
            skip = !(p > 0.0);
            pinv = skip ? 0.0 : 1.0 / p;
        }
        __syncthreads();
        if (skip) {
            for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) {
                a[k * n + t] = 0.0;
                a[t * n + k] = 0.0;
            }
            __syncthreads();
            continue;
        }
        // row k scaled: a[k][j] *= pinv (j != k), a[k][k] = pinv
        for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) a[k * n + j] = (j == k) ? pinv : a[k * n + j] * pinv;
        __syncthreads();
        // other rows: a[i][j] -= a[i][k] * a[k][j] (j != k), a[i][k] = -a[i][k] * pinv
        for (uint32_t t = threadIdx.x; t < n * n; t += blockDim.x) {
            const uint32_t i = t / n, j = t % n;
            if (i == k || j == k) continue;
            a[t] -= a[i * n + k] * a[k * n + j];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
            if (i != k) a[i * n + k] = -a[i * n + k] * pinv;
        __syncthreads();
    }
    for (uint32_t t = threadIdx.x; t < n * n; t += blockDim.x) inv[t] = float(a[t]);
}

__global__ void k_amg_d2f(uint32_t n, const double *__restrict__ src, float *__restrict__ dst)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = float(src[i]);
}
__global__ void k_amg_f2d(uint32_t n, const float *__restrict__ src, double *__restrict__ dst)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = double(src[i]);
}

// ---------------------------------------------------------------- V-cycle kernels -----------

// Source of the iterate a sweep starts from (x in x + dw (b - A x)):
//   kSrcDwB:     x = dw b             (the first sweep from x = 0, never stored)
//   kSrcX:       x = xs               (a stored iterate)
//   kSrcDwBCorr: x = dw b + s P e_c   (one sweep per side: coarse correction of the pre-smoothed x)
//   kSrcXCorr:   x = xs + s P e_c     (two sweeps per side)
enum { kSrcDwB = 0, kSrcX = 1, kSrcDwBCorr = 2, kSrcXCorr = 3 };
// Output: kOutRes writes r = b - A x, kOutSmooth writes x + dw (b - A x).
enum { kOutRes = 0, kOutSmooth = 1 };

//   kSrcXCorrK:  x = xs + P (g1 c1 + a2 c2) -- the correction from a K-cycle level, whose two
//                flexible-CG directions are combined here with the coefficients of its device scalars
enum { kSrcXCorrK = 4 };

struct SweepArgs {
    const float *b, *dw, *xs, *ec;
    const uint32_t *agg;
    float s;
    float *out;
    const float *ec2 = nullptr;   // kSrcXCorrK: the second direction (ec holds the first)
    const double *kc = nullptr;   // kSrcXCorrK: the K-cycle level's scalars
    float s2 = 0.f;
};

// Coefficients of the two-step flexible-CG approximation e = g1 c1 + a2 c2 from the scalars
// sc = {c1.v1, c1.b, c2.v2, c2.v1, c2.r2} (v = A c): a1 = c1.b / c1.v1, b2 = c2.v2 - (c2.v1)^2 / c1.v1,
// a2 = c2.r2 / b2, g1 = a1 - (c2.v1) a2 / c1.v1.
// Loads of vectors: COH (the persistent coarse-level kernel, whose phases read what other CTAs wrote
// earlier in the same launch) reads through L2 (ld.global.cg); the separate kernels load plainly.
template <bool COH, typename T>
__device__ __forceinline__ T ldv(const T *p)
{
    if constexpr (COH) return __ldcg(p);
    else return *p;
}

template <bool COH = false>
__device__ __forceinline__ void kc_coefficients(const double *sc, float &g1, float &a2)
{
    const double d1 = ldv<COH>(sc), t1 = ldv<COH>(sc + 1), d2 = ldv<COH>(sc + 2), g = ldv<COH>(sc + 3),
                 t2 = ldv<COH>(sc + 4);
    double c1 = 0.0, c2 = 0.0;
    if (d1 > 0.0) {
        const double b2 = d2 - g * g / d1;
        c2 = b2 > 0.0 ? t2 / b2 : 0.0;
        c1 = t1 / d1 - g * c2 / d1;
    }
    g1 = float(c1);
    a2 = float(c2);
}

template <int SRC, bool COH = false>
__device__ __forceinline__ float sweep_x(const SweepArgs &a, uint32_t c)
{
    float x = (SRC == kSrcDwB || SRC == kSrcDwBCorr) ? a.dw[c] * ldv<COH>(a.b + c) : ldv<COH>(a.xs + c);
    if (SRC == kSrcDwBCorr || SRC == kSrcXCorr) x = fmaf(a.s, ldv<COH>(a.ec + a.agg[c]), x);
    if (SRC == kSrcXCorrK) {
        const uint32_t g = a.agg[c];
        x = fmaf(a.s, ldv<COH>(a.ec + g), fmaf(a.s2, ldv<COH>(a.ec2 + g), x));
    }
    return x;
}

// rz = r^T z of the new preconditioned residual; qz = q^T z with q = A p of the last step.  The cycle
// is a variable preconditioner (its K-cycle levels run flexible-CG steps whose coefficients depend on
// the input), so the direction update is the flexible (Polak-Ribiere) one: with r_new = r_old - alpha q,
// beta = z^T (r_new - r_old) / rho = -alpha q^T z / rho.  After a true-residual refresh (r replaced)
// the mixed-precision refresh rule applies (finalize_check_mixed).
__device__ __forceinline__ void amg_finalize(CgState *st, double rz, double qz, int mode, double *rz_out)
{
    if (!st) {
        if (rz_out) *rz_out = rz;
        return;
    }
    if (mode == 0) {
        st->rho_new = rz;
        st->rho = rz;
        st->beta = 0.0;
    } else if (st->need_check) {
        finalize_check_mixed(st, rz, st->check_rn);
    } else {
        st->rho_new = rz;
        st->beta = -st->alpha * qz / st->rho;
    }
}

// Sweep over the finest level (the caller's matrix, FP32 copy).  FINAL: the output is z of the
// preconditioner; r^T z is reduced and the CG state finalized.
template <int RPW, int SRC, int OUT, bool FINAL>
__global__ void __launch_bounds__(kBlock) k_amg_fine(Csr<float> M, Sell<float> S, int use_sell, SweepArgs a,
                                                     const float *qv, double *partials, unsigned int *ticket,
                                                     CgState *st, int mode, double *rz_out)
{
    pdl_wait();
    pdl_release();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double sh[64];
    if (st && st->done) return;
    Dot2 rz, qz;
    auto gx = [&](uint32_t c) { return sweep_x<SRC>(a, c); };
    auto epi = [&](uint32_t row, float ax) {
        const float res = a.b[row] - ax;
        float o;
        if (OUT == kOutRes) o = res;
        else o = fmaf(a.dw[row], res, sweep_x<SRC>(a, row));
        a.out[row] = o;
        if (FINAL) {
            rz.add_prod(a.b[row], o);
            if (qv) qz.add_prod(qv[row], o);
        }
    };
    unsigned int *errw = st ? &st->ticket[7] : (ticket ? ticket + 1 : nullptr);
    for_rows_any<float, RPW>(M, S, use_sell != 0, gx, epi, smem_raw, errw, true);
    if (FINAL) {
        double acc[2] = {rz.value(), qz.value()};
        double tot[2];
        if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0)
            amg_finalize(st, tot[0], tot[1], mode, rz_out);
    }
}

// x_out = xs + s P e_c (the prolongated, scaled coarse correction), one streaming pass; with kc given
// (a K-cycle coarse level) x_out = xs + P (g1 c1 + a2 c2), ec = c1, ec2 = c2.
__global__ void k_amg_prolong(uint32_t n, const float *__restrict__ xs, const uint32_t *__restrict__ agg,
                              const float *__restrict__ ec, const float *__restrict__ ec2, const double *kc, float s,
                              float *__restrict__ out, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    float g1 = s, a2 = 0.f;
    if (kc) kc_coefficients(kc, g1, a2);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t g = agg[i];
        out[i] = kc ? fmaf(g1, ec[g], fmaf(a2, ec2[g], xs[i])) : fmaf(g1, ec[g], xs[i]);
    }
}

// Sweep over a coarse level (CSR, kLanes lanes per row).  Coarse levels are small and latency-bound:
// each lane first loads up to kChunk column indexes and values of its row, then issues all the
// gathers, then the multiply-adds, so that a row costs a few round trips instead of one per entry.
constexpr int kLanes = 4;
constexpr int kChunk = 8;  // entries per lane per round: rows of up to kLanes * kChunk entries in one round

template <class GX>
__device__ __forceinline__ float csr_row_dot(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                                             const float *__restrict__ val, uint32_t row, bool valid, int lane,
                                             GX &gx)
{
    float acc = 0.f;
    const uint32_t beg = valid ? rp[row] : 0u, end = valid ? rp[row + 1] : 0u;
    for (uint32_t j0 = beg; j0 < end; j0 += kLanes * kChunk) {
        uint32_t c[kChunk];
        float v[kChunk], x[kChunk];
#pragma unroll
        for (int t = 0; t < kChunk; t++) {
            const uint32_t j = j0 + uint32_t(lane) + uint32_t(kLanes * t);
            const bool ok = j < end;
            c[t] = ok ? ci[j] : row;
            v[t] = ok ? val[j] : 0.f;
        }
#pragma unroll
        for (int t = 0; t < kChunk; t++) x[t] = v[t] != 0.f ? gx(c[t]) : 0.f;
#pragma unroll
        for (int t = 0; t < kChunk; t++) acc = fmaf(v[t], x[t], acc);
    }
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// The rows of one sweep, warp gw of warps (kLanes lanes per row).
template <int SRC, int OUT, bool COH = false>
__device__ __forceinline__ void coarse_rows(uint32_t n, const uint32_t *__restrict__ rp,
                                            const uint32_t *__restrict__ ci, const float *__restrict__ val,
                                            const SweepArgs &a, uint32_t gw, uint32_t warps)
{
    const int lane = threadIdx.x & (kLanes - 1);
    const uint32_t sub = (threadIdx.x & 31) / kLanes;  // row within the warp's group
    auto gx = [&](uint32_t c) { return sweep_x<SRC, COH>(a, c); };
    for (uint32_t base = gw * (32 / kLanes); base < n; base += warps * (32 / kLanes)) {
        const uint32_t row = base + sub;
        const bool valid = row < n;
        const float acc = csr_row_dot(rp, ci, val, row, valid, lane, gx);
        if (lane == 0 && valid) {
            const float res = ldv<COH>(a.b + row) - acc;
            a.out[row] = OUT == kOutRes ? res : fmaf(a.dw[row], res, sweep_x<SRC, COH>(a, row));
        }
    }
}

template <int SRC, int OUT>
__global__ void __launch_bounds__(kBlock) k_amg_coarse(uint32_t n, const uint32_t *__restrict__ rp,
                                                       const uint32_t *__restrict__ ci, const float *__restrict__ val,
                                                       SweepArgs a, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    if (SRC == kSrcXCorrK) kc_coefficients(a.kc, a.s, a.s2);
    coarse_rows<SRC, OUT>(n, rp, ci, val, a, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                          (gridDim.x * blockDim.x) >> 5);
}

// Residual and restriction in one pass over a coarse level: b_c[I] = sum over the aggregate's rows i
// of (b_i - (A xs)_i), and x0_c[I] = dw_c[I] b_c[I].  One warp per aggregate: eight row slots of four
// lanes, a slot taking every eighth row of the aggregate and its four lanes every fourth entry of the
// row (indexes and values loaded a chunk ahead of the gathers); a fixed shuffle tree adds the lanes.
// The aggregates of one restriction, warp gw of warps; the restricted residual of aggregate I goes
// to bc[I] (and x0c[I] = dwc[I] bc[I] when x0c is given).
template <bool COH = false>
__device__ __forceinline__ void res_restrict_rows(uint32_t nc, const uint32_t *__restrict__ ptr,
                                                  const uint32_t *__restrict__ rows, const uint32_t *__restrict__ rp,
                                                  const uint32_t *__restrict__ ci, const float *__restrict__ val,
                                                  const float *b, const float *xs, const float *__restrict__ dwc,
                                                  float *bc, float *x0c, uint32_t gw, uint32_t warps)
{
    const int lane = threadIdx.x & 31, slot = lane >> 2, q = lane & 3;
    for (uint32_t I = gw; I < nc; I += warps) {
        float part = 0.f;
        const uint32_t k1 = ptr[I + 1];
        for (uint32_t k = ptr[I] + slot; k < k1; k += 8) {
            const uint32_t row = rows[k];
            const uint32_t end = rp[row + 1];
            float acc = 0.f;
            for (uint32_t j0 = rp[row] + q; j0 < end; j0 += 4 * kChunk) {
                uint32_t c[kChunk];
                float v[kChunk], x[kChunk];
#pragma unroll
                for (int t = 0; t < kChunk; t++) {
                    const bool ok = j0 + 4 * t < end;
                    c[t] = ok ? ci[j0 + 4 * t] : row;
                    v[t] = ok ? val[j0 + 4 * t] : 0.f;
                }
#pragma unroll
                for (int t = 0; t < kChunk; t++) x[t] = v[t] != 0.f ? ldv<COH>(xs + c[t]) : 0.f;
#pragma unroll
                for (int t = 0; t < kChunk; t++) acc = fmaf(v[t], x[t], acc);
            }
            part += (q == 0 ? ldv<COH>(b + row) : 0.f) - acc;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) {
            bc[I] = part;
            if (x0c) x0c[I] = dwc[I] * part;
        }
    }
}

__global__ void __launch_bounds__(kBlock) k_amg_res_restrict(uint32_t nc, const uint32_t *__restrict__ ptr,
                                                             const uint32_t *__restrict__ rows,
                                                             const uint32_t *__restrict__ rp,
                                                             const uint32_t *__restrict__ ci,
                                                             const float *__restrict__ val,
                                                             const float *__restrict__ b,
                                                             const float *__restrict__ xs,
                                                             const float *__restrict__ dwc, float *__restrict__ bc,
                                                             float *__restrict__ x0c, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    res_restrict_rows(nc, ptr, rows, rp, ci, val, b, xs, dwc, bc, x0c, (blockIdx.x * blockDim.x + threadIdx.x) >> 5,
                      (gridDim.x * blockDim.x) >> 5);
}

// k_amg_kc_r2 folded into the restriction that follows it (one sweep per side): the K-cycle's second
// right-hand side r2 = b - a1 v1 and its first smoothing step x1 = dw r2 are formed where the
// restriction reads them -- for the gathered columns on the fly, for the aggregate's own rows also
// stored (each row belongs to one aggregate) for the cycle's later steps.  The same expressions as
// k_amg_kc_r2, so the same bits.
__global__ void __launch_bounds__(kBlock) k_amg_res_restrict_kc(uint32_t nc, const uint32_t *__restrict__ ptr,
                                                                const uint32_t *__restrict__ rows,
                                                                const uint32_t *__restrict__ rp,
                                                                const uint32_t *__restrict__ ci,
                                                                const float *__restrict__ val,
                                                                const float *__restrict__ b,
                                                                const float *__restrict__ v1,
                                                                const double *__restrict__ sc,
                                                                const float *__restrict__ dw,
                                                                const float *__restrict__ dwc, float *__restrict__ bc,
                                                                float *__restrict__ x0c, float *__restrict__ r2,
                                                                float *__restrict__ x1, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    const double d1 = sc[0];
    const float a1 = d1 > 0.0 ? float(sc[1] / d1) : 0.f;
    const int lane = threadIdx.x & 31, slot = lane >> 2, q = lane & 3;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; I < nc; I += warps) {
        float part = 0.f;
        const uint32_t k1 = ptr[I + 1];
        for (uint32_t k = ptr[I] + slot; k < k1; k += 8) {
            const uint32_t row = rows[k];
            const uint32_t end = rp[row + 1];
            float acc = 0.f;
            for (uint32_t j0 = rp[row] + q; j0 < end; j0 += 4 * kChunk) {
                uint32_t c[kChunk];
                float v[kChunk], x[kChunk];
#pragma unroll
                for (int t = 0; t < kChunk; t++) {
                    const bool ok = j0 + 4 * t < end;
                    c[t] = ok ? ci[j0 + 4 * t] : row;
                    v[t] = ok ? val[j0 + 4 * t] : 0.f;
                }
#pragma unroll
                for (int t = 0; t < kChunk; t++) x[t] = v[t] != 0.f ? dw[c[t]] * fmaf(-a1, v1[c[t]], b[c[t]]) : 0.f;
#pragma unroll
                for (int t = 0; t < kChunk; t++) acc = fmaf(v[t], x[t], acc);
            }
            float r = 0.f;
            if (q == 0) {
                r = fmaf(-a1, v1[row], b[row]);
                r2[row] = r;
                x1[row] = dw[row] * r;
            }
            part += r - acc;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) {
            bc[I] = part;
            x0c[I] = dwc[I] * part;
        }
    }
}

// The bottom of the hierarchy in one CTA: the cycle on the last smoothed level l (at most
// kBottomRows rows), whose next level is inverted densely -- pre-smoothing (two sweeps), residual and
// restriction into shared memory, the dense coarse solve, the corrected post-smoothing.  Same
// arithmetic as the separate kernels; __syncthreads orders the phases.
constexpr uint32_t kBottomRows = 1024;
constexpr int kBottomThreads = 1024;
struct BottomArgs {
    uint32_t n, nc;
    const uint32_t *rp, *ci, *agg, *ptr, *rows;
    const float *val, *dw, *inv;
    const float *b;
    float *x1, *x2, *out;
    float s;
};
// Words of shared memory the staged form needs (matrix, aggregate lists and the level's vectors).
inline size_t bottom_stage_words(uint32_t n, uint32_t nc, uint64_t nnz) { return size_t(n) * 7 + 2 * nnz + nc + 8; }
constexpr size_t kBottomStageBytes = 160 * 1024;

// STAGE: the level's matrix, aggregate lists, diagonal weights and vectors are first copied into
// shared memory by the whole CTA (the static parts before waiting on the previous kernel, so the
// copy overlaps its tail), and every phase then reads shared memory instead of chaining L2 round
// trips.  Same arithmetic either way.
template <int SWEEPS, bool STAGE>
__global__ void __launch_bounds__(kBottomThreads) k_amg_bottom(BottomArgs B, const CgState *st)
{
    extern __shared__ __align__(16) uint32_t stage[];
    if (STAGE) {
        const uint32_t n = B.n, nc = B.nc, nnz = B.rp[n] - B.rp[0], r0 = B.rp[0];
        uint32_t *rp = stage, *ci = rp + n + 1, *agg = ci + nnz, *ptr = agg + n, *rows = ptr + nc + 1;
        float *val = reinterpret_cast<float *>(rows + n), *dw = val + nnz, *b = dw + n, *x1 = b + n, *x2 = x1 + n;
        for (uint32_t i = threadIdx.x; i <= n; i += blockDim.x) rp[i] = B.rp[i] - r0;
        for (uint32_t j = threadIdx.x; j < nnz; j += blockDim.x) {
            ci[j] = B.ci[r0 + j];
            val[j] = B.val[r0 + j];
        }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            agg[i] = B.agg[i];
            rows[i] = B.rows[i];
            dw[i] = B.dw[i];
        }
        for (uint32_t i = threadIdx.x; i <= nc; i += blockDim.x) ptr[i] = B.ptr[i];
        pdl_wait();
        pdl_release();
        if (st && st->done) return;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            b[i] = B.b[i];
            x1[i] = B.x1[i];
        }
        __syncthreads();
        B.rp = rp;
        B.ci = ci;
        B.agg = agg;
        B.ptr = ptr;
        B.rows = rows;
        B.val = val;
        B.dw = dw;
        B.b = b;
        B.x1 = x1;
        B.x2 = x2;
    } else {
        pdl_wait();
        pdl_release();
        if (st && st->done) return;
    }
    __shared__ float sb[kAmgCoarsest], se[kAmgCoarsest];
    const uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    float *b = const_cast<float *>(B.b);
    const float *xs = B.x1;
    if (SWEEPS == 2) {
        SweepArgs a{b, B.dw, B.x1, nullptr, nullptr, 0.f, B.x2};
        coarse_rows<kSrcX, kOutSmooth>(B.n, B.rp, B.ci, B.val, a, w, nw);
        __syncthreads();
        xs = B.x2;
    }
    res_restrict_rows(B.nc, B.ptr, B.rows, B.rp, B.ci, B.val, B.b, xs, nullptr, sb, nullptr, w, nw);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (uint32_t i = w; i < B.nc; i += nw) {
        float v[kAmgCoarsest / 32];
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            v[t] = j < B.nc ? B.inv[size_t(i) * B.nc + j] : 0.f;
        }
        float acc = 0.f;
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            if (j < B.nc) acc = fmaf(v[t], sb[j], acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) se[i] = acc;
    }
    __syncthreads();
    SweepArgs u{b, B.dw, const_cast<float *>(xs), se, B.agg, B.s, SWEEPS == 2 ? B.x1 : B.out};
    coarse_rows<kSrcXCorr, kOutSmooth>(B.n, B.rp, B.ci, B.val, u, w, nw);
    if (SWEEPS == 2) {
        __syncthreads();
        SweepArgs u2{b, B.dw, B.x1, nullptr, nullptr, 0.f, B.out};
        coarse_rows<kSrcX, kOutSmooth>(B.n, B.rp, B.ci, B.val, u2, w, nw);
    }
}

// ---- K-cycle: two flexible-CG steps on a coarse level (Notay's K-cycle) ----
// v = A c (CSR, kLanes lanes per row), with the dot products c.v, c.y1 and (y2 given) c.y2 reduced
// over the grid into sc[o0], sc[o1], sc[o2].
template <int NDOT>
__global__ void __launch_bounds__(kBlock) k_amg_kc_spmv(uint32_t n, const uint32_t *__restrict__ rp,
                                                        const uint32_t *__restrict__ ci, const float *__restrict__ val,
                                                        const float *__restrict__ c, float *__restrict__ v,
                                                        const float *__restrict__ y1, const float *__restrict__ y2,
                                                        double *partials, unsigned int *ticket, double *sc, int o0,
                                                        int o1, int o2, const CgState *st)
{
    pdl_wait();
    pdl_release();
    __shared__ double sh[3 * 32];
    if (st && st->done) return;
    const int lane = threadIdx.x & (kLanes - 1);
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t sub = (threadIdx.x & 31) / kLanes;
    Dot2 d0, d1, d2;
    auto gx = [&](uint32_t col) { return c[col]; };
    for (uint32_t base = gw * (32 / kLanes); base < n; base += warps * (32 / kLanes)) {
        const uint32_t row = base + sub;
        const float acc = csr_row_dot(rp, ci, val, row, row < n, lane, gx);
        if (lane == 0 && row < n) {
            v[row] = acc;
            const float ci_ = c[row];
            d0.add_prod(ci_, acc);
            d1.add_prod(ci_, y1[row]);
            if (NDOT == 3) d2.add_prod(ci_, y2[row]);
        }
    }
    double accd[3] = {d0.value(), d1.value(), d2.value()};
    double tot[3];
    if (grid_sum<3>(accd, partials, ticket, sh, tot) && threadIdx.x == 0) {
        sc[o0] = tot[0];
        sc[o1] = tot[1];
        if (NDOT == 3) sc[o2] = tot[2];
    }
}

// r2 = b - alpha1 v1 with alpha1 = (c1.b) / (c1.v1); x1 = dw r2 (the next cycle's first smoothing step).
__global__ void k_amg_kc_r2(uint32_t n, const float *__restrict__ b, const float *__restrict__ v1,
                            const double *__restrict__ sc, const float *__restrict__ dw, float *__restrict__ r2,
                            float *__restrict__ x1, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    const double d1 = sc[0];
    const float a1 = d1 > 0.0 ? float(sc[1] / d1) : 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float r = fmaf(-a1, v1[i], b[i]);
        r2[i] = r;
        x1[i] = dw[i] * r;
    }
}

// b_c[I] = sum of r over the aggregate's rows (ascending order), and the coarse level's first
// smoothing step x0_c = dw_c b_c.
__global__ void k_amg_restrict(uint32_t nc, const uint32_t *__restrict__ ptr, const uint32_t *__restrict__ rows,
                               const float *__restrict__ r, const float *__restrict__ dwc, float *__restrict__ bc,
                               float *__restrict__ x0c, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    for (uint32_t I = blockIdx.x * blockDim.x + threadIdx.x; I < nc; I += gridDim.x * blockDim.x) {
        float s = 0.f;
        const uint32_t beg = ptr[I], end = ptr[I + 1];
        for (uint32_t k0 = beg; k0 < end; k0 += 8) {  // indexes first, then the gathers (in order)
            uint32_t ix[8];
            float v[8];
#pragma unroll
            for (int t = 0; t < 8; t++) ix[t] = k0 + t < end ? rows[k0 + t] : 0u;
#pragma unroll
            for (int t = 0; t < 8; t++) v[t] = k0 + t < end ? r[ix[t]] : 0.f;
#pragma unroll
            for (int t = 0; t < 8; t++)
                if (k0 + t < end) s += v[t];
        }
        bc[I] = s;
        x0c[I] = dwc[I] * s;
    }
}

// e = inv b on the coarsest level (dense, one CTA).
__global__ void k_amg_dense_apply(uint32_t n, const float *__restrict__ inv, const float *__restrict__ b,
                                  float *__restrict__ e, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    __shared__ float sb[kAmgCoarsest];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sb[i] = b[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t i = warp; i < n; i += nw) {
        float v[kAmgCoarsest / 32];
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            v[t] = j < n ? inv[size_t(i) * n + j] : 0.f;
        }
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            if (j < n) s = fmaf(v[t], sb[j], s);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) e[i] = s;
    }
}

// Single-level fallbacks (a matrix with no coarse level): z = inv r when the matrix itself is
// small enough to invert densely, else one damped-Jacobi step z = dw r; then r^T z.
__global__ void k_amg_jacobi(uint32_t n, const float *__restrict__ dw, const float *__restrict__ r,
                             float *__restrict__ z, const CgState *st)
{
    pdl_wait();
    pdl_release();
    if (st && st->done) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = dw[i] * r[i];
}

__global__ void k_amg_rz(uint32_t n, const float *__restrict__ r, const float *__restrict__ z, const float *qv,
                         double *partials, unsigned int *ticket, CgState *st, int mode, double *rz_out)
{
    pdl_wait();
    pdl_release();
    __shared__ double sh[64];
    if (st && st->done) return;
    Dot2 rz, qz;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        rz.add_prod(r[i], z[i]);
        if (qv) qz.add_prod(qv[i], z[i]);
    }
    double acc[2] = {rz.value(), qz.value()};
    double tot[2];
    if (grid_sum<2>(acc, partials, ticket, sh, tot) && threadIdx.x == 0) amg_finalize(st, tot[0], tot[1], mode, rz_out);
}

// ---- the coarse levels of one cycle in one persistent kernel ----
// Below kCoarsePersistRows rows a level's kernels are chains of a few L2 round trips each; launched
// one by one, the launch and the wait for the predecessor cost as much as the work.  From the first
// level at or below that size, solve_level's whole recursion (cycles, K-cycle steps, the dense coarse
// solve) runs as one cooperative launch: the host records the phases it would launch, in order, as a
// program (CoarsePhase), and the kernel runs them with a grid barrier between phases.  Each phase does
// what the separate kernel does, with the same per-row (per-aggregate) arithmetic; the K-cycle dot
// products keep the separate kernel's grid as virtual blocks and its per-block partial sums, and the
// last CTA at the barrier adds the partials in the separate kernel's order (grid_sum), so the cycle
// gives the same bits either way.  The bottom level's cycle runs as its separate phases (restriction,
// dense solve, corrected sweep), the same arithmetic as the fused one-CTA kernel.
#ifndef RSG_COARSE_CTAS_PER_SM
#define RSG_COARSE_CTAS_PER_SM 1
#endif
constexpr int kCoarseCtasPerSm = RSG_COARSE_CTAS_PER_SM;
constexpr uint32_t kCoarsePersistRows = 32768;

enum CoarseOp : uint32_t {
    CP_SWEEP_X = 0,   // coarse_rows<kSrcX, kOutSmooth>
    CP_SWEEP_CORR,    // coarse_rows<kSrcXCorr, kOutSmooth>
    CP_SWEEP_CORRK,   // coarse_rows<kSrcXCorrK, kOutSmooth> (coefficients from a.kc)
    CP_RES_RESTRICT,  // res_restrict_rows: a.b, a.xs -> bc, x0c
    CP_DENSE,         // dense coarse solve: a.out = inv a.b
    CP_KC_SPMV2,      // K-cycle: v = A c, sc[o0] = c.v, sc[o1] = c.y1
    CP_KC_SPMV3,      //          ... and sc[o2] = c.y2
    CP_KC_R2,         // K-cycle: r2 = a.b - a1 v1 (a1 from sc), x1 = dw r2
};

struct CoarsePhase {
    uint32_t op, n, nc, vgrid;          // rows; coarse rows (restriction); the K-cycle SpMV's grid
    const uint32_t *rp, *ci;            // the level's matrix
    const float *val;
    const uint32_t *ptr, *rows;         // restriction: aggregate lists
    const float *dwc;                   // restriction: the coarse level's weights
    float *bc, *x0c;                    // restriction outputs; K-cycle r2: r2 and x1
    const float *inv;                   // dense solve
    const float *c, *y1, *y2;           // K-cycle SpMV operands (r2: c = v1)
    float *v;                           // K-cycle SpMV output
    double *sc;                         // K-cycle scalars of the level
    int32_t o0, o1, o2, pad;
    SweepArgs a;
};

__device__ __forceinline__ void dense_rows(uint32_t n, const float *__restrict__ inv, const float *b, float *e,
                                           float *sb, uint32_t gw, uint32_t warps)
{
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) sb[i] = __ldcg(b + i);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (uint32_t i = gw; i < n; i += warps) {
        float v[kAmgCoarsest / 32];
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            v[t] = j < n ? inv[size_t(i) * n + j] : 0.f;
        }
        float s = 0.f;
#pragma unroll
        for (int t = 0; t < int(kAmgCoarsest / 32); t++) {
            const uint32_t j = uint32_t(lane) + 32u * uint32_t(t);
            if (j < n) s = fmaf(v[t], sb[j], s);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) e[i] = s;
    }
}

// k_amg_kc_spmv's work for its virtual blocks vb = blockIdx.x, blockIdx.x + gridDim.x, ... < vgrid:
// the same rows per thread, the same compensated sums, the block's partials at part[3 vb + k].
template <int NDOT>
__device__ __forceinline__ void kc_spmv_blocks(const CoarsePhase &p, double *part, double *sh)
{
    const int lane = threadIdx.x & (kLanes - 1);
    const uint32_t sub = (threadIdx.x & 31) / kLanes, vwarps = (p.vgrid * blockDim.x) >> 5;
    const float *c = p.c;
    auto gx = [&](uint32_t col) { return __ldcg(c + col); };
    for (uint32_t vb = blockIdx.x; vb < p.vgrid; vb += gridDim.x) {
        const uint32_t gw = (vb * blockDim.x + threadIdx.x) >> 5;
        Dot2 d0, d1, d2;
        for (uint32_t base = gw * (32 / kLanes); base < p.n; base += vwarps * (32 / kLanes)) {
            const uint32_t row = base + sub;
            const float acc = csr_row_dot(p.rp, p.ci, p.val, row, row < p.n, lane, gx);
            if (lane == 0 && row < p.n) {
                p.v[row] = acc;
                const float ci_ = __ldcg(c + row);
                d0.add_prod(ci_, acc);
                d1.add_prod(ci_, __ldcg(p.y1 + row));
                if (NDOT == 3) d2.add_prod(ci_, __ldcg(p.y2 + row));
            }
        }
        double accd[3] = {d0.value(), d1.value(), d2.value()};
        block_sum<3>(accd, sh);
        if (threadIdx.x == 0)
#pragma unroll
            for (int k = 0; k < 3; k++) part[size_t(vb) * 3 + k] = accd[k];
    }
}

__global__ void __launch_bounds__(kBlock) k_amg_coarse_persist(const CoarsePhase *prog, uint32_t n_phases,
                                                               double *part, unsigned int *bar, const CgState *st,
                                                               unsigned int *err)
{
    __shared__ __align__(16) unsigned char ph_raw[sizeof(CoarsePhase)];
    __shared__ double sh[3 * 32];
    __shared__ float sb[kAmgCoarsest];
    if (st && st->done) return;  // written before this launch only: the same answer in every CTA
    const CoarsePhase &p = *reinterpret_cast<const CoarsePhase *>(ph_raw);
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = 0; i < n_phases; i++) {
        __syncthreads();
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(prog + i);
            uint32_t *dst = reinterpret_cast<uint32_t *>(ph_raw);
            for (uint32_t w = threadIdx.x; w < uint32_t(sizeof(CoarsePhase) / 4); w += blockDim.x) dst[w] = src[w];
        }
        __syncthreads();
        const uint32_t op = p.op;
        if (op == CP_SWEEP_X) {
            coarse_rows<kSrcX, kOutSmooth, true>(p.n, p.rp, p.ci, p.val, p.a, gw, warps);
        } else if (op == CP_SWEEP_CORR) {
            coarse_rows<kSrcXCorr, kOutSmooth, true>(p.n, p.rp, p.ci, p.val, p.a, gw, warps);
        } else if (op == CP_SWEEP_CORRK) {
            SweepArgs a = p.a;
            kc_coefficients<true>(a.kc, a.s, a.s2);
            coarse_rows<kSrcXCorrK, kOutSmooth, true>(p.n, p.rp, p.ci, p.val, a, gw, warps);
        } else if (op == CP_RES_RESTRICT) {
            res_restrict_rows<true>(p.nc, p.ptr, p.rows, p.rp, p.ci, p.val, p.a.b, p.a.xs, p.dwc, p.bc, p.x0c, gw,
                                    warps);
        } else if (op == CP_DENSE) {
            dense_rows(p.n, p.inv, p.a.b, p.a.out, sb, gw, warps);
        } else if (op == CP_KC_SPMV2 || op == CP_KC_SPMV3) {
            if (op == CP_KC_SPMV2) kc_spmv_blocks<2>(p, part, sh);
            else kc_spmv_blocks<3>(p, part, sh);
            // the last CTA to arrive adds the partials in grid_sum's order and stores the scalars
            auto last = [&]() {
                double acc[3] = {0.0, 0.0, 0.0};
                for (uint32_t b = threadIdx.x; b < p.vgrid; b += blockDim.x)
#pragma unroll
                    for (int k = 0; k < 3; k++) acc[k] += __ldcg(&part[size_t(b) * 3 + k]);
                block_sum<3>(acc, sh);
                if (threadIdx.x == 0) {
                    p.sc[p.o0] = acc[0];
                    p.sc[p.o1] = acc[1];
                    if (op == CP_KC_SPMV3) p.sc[p.o2] = acc[2];
                }
            };
            if (!grid_barrier(bar, err, last)) return;
            continue;
        } else if (op == CP_KC_R2) {
            const double d1 = __ldcg(p.sc), t1 = __ldcg(p.sc + 1);
            const float a1 = d1 > 0.0 ? float(t1 / d1) : 0.f;
            for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < p.n; k += gridDim.x * blockDim.x) {
                const float r = fmaf(-a1, __ldcg(p.c + k), __ldcg(p.a.b + k));
                p.bc[k] = r;
                p.x0c[k] = p.a.dw[k] * r;
            }
        }
        if (i + 1 < n_phases && !grid_barrier(bar, err)) return;
    }
}

// ---------------------------------------------------------------- host: set-up --------------

rsg_status read_flags(rsg_context *ctx, AmgHierarchy *H, int count)
{
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(H->flags_h, H->flags, count * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                        ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return RSG_OK;
}

rsg_status read_u32(rsg_context *ctx, AmgHierarchy *H, const uint32_t *dev, uint32_t *host)
{
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(H->flags_h + 8, dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *host = H->flags_h[8];
    return RSG_OK;
}

// Aggregates of level l (sets F.agg, F.agg_ptr, F.agg_rows and the next level's size).
rsg_status build_aggregates(rsg_context *ctx, AmgHierarchy *H, AmgLevel &F, uint32_t *n_coarse, uint32_t *max_entries,
                            uint32_t *max_size)
{
    const uint32_t n = F.n;
    const int g = grid_rows(n);
    cudaStream_t s = ctx->stream;
    if (!H->T.ensure(n) || !H->M1.ensure(n) || !H->smask.ensure(F.nnz + 1) ||
        !H->u1.ensure(size_t(n) + 1) || !H->u2.ensure(size_t(n) + 1) || !H->u3.ensure(size_t(n) + 1) ||
        !F.agg.ensure(n))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: set-up workspace");
    count_launch();
    k_amg_strength<<<grid_groups(n), kBlock, 0, s>>>(n, F.rp, F.ci, F.val, F.diag.p, kAmgTheta, H->smask.p);
    count_launch();
    k_amg_mis_init<<<g, kBlock, 0, s>>>(n, H->T.p);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    if (n <= kMisCtaRows) {  // a small level: every round in one CTA, one synchronisation
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->flags + 10, 0, 2 * sizeof(unsigned int), s));
        count_launch();
        k_amg_mis_cta<<<1, kMisCtaThreads, 0, s>>>(n, F.rp, F.ci, H->smask.p, H->T.p, H->M1.p, H->flags + 10);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        RSG_TRY(read_flags(ctx, H, 12));
        if (H->flags_h[11] != 0) return set_error(ctx, RSG_ERR_CUDA, "amg: independent set did not converge");
        H->mis_rounds += H->flags_h[10];
    } else {
        // synchronous rounds until no node is undecided: launched in batches of kRoundBatch with one
        // undecided-node counter per round (rounds after the last one needed return at once); the host
        // reads the batch's last counter
        constexpr uint32_t kRoundBatch = 8;
        if (!H->rounds.ensure(kMisMaxRounds)) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: round counters");
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->rounds.p, 0, kMisMaxRounds * sizeof(unsigned int), s));
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->u3.p, 0, size_t(n) * sizeof(uint32_t), s));  // round stamps
        uint32_t round = 0;
        for (;;) {
            for (uint32_t k = 0; k < kRoundBatch; k++, round++) {
                const unsigned int *prev = round ? H->rounds.p + round - 1 : nullptr;
                count_launch();
                k_amg_nbmax<<<g, kBlock, 0, s>>>(n, F.rp, F.ci, H->smask.p, H->T.p, H->M1.p, H->u3.p, round, prev);
                count_launch();
                k_amg_mis_round2<<<g, kBlock, 0, s>>>(n, F.rp, F.ci, H->smask.p, H->M1.p, H->T.p, H->u3.p, round,
                                                      prev, H->rounds.p + round);
            }
            RSG_CHECK_CUDA(ctx, cudaGetLastError());
            RSG_TRY(read_u32(ctx, H, H->rounds.p + round - 1, &H->flags_h[0]));
            if (H->flags_h[0] == 0) break;
            if (round + kRoundBatch > kMisMaxRounds)
                return set_error(ctx, RSG_ERR_CUDA, "amg: independent set did not converge");
        }
        H->mis_rounds += round;
    }
    // root numbering, joins
    count_launch();
    k_amg_root_flags<<<g, kBlock, 0, s>>>(n, H->T.p, H->u1.p);
    RSG_TRY(scan_u32(ctx, H, H->u1.p, n, H->u2.p));
    count_launch();
    k_amg_join1<<<g, kBlock, 0, s>>>(n, F.rp, F.ci, H->smask.p, H->T.p, H->u2.p, H->u1.p);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->flags, 0, 4 * sizeof(unsigned int), s));
    count_launch();
    k_amg_join2<<<g, kBlock, 0, s>>>(n, F.rp, F.ci, H->smask.p, H->u1.p, F.agg.p, H->flags);
    // one synchronisation for the number of roots and the nodes left without an aggregate
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(H->flags_h + 8, H->u2.p + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RSG_TRY(read_flags(ctx, H, 2));
    uint32_t nc = H->flags_h[8];
    if (H->flags_h[1] > 0) {  // singletons for nodes without any strong path to a root
        count_launch();
        k_amg_unset_flags<<<g, kBlock, 0, s>>>(n, F.agg.p, H->u1.p);
        RSG_TRY(scan_u32(ctx, H, H->u1.p, n, H->u2.p));
        count_launch();
        k_amg_singletons<<<g, kBlock, 0, s>>>(n, nc, H->u2.p, F.agg.p);
        nc += H->flags_h[1];
    }
    // aggregate lists
    if (!F.agg_ptr.ensure(size_t(nc) + 1) || !F.agg_rows.ensure(n) || !H->u3.ensure(size_t(nc) + 1))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: aggregate lists");
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->u3.p, 0, size_t(nc) * sizeof(uint32_t), s));
    count_launch();
    k_amg_count<<<g, kBlock, 0, s>>>(n, F.agg.p, H->u3.p);
    RSG_TRY(scan_u32(ctx, H, H->u3.p, nc, F.agg_ptr.p));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->u3.p, 0, size_t(nc) * sizeof(uint32_t), s));
    count_launch();
    k_amg_fill<<<g, kBlock, 0, s>>>(n, F.agg.p, F.agg_ptr.p, H->u3.p, F.agg_rows.p);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->flags + 2, 0, 2 * sizeof(unsigned int), s));
    count_launch();
    k_amg_sort_agg<<<grid_rows(nc), kBlock, 0, s>>>(nc, F.agg_ptr.p, F.agg_rows.p, F.rp, H->u3.p, H->flags);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    RSG_TRY(read_flags(ctx, H, 4));
    *n_coarse = nc;
    *max_entries = H->flags_h[2];
    *max_size = H->flags_h[3];
    return RSG_OK;
}

// Coarse matrix C = P^T A P of level F into level Cl (F.agg_* and H->u3 = entries per coarse row).
rsg_status build_galerkin(rsg_context *ctx, AmgHierarchy *H, AmgLevel &F, AmgLevel &Cl, uint32_t nc, uint32_t emax,
                          uint32_t max_size)
{
    cudaStream_t s = ctx->stream;
    // staging offsets (one slot per fine entry)
    if (!H->u1.ensure(size_t(nc) + 1) || !H->u2.ensure(size_t(nc) + 1) || !H->tcol.ensure(F.nnz + 1) ||
        !H->tval.ensure(F.nnz + 1))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: Galerkin staging");
    RSG_TRY(scan_u32(ctx, H, H->u3.p, nc, H->u1.p));  // eoff
    uint32_t P = 32;
    while (P < emax) P <<= 1;
    // keys and values (16 bytes per padded slot), then the staging offsets of the aggregate's rows
    const size_t smem = size_t(P) * 16 + (size_t(max_size) + 1) * sizeof(uint32_t);
    // one warp per coarse row; rows with more distinct columns than the warp kernel keeps fall back to
    // the sorting kernel (one CTA per row) for the whole level
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->flags + 5, 0, sizeof(unsigned int), s));
    count_launch();
    k_amg_galerkin_warp<<<int(std::min<uint64_t>((nc + kGalWarps - 1) / kGalWarps, 65535ull * 8)), 32 * kGalWarps, 0,
                          s>>>(nc, F.agg_ptr.p, F.agg_rows.p, F.rp, F.ci, F.val, F.agg.p, H->u1.p, H->tcol.p,
                               H->tval.p, H->u2.p, H->flags);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    // coarse row pointer; one synchronisation for the coarse nnz and the overflow flag
    if (!Cl.own_rp.ensure(size_t(nc) + 1)) return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: coarse matrix");
    RSG_TRY(scan_u32(ctx, H, H->u2.p, nc, Cl.own_rp.p));
    RSG_CHECK_CUDA(ctx, cudaMemcpyAsync(H->flags_h + 9, Cl.own_rp.p + nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RSG_TRY(read_flags(ctx, H, 6));
    if (H->flags_h[5]) {
        cudaFuncSetAttribute(k_amg_galerkin, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        count_launch();
        k_amg_galerkin<<<nc, kGalThreads, smem, s>>>(nc, F.agg_ptr.p, F.agg_rows.p, F.rp, F.ci, F.val, F.agg.p,
                                                      H->u1.p, H->tcol.p, H->tval.p, H->u2.p);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
        RSG_TRY(scan_u32(ctx, H, H->u2.p, nc, Cl.own_rp.p));
        RSG_TRY(read_u32(ctx, H, Cl.own_rp.p + nc, &H->flags_h[9]));
    }
    const uint32_t nnz = H->flags_h[9];
    if (!Cl.own_ci.ensure(size_t(nnz) + 1) || !Cl.own_val.ensure(size_t(nnz) + 1) || !Cl.own_val32.ensure(size_t(nnz) + 1))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: coarse matrix");
    count_launch();
    k_amg_compact<<<grid_groups(nc), kBlock, 0, s>>>(nc, H->u1.p, H->u2.p, Cl.own_rp.p, H->tcol.p, H->tval.p,
                                                   Cl.own_ci.p, Cl.own_val.p, Cl.own_val32.p);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    Cl.n = nc;
    Cl.nnz = nnz;
    Cl.rp = Cl.own_rp.p;
    Cl.ci = Cl.own_ci.p;
    Cl.val = Cl.own_val.p;
    Cl.val32 = Cl.own_val32.p;
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

rsg_status level_vectors(rsg_context *ctx, AmgLevel &l, bool k_buffers)
{
    if (!l.diag.ensure(l.n) || !l.dw.ensure(l.n) || !l.b.ensure(l.n) || !l.r.ensure(l.n) || !l.x1.ensure(l.n) ||
        !l.x2.ensure(l.n) || !l.e.ensure(l.n))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: level vectors");
    if (k_buffers && (!l.c1.ensure(l.n) || !l.c2.ensure(l.n) || !l.v1.ensure(l.n) || !l.v2.ensure(l.n) ||
                      !l.r2.ensure(l.n)))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: K-cycle vectors");
    count_launch();
    k_amg_diag<<<grid_rows(l.n), kBlock, 0, ctx->stream>>>(l.n, l.rp, l.ci, l.val, l.diag.p, l.dw.p);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}

}  // namespace

void amg_free(AmgHierarchy *H)
{
    if (!H) return;
    for (auto &l : H->L) {
        l.own_rp.release();
        l.own_ci.release();
        l.own_val.release();
        l.own_val32.release();
        l.diag.release();
        l.dw.release();
        l.agg.release();
        l.agg_ptr.release();
        l.agg_rows.release();
        l.b.release();
        l.r.release();
        l.x1.release();
        l.x2.release();
        l.e.release();
        l.c1.release();
        l.c2.release();
        l.v1.release();
        l.v2.release();
        l.r2.release();
    }
    H->coarse_inv.release();
    H->T.release();
    H->M1.release();
    H->smask.release();
    H->u1.release();
    H->u2.release();
    H->u3.release();
    H->scan_blocks.release();
    H->kc_part.release();
    H->persist_prog.release();
    H->persist_bar.release();
    H->kc_ticket.release();
    H->kc_sc.release();
    H->rounds.release();
    H->tcol.release();
    H->tval.release();
    if (H->flags) cudaFree(H->flags);
    if (H->flags_h) cudaFreeHost(H->flags_h);
    delete H;
}

void amg_release(void *h) { amg_free(static_cast<AmgHierarchy *>(h)); }

AmgHierarchy *amg_of(const rsg_csr *A) { return static_cast<AmgHierarchy *>(A->amg); }

namespace {
rsg_status build_persist(rsg_context *ctx, AmgHierarchy *H, bool want);
}  // namespace

rsg_status amg_setup(rsg_context *ctx, rsg_csr *A, bool persistent)
{
    const auto t0 = std::chrono::steady_clock::now();
    const uint32_t launches0 = t_launches;
    AmgHierarchy *H = amg_of(A);
    if (!H) {
        H = new AmgHierarchy;
        if (cudaMalloc(&H->flags, 16 * sizeof(unsigned int)) != cudaSuccess ||
            cudaMallocHost(&H->flags_h, 16 * sizeof(unsigned int)) != cudaSuccess || !H->kc_part.ensure(3 * kMaxGrid) ||
            !H->kc_ticket.ensure(1) || !H->kc_sc.ensure(8 * kAmgMaxLevels)) {
            amg_free(H);
            return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: counters");
        }
        A->amg = H;
        RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->kc_ticket.p, 0, sizeof(unsigned int), ctx->stream));
    }
    H->mis_rounds = 0;
    H->levels = 1;
    H->dense_coarsest = false;
    AmgLevel &L0 = H->L[0];
    L0.n = A->n;
    L0.nnz = A->nnz;
    L0.rp = A->rp;
    L0.ci = A->ci;
    L0.val = A->val;
    L0.val32 = A->val32;
    RSG_TRY(level_vectors(ctx, L0, false));
    while (H->levels < kAmgMaxLevels) {
        AmgLevel &F = H->L[H->levels - 1];
        if (F.n <= kAmgCoarsest) {
            H->dense_coarsest = true;
            break;
        }
        uint32_t nc = 0, emax = 0, max_size = 0;
        RSG_TRY(build_aggregates(ctx, H, F, &nc, &emax, &max_size));
        // stop when coarsening stalls or a coarse row would not fit the staging buffer
        if (nc == 0 || uint64_t(nc) * 10 > uint64_t(F.n) * 9 || emax > kAmgMaxEntries || max_size > kAmgMaxEntries)
            break;
        AmgLevel &Cl = H->L[H->levels];
        RSG_TRY(build_galerkin(ctx, H, F, Cl, nc, emax, max_size));
        RSG_TRY(level_vectors(ctx, Cl, H->levels <= kAmgKLevels));
        H->levels++;
    }
    AmgLevel &last = H->L[H->levels - 1];
    if (H->dense_coarsest) {
        if (!H->coarse_inv.ensure(size_t(kAmgCoarsest) * kAmgCoarsest))
            return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: coarse inverse");
        const size_t smem = size_t(last.n) * last.n * sizeof(double);
        cudaFuncSetAttribute(k_amg_dense_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        count_launch();
        k_amg_dense_inverse<<<1, 512, smem, ctx->stream>>>(last.n, last.rp, last.ci, last.val, H->coarse_inv.p);
        RSG_CHECK_CUDA(ctx, cudaGetLastError());
    }
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    H->seconds_setup = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    H->setup_launches = t_launches - launches0;
    RSG_TRY(build_persist(ctx, H, persistent));
    // launches of one cycle as the CG loop applies it, for one and two sweeps (dry runs: nothing launched)
    for (int nu = 1; nu <= 2; nu++) {
        const uint32_t c0 = t_launches;
        t_dry = true;
        const rsg_status st = amg_vcycle(ctx, A, H, nullptr, H->L[0].x1.p, nullptr, nullptr, nu, nullptr, nullptr,
                                         nullptr, 1, nullptr, true);
        t_dry = false;
        RSG_TRY(st);
        H->cycle_launches[nu - 1] = t_launches - c0;
    }
    return RSG_OK;
}

// ---------------------------------------------------------------- host: V-cycle -------------

namespace {

int coarse_grid(rsg_context *ctx, uint32_t n)
{
    const long long threads = (long long)n * kLanes;
    return std::max(1, std::min<int>(int((threads + kBlock - 1) / kBlock), ctx->num_sms * 8));
}

template <int RPW>
struct FineLaunch {
    Csr<float> M;
    Sell<float> S;
    int use_sell, grid;
    size_t smem;
};

template <int RPW, int SRC, int OUT, bool FINAL>
void fine_sweep(rsg_context *ctx, const FineLaunch<RPW> &f, const SweepArgs &a, const float *qv, double *partials,
                unsigned int *ticket, CgState *st, int mode, double *rz_out, bool pdl)
{
    amg_launch(ctx->stream, pdl, k_amg_fine<RPW, SRC, OUT, FINAL>, f.grid, kBlock, f.smem, f.M, f.S, f.use_sell, a, qv,
             partials, ticket, st, mode, rz_out);
}

// Coarse levels run on the whole GPU: CSR with kLanes lanes per row.  (A SELL-32 copy leaves one warp
// per 32 rows, too few warps for these levels: measured slower.  One thread-block cluster of 8 CTAs
// running all levels of up to 32k rows with cluster barriers between steps was slower still: 8 SMs
// lack the memory-level parallelism for the 276k-entry third level.)
template <int SRC, int OUT>
void coarse_sweep(rsg_context *ctx, const AmgLevel &l, const SweepArgs &a, const CgState *st, bool pdl)
{
    amg_launch(ctx->stream, pdl, k_amg_coarse<SRC, OUT>, coarse_grid(ctx, l.n), kBlock, 0, l.n, l.rp, l.ci, l.val32, a,
             st);
}

// Restriction of the finest level's residual (written by the fine sweep into r) to level 1's b and x0.
void down_restrict(rsg_context *ctx, const AmgHierarchy *H, int l, const CgState *st, bool pdl)
{
    const AmgLevel &F = H->L[l], &C = H->L[l + 1];
    amg_launch(ctx->stream, pdl, k_amg_restrict, grid_rows(C.n), kBlock, 0, C.n, (const uint32_t *)F.agg_ptr.p,
             (const uint32_t *)F.agg_rows.p, (const float *)F.r.p, (const float *)C.dw.p, C.b.p, C.x1.p, st);
}

bool k_level(const AmgHierarchy *H, int l) { return l >= 1 && l <= kAmgKLevels && l < H->levels - 1; }

// Scale of the prolongated correction from level l: the K-cycle's flexible-CG steps already scale it.
float corr_scale(const AmgHierarchy *H, int l, int sweeps)
{
    return k_level(H, l) ? 1.f : (sweeps == 2 ? kAmgScale2 : kAmgScale1);
}

void solve_level(rsg_context *ctx, const AmgHierarchy *H, int l, const float *b, float *e, int sweeps,
                 const CgState *st, bool pdl);

// The prolongated correction from coarse level c into SweepArgs: a K-cycle level's two flexible-CG
// directions with their coefficients, else the level's e scaled by s.
void set_correction(const AmgHierarchy *H, int c, int sweeps, SweepArgs &a)
{
    const AmgLevel &C = H->L[c];
    if (k_level(H, c)) {
        a.ec = C.c1.p;
        a.ec2 = C.c2.p;
        a.kc = H->kc_sc.p + 8 * c;
    } else {
        a.ec = C.e.p;
        a.s = sweeps == 2 ? kAmgScale2 : kAmgScale1;
    }
}

template <int OUT>
void coarse_sweep_corr(rsg_context *ctx, const AmgHierarchy *H, int l, SweepArgs a, int sweeps, const CgState *st,
                       bool pdl)
{
    const AmgLevel &F = H->L[l];
    a.agg = F.agg.p;
    set_correction(H, l + 1, sweeps, a);
    if (k_level(H, l + 1)) coarse_sweep<kSrcXCorrK, OUT>(ctx, F, a, st, pdl);
    else coarse_sweep<kSrcXCorr, OUT>(ctx, F, a, st, pdl);
}

// Residual of level l from iterate xs, restricted to the next level's b and x0 (one pass).
void res_restrict(rsg_context *ctx, const AmgHierarchy *H, int l, const float *b, const float *xs, const CgState *st,
                  bool pdl)
{
    const AmgLevel &F = H->L[l], &C = H->L[l + 1];
    const int g = std::max(1, std::min<int>(int((uint64_t(C.n) * 32 + kBlock - 1) / kBlock), ctx->num_sms * 8));
    amg_launch(ctx->stream, pdl, k_amg_res_restrict, g, kBlock, 0, C.n, (const uint32_t *)F.agg_ptr.p,
             (const uint32_t *)F.agg_rows.p, F.rp, F.ci, F.val32, b, xs, (const float *)C.dw.p, C.b.p, C.x1.p, st);
}

// Whether the cycle on level l runs as the one-CTA bottom kernel.
bool bottom_cycle(const AmgHierarchy *H, int l)
{
    return l + 1 == H->levels - 1 && H->dense_coarsest && H->L[l].n <= kBottomRows;
}

// One cycle on coarse level l >= 1: out ~ A_l^-1 b, with x0 = dw b already in x1 (written by the
// restriction): pre-smoothing, residual and restriction in one pass, the coarser levels, the
// prolongated correction fused into the first post-smoothing sweep.  With two sweeps x2 holds the
// pre-smoothed iterate.  kc_b (one sweep, not the bottom cycle): b is the K-cycle's r2 = kc_b - a1 v1,
// still to be formed together with x1 by the restriction (k_amg_res_restrict_kc).
void cycle(rsg_context *ctx, const AmgHierarchy *H, int l, const float *b, float *out, int sweeps, const CgState *st,
           bool pdl, const float *kc_b = nullptr)
{
    const AmgLevel &F = H->L[l], &C = H->L[l + 1];
    float *bb = const_cast<float *>(b);
    if (kc_b) {
        const int g = std::max(1, std::min<int>(int((uint64_t(C.n) * 32 + kBlock - 1) / kBlock), ctx->num_sms * 8));
        amg_launch(ctx->stream, pdl, k_amg_res_restrict_kc, g, kBlock, 0, C.n, (const uint32_t *)F.agg_ptr.p,
                   (const uint32_t *)F.agg_rows.p, F.rp, F.ci, F.val32, kc_b, (const float *)F.v1.p,
                   (const double *)(H->kc_sc.p + 8 * l), (const float *)F.dw.p, (const float *)C.dw.p, C.b.p, C.x1.p,
                   F.r2.p, F.x1.p, st);
        solve_level(ctx, H, l + 1, C.b.p, C.e.p, sweeps, st, pdl);
        SweepArgs u1{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, out};
        coarse_sweep_corr<kOutSmooth>(ctx, H, l, u1, sweeps, st, pdl);
        return;
    }
    if (bottom_cycle(H, l)) {
        const BottomArgs B{F.n, C.n, F.rp, F.ci, F.agg.p, F.agg_ptr.p, F.agg_rows.p, F.val32, F.dw.p, H->coarse_inv.p,
                           b, F.x1.p, F.x2.p, out, sweeps == 2 ? kAmgScale2 : kAmgScale1};
        const size_t sm = bottom_stage_words(F.n, C.n, F.nnz) * sizeof(uint32_t);
        if (sm <= kBottomStageBytes) {
            auto k = sweeps == 2 ? k_amg_bottom<2, true> : k_amg_bottom<1, true>;
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kBottomStageBytes));
            amg_launch(ctx->stream, pdl, k, 1, kBottomThreads, sm, B, st);
        } else {
            amg_launch(ctx->stream, pdl, sweeps == 2 ? k_amg_bottom<2, false> : k_amg_bottom<1, false>, 1,
                       kBottomThreads, 0, B, st);
        }
        return;
    }
    if (sweeps == 2) {
        SweepArgs a1{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, F.x2.p};
        coarse_sweep<kSrcX, kOutSmooth>(ctx, F, a1, st, pdl);
        res_restrict(ctx, H, l, b, F.x2.p, st, pdl);
    } else {
        res_restrict(ctx, H, l, b, F.x1.p, st, pdl);
    }
    solve_level(ctx, H, l + 1, C.b.p, C.e.p, sweeps, st, pdl);
    if (sweeps == 2) {
        SweepArgs u1{bb, F.dw.p, F.x2.p, nullptr, nullptr, 0.f, F.x1.p};
        coarse_sweep_corr<kOutSmooth>(ctx, H, l, u1, sweeps, st, pdl);
        SweepArgs u2{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, out};
        coarse_sweep<kSrcX, kOutSmooth>(ctx, F, u2, st, pdl);
    } else {
        SweepArgs u1{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, out};
        coarse_sweep_corr<kOutSmooth>(ctx, H, l, u1, sweeps, st, pdl);
    }
}

// e ~ A_l^-1 b on coarse level l (x0 = dw b already in x1): the dense inverse on the last level, one
// cycle on an ordinary level.  On a K-cycle level two flexible-CG steps preconditioned by the cycle
// leave their directions in c1, c2 and the scalars in the level's kc_sc slots; the caller's
// prolongation combines them (e is not written).
void coarse_persist(rsg_context *ctx, const AmgHierarchy *H, int sweeps, const CgState *st);

void solve_level(rsg_context *ctx, const AmgHierarchy *H, int l, const float *b, float *e, int sweeps,
                 const CgState *st, bool pdl)
{
    const AmgLevel &F = H->L[l];
    if (l == H->persist_level && b == F.b.p && e == F.e.p) {  // the recorded program of this visit
        coarse_persist(ctx, H, sweeps, st);
        return;
    }
    if (l == H->levels - 1) {
        if (H->dense_coarsest) {
            amg_launch(ctx->stream, pdl, k_amg_dense_apply, 1, 1024, 0, F.n, (const float *)H->coarse_inv.p, b, e, st);
        } else {  // coarsening stalled above the dense limit: nine damped-Jacobi sweeps from zero
            float *src = F.x1.p, *dst = F.x2.p, *bb = const_cast<float *>(b);
            for (int k = 0; k < 7; k++) {
                SweepArgs a{bb, F.dw.p, src, nullptr, nullptr, 0.f, dst};
                coarse_sweep<kSrcX, kOutSmooth>(ctx, F, a, st, pdl);
                std::swap(src, dst);
            }
            SweepArgs a{bb, F.dw.p, src, nullptr, nullptr, 0.f, e};
            coarse_sweep<kSrcX, kOutSmooth>(ctx, F, a, st, pdl);
        }
        return;
    }
    if (!k_level(H, l)) {
        cycle(ctx, H, l, b, e, sweeps, st, pdl);
        return;
    }
    double *sc = H->kc_sc.p + 8 * l;
    const int gs = coarse_grid(ctx, F.n), gv = grid_rows(F.n);
    cycle(ctx, H, l, b, F.c1.p, sweeps, st, pdl);
    amg_launch(ctx->stream, pdl, k_amg_kc_spmv<2>, gs, kBlock, 0, F.n, F.rp, F.ci, F.val32, (const float *)F.c1.p,
             F.v1.p, b, (const float *)nullptr, H->kc_part.p, H->kc_ticket.p, sc, 0, 1, 0, st);
    // with one sweep the next cycle starts with the restriction, which forms r2 and x1 itself
    const bool fold = sweeps == 1 && !bottom_cycle(H, l);
    if (!fold)
        amg_launch(ctx->stream, pdl, k_amg_kc_r2, gv, kBlock, 0, F.n, b, (const float *)F.v1.p, (const double *)sc,
                   (const float *)F.dw.p, F.r2.p, F.x1.p, st);
    cycle(ctx, H, l, F.r2.p, F.c2.p, sweeps, st, pdl, fold ? b : nullptr);
    amg_launch(ctx->stream, pdl, k_amg_kc_spmv<3>, gs, kBlock, 0, F.n, F.rp, F.ci, F.val32, (const float *)F.c2.p,
             F.v2.p, (const float *)F.v1.p, (const float *)F.r2.p, H->kc_part.p, H->kc_ticket.p, sc, 2, 3, 4, st);
}

// ---- the small coarse levels as one persistent kernel: program recording, probe, launch ----

// Records, in launch order, the phases solve_level(l) launches (the bottom level's cycle as its
// separate phases).  Mirrors cycle / solve_level / coarse_sweep_corr / res_restrict above.
struct CoarseProgram {
    rsg_context *ctx;
    const AmgHierarchy *H;
    int sweeps;
    std::vector<CoarsePhase> ph;

    void sweep(int src, const AmgLevel &l, const SweepArgs &a)
    {
        CoarsePhase p{};
        p.op = src == kSrcX ? CP_SWEEP_X : src == kSrcXCorr ? CP_SWEEP_CORR : CP_SWEEP_CORRK;
        p.n = l.n;
        p.rp = l.rp;
        p.ci = l.ci;
        p.val = l.val32;
        p.a = a;
        ph.push_back(p);
    }
    void sweep_corr(int l, SweepArgs a)
    {
        const AmgLevel &F = H->L[l];
        a.agg = F.agg.p;
        set_correction(H, l + 1, sweeps, a);
        sweep(k_level(H, l + 1) ? kSrcXCorrK : kSrcXCorr, F, a);
    }
    void res_restrict(int l, const float *b, const float *xs)
    {
        const AmgLevel &F = H->L[l], &C = H->L[l + 1];
        CoarsePhase p{};
        p.op = CP_RES_RESTRICT;
        p.n = F.n;
        p.nc = C.n;
        p.rp = F.rp;
        p.ci = F.ci;
        p.val = F.val32;
        p.ptr = F.agg_ptr.p;
        p.rows = F.agg_rows.p;
        p.dwc = C.dw.p;
        p.bc = C.b.p;
        p.x0c = C.x1.p;
        p.a.b = b;
        p.a.xs = xs;
        ph.push_back(p);
    }
    void kc_spmv(const AmgLevel &F, int ndot, const float *c, float *v, const float *y1, const float *y2, double *sc,
                 int o0, int o1, int o2)
    {
        CoarsePhase p{};
        p.op = ndot == 2 ? CP_KC_SPMV2 : CP_KC_SPMV3;
        p.n = F.n;
        p.vgrid = uint32_t(coarse_grid(ctx, F.n));
        p.rp = F.rp;
        p.ci = F.ci;
        p.val = F.val32;
        p.c = c;
        p.v = v;
        p.y1 = y1;
        p.y2 = y2;
        p.sc = sc;
        p.o0 = o0;
        p.o1 = o1;
        p.o2 = o2;
        ph.push_back(p);
    }
    void cycle(int l, const float *b, float *out)
    {
        const AmgLevel &F = H->L[l], &C = H->L[l + 1];
        float *bb = const_cast<float *>(b);
        if (sweeps == 2) {
            sweep(kSrcX, F, SweepArgs{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, F.x2.p});
            res_restrict(l, b, F.x2.p);
        } else {
            res_restrict(l, b, F.x1.p);
        }
        solve_level(l + 1, C.b.p, C.e.p);
        if (sweeps == 2) {
            sweep_corr(l, SweepArgs{bb, F.dw.p, F.x2.p, nullptr, nullptr, 0.f, F.x1.p});
            sweep(kSrcX, F, SweepArgs{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, out});
        } else {
            sweep_corr(l, SweepArgs{bb, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, out});
        }
    }
    void solve_level(int l, const float *b, float *e)
    {
        const AmgLevel &F = H->L[l];
        if (l == H->levels - 1) {
            if (H->dense_coarsest) {
                CoarsePhase p{};
                p.op = CP_DENSE;
                p.n = F.n;
                p.inv = H->coarse_inv.p;
                p.a.b = b;
                p.a.out = e;
                ph.push_back(p);
            } else {
                float *src = F.x1.p, *dst = F.x2.p, *bb = const_cast<float *>(b);
                for (int k = 0; k < 7; k++) {
                    sweep(kSrcX, F, SweepArgs{bb, F.dw.p, src, nullptr, nullptr, 0.f, dst});
                    std::swap(src, dst);
                }
                sweep(kSrcX, F, SweepArgs{bb, F.dw.p, src, nullptr, nullptr, 0.f, e});
            }
            return;
        }
        if (!k_level(H, l)) {
            cycle(l, b, e);
            return;
        }
        double *sc = H->kc_sc.p + 8 * l;
        cycle(l, b, F.c1.p);
        kc_spmv(F, 2, F.c1.p, F.v1.p, b, nullptr, sc, 0, 1, 0);
        CoarsePhase r{};
        r.op = CP_KC_R2;
        r.n = F.n;
        r.a.b = b;
        r.a.dw = F.dw.p;
        r.c = F.v1.p;
        r.sc = sc;
        r.bc = F.r2.p;
        r.x0c = F.x1.p;
        ph.push_back(r);
        cycle(l, F.r2.p, F.c2.p);
        kc_spmv(F, 3, F.c2.p, F.v2.p, F.v1.p, F.r2.p, sc, 2, 3, 4);
    }
};

__global__ void k_coop_probe(unsigned int *) {}

// Whether this device runs a cooperative launch captured in a CUDA graph (the CG loop's body is one):
// one tiny captured launch on a private stream, cached in the context.
bool coop_graph_supported(rsg_context *ctx)
{
    if (ctx->coop_graph >= 0) return ctx->coop_graph != 0;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device);
    bool ok = coop != 0;
    cudaStream_t s = nullptr;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    if (ok) ok = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
        cudaLaunchAttribute at;
        at.id = cudaLaunchAttributeCooperative;
        at.val.cooperative = 1;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2);
        cfg.blockDim = dim3(32);
        cfg.stream = s;
        cfg.attrs = &at;
        cfg.numAttrs = 1;
        const cudaError_t le = cudaLaunchKernelEx(&cfg, k_coop_probe, (unsigned int *)nullptr);
        const cudaError_t ee = cudaStreamEndCapture(s, &g);
        ok = le == cudaSuccess && ee == cudaSuccess && g && cudaGraphInstantiate(&ge, g, 0) == cudaSuccess &&
             cudaGraphLaunch(ge, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
    }
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    if (s) cudaStreamDestroy(s);
    (void)cudaGetLastError();
    ctx->coop_graph = ok ? 1 : 0;
    return ok;
}

// Picks the first level (below the finest) of at most kCoarsePersistRows rows that has a coarser
// level, records its programs for one and two sweeps and uploads them; persist_level stays 0 when
// the kernel is not wanted or cannot run.
rsg_status build_persist(rsg_context *ctx, AmgHierarchy *H, bool want)
{
    H->persist_level = 0;
    H->persist_grid = 0;
    if (!want) return RSG_OK;
    int l0 = 0;
    for (int l = 1; l + 1 < H->levels; l++)
        if (H->L[l].n <= kCoarsePersistRows) {
            l0 = l;
            break;
        }
    if (l0 == 0 || !coop_graph_supported(ctx)) return RSG_OK;
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_amg_coarse_persist, kBlock, 0) != cudaSuccess || occ < 1) {
        (void)cudaGetLastError();
        return RSG_OK;
    }
    std::vector<CoarsePhase> all;
    for (int nu = 1; nu <= 2; nu++) {
        CoarseProgram P{ctx, H, nu, {}};
        P.solve_level(l0, H->L[l0].b.p, H->L[l0].e.p);
        H->persist_len[nu - 1] = uint32_t(P.ph.size());
        all.insert(all.end(), P.ph.begin(), P.ph.end());
    }
    const size_t bytes = all.size() * sizeof(CoarsePhase);
    if (!H->persist_prog.ensure(bytes) || !H->persist_bar.ensure(4))
        return set_error(ctx, RSG_ERR_OUT_OF_MEMORY, "amg: persistent cycle program");
    RSG_CHECK_CUDA(ctx, cudaMemcpy(H->persist_prog.p, all.data(), bytes, cudaMemcpyHostToDevice));
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(H->persist_bar.p, 0, 4 * sizeof(unsigned int), ctx->stream));
    H->persist_grid = std::min(occ, kCoarseCtasPerSm) * ctx->num_sms;
    H->persist_level = l0;
    return RSG_OK;
}

// solve_level(l) from the recorded program: one cooperative launch (counted like the others).
void coarse_persist(rsg_context *ctx, const AmgHierarchy *H, int sweeps, const CgState *st)
{
    ++t_launches;
    if (t_dry) return;
    const uint32_t k = sweeps == 2 ? 1 : 0;
    const CoarsePhase *prog = reinterpret_cast<const CoarsePhase *>(H->persist_prog.p) + (k ? H->persist_len[0] : 0);
    unsigned int *err = st ? const_cast<unsigned int *>(&st->ticket[7]) : ctx->errw;
    cudaLaunchAttribute at;
    at.id = cudaLaunchAttributeCooperative;
    at.val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(H->persist_grid));
    cfg.blockDim = dim3(kBlock);
    cfg.stream = ctx->stream;
    cfg.attrs = &at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_amg_coarse_persist, prog, H->persist_len[k], H->kc_part.p, H->persist_bar.p, st, err);
}

template <int RPW>
FineLaunch<RPW> fine_launch(rsg_context *ctx, const rsg_csr *A)
{
    FineLaunch<RPW> f;
    f.M = view<float>(A, true);
    f.S = sell_view<float>(A);
    f.use_sell = A->use_sell;
    f.smem = A->use_sell ? 0 : tma_smem<float>();
    if (!A->use_sell) {
        const int sm = int(f.smem);
        cudaFuncSetAttribute(k_amg_fine<RPW, kSrcX, kOutRes, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(k_amg_fine<RPW, kSrcX, kOutSmooth, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(k_amg_fine<RPW, kSrcXCorr, kOutSmooth, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(k_amg_fine<RPW, kSrcX, kOutSmooth, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        cudaFuncSetAttribute(k_amg_fine<RPW, kSrcXCorr, kOutSmooth, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    f.grid = spmv_grid(ctx, A, (const void *)k_amg_fine<RPW, kSrcX, kOutSmooth, true>, f.smem, RPW);
    return f;
}

// x0 (= dw r) in the finest level's x1 buffer, computed by the caller or here.
template <int RPW>
rsg_status vcycle_typed(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, const float *x0,
                        const float *q, float *z, int sweeps, double *partials, unsigned int *ticket, CgState *st,
                        int mode, double *rz_out, bool pdl)
{
    const AmgLevel &F = H->L[0];
    if (!x0) {
        amg_launch(ctx->stream, pdl, k_amg_jacobi, grid_rows(F.n), kBlock, 0, F.n, (const float *)F.dw.p, r, F.x1.p,
                 (const CgState *)st);
        x0 = F.x1.p;
    }
    if (H->levels < 2) {
        if (H->dense_coarsest)
            amg_launch(ctx->stream, pdl, k_amg_dense_apply, 1, 1024, 0, F.n, (const float *)H->coarse_inv.p, r, z,
                     (const CgState *)st);
        else
            amg_launch(ctx->stream, pdl, k_amg_jacobi, grid_rows(F.n), kBlock, 0, F.n, (const float *)F.dw.p, r, z,
                     (const CgState *)st);
        const int g = std::min(grid_rows(F.n), kMaxGrid);
        amg_launch(ctx->stream, pdl, k_amg_rz, g, kBlock, 0, F.n, r, (const float *)z, q, partials, ticket, st, mode,
                 rz_out);
        return RSG_OK;
    }
    const FineLaunch<RPW> f = fine_launch<RPW>(ctx, A);
    const AmgLevel &C = H->L[1];
    float *x1 = F.x1.p, *x2 = F.x2.p;
    if (sweeps == 2) {
        SweepArgs a1{r, F.dw.p, x0, nullptr, nullptr, 0.f, x2};
        fine_sweep<RPW, kSrcX, kOutSmooth, false>(ctx, f, a1, nullptr, partials, ticket, st, mode, rz_out, pdl);
        SweepArgs a2{r, F.dw.p, x2, nullptr, nullptr, 0.f, F.r.p};
        fine_sweep<RPW, kSrcX, kOutRes, false>(ctx, f, a2, nullptr, partials, ticket, st, mode, rz_out, pdl);
    } else {
        SweepArgs a1{r, F.dw.p, x0, nullptr, nullptr, 0.f, F.r.p};
        fine_sweep<RPW, kSrcX, kOutRes, false>(ctx, f, a1, nullptr, partials, ticket, st, mode, rz_out, pdl);
    }
    down_restrict(ctx, H, 0, st, pdl);
    solve_level(ctx, H, 1, C.b.p, C.e.p, sweeps, st, pdl);
    const bool kc1 = k_level(H, 1);
    const float s = corr_scale(H, 1, sweeps);
    const float *ec = kc1 ? C.c1.p : C.e.p, *ec2 = kc1 ? C.c2.p : nullptr;
    const double *kc = kc1 ? H->kc_sc.p + 8 : nullptr;
    // the coarse correction in its own streaming pass, so that the post-smoothing sweeps gather one vector
    const int gp = std::min(grid_rows(F.n), kMaxGrid);
    if (sweeps == 2) {
        amg_launch(ctx->stream, pdl, k_amg_prolong, gp, kBlock, 0, F.n, (const float *)x2, (const uint32_t *)F.agg.p, ec,
                 ec2, kc, s, x1, (const CgState *)st);
        SweepArgs u1{r, F.dw.p, x1, nullptr, nullptr, 0.f, x2};
        fine_sweep<RPW, kSrcX, kOutSmooth, false>(ctx, f, u1, nullptr, partials, ticket, st, mode, rz_out, pdl);
        SweepArgs u2{r, F.dw.p, x2, nullptr, nullptr, 0.f, z};
        fine_sweep<RPW, kSrcX, kOutSmooth, true>(ctx, f, u2, q, partials, ticket, st, mode, rz_out, pdl);
    } else {
        amg_launch(ctx->stream, pdl, k_amg_prolong, gp, kBlock, 0, F.n, x0, (const uint32_t *)F.agg.p, ec, ec2, kc, s,
                 x2, (const CgState *)st);
        SweepArgs u1{r, F.dw.p, x2, nullptr, nullptr, 0.f, z};
        fine_sweep<RPW, kSrcX, kOutSmooth, true>(ctx, f, u1, q, partials, ticket, st, mode, rz_out, pdl);
    }
    return RSG_OK;
}

}  // namespace

namespace {
template <int RPW>
rsg_status profile_typed_sweep(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, float *z)
{
    const FineLaunch<RPW> f = fine_launch<RPW>(ctx, A);
    const AmgLevel &F = H->L[0];
    SweepArgs a{r, F.dw.p, F.x1.p, nullptr, nullptr, 0.f, z};
    fine_sweep<RPW, kSrcX, kOutSmooth, false>(ctx, f, a, nullptr, nullptr, nullptr, nullptr, 0, nullptr, false);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    return RSG_OK;
}
}  // namespace

rsg_status amg_profile_launch(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, float *z)
{
    if (!H || H->levels < 2) return set_error(ctx, RSG_ERR_UNSUPPORTED, "amg: the matrix has no coarse level");
    RSG_RPW_DISPATCH(pick_rpw(A), return profile_typed_sweep<RPW>(ctx, A, H, r, z));
    return RSG_ERR_UNSUPPORTED;
}

rsg_status amg_vcycle(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, const float *x0,
                      const float *q, float *z, int sweeps, double *partials, unsigned int *ticket, CgState *st,
                      int mode, double *rz_out, bool pdl)
{
    if (!H || H->levels < 1) return set_error(ctx, RSG_ERR_INVALID_ARG, "amg: no hierarchy");
    // The V-cycle is a chain of short kernels (the coarse levels' sweeps run a few microseconds), so
    // each is launched with programmatic dependent launch whatever the caller chose for its own loop
    // kernels: the next kernel's blocks are scheduled while the current one drains.
    (void)pdl;
    pdl = true;
    RSG_RPW_DISPATCH(pick_rpw(A),
                     return vcycle_typed<RPW>(ctx, A, H, r, x0, q, z, sweeps, partials, ticket, st, mode, rz_out,
                                              pdl));
    return RSG_ERR_UNSUPPORTED;
}

}  // namespace rsg

// ---------------------------------------------------------------- C ABI -----------------------

using namespace rsg;

extern "C" {

rsg_status rsg_amg_setup(rsg_context *ctx, rsg_csr *A, rsg_amg_info *info)
{
    return rsg_amg_setup_conf(ctx, A, nullptr, info);
}

rsg_status rsg_amg_setup_conf(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf, rsg_amg_info *info)
{
    if (!ctx || !A) return set_error(ctx, RSG_ERR_INVALID_ARG, "amg_setup: bad arguments");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_TRY(amg_setup(ctx, A, conf && conf->persistent > 0));
    if (info) {
        const AmgHierarchy *H = amg_of(A);
        std::memset(info, 0, sizeof(*info));
        info->levels = uint32_t(H->levels);
        info->dense_coarsest = H->dense_coarsest ? 1u : 0u;
        for (int l = 0; l < H->levels && l < 16; l++) {
            info->rows[l] = H->L[l].n;
            info->nnz[l] = H->L[l].nnz;
        }
        info->mis_rounds = H->mis_rounds;
        info->setup_launches = H->setup_launches;
        info->seconds_setup = H->seconds_setup;
        info->cycle_launches[0] = H->cycle_launches[0];
        info->cycle_launches[1] = H->cycle_launches[1];
        info->persist_level = uint32_t(H->persist_level);
    }
    return RSG_OK;
}

rsg_status rsg_amg_level(rsg_context *ctx, const rsg_csr *A, uint32_t level, uint32_t *agg, uint32_t *row_ptr,
                         uint32_t *col_idx, double *values)
{
    const AmgHierarchy *H = A ? amg_of(A) : nullptr;
    if (!ctx || !H || level >= uint32_t(H->levels)) return set_error(ctx, RSG_ERR_INVALID_ARG, "amg_level: bad level");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    const AmgLevel &l = H->L[level];
    if (agg) {
        if (int(level) + 1 >= H->levels) return set_error(ctx, RSG_ERR_INVALID_ARG, "amg_level: the last level has no aggregates");
        RSG_CHECK_CUDA(ctx, cudaMemcpy(agg, l.agg.p, size_t(l.n) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    }
    if (row_ptr) RSG_CHECK_CUDA(ctx, cudaMemcpy(row_ptr, l.rp, (size_t(l.n) + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (col_idx) RSG_CHECK_CUDA(ctx, cudaMemcpy(col_idx, l.ci, size_t(l.nnz) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (values) RSG_CHECK_CUDA(ctx, cudaMemcpy(values, l.val, size_t(l.nnz) * sizeof(double), cudaMemcpyDeviceToHost));
    return RSG_OK;
}

rsg_status rsg_amg_apply(rsg_context *ctx, rsg_csr *A, const double *r, double *z, uint32_t sweeps)
{
    AmgHierarchy *H = A ? amg_of(A) : nullptr;
    if (!ctx || !H || !r || !z || (sweeps != 1 && sweeps != 2))
        return set_error(ctx, RSG_ERR_INVALID_ARG, "amg_apply: bad arguments (call rsg_amg_setup first)");
    RSG_CHECK_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t n = A->n;
    // FP32 copies of r and z in level 0's b and e (unused by the V-cycle on the finest level)
    AmgLevel &L0 = H->L[0];
    const size_t red = arena_bytes(kMaxGrid, sizeof(double)) + arena_bytes(8, sizeof(double));
    RSG_TRY(arena_reserve(ctx, red));
    double *partials = arena_take<double>(ctx, kMaxGrid);
    double *scal = arena_take<double>(ctx, 8);
    unsigned int *ticket = reinterpret_cast<unsigned int *>(scal + 4);
    RSG_CHECK_CUDA(ctx, cudaMemsetAsync(scal, 0, 8 * sizeof(double), ctx->stream));
    const int g = std::min(grid_rows(n), kMaxGrid);
    count_launch();
    k_amg_d2f<<<g, kBlock, 0, ctx->stream>>>(n, r, L0.b.p);
    RSG_TRY(amg_vcycle(ctx, A, H, L0.b.p, nullptr, nullptr, L0.e.p, int(sweeps), partials, ticket, nullptr, 0, scal,
                       false));
    count_launch();
    k_amg_f2d<<<g, kBlock, 0, ctx->stream>>>(n, L0.e.p, z);
    RSG_CHECK_CUDA(ctx, cudaGetLastError());
    RSG_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return RSG_OK;
}

}  // extern "C"
