// Internal interface of the multilevel aggregation preconditioner (RSG_PREC_AMG).
//
// No counterpart in the reference, whose preconditioners are NONE / JACOBI / BLOCK_JACOBI
// (src/rmatrixpreconditioner.cpp).  The hierarchy is built on the GPU from the matrix's current
// values (strength of connection, aggregates rooted at a distance-2 independent set of hashed
// priorities, piecewise-constant prolongation, Galerkin coarse matrices summed in a fixed order,
// dense inverse of the coarsest level) and applied as an FP32 cycle with damped-Jacobi smoothing and a
// scaled coarse correction; levels 1..kAmgKLevels are solved by two flexible-CG steps each (K-cycle),
// so the outer CG uses the flexible direction update.
#pragma once

#include "krylov.cuh"

namespace rsg {

constexpr int kAmgMaxLevels = 12;
constexpr uint32_t kAmgCoarsest = 128;     // rows at or below which a level is inverted densely
constexpr uint32_t kAmgMaxEntries = 4096;  // fine entries gathered into one coarse row (Galerkin staging)
constexpr double kAmgTheta = 0.08;         // strength threshold |a_ij| >= theta sqrt(|a_ii a_jj|)
constexpr float kAmgOmega = 2.0f / 3.0f;   // damped-Jacobi weight of the smoother
constexpr float kAmgScale1 = 1.6f;         // coarse-correction scale, one smoothing sweep per side
constexpr float kAmgScale2 = 1.8f;         // coarse-correction scale, two sweeps per side
#ifndef RSG_AMG_KLEVELS
#define RSG_AMG_KLEVELS 2
#endif
constexpr int kAmgKLevels = RSG_AMG_KLEVELS;  // levels 1..kAmgKLevels are solved by two flexible-CG steps (K-cycle)
constexpr uint32_t kAmgUnset = 0xffffffffu;

// Device buffer that only grows (reallocated when a larger size is asked for).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    bool ensure(size_t count)
    {
        if (count <= cap && p) return true;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = count + count / 4 + 64;
        if (cudaMalloc(&p, want * sizeof(T)) != cudaSuccess) return false;
        cap = want;
        return true;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct AmgLevel {
    uint32_t n = 0;
    uint64_t nnz = 0;
    // the level's matrix: level 0 points at the caller's matrix, coarser levels use the owned buffers
    const uint32_t *rp = nullptr, *ci = nullptr;
    const double *val = nullptr;
    const float *val32 = nullptr;
    DevBuf<uint32_t> own_rp, own_ci;
    DevBuf<double> own_val;
    DevBuf<float> own_val32;
    DevBuf<double> diag;                   // a_ii (FP64, strength test)
    DevBuf<float> dw;                      // omega / a_ii (0 for a zero diagonal)
    DevBuf<uint32_t> agg;                  // row of this level -> row of the next level
    DevBuf<uint32_t> agg_ptr, agg_rows;    // next-level row -> rows of this level (ascending)
    DevBuf<float> b, r, x1, x2, e;         // V-cycle vectors; x1 starts as x0 = dw b (b and e unused on level 0)
    DevBuf<float> c1, c2, v1, v2, r2;      // K-cycle levels: the two flexible-CG steps
};

struct AmgHierarchy {
    int levels = 0;                 // levels in use, the finest included
    AmgLevel L[kAmgMaxLevels];
    bool dense_coarsest = false;    // the last level is applied through coarse_inv
    DevBuf<float> coarse_inv;       // dense inverse of the last level (row-major)
    // setup scratch
    DevBuf<uint64_t> T, M1;         // independent-set tuples and their neighbourhood maxima
    DevBuf<uint8_t> smask;          // strong-connection flag per stored entry
    DevBuf<uint32_t> u1, u2, u3;    // per-row counters / scan output
    DevBuf<uint32_t> scan_blocks;   // scan workspace
    DevBuf<unsigned int> rounds;    // undecided nodes after each independent-set round
    DevBuf<uint32_t> tcol;          // Galerkin staging: columns
    DevBuf<double> tval;            // Galerkin staging: values
    DevBuf<double> kc_part;         // K-cycle: grid-reduction partials
    DevBuf<unsigned int> kc_ticket; // K-cycle: grid-reduction counter (zero between uses)
    DevBuf<double> kc_sc;           // K-cycle: 8 scalars per level (c1.v1, c1.b, c2.v2, c2.v1, c2.r2)
    unsigned int *flags = nullptr;  // device counters read back by the host (16 words)
    unsigned int *flags_h = nullptr;  // pinned host copy
    double seconds_setup = 0.0;
    uint32_t mis_rounds = 0;
    uint32_t setup_launches = 0;         // kernel launches of the last set-up
    uint32_t cycle_launches[2] = {0, 0};  // kernel launches of one cycle inside CG, one / two sweeps
    // Levels from persist_level on (0: none) run as one persistent cooperative kernel per visit: the
    // phase programs it runs for one and two sweeps (recorded from the cycle's own recursion), its
    // CTA count and its barrier words.
    int persist_level = 0;
    int persist_grid = 0;
    DevBuf<uint8_t> persist_prog;
    uint32_t persist_len[2] = {0, 0};
    DevBuf<unsigned int> persist_bar;
};

void amg_free(AmgHierarchy *H);
// (Re)builds A's hierarchy from A's current values; A owns it afterwards (freed with A).
// persistent: run the small coarse levels of each cycle as one persistent kernel (when the device
// can capture a cooperative launch in a graph); false (the default) launches their kernels one by one.
rsg_status amg_setup(rsg_context *ctx, rsg_csr *A, bool persistent = false);
AmgHierarchy *amg_of(const rsg_csr *A);

// z = M(r), one cycle, on the context stream (FP32; sweeps = 1 or 2 smoothing sweeps per side;
// levels 1..kAmgKLevels solved by two flexible-CG steps, so M varies with r).  The final kernel adds
// r^T z and q^T z (compensated) over its grid and, when st is given, finalizes the CG state: mode 0
// starts the recurrence (rho = r^T z, beta = 0), mode 1 continues it with the flexible update
// beta = -alpha q^T z / rho (or the residual-replacement rule after a true-residual check).  Without st
// r^T z goes to *rz_out.  partials holds >= 2 kMaxGrid doubles; ticket is a zeroed counter.
// x0 = (omega / a_ii) r, the first smoothing step, computed by the caller's streaming pass (the CG
// update / check kernels) in the finest level's x0 buffer (amg_finest_x0), or NULL to compute it here.
// q (mode 1): the CG's q = A p of the last step, for the flexible direction update.
rsg_status amg_vcycle(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, const float *x0,
                      const float *q, float *z, int sweeps, double *partials, unsigned int *ticket, CgState *st,
                      int mode, double *rz_out, bool pdl);
inline const float *amg_finest_weights(const AmgHierarchy *H) { return H->L[0].dw.p; }
inline float *amg_finest_x0(const AmgHierarchy *H) { return H->L[0].x1.p; }

// One launch of a finest-level smoothing sweep (z = x + dw (r - A x)), for kernel timing.
rsg_status amg_profile_launch(rsg_context *ctx, const rsg_csr *A, const AmgHierarchy *H, const float *r, float *z);

}  // namespace rsg
