/*
 * rsg.h -- C ABI of the B200 sparse linear-solve library (librsg.so).
 *
 * Plain C types only: pointers, sizes, status codes.  No exceptions cross this
 * boundary.  Every entry point names the reference interface it replaces
 * (paths relative to the reference project, Range-Software/range-solver-lib).
 *
 * Memory: arrays passed with RSG_MEM_HOST are caller-owned host buffers
 * (copied during the call); arrays passed with RSG_MEM_DEVICE are device
 * pointers on the context's GPU.  Matrices, preconditioners, assembly plans
 * and learned models live in library-owned device memory behind opaque
 * handles.  Each context owns one CUDA stream; calls on one context are
 * serialised by the caller (like the reference, which is not re-entrant for
 * one matrix); different contexts may be used from different threads.
 */
#ifndef RSG_H
#define RSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define RSG_API __attribute__((visibility("default")))
#else
#define RSG_API
#endif

typedef enum {
    RSG_OK = 0,
    RSG_NOT_CONVERGED = 1,      /* iteration limit reached (the reference returns silently) */
    RSG_BREAKDOWN = 2,          /* non-finite residual / zero search direction */
    RSG_ERR_INVALID_ARG = -1,
    RSG_ERR_CUDA = -2,
    RSG_ERR_OUT_OF_MEMORY = -3,
    RSG_ERR_UNSUPPORTED = -4,
    RSG_ERR_SINGULAR = -5,      /* singular block in block-Jacobi (RRMatrix::invert failure); a zero norm
                                   (breakdown) in an eigenvalue driver */
    RSG_ERR_TIMEOUT = -6
} rsg_status;

/* RMatrixSolverConf::Type (range-model-lib; used at src/rmatrixsolver.cpp:186-196) */
typedef enum { RSG_SOLVER_CG = 0, RSG_SOLVER_GMRES = 1 } rsg_solver_type;

/* RMatrixPreconditionerType (include/rmatrixpreconditioner.h:7-16), plus two without a reference
 * counterpart: the learned one and a multilevel aggregation preconditioner (rsg_amg_*). */
typedef enum {
    RSG_PREC_NONE = 0,
    RSG_PREC_JACOBI = 1,
    RSG_PREC_BLOCK_JACOBI = 2,
    RSG_PREC_LEARNED = 3,
    RSG_PREC_AMG = 4
} rsg_prec_type;

typedef enum {
    RSG_STOP_REFERENCE = 0,     /* RIterationInfo::hasConverged on ||r||/(||A||_F||x||+||b||) */
    RSG_STOP_TRUE_RELRES = 1    /* FP64 true ||b-Ax||/||b|| <= rtol, recomputed before stopping */
} rsg_stop_rule;

typedef enum {
    RSG_PRECISION_FP64 = 0,     /* everything in FP64 */
    RSG_PRECISION_MIXED = 1,    /* FP32 inner Krylov, FP64 residual/solution (reliable updates) */
    RSG_PRECISION_AUTO = 2      /* CG: mixed precision, continuing in FP64 from the current x when a residual
                                   refresh finds the FP32 recurrence more than 2x off the true residual (stiff
                                   systems, where FP32 matrix values cost iterations); TRUE_RELRES rule.  It
                                   recovers part of mixed precision's loss there; FP64 stays the choice when
                                   the system is known to be stiff */
} rsg_precision;

typedef enum { RSG_MEM_HOST = 0, RSG_MEM_DEVICE = 1 } rsg_memory;

/* Mirrors RMatrixSolverConf fields read by src/rmatrixsolver.cpp:125-128 plus
 * the GPU-specific options.  Fill with rsg_conf_default() first. */
typedef struct {
    int32_t  solver_type;       /* rsg_solver_type */
    uint32_t n_outer;           /* nOuterIterations: CG iteration cap / GMRES restart cap */
    uint32_t n_inner;           /* nInnerIterations: GMRES restart length */
    double   cvg;               /* solverCvgValue (reference stopping rule) */
    uint32_t output_frequency;  /* 0 = silent, like RIterationInfo */
    const char *output_file;    /* convergence log "Iteration number|Solver residual|Solver convergence"; NULL = none */
    double   eps;               /* stand-in for RConstants::eps (clamps and stagnation test) */
    int32_t  stop_rule;         /* rsg_stop_rule */
    double   rtol;              /* for RSG_STOP_TRUE_RELRES */
    int32_t  precision;         /* rsg_precision */
    int32_t  scale_equations;   /* 1 = reference's equation scaling 1e9*||A||_F/||b|| (src/rmatrixsolver.cpp:164-184) */
    double   reliable_delta;    /* mixed precision: refresh the FP64 residual when ||r|| drops by this factor
                                   (default 1e-3) */
    int32_t  flexible;          /* GMRES: store Z (flexible / variable preconditioner) */
    int32_t  use_graph;         /* 1 = device-driven loop in one CUDA graph launch (default) */
    uint32_t check_interval;    /* host-driven loop: iterations per convergence poll */
    const void *learned;        /* rsg_learned* for RSG_PREC_LEARNED / learned initial guess */
    int32_t  learned_initial_guess;
    int32_t  l2_resident_f32;   /* mixed, CSR-stream layout only: FP32 matrix loads with L2 evict_last
                                   (slower than evict_first on SELL-32 in measurements, so not applied there) */
    int32_t  autotune;          /* 1: autotune A's launch shapes on its first solve (rsg_autotune, with the
                                   cache file named by the RSG_TUNE_CACHE environment variable if set) */
    int32_t  amg_sweeps;        /* RSG_PREC_AMG: damped-Jacobi sweeps per side of the cycle, 1 or 2 (0: 1) */
    int32_t  persistent;        /* CG with none / Jacobi in graph mode: run the loop as one persistent cooperative
                                   kernel (same results bit for bit): 0 = for systems up to 131,072 rows,
                                   1 = whenever the device allows it, -1 = never */
    int32_t  reserved[3];
} rsg_solver_conf;

typedef struct {
    uint32_t iterations;        /* CG iterations or GMRES inner steps in total */
    uint32_t outer;             /* GMRES restarts / mixed-precision residual refreshes */
    double   error;             /* last reference-style error */
    double   trend;
    double   true_relres;       /* FP64 ||b - A x|| / ||b|| of the returned x, recomputed on the GPU */
    double   equation_scale;
    double   norm_a;            /* ||A||_F */
    double   norm_b;
    double   seconds_setup;     /* preconditioner build, uploads (device-timed) */
    double   seconds_solve;     /* iterations (device-timed) */
    int32_t  converged;
    int32_t  status;            /* rsg_status of the solve */
    uint32_t fallbacks;         /* learned preconditioner: steps that fell back to Jacobi */
    uint32_t fp64_iterations;   /* RSG_PRECISION_AUTO: iterations run in FP64 after the switch (0: none) */
    uint32_t reserved[4];
} rsg_stats;

typedef struct rsg_context rsg_context;
typedef struct rsg_csr rsg_csr;
typedef struct rsg_learned rsg_learned;
typedef struct rsg_batch rsg_batch;

/* ---- context ---- */
RSG_API rsg_status rsg_context_create(int device, rsg_context **out);
RSG_API void       rsg_context_destroy(rsg_context *ctx);
RSG_API const char *rsg_status_string(rsg_status s);
RSG_API const char *rsg_last_error(const rsg_context *ctx);
RSG_API rsg_status rsg_context_set_stream(rsg_context *ctx, void *cuda_stream); /* NULL = own stream */
RSG_API rsg_status rsg_synchronize(rsg_context *ctx);
RSG_API void       rsg_conf_default(rsg_solver_conf *conf);

/* ---- CSR matrices ----
 * Replaces SparseMatrixCache + buildSparseMatrixCache (src/rmatrixsolver.cpp:14-54):
 * upload the CSR once (uint32 row pointer and column indexes, FP64 values),
 * compute ||A||_F, and derive the kernels' internal formats (FP32 values,
 * 16-bit column offsets) on the GPU. */
RSG_API rsg_status rsg_csr_create(rsg_context *ctx, uint32_t n_rows, const uint32_t *row_ptr,
                                  const uint32_t *col_idx, const double *values, int32_t memory,
                                  rsg_csr **out);
/* Replaces refreshSparseMatrixCache (src/rmatrixsolver.cpp:56-97): same pattern, new values. */
RSG_API rsg_status rsg_csr_update_values(rsg_context *ctx, rsg_csr *A, const double *values, int32_t memory);
RSG_API void       rsg_csr_destroy(rsg_context *ctx, rsg_csr *A);
RSG_API rsg_status rsg_csr_info(const rsg_csr *A, uint32_t *n_rows, uint64_t *nnz, double *frobenius);
/* Device pointers to the stored CSR (row_ptr, col_idx, values) for callers that read it back. */
RSG_API rsg_status rsg_csr_device_arrays(const rsg_csr *A, const uint32_t **row_ptr, const uint32_t **col_idx,
                                         const double **values);

/* Copy the stored CSR back to caller-owned host arrays (n_rows+1, nnz, nnz entries);
 * the assembled system in the reference lives in host memory (RSparseMatrix). */
RSG_API rsg_status rsg_csr_copy_to_host(rsg_context *ctx, const rsg_csr *A, uint32_t *row_ptr, uint32_t *col_idx,
                                        double *values);

/* y = A x in FP64 (multiplyRow, src/rmatrixsolver.cpp:111-119, over all rows).  Device pointers. */
RSG_API rsg_status rsg_spmv(rsg_context *ctx, const rsg_csr *A, const double *x, double *y);
/* y = A x with the FP32 copy of the values (mixed-precision inner product).  Device pointers. */
RSG_API rsg_status rsg_spmv_f32(rsg_context *ctx, const rsg_csr *A, const float *x, float *y);
/* Jacobi inverse diagonal d_i = 1/A_ii (0 when absent or zero): constructJacobi,
 * src/rmatrixpreconditioner.cpp:78-94.  Device output. */
RSG_API rsg_status rsg_jacobi_build(rsg_context *ctx, const rsg_csr *A, double *inv_diag);
/* Block-Jacobi inverse blocks (n_rows x width, row-major per block row):
 * constructBlockJacobi, src/rmatrixpreconditioner.cpp:96-148.  Device output. */
RSG_API rsg_status rsg_block_jacobi_build(rsg_context *ctx, const rsg_csr *A, uint32_t block_size,
                                          double *blocks, uint32_t *width_out);

/* ---- solve ----
 * Replaces RMatrixSolver::solve (src/rmatrixsolver.cpp:158-201) with its CG
 * (:208-355) and GMRES (:357-581).  x is in/out: its incoming values are the
 * initial guess, like the reference (callers zero it).  b and x are host or
 * device arrays of n_rows doubles according to `memory`. */
RSG_API rsg_status rsg_solve(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf, int32_t prec_type,
                             uint32_t block_size, const double *b, double *x, int32_t memory, rsg_stats *stats);

/* Diagnostic (no reference counterpart): average device time in seconds of one
 * of the solver's kernels on matrix A over `reps` launches on the context
 * stream, measured with CUDA events.  flush_l2 != 0 writes a buffer larger
 * than L2 before every launch (excluded from the timing), giving the
 * HBM-bound time; 0 measures back-to-back launches as inside a solve.  The CG
 * kernels are launched with the solve loop's shapes (A's autotuned grids when it
 * has them, else the built-in defaults). */
typedef enum {
    RSG_KERNEL_CG_DIR_FP64 = 0,    /* p = z + beta p, q = A p, p^T q   (FP64 CSR) */
    RSG_KERNEL_CG_DIR_MIXED = 1,   /* same with FP32 values and 16-bit column offsets */
    RSG_KERNEL_CG_UPDATE_FP64 = 2, /* x, r update + Jacobi + dots */
    RSG_KERNEL_CG_UPDATE_MIXED = 3,
    RSG_KERNEL_SPMV_FP64 = 4,
    RSG_KERNEL_SPMV_FP32 = 5,
    RSG_KERNEL_AMG_SWEEP = 6       /* RSG_PREC_AMG: a finest-level smoothing sweep x + dw (r - A x) of the
                                      V-cycle (builds A's hierarchy first if it has none) */
} rsg_kernel_id;
RSG_API rsg_status rsg_profile_kernel(rsg_context *ctx, const rsg_csr *A, int32_t kernel, uint32_t reps,
                                      int32_t flush_l2, double *seconds);

/* Several right-hand sides of one matrix (replaces k RMatrixSolver::solve calls
 * with the same A, src/rmatrixsolver.cpp:158-201, e.g. load cases or
 * REigenValueSolver's repeated solves, src/reigenvaluesolver.cpp:119-392):
 * FP64 CG with JACOBI or NONE, every column with its own recurrences and the
 * RSG_STOP_TRUE_RELRES rule (conf->stop_rule must be TRUE_RELRES, precision
 * FP64; no equation scaling is applied -- the true-residual rule does not
 * depend on it).  One pass over the matrix per iteration serves all columns.
 * B and X hold k columns of n values each (column j at offset j*n), X is
 * in/out (initial guesses), host or device memory as `memory` says; 1 <= k <= 16.
 * per_rhs (k entries) and summary (worst case over the columns) may be NULL. */
RSG_API rsg_status rsg_solve_multi(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf, int32_t prec_type,
                                   uint32_t k, const double *B, double *X, int32_t memory, rsg_stats *per_rhs,
                                   rsg_stats *summary);

/* ---- pattern-cached assembly of caller-computed element matrices ----
 * Replaces RSolverFluid::buildSparseMatrixPattern / assemblyMatrix (src/rsolverfluid.cpp:2305-2419),
 * the fluid solver's assembly of its element matrices (4 DOFs per node there; any count here).
 * rsg_scatter_plan_create builds, on the host, the CSR pattern of every active element's enabled DOFs
 * (rows and columns ascending, values zero) and, for every stored entry and every right-hand-side
 * row, the list of element contributions in element order; rsg_scatter_assemble then forms the values
 * on the GPU, one thread per entry adding its contributions in that order -- the order of the
 * reference's serial element loop, so the result is the same bit for bit (no atomics).
 * Mesh: element e has nodes elem_nodes[elem_begin[e] .. elem_begin[e+1]); elem_active[e] != 0 marks
 * the elements the reference assembles (computable volumes, surfaces with a free-pressure condition).
 * book[node * dofs_per_node + c]: the DOF's equation number (< n_free), or 0xffffffff when disabled.
 * Ae / fe (host or device per `memory`): for every ACTIVE element in element order, its dense
 * (dofs_per_node * nodes)^2 matrix (row-major, local DOF = node slot * dofs_per_node + component) and
 * its (dofs_per_node * nodes) vector, concatenated; rsg_scatter_plan_info gives the two totals. */
typedef struct rsg_scatter_plan rsg_scatter_plan;
RSG_API rsg_status rsg_scatter_plan_create(rsg_context *ctx, uint32_t dofs_per_node, uint32_t n_elements,
                                           const uint32_t *elem_begin, const uint32_t *elem_nodes,
                                           const uint8_t *elem_active, uint32_t n_nodes, const uint32_t *book,
                                           uint32_t n_free, rsg_scatter_plan **out);
RSG_API rsg_status rsg_scatter_plan_info(const rsg_scatter_plan *plan, uint64_t *ae_values, uint64_t *fe_values,
                                         uint64_t *nnz);
/* A: created on the first call (*A == NULL), its values replaced afterwards (same pattern); b_device:
 * n_free doubles, overwritten. */
RSG_API rsg_status rsg_scatter_assemble(rsg_context *ctx, rsg_scatter_plan *plan, const double *Ae,
                                        const double *fe, int32_t memory, rsg_csr **A, double *b_device);
RSG_API void       rsg_scatter_plan_destroy(rsg_context *ctx, rsg_scatter_plan *plan);

/* ---- eigenvalues of the pencil (M, K) ----
 * Replaces REigenValueSolver::solve (src/reigenvaluesolver.cpp:40-110) with its three methods:
 * Lanczos (:119-210, with qlDecomposition :420-497), Arnoldi (:211-294, with qrDecomposition
 * :499-592) and the Rayleigh quotient iteration (:295-392).  Every solve of a step is rsg_solve with
 * *conf and Jacobi (as the reference passes R_MATRIX_PRECONDITIONER_JACOBI), its x the previous
 * step's vector as the reference's is; the vectors stay on the device.  Results follow the
 * reference's solve(): with more than one value, d_i = |1/d_i| sorted ascending (after the
 * reference's swap of the first two) and the eigenvectors reordered by the same permutation; the
 * Lanczos values are the Lanczos diagonal (the reference's QL step ends before any rotation);
 * Rayleigh returns its shift mu and vector.  M and K: CSR handles of one size (Rayleigh: one
 * pattern).  start: n host values, the reference's random start vector rand()/RAND_MAX (normalised
 * here).  values: n_eigen (Rayleigh: 1) host doubles; vectors (Arnoldi, Rayleigh; may be NULL):
 * the same count of rows of n doubles.  A zero norm met on the way returns RSG_ERR_SINGULAR. */
typedef enum {
    RSG_EIGEN_LANCZOS = 0,      /* REigenValueSolverConf::Lanczos */
    RSG_EIGEN_ARNOLDI = 1,      /* REigenValueSolverConf::Arnoldi */
    RSG_EIGEN_RAYLEIGH = 2      /* REigenValueSolverConf::Rayleigh */
} rsg_eigen_method;
typedef struct {
    int32_t  method;            /* rsg_eigen_method */
    uint32_t n_eigen;           /* getNEigenValues (Lanczos, Arnoldi) */
    uint32_t n_iterations;      /* getNIterations: QR sweeps (Arnoldi), iterations (Rayleigh) */
    uint32_t reserved;
    double   cvg;               /* getSolverCvgValue: QR subdiagonal bound, Rayleigh |mu - mu_old| */
    double   mu0;               /* Rayleigh: the first shift (the reference draws 1e9 rand()/RAND_MAX) */
} rsg_eigen_conf;
typedef struct {
    uint32_t n_values;          /* values written */
    uint32_t solves;            /* linear solves run */
    uint64_t iterations;        /* their Krylov iterations in total */
} rsg_eigen_stats;
RSG_API rsg_status rsg_eigen_solve(rsg_context *ctx, const rsg_csr *M, rsg_csr *K, const rsg_eigen_conf *econf,
                                   const rsg_solver_conf *conf, const double *start, double *values,
                                   double *vectors, rsg_eigen_stats *stats);

/* Autotuner (no counterpart in the reference, whose loops are OpenMP).  Picks
 * A's layout (SELL-32, or the CSR stream with a rows-per-warp chunk) and the
 * grid sizes of the CG loop's two kernels per iteration (fused direction +
 * SpMV, and update) by timing short fixed-length Jacobi-PCG solves of A itself
 * in FP64 and mixed precision for each candidate; the built-in defaults are a
 * candidate too.  The choice stays with A for every later solve.  cache_path
 * (may be NULL): a text file keyed by device, matrix shape and layout; a
 * matching line is used without timing, a new result is appended.  Tuning
 * allocates two n-vectors for the duration of the call.  After the grids, the
 * tuner also times the loop with programmatic dependent launch switched the other
 * way from its default (on for n <= 262144 rows, where launch latency dominates). */
typedef struct rsg_tune_info {
    int32_t  tuned;                  /* 1 when A carries autotuned shapes */
    int32_t  from_cache;
    int32_t  format;                 /* 1 SELL-32, 0 CSR stream */
    uint32_t rows_per_warp;          /* CSR stream chunk (32 for SELL-32) */
    uint32_t grid_dir_fp64, grid_dir_fp32, grid_update_fp64, grid_update_fp32;  /* 0 = built-in default */
    double   seconds_iter_fp64, seconds_iter_fp32;                   /* per CG iteration, chosen shapes */
    double   seconds_iter_fp64_default, seconds_iter_fp32_default;   /* per CG iteration, built-in shapes */
    uint32_t candidates;             /* timed solves */
    int32_t  pdl_fp64, pdl_fp32;     /* 1: the CG loop's kernels use programmatic dependent launch */
    int32_t  reserved[1];
} rsg_tune_info;
RSG_API rsg_status rsg_autotune(rsg_context *ctx, rsg_csr *A, const char *cache_path, rsg_tune_info *out);
RSG_API rsg_status rsg_tune_get(const rsg_csr *A, rsg_tune_info *out);
/* The same for a batch (rsg_batch_create): the grid of the batch loop's slice kernels
 * per precision, by timing 32-iteration batch solves (grid_dir_* = grid_update_*). */
RSG_API rsg_status rsg_batch_autotune(rsg_context *ctx, rsg_batch *batch, rsg_tune_info *out);

/* CSR/RHS dump (no counterpart in the reference): the matrix as the solver holds
 * it, and optionally a right-hand side (b_device, n doubles, may be NULL), in a
 * little-endian binary file with a 64-byte "RSGCSR01" header -- reproducible
 * benchmark and regression inputs.  rsg_csr_load creates *A and, when the file
 * has a right-hand side and b_device is given, copies it there. */
RSG_API rsg_status rsg_csr_save(rsg_context *ctx, const rsg_csr *A, const double *b_device, const char *path);
RSG_API rsg_status rsg_csr_load(rsg_context *ctx, const char *path, rsg_csr **A, double *b_device, uint32_t *n_rows,
                                uint64_t *nnz, int32_t *has_b);

/* Failure-detection self-test (no counterpart in the reference): a kernel waits,
 * with the library's bounded mbarrier wait limited to `polls` polls (0: 1024),
 * for a completion that never comes; it flags the context's error word and
 * returns, so this call returns RSG_ERR_TIMEOUT and the context stays usable.
 * Nothing faults or hangs. */
RSG_API rsg_status rsg_selftest_wait_timeout(rsg_context *ctx, uint32_t polls);

/* ---- multilevel aggregation preconditioner (RSG_PREC_AMG) ----
 * No counterpart in the reference (its preconditioners are NONE / JACOBI / BLOCK_JACOBI); it fills
 * the same slot, P.compute(r, z) in solveCG (src/rmatrixsolver.cpp:258).  Built on the GPU from the
 * matrix's current values at every rsg_solve that asks for it: aggregates rooted at a distance-2
 * independent set of the strength graph (|a_ij| >= 0.08 sqrt(|a_ii a_jj|)), piecewise-constant
 * prolongation, Galerkin coarse matrices added in a fixed order (deterministic), down to at most
 * 128 rows, inverted densely.  Applied as an FP32 cycle (damped Jacobi, weight 2/3, with
 * conf.amg_sweeps sweeps per side and a coarse correction scaled by 1.6 / 1.8; levels 1 and 2 solved
 * by two flexible-CG steps each, a K-cycle) inside the mixed-precision CG (precision MIXED, stop_rule
 * TRUE_RELRES), whose direction update is then the flexible one; the result keeps FP64 accuracy. */
typedef struct {
    uint32_t levels;            /* levels including the finest */
    uint32_t dense_coarsest;    /* 1: the last level is applied through its dense inverse */
    uint32_t rows[16];
    uint64_t nnz[16];
    uint32_t mis_rounds;        /* synchronous rounds of the independent-set construction, all levels */
    uint32_t setup_launches;    /* kernel launches of the set-up */
    double   seconds_setup;     /* wall time of the set-up */
    uint32_t cycle_launches[2]; /* kernel launches of one cycle inside CG, with 1 / 2 smoothing sweeps */
    uint32_t persist_level;     /* first level (<= 32768 rows) whose visits run as one persistent
                                   cooperative kernel each (rsg_amg_setup_conf with persistent > 0);
                                   0 when every cycle kernel is launched */
} rsg_amg_info;
/* Build (or rebuild) A's hierarchy from A's current values; info may be NULL. */
RSG_API rsg_status rsg_amg_setup(rsg_context *ctx, rsg_csr *A, rsg_amg_info *info);
/* The same, built as rsg_solve builds it for conf (conf->persistent > 0: the levels of at most 32768
 * rows below the finest run as one persistent cooperative kernel per visit; NULL: as rsg_amg_setup). */
RSG_API rsg_status rsg_amg_setup_conf(rsg_context *ctx, rsg_csr *A, const rsg_solver_conf *conf,
                                      rsg_amg_info *info);
/* Copy level `level` of the last hierarchy to host arrays (any may be NULL): agg (rows of the level)
 * maps each row to its aggregate, the row of level + 1 (not for the last level); row_ptr / col_idx /
 * values are the level's CSR (level 0: A itself). */
RSG_API rsg_status rsg_amg_level(rsg_context *ctx, const rsg_csr *A, uint32_t level, uint32_t *agg, uint32_t *row_ptr,
                                 uint32_t *col_idx, double *values);
/* z = one V-cycle applied to r (device arrays of n_rows doubles; FP32 inside), sweeps 1 or 2. */
RSG_API rsg_status rsg_amg_apply(rsg_context *ctx, rsg_csr *A, const double *r, double *z, uint32_t sweeps);

/* FP64 true relative residual ||b - A x|| / ||b|| (device pointers). */
RSG_API rsg_status rsg_true_relres(rsg_context *ctx, const rsg_csr *A, const double *b, const double *x,
                                   double *relres);

/* No counterpart in the reference.  The FP64 true relative residual of
 * rsg_true_relres for callers that cannot allocate device memory -- host
 * applications that give all device memory to their own pool allocator, or
 * that cannot accept the device-wide synchronisation of cudaMalloc/cudaFree
 * inside their loop.  It creates no context or handle and allocates nothing:
 * row_ptr (n_rows+1), col_idx, values, b, x and out3 are caller-owned device
 * arrays, out3 receives {||b - A x||, ||b||, ||b - A x|| / ||b||}, and the
 * kernel runs on `stream` (NULL = legacy default stream) without waiting for it.
 * Its scratch is a fixed 1 MiB array inside the library, held by every GPU that
 * loads the library until the process exits; n_rows above
 * RSG_NOALLOC_MAX_ROWS is rejected with RSG_ERR_INVALID_ARG.  Calls share that
 * array: calls whose kernels overlap on the GPU race and give wrong results,
 * so order them on one stream.  Each call looks up the array's address on
 * the current device (no allocation), so the entry point stays usable after
 * the application calls cudaDeviceReset; the first call on a device may load
 * the library's device code there, so make it before any stream capture.  A
 * column index >= n_rows is not read and makes the result NaN. */
#define RSG_NOALLOC_MAX_ROWS 2097152u
RSG_API rsg_status rsg_true_relres_noalloc(uint32_t n_rows, const uint32_t *row_ptr, const uint32_t *col_idx,
                                           const double *values, const double *b, const double *x, double *out3,
                                           void *stream);

/* ---- batched solves ----
 * Many independent systems of uneven size solved together (the reference
 * solves one system per RMatrixSolver::solve call, src/rmatrixsolver.cpp:158-201,
 * e.g. once per load case or per mesh).  The caller passes the systems as one
 * block-diagonal CSR (host arrays): system s owns rows and columns
 * [sys_row_begin[s], sys_row_begin[s+1]).  Each system is solved with CG (NONE
 * or JACOBI) to the FP64 true relative residual conf->rtol (stop_rule must be
 * RSG_STOP_TRUE_RELRES), in FP64 or mixed precision, with its own iteration
 * count and convergence; the whole batch is one device-driven loop. */
RSG_API rsg_status rsg_batch_create(rsg_context *ctx, uint32_t n_systems, const uint32_t *sys_row_begin,
                                    const uint32_t *row_ptr, const uint32_t *col_idx, const double *values,
                                    rsg_batch **out);
RSG_API void       rsg_batch_destroy(rsg_context *ctx, rsg_batch *batch);
RSG_API rsg_status rsg_batch_info(const rsg_batch *batch, uint32_t *n_systems, uint32_t *rows,
                                  uint32_t *padded_rows, uint64_t *nnz);
/* b and x: concatenated per system (rows of sys_row_begin), host or device per `memory`; x is in/out.
 * per_system (n_systems entries) and summary may be NULL. */
RSG_API rsg_status rsg_batch_solve(rsg_context *ctx, rsg_batch *batch, const rsg_solver_conf *conf, int32_t prec_type,
                                   const double *b, double *x, int32_t memory, rsg_stats *per_system,
                                   rsg_stats *summary);

/* ---- learned preconditioner ----
 * No counterpart in the reference (its preconditioners are NONE / JACOBI /
 * BLOCK_JACOBI, src/rmatrixpreconditioner.cpp).  A message-passing network over
 * the matrix graph maps a residual r to z = M(r) ~ A^{-1} r: node features are
 * the Jacobi-scaled residual, the diagonal, the row-sum ratio (non-zero next to
 * Dirichlet boundaries) and optional node coordinates; edge weights are the
 * normalised off-diagonals.  It is used as RSG_PREC_LEARNED (flexible CG, or
 * GMRES with flexible = 1) with Jacobi as fallback, and as an initial guess
 * (conf.learned_initial_guess).  All device arrays; xyz (3 per row) may be NULL.
 * Training minimises ||r - A M(r)||^2 / ||r||^2 with Adam on the GPU. */
RSG_API rsg_status rsg_learned_create(rsg_context *ctx, uint32_t layers, uint64_t seed, rsg_learned **out);
RSG_API void       rsg_learned_destroy(rsg_context *ctx, rsg_learned *model);
RSG_API rsg_status rsg_learned_info(const rsg_learned *model, uint32_t *layers, uint32_t *hidden, uint64_t *n_params,
                                    uint64_t *step);
/* which: 0 = parameters, 1 = last gradient, 2 = Adam first moment, 3 = Adam second moment (n_params floats) */
RSG_API rsg_status rsg_learned_get_params(rsg_context *ctx, const rsg_learned *model, float *host, int32_t which);
RSG_API rsg_status rsg_learned_set_params(rsg_context *ctx, rsg_learned *model, const float *host, int32_t which);
RSG_API rsg_status rsg_learned_set_step(rsg_learned *model, uint64_t step);
/* Training checkpoint (parameters, Adam moments, step) in a binary file with a
 * 64-byte "RSGGNN01" header (version, layers, width, features, parameter count). */
RSG_API rsg_status rsg_learned_save(rsg_context *ctx, const rsg_learned *model, const char *path);
RSG_API rsg_status rsg_learned_load(rsg_context *ctx, const char *path, rsg_learned **out);
/* z = M(r); tensor_cores != 0 runs the dense layers as BF16 MMA with FP32 accumulation, else FP32 */
RSG_API rsg_status rsg_learned_apply(rsg_context *ctx, rsg_learned *model, const rsg_csr *A, const double *r,
                                     double *z, const double *xyz, int32_t tensor_cores);
/* loss and gradient (into the model's gradient buffer) for one residual, no update */
RSG_API rsg_status rsg_learned_loss_grad(rsg_context *ctx, rsg_learned *model, const rsg_csr *A, const double *r,
                                         const double *xyz, int32_t tensor_cores, double *loss);
/* forward (tensor cores) + backward + one Adam step with learning rate lr */
RSG_API rsg_status rsg_learned_train_step(rsg_context *ctx, rsg_learned *model, const rsg_csr *A, const double *r,
                                          const double *xyz, float lr, double *loss);

/* ---- node books (DOF numbering) ----
 * The model's elements and element groups as plain arrays (host memory): element e has the nodes
 * elem_nodes[elem_begin[e] .. elem_begin[e+1]) -- any element type (points, lines, triangles,
 * tetrahedra); group g holds the elements group_elems[group_begin[g] .. group_begin[g+1]).
 * computable (n_elements flags) marks the elements the solver computes (RSolverGeneric's
 * computableElements); NULL = all.  Indexes out of range or decreasing begin arrays are rejected
 * with RSG_ERR_INVALID_ARG.  The book receives the free position of every DOF in index order, or
 * 0xffffffff (RConstants::eod) for a disabled one; *n_free the number of free DOFs.  These run on the
 * host and need no context. */
typedef struct {
    uint32_t n_nodes;
    uint32_t n_elements;
    const uint32_t *elem_begin;   /* n_elements + 1 */
    const uint32_t *elem_nodes;
    uint32_t n_groups;
    const uint32_t *group_begin;  /* n_groups + 1 */
    const uint32_t *group_elems;
    const uint8_t *computable;    /* n_elements, or NULL */
} rsg_model_groups;

/* RSolverGeneric::generateNodeBook + rebuildNodeBook (src/rsolvergeneric.cpp:498-582): one DOF per
 * node; the nodes of every group with group_explicit_bc[g] != 0 (an explicit boundary condition of
 * the problem type) and the nodes no computable element touches are disabled.  book: n_nodes. */
RSG_API rsg_status rsg_node_book_generic(const rsg_model_groups *model, const uint8_t *group_explicit_bc,
                                         uint32_t *book, uint32_t *n_free);

/* Displacement conditions of an element group for rsg_node_book_stress (bit mask: a group may carry several). */
enum {
    RSG_BC_DISPLACEMENT = 1,         /* R_BOUNDARY_CONDITION_DISPLACEMENT: all three components */
    RSG_BC_DISPLACEMENT_NORMAL = 2,  /* R_BOUNDARY_CONDITION_DISPLACEMENT_NORMAL: all three components */
    RSG_BC_DISPLACEMENT_ROLLER = 4   /* R_BOUNDARY_CONDITION_DISPLACEMENT_ROLLER: y and z on a line group, else x */
};
/* RSolverStress::generateNodeBook (src/rsolverstress.cpp:1564-1652): three interleaved DOFs per node
 * (position 3 node + component); group_bc[g] is a mask of RSG_BC_* and group_is_line[g] != 0 marks a
 * line (edge) group.  Nodes no computable element touches lose all three components.  book: 3 n_nodes. */
RSG_API rsg_status rsg_node_book_stress(const rsg_model_groups *model, const uint8_t *group_bc,
                                        const uint8_t *group_is_line, uint32_t *book, uint32_t *n_free);

/* ---- assembly (RSolverHeat / RSolverStress prepare + assemblyMatrix) ----
 * A plan is the sparsity pattern of the free-DOF system plus the
 * element-to-nonzero scatter map (the reference precedent is
 * RSolverFluid::buildSparseMatrixPattern, src/rsolverfluid.cpp:2305-2397).  It
 * is built once per mesh and node book; numeric assembly then runs on the GPU
 * without atomics and in a fixed order, so repeated assemblies are bitwise
 * identical. */
typedef struct rsg_assembly rsg_assembly;

typedef struct {
    int32_t transient;   /* time solver enabled */
    double  alpha;       /* time-march approximation coefficient (1 = backward Euler) */
    double  dt;
} rsg_time;

/* Heat: 1 DOF per node; book[i] = free position or 0xffffffff (RSolverGeneric::generateNodeBook,
 * src/rsolvergeneric.cpp:498-582).  All arrays host memory. */
RSG_API rsg_status rsg_assembly_create_heat(rsg_context *ctx, uint32_t n_nodes, const double *xyz,
                                            uint32_t n_tets, const uint32_t *tets, const uint32_t *book,
                                            uint32_t n_free, rsg_assembly **out);
/* Elasticity: 3 interleaved DOFs per node (RSolverStress::generateNodeBook,
 * src/rsolverstress.cpp:1564-1652); traction triangles add RHS only. */
RSG_API rsg_status rsg_assembly_create_stress(rsg_context *ctx, uint32_t n_nodes, const double *xyz,
                                              uint32_t n_tets, const uint32_t *tets, uint32_t n_tris,
                                              const uint32_t *tris, const uint32_t *book, uint32_t n_free,
                                              rsg_assembly **out);
/* Magnetostatics (vector potential): 3 interleaved DOFs per node (3 * position + component) with a
 * node's three DOFs enabled or disabled together -- one node book position per node, as
 * RSolverMagnetostatics::prepare/assemblyMatrix use it (src/rsolvermagnetostatics.cpp:46, :245, :261);
 * a book that disables some but not all of a node's components, or places them elsewhere than at
 * 3 * position + c, is rejected.  The pattern holds full
 * 3x3 blocks per node pair, the reference's zero entries between components included (:272-282). */
RSG_API rsg_status rsg_assembly_create_magnetostatics(rsg_context *ctx, uint32_t n_nodes, const double *xyz,
                                                      uint32_t n_tets, const uint32_t *tets, const uint32_t *book,
                                                      uint32_t n_free, rsg_assembly **out);
RSG_API void       rsg_assembly_destroy(rsg_context *ctx, rsg_assembly *plan);
RSG_API rsg_status rsg_assembly_info(const rsg_assembly *plan, uint32_t *n_free, uint64_t *nnz);
/* Solution back into the nodal field (device arrays): node_values[node*dofs + c] =
 * x[book[node*dofs + c]] for every free DOF, Dirichlet entries untouched -- the map
 * RSolverHeat/RSolverStress apply after solve (src/rsolverheat.cpp:466-483); with it
 * a transient step (assemble, solve, scatter) stays on the GPU. */
RSG_API rsg_status rsg_assembly_scatter(rsg_context *ctx, const rsg_assembly *plan, const double *x_device,
                                        double *node_values_device);

/* Heat numeric assembly, src/rsolverheat.cpp:361-455 (element loop) and :755-820
 * (theta scheme, Dirichlet lifting, scatter).  Per-tet arrays k_e, q_e, rhoc_e;
 * per-node node_t (prescribed values at disabled nodes, previous T when
 * transient).  Inputs in `memory`; writes the values of *A (created on the
 * first call, same pattern afterwards) and b (device, n_free doubles). */
RSG_API rsg_status rsg_assemble_heat(rsg_context *ctx, rsg_assembly *plan, const double *k_e, const double *q_e,
                                     const double *rhoc_e, const double *node_t, const rsg_time *time,
                                     int32_t memory, rsg_csr **A, double *b_device);

/* Elasticity numeric assembly, src/rsolverstress.cpp:384-715 and :1654-1772.
 * Per-tet e_mod, nu, rho_e, texp_e, dtemp_e; gravity[3]; per-triangle traction[3];
 * node_u (3 per node: prescribed displacement / previous displacement). */
RSG_API rsg_status rsg_assemble_stress(rsg_context *ctx, rsg_assembly *plan, const double *e_mod, const double *nu,
                                       const double *rho_e, const double *gravity, const double *texp_e,
                                       const double *dtemp_e, const double *traction, const double *node_u,
                                       const rsg_time *time, int32_t memory, rsg_csr **A, double *b_device);

/* Magnetostatic numeric assembly, src/rsolvermagnetostatics.cpp:57-137 (element loop) and
 * :234-287 (lifting, scatter): per tet and node pair -(grad N_m . grad N_n) V on each component,
 * right-hand side e0 V/4 (grad N_m x J_m) with J the nodal current density.  node_j: current
 * density (3 per node, the reference's convertElementToNodeVector output, :38-40); node_a:
 * prescribed potential at disabled nodes (3 per node).  Inputs in `memory`; writes *A and b
 * as rsg_assemble_heat. */
RSG_API rsg_status rsg_assemble_magnetostatics(rsg_context *ctx, rsg_assembly *plan, const double *node_j,
                                               const double *node_a, int32_t memory, rsg_csr **A,
                                               double *b_device);

#ifdef __cplusplus
}
#endif
#endif /* RSG_H */
