/*
 * CPU oracle for the sparse linear-solve path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain C++17 + OpenMP restatement of the reference library's
 * algorithms for the hot path.  It is the checker for the CUDA library, and
 * the timed CPU baseline in bench.py.  Nothing in the product (the CUDA
 * library under range-solver-lib_b200/) links, loads or calls it.
 *
 * Reference files restated (paths relative to the reference project):
 *   src/rmatrixsolver.cpp           CSR cache, Frobenius norm, row product,
 *                                   equation scaling, PCG, restarted GMRES
 *   src/rmatrixpreconditioner.cpp   Jacobi and block-Jacobi construct/apply
 *   src/riterationinfo.cpp          stopping rule (setError / hasConverged)
 *   src/rsolvergeneric.cpp          DOF numbering (node book)
 *   src/rsolverheat.cpp             P1 tet heat element + theta scheme + lifting
 *   src/rsolverstress.cpp           P1 tet elasticity element, traction, lifting
 *   src/rsolvermagnetostatics.cpp   P1 tet vector-potential element, curl source, lifting
 *
 * Parity pins: the reference's only known-answer tests
 * (tests/tst_matrix_solver.cpp:33-54 and :56-77) are reproduced by
 * tests/test_oracle.py.  Element formulas come from the absent range-model-lib
 * (shape functions, findJacobian) and are restated as the textbook linear
 * tetrahedron; those are pinned by manufactured-solution tests, not by the
 * reference ("parity unpinned" for quadrature details).
 */
#ifndef RSG_ORACLE_H
#define RSG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors RMatrixSolverConf fields read by src/rmatrixsolver.cpp:125-128,186. */
typedef struct {
    int32_t  solver_type;     /* 0 = CG, 1 = GMRES */
    uint32_t n_outer;         /* nOuterIterations */
    uint32_t n_inner;         /* nInnerIterations (GMRES restart length) */
    double   cvg;             /* solverCvgValue */
    double   eps;             /* stand-in for RConstants::eps (range-base-lib, absent) */
    int32_t  stop_rule;       /* 0 = RIterationInfo::hasConverged, 1 = true relative residual <= rtol */
    double   rtol;
    int32_t  scale_equations; /* 1 = reference's 1e9 equation scaling (rmatrixsolver.cpp:164-184) */
    int32_t  n_threads;       /* 0 = OpenMP default */
} orc_conf;

typedef struct {
    uint32_t iterations;      /* CG iterations, or GMRES inner steps in total */
    uint32_t outer;           /* GMRES restart cycles */
    double   error;           /* last reference error ||r||/(||A||_F ||x|| + ||b||) */
    double   trend;
    double   true_relres;     /* ||b - A x|| / ||b|| recomputed in long double */
    double   equation_scale;
    double   norm_a;
    double   norm_b;
    double   seconds;         /* wall time of the solve proper */
    int32_t  converged;
    int32_t  status;          /* 0 ok, <0 error */
} orc_stats;

/* a1 */ double orc_csr_frobenius(uint32_t n, const uint32_t *rp, const double *val);
/* a3 */ void   orc_spmv(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                         const double *x, double *y);
/* a7 */ void   orc_jacobi_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                                 double *d);
/* f1 */ int    orc_block_jacobi_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                                       uint32_t block_size, double *data, uint32_t *width_out);
/* a4-a9 */ int orc_solve(const orc_conf *conf, uint32_t n, const uint32_t *rp, const uint32_t *ci,
                          const double *val, int32_t prec_type, uint32_t block_size,
                          const double *b, double *x, orc_stats *stats);
double orc_true_relres(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val,
                       const double *b, const double *x);

/* a10: node book (RSolverGeneric::rebuildNodeBook).  book[i] = position or 0xffffffff. */
uint32_t orc_node_book(uint32_t n, const uint8_t *disabled, uint32_t *book);
/* RSolverGeneric::generateNodeBook (src/rsolvergeneric.cpp:498-561) + rebuildNodeBook: elements
 * e have nodes elem_nodes[elem_begin[e]..elem_begin[e+1]); group g holds group_elems[group_begin[g]..];
 * explicit_bc per group; computable per element (NULL = all).  Returns n_free. */
uint32_t orc_node_book_generic(uint32_t n_nodes, uint32_t n_elements, const uint32_t *elem_begin,
                               const uint32_t *elem_nodes, uint32_t n_groups, const uint32_t *group_begin,
                               const uint32_t *group_elems, const uint8_t *computable, const uint8_t *explicit_bc,
                               uint32_t *book);
/* RSolverStress::generateNodeBook (src/rsolverstress.cpp:1564-1652): bc bit mask per group
 * (1 displacement, 2 normal displacement, 4 roller), is_line per group.  book: 3 n_nodes. */
uint32_t orc_node_book_stress(uint32_t n_nodes, uint32_t n_elements, const uint32_t *elem_begin,
                              const uint32_t *elem_nodes, uint32_t n_groups, const uint32_t *group_begin,
                              const uint32_t *group_elems, const uint8_t *computable, const uint8_t *bc,
                              const uint8_t *is_line, uint32_t *book);

/* Assembled system handle (CSR with sorted columns + RHS). */
typedef struct orc_system orc_system;
uint32_t orc_system_n(const orc_system *s);
uint64_t orc_system_nnz(const orc_system *s);
void     orc_system_copy(const orc_system *s, uint32_t *rp, uint32_t *ci, double *val, double *b);
void     orc_system_free(orc_system *s);

/* a11/a12: heat conduction on linear tetrahedra. */
typedef struct {
    int32_t transient;        /* time solver enabled */
    double  alpha;            /* time-march approximation coefficient (1 = backward Euler) */
    double  dt;
    int32_t mass_rule;        /* quadrature of the mass integral N N^T over a tetrahedron: 0 exact
                                 (V (1 + d_mn) / 20, any rule of degree >= 2), 1 one centroid point
                                 (V / 16 for every pair), 2 row-sum lumped (V / 4 on the diagonal) */
} orc_time;

orc_system *orc_assemble_heat(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                              const double *k_e, const double *q_e, const double *rhoc_e,
                              const double *node_t, const uint32_t *book, uint32_t n_free,
                              const orc_time *time);

/* a14-a17: linear elasticity on linear tetrahedra (3 dofs per node, interleaved). */
orc_system *orc_assemble_stress(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                                const double *e_mod, const double *nu, const double *rho_e,
                                const double *gravity /* 3 */, const double *texp_e, const double *dtemp_e,
                                uint32_t n_tris, const uint32_t *tris, const double *traction /* n_tris*3 */,
                                const double *node_u /* 3*n_nodes */, const uint32_t *book /* 3*n_nodes */,
                                uint32_t n_free, const orc_time *time);

/* f4: magnetostatics (vector potential, 3 dofs per node interleaved, a node's three dofs enabled or
 * disabled together); node_j = nodal current density, node_a = prescribed potential (3*n_nodes each). */
orc_system *orc_assemble_magnetostatics(uint32_t n_nodes, const double *xyz, uint32_t n_tets, const uint32_t *tets,
                                        const double *node_j, const double *node_a, const uint32_t *book,
                                        uint32_t n_free);

/* Multilevel aggregation preconditioner (no reference counterpart; the checker of the CUDA
 * library's RSG_PREC_AMG): the same aggregation (strength threshold, distance-2 independent roots
 * of hashed priorities in synchronous rounds, joins, singletons), the same Galerkin summation order
 * and stopping rule of the coarsening, and the cycle in FP64 (levels 1 and 2 solved by two
 * flexible-CG steps each: a K-cycle). */
typedef struct orc_amg orc_amg;
orc_amg *orc_amg_build(uint32_t n, const uint32_t *rp, const uint32_t *ci, const double *val);
uint32_t orc_amg_levels(const orc_amg *h);
int32_t orc_amg_dense_coarsest(const orc_amg *h);
uint32_t orc_amg_rows(const orc_amg *h, uint32_t level);
uint64_t orc_amg_nnz(const orc_amg *h, uint32_t level);
/* agg (rows of the level; not for the last level), row_ptr, col_idx, values: any may be NULL */
void orc_amg_level(const orc_amg *h, uint32_t level, uint32_t *agg, uint32_t *row_ptr, uint32_t *col_idx,
                   double *values);
/* z = one cycle applied to r (FP64), sweeps 1 or 2 per side */
void orc_amg_apply(const orc_amg *h, const double *r, double *z, uint32_t sweeps);
void orc_amg_free(orc_amg *h);

/* RSolverFluid::buildSparseMatrixPattern + assemblyMatrix (src/rsolverfluid.cpp:2305-2419): the pattern
 * of the active elements' enabled DOFs, then every active element's Ae / fe added in element order.
 * Returns nnz; rp / ci / val / b are filled when non-NULL (call once with NULLs to size them). */
uint64_t orc_scatter_assemble(uint32_t d, uint32_t n_elements, const uint32_t *elem_begin, const uint32_t *elem_nodes,
                              const uint8_t *elem_active, uint32_t n_nodes, const uint32_t *book, uint32_t n_free,
                              const double *Ae, const double *fe, uint32_t *rp, uint32_t *ci, double *val, double *b);

#ifdef __cplusplus
}
#endif
#endif
