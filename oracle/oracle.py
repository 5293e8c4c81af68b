"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker / the timed CPU baseline.  The CUDA library
never calls it.  Build with `make -C oracle` (done by __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

EOD = 0xFFFFFFFF


class OrcConf(C.Structure):
    _fields_ = [
        ("solver_type", C.c_int32),
        ("n_outer", C.c_uint32),
        ("n_inner", C.c_uint32),
        ("cvg", C.c_double),
        ("eps", C.c_double),
        ("stop_rule", C.c_int32),
        ("rtol", C.c_double),
        ("scale_equations", C.c_int32),
        ("n_threads", C.c_int32),
    ]


class OrcStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_uint32),
        ("outer", C.c_uint32),
        ("error", C.c_double),
        ("trend", C.c_double),
        ("true_relres", C.c_double),
        ("equation_scale", C.c_double),
        ("norm_a", C.c_double),
        ("norm_b", C.c_double),
        ("seconds", C.c_double),
        ("converged", C.c_int32),
        ("status", C.c_int32),
    ]


class OrcTime(C.Structure):
    _fields_ = [("transient", C.c_int32), ("alpha", C.c_double), ("dt", C.c_double), ("mass_rule", C.c_int32)]


# quadrature of the P1 mass integral (orc_time.mass_rule)
MASS_EXACT, MASS_CENTROID, MASS_LUMPED = 0, 1, 2


_P = C.c_void_p


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(path)
        L.orc_csr_frobenius.restype = C.c_double
        L.orc_csr_frobenius.argtypes = [C.c_uint32, _P, _P]
        L.orc_spmv.argtypes = [C.c_uint32, _P, _P, _P, _P, _P]
        L.orc_jacobi_build.argtypes = [C.c_uint32, _P, _P, _P, _P]
        L.orc_block_jacobi_build.restype = C.c_int
        L.orc_block_jacobi_build.argtypes = [C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.POINTER(C.c_uint32)]
        L.orc_solve.restype = C.c_int
        L.orc_solve.argtypes = [C.POINTER(OrcConf), C.c_uint32, _P, _P, _P, C.c_int32, C.c_uint32, _P, _P,
                                C.POINTER(OrcStats)]
        L.orc_true_relres.restype = C.c_double
        L.orc_true_relres.argtypes = [C.c_uint32, _P, _P, _P, _P, _P]
        L.orc_node_book.restype = C.c_uint32
        L.orc_node_book.argtypes = [C.c_uint32, _P, _P]
        L.orc_amg_build.restype = C.c_void_p
        L.orc_amg_build.argtypes = [C.c_uint32, _P, _P, _P]
        L.orc_amg_levels.restype = C.c_uint32
        L.orc_amg_levels.argtypes = [_P]
        L.orc_amg_dense_coarsest.restype = C.c_int32
        L.orc_amg_dense_coarsest.argtypes = [_P]
        L.orc_amg_rows.restype = C.c_uint32
        L.orc_amg_rows.argtypes = [_P, C.c_uint32]
        L.orc_amg_nnz.restype = C.c_uint64
        L.orc_amg_nnz.argtypes = [_P, C.c_uint32]
        L.orc_amg_level.argtypes = [_P, C.c_uint32, _P, _P, _P, _P]
        L.orc_amg_apply.argtypes = [_P, _P, _P, C.c_uint32]
        L.orc_amg_free.argtypes = [_P]
        L.orc_node_book_generic.restype = C.c_uint32
        L.orc_node_book_generic.argtypes = [C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P, _P, _P]
        L.orc_scatter_assemble.restype = C.c_uint64
        L.orc_scatter_assemble.argtypes = [C.c_uint32, C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.c_uint32, _P, _P,
                                           _P, _P, _P, _P]
        L.orc_node_book_stress.restype = C.c_uint32
        L.orc_node_book_stress.argtypes = [C.c_uint32, C.c_uint32, _P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P]
        L.orc_system_n.restype = C.c_uint32
        L.orc_system_n.argtypes = [_P]
        L.orc_system_nnz.restype = C.c_uint64
        L.orc_system_nnz.argtypes = [_P]
        L.orc_system_copy.argtypes = [_P, _P, _P, _P, _P]
        L.orc_system_free.argtypes = [_P]
        L.orc_assemble_heat.restype = _P
        L.orc_assemble_heat.argtypes = [C.c_uint32, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint32,
                                        C.POINTER(OrcTime)]
        L.orc_assemble_stress.restype = _P
        L.orc_assemble_stress.argtypes = [C.c_uint32, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, _P, C.c_uint32, _P,
                                          _P, _P, _P, C.c_uint32, C.POINTER(OrcTime)]
        L.orc_assemble_magnetostatics.restype = _P
        L.orc_assemble_magnetostatics.argtypes = [C.c_uint32, _P, C.c_uint32, _P, _P, _P, _P, C.c_uint32]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class CSR:
    n: int
    rp: np.ndarray  # uint32 (n+1)
    ci: np.ndarray  # uint32
    val: np.ndarray  # float64

    @property
    def nnz(self) -> int:
        return int(self.ci.shape[0])

    def to_dense(self) -> np.ndarray:
        A = np.zeros((self.n, self.n))
        for i in range(self.n):
            A[i, self.ci[self.rp[i]:self.rp[i + 1]]] += self.val[self.rp[i]:self.rp[i + 1]]
        return A


def csr_from_dense(A: np.ndarray) -> CSR:
    n = A.shape[0]
    rp = [0]
    ci = []
    val = []
    for i in range(n):
        for j in range(n):
            if A[i, j] != 0.0:
                ci.append(j)
                val.append(A[i, j])
        rp.append(len(ci))
    return CSR(n, np.asarray(rp, np.uint32), np.asarray(ci, np.uint32), np.asarray(val, np.float64))


def frobenius(A: CSR) -> float:
    return lib().orc_csr_frobenius(A.n, _ptr(A.rp), _ptr(A.val))


def spmv(A: CSR, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float64)
    y = np.empty(A.n)
    lib().orc_spmv(A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val), _ptr(x), _ptr(y))
    return y


def jacobi(A: CSR) -> np.ndarray:
    d = np.empty(A.n)
    lib().orc_jacobi_build(A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val), _ptr(d))
    return d


def block_jacobi(A: CSR, block_size: int):
    data = np.empty(A.n * max(block_size, 1))
    w = C.c_uint32(0)
    rc = lib().orc_block_jacobi_build(A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val), block_size, _ptr(data), C.byref(w))
    if rc != 0:
        raise RuntimeError("singular diagonal block")
    return data[: A.n * w.value].reshape(A.n, w.value), w.value


def true_relres(A: CSR, b: np.ndarray, x: np.ndarray) -> float:
    b = np.ascontiguousarray(b, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    return lib().orc_true_relres(A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val), _ptr(b), _ptr(x))


def make_conf(solver: str = "cg", n_outer: int = 1000, n_inner: int = 30, cvg: float = 1e-13, eps: float = 1e-14,
              stop_rule: str = "reference", rtol: float = 1e-10, scale: bool = True, threads: int = 0) -> OrcConf:
    return OrcConf(0 if solver == "cg" else 1, n_outer, n_inner, cvg, eps, 0 if stop_rule == "reference" else 1,
                   rtol, 1 if scale else 0, threads)


def solve(A: CSR, b: np.ndarray, x0: np.ndarray | None = None, *, prec: int = 1, block_size: int = 1,
          conf: OrcConf | None = None, **kw):
    """RMatrixSolver::solve restated: returns (x, stats)."""
    conf = conf or make_conf(**kw)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n) if x0 is None else np.array(x0, np.float64, copy=True)
    st = OrcStats()
    rc = lib().orc_solve(C.byref(conf), A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val), prec, block_size, _ptr(b), _ptr(x),
                         C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle solve failed: {rc}")
    return x, st


def node_book_generic(n_nodes, elem_begin, elem_nodes, group_begin, group_elems, explicit_bc, computable=None):
    """RSolverGeneric::generateNodeBook (src/rsolvergeneric.cpp:498-582): (book, n_free)."""
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (elem_begin, elem_nodes, group_begin, group_elems)]
    flags = np.ascontiguousarray(explicit_bc, np.uint8)
    comp = None if computable is None else np.ascontiguousarray(computable, np.uint8)
    book = np.empty(n_nodes, np.uint32)
    n_free = lib().orc_node_book_generic(n_nodes, len(arrs[0]) - 1, _ptr(arrs[0]), _ptr(arrs[1]), len(arrs[2]) - 1,
                                         _ptr(arrs[2]), _ptr(arrs[3]), None if comp is None else _ptr(comp),
                                         _ptr(flags), _ptr(book))
    return book, int(n_free)


def node_book_stress(n_nodes, elem_begin, elem_nodes, group_begin, group_elems, bc, is_line, computable=None):
    """RSolverStress::generateNodeBook (src/rsolverstress.cpp:1564-1652): (book of 3 n_nodes, n_free)."""
    arrs = [np.ascontiguousarray(a, np.uint32) for a in (elem_begin, elem_nodes, group_begin, group_elems)]
    bcs = np.ascontiguousarray(bc, np.uint8)
    line = np.ascontiguousarray(is_line, np.uint8)
    comp = None if computable is None else np.ascontiguousarray(computable, np.uint8)
    book = np.empty(3 * n_nodes, np.uint32)
    n_free = lib().orc_node_book_stress(n_nodes, len(arrs[0]) - 1, _ptr(arrs[0]), _ptr(arrs[1]), len(arrs[2]) - 1,
                                        _ptr(arrs[2]), _ptr(arrs[3]), None if comp is None else _ptr(comp),
                                        _ptr(bcs), _ptr(line), _ptr(book))
    return book, int(n_free)


class Amg:
    """The multilevel aggregation preconditioner built on the host (the checker of RSG_PREC_AMG)."""

    def __init__(self, A: CSR):
        self.h = C.c_void_p(lib().orc_amg_build(A.n, _ptr(A.rp), _ptr(A.ci), _ptr(A.val)))
        L = lib()
        self.levels = int(L.orc_amg_levels(self.h))
        self.dense_coarsest = bool(L.orc_amg_dense_coarsest(self.h))
        self.rows = [int(L.orc_amg_rows(self.h, l)) for l in range(self.levels)]
        self.nnz = [int(L.orc_amg_nnz(self.h, l)) for l in range(self.levels)]

    def level(self, l: int):
        """(agg or None, CSR) of level l."""
        n, nnz = self.rows[l], self.nnz[l]
        agg = np.empty(n, np.uint32) if l + 1 < self.levels else None
        rp = np.empty(n + 1, np.uint32)
        ci = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        lib().orc_amg_level(self.h, l, None if agg is None else _ptr(agg), _ptr(rp), _ptr(ci), _ptr(val))
        return agg, CSR(n, rp, ci, val)

    def apply(self, r: np.ndarray, sweeps: int = 2) -> np.ndarray:
        r = np.ascontiguousarray(r, np.float64)
        z = np.empty_like(r)
        lib().orc_amg_apply(self.h, _ptr(r), _ptr(z), sweeps)
        return z

    def close(self):
        if self.h:
            lib().orc_amg_free(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _system(h) -> tuple[CSR, np.ndarray]:
    L = lib()
    n = L.orc_system_n(h)
    nnz = L.orc_system_nnz(h)
    rp = np.empty(n + 1, np.uint32)
    ci = np.empty(nnz, np.uint32)
    val = np.empty(nnz, np.float64)
    b = np.empty(n, np.float64)
    L.orc_system_copy(h, _ptr(rp), _ptr(ci), _ptr(val), _ptr(b))
    L.orc_system_free(h)
    return CSR(n, rp, ci, val), b


def assemble_heat(p, mass_rule: int = MASS_EXACT) -> tuple[CSR, np.ndarray]:
    """RSolverHeat::prepare + assemblyMatrix restated for a rsg.workloads.HeatProblem.  mass_rule picks
    the quadrature of the transient mass integral, which the reference takes from range-model-lib's
    tetrahedron rule (absent here): exact (the default, as the GPU assembly), centroid or lumped."""
    m = p.mesh
    xyz = np.ascontiguousarray(m.xyz, np.float64)
    tets = np.ascontiguousarray(m.tets, np.uint32)
    k = np.ascontiguousarray(p.k_e, np.float64)
    q = np.ascontiguousarray(p.q_e, np.float64)
    rc = np.ascontiguousarray(p.rhoc_e, np.float64)
    nt = np.ascontiguousarray(p.node_t, np.float64)
    book = np.ascontiguousarray(p.book, np.uint32)
    tm = OrcTime(1 if p.transient else 0, p.alpha, p.dt, mass_rule)
    h = lib().orc_assemble_heat(m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets), _ptr(k), _ptr(q), _ptr(rc), _ptr(nt),
                                _ptr(book), p.n_free, C.byref(tm))
    return _system(h)


def transient_heat(p, steps: int, *, mass_rule: int = MASS_EXACT, rtol: float = 1e-12) -> list[np.ndarray]:
    """The reference's transient time loop for heat (src/rsolver.cpp:106-144: every step re-assembles
    with the previous step's temperatures, src/rsolverheat.cpp:768-779, and solves with CG + Jacobi,
    the previous solution as the initial guess).  Returns the node temperatures after each step; p is
    not modified."""
    import copy
    q = copy.copy(p)
    q.node_t = np.array(p.node_t, np.float64, copy=True)
    free = q.book != 0xFFFFFFFF
    idx = q.book[free].astype(np.int64)
    out = []
    for _ in range(steps):
        A, b = assemble_heat(q, mass_rule)
        x0 = np.empty(A.n)
        x0[idx] = q.node_t[free]
        x, st = solve(A, b, x0, prec=1, n_outer=100000, stop_rule="true", rtol=rtol)
        q.node_t[free] = x[idx]
        out.append(q.node_t.copy())
    return out


def assemble_stress(p, mass_rule: int = MASS_EXACT) -> tuple[CSR, np.ndarray]:
    """RSolverStress::prepare + assemblyMatrix restated for a rsg.workloads.StressProblem (mass_rule as
    for assemble_heat)."""
    m = p.mesh
    arrs = [np.ascontiguousarray(a, np.float64) for a in (m.xyz, p.e_mod, p.nu, p.rho_e, p.gravity, p.texp_e,
                                                          p.dtemp_e, p.traction, p.node_u)]
    xyz, e, nu, rho, g, te, dte, tr, nu_ = arrs
    tets = np.ascontiguousarray(m.tets, np.uint32)
    tris = np.ascontiguousarray(p.tris, np.uint32)
    book = np.ascontiguousarray(p.book, np.uint32)
    tm = OrcTime(1 if p.transient else 0, p.alpha, p.dt, mass_rule)
    h = lib().orc_assemble_stress(m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets), _ptr(e), _ptr(nu), _ptr(rho), _ptr(g),
                                  _ptr(te), _ptr(dte), tris.shape[0], _ptr(tris), _ptr(tr), _ptr(nu_), _ptr(book),
                                  p.n_free, C.byref(tm))
    return _system(h)


def assemble_magnetostatics(p) -> tuple[CSR, np.ndarray]:
    """RSolverMagnetostatics::prepare + assemblyMatrix restated for a rsg.workloads.MagnetostaticProblem."""
    m = p.mesh
    xyz = np.ascontiguousarray(m.xyz, np.float64)
    tets = np.ascontiguousarray(m.tets, np.uint32)
    j = np.ascontiguousarray(p.node_j, np.float64)
    a = np.ascontiguousarray(p.node_a, np.float64)
    book = np.ascontiguousarray(p.book, np.uint32)
    h = lib().orc_assemble_magnetostatics(m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets), _ptr(j), _ptr(a), _ptr(book),
                                          p.n_free)
    return _system(h)


# ---- eigenvalues of the pencil (M, K): REigenValueSolver restated (src/reigenvaluesolver.cpp) ----
EIGEN_LANCZOS, EIGEN_ARNOLDI, EIGEN_RAYLEIGH = 0, 1, 2


def _sdot(x: np.ndarray, y: np.ndarray) -> float:
    """Sum of products in index order (RRVector::dot)."""
    return float(np.cumsum(x * y)[-1]) if len(x) else 0.0


def _qr_iteration(H: np.ndarray, n_iterations: int, cvg: float):
    """qrDecomposition (src/reigenvaluesolver.cpp:499-592): unshifted QR iteration by classical
    Gram-Schmidt, A <- R Q, V <- V Q, until every subdiagonal entry is at most cvg."""
    m = H.shape[0]
    A = H.copy()
    V = np.zeros((m, m))
    Q = np.zeros((m, m))
    R = np.zeros((m, m))
    for it in range(n_iterations):
        for i in range(m):
            a = A[:, i].copy()
            u = a.copy()
            for j in range(i):
                e = Q[:, j]
                u = u - _sdot(a, e) * e
            nu = np.sqrt(_sdot(u, u))
            if nu == 0.0:
                raise RuntimeError("QR iteration met a dependent column")
            Q[:, i] = u * (1.0 / nu)
        for i in range(m):
            e = Q[:, i]
            for j in range(i, m):
                R[i, j] = _sdot(A[:, j], e)
        A = np.array([[_sdot(R[r, :], Q[:, c]) for c in range(m)] for r in range(m)])
        V = Q.copy() if it == 0 else np.array([[_sdot(V[r, :], Q[:, c]) for c in range(m)] for r in range(m)])
        if all(abs(A[i, i - 1]) <= cvg for i in range(1, m)):
            break
    return np.diag(A).copy(), V


def eigen_solve(M: CSR, K: CSR, method: int, n_eigen: int, start: np.ndarray, *, mu0: float = 0.0,
                n_iterations: int = 100, eig_cvg: float = 1e-8, **solve_kw):
    """REigenValueSolver::solve restated (src/reigenvaluesolver.cpp:40-110 and the three methods);
    every linear solve is the oracle's RMatrixSolver::solve with Jacobi and solve_kw, its x the
    previous vector as in the reference.  start: the n start values (normalised here); eig_cvg: the
    eigenvalue solver's own bound (QR subdiagonal, Rayleigh |mu - mu_old|).  Returns
    (values, vectors or None, number of solves)."""
    conf = make_conf(**solve_kw)
    n = K.n
    v = np.array(start, np.float64, copy=True)
    v = v / np.sqrt(_sdot(v, v))
    solves = 0
    vec = None
    if method == EIGEN_LANCZOS:  # :119-210; qlDecomposition (:420-497) leaves d unchanged
        ne = min(n_eigen, n)
        d, e = np.zeros(ne), np.zeros(ne + 1)
        vo, w = np.zeros(n), np.zeros(n)
        for i in range(ne):
            b = spmv(M, v)
            if i > 0:
                b = b - spmv(K, vo) * e[i]
            w, _ = solve(K, b, w, prec=1, conf=conf)
            solves += 1
            d[i] = _sdot(w, v)
            if i + 1 < ne:
                w = w - d[i] * v
                e[i + 1] = np.sqrt(_sdot(w, w))
                vo = v
                v = w / e[i + 1]
    elif method == EIGEN_ARNOLDI:  # :211-294
        ne = min(n_eigen, n)
        H = np.zeros((ne, ne))
        Qa = np.zeros((n, ne))
        Qa[:, 0] = v
        q = v.copy()
        for i in range(1, ne + 1):
            q, _ = solve(K, spmv(M, Qa[:, i - 1].copy()), q, prec=1, conf=conf)
            solves += 1
            for j in range(i):
                H[j, i - 1] = _sdot(Qa[:, j], q)
                q = q - H[j, i - 1] * Qa[:, j]
            if i < ne:
                H[i, i - 1] = np.sqrt(_sdot(q, q))
                Qa[:, i] = q / H[i, i - 1]
        d, V = _qr_iteration(H, n_iterations, eig_cvg)
        vec = (Qa @ V).T.copy()
    else:  # Rayleigh quotient iteration, :295-392 (M and K on one pattern)
        m2 = M.val.copy()
        c, dd = np.zeros(n), np.zeros(n)
        b = v
        mu = mu0
        for it in range(n_iterations):
            muo = mu
            kv = K.val * mu
            m2 = np.where(kv != 0.0, m2 + kv, m2)
            f = spmv(CSR(n, K.rp, K.ci, kv), b)
            c, _ = solve(CSR(n, M.rp, M.ci, m2), f, c, prec=1, conf=conf)
            f = f * (1.0 / np.sqrt(_sdot(c, c)))
            b, _ = solve(M, f, b, prec=1, conf=conf)
            kv = -1.0 * K.val * mu
            m2 = np.where(kv != 0.0, m2 + kv, m2)
            dd, _ = solve(K, spmv(CSR(n, M.rp, M.ci, m2), b), dd, prec=1, conf=conf)
            solves += 3
            mu = _sdot(dd, b) / _sdot(b, b)
            if it > 0 and abs(muo - mu) < eig_cvg:
                break
        d = np.array([mu])
        vec = b[None, :].copy()
    if len(d) > 1:  # solve(), :90-110
        d = np.abs(1.0 / d)
        d[0], d[1] = d[1], d[0]
        order = np.argsort(d, kind="stable")
        d = d[order]
        if vec is not None:
            vec = vec[order]
    return d, vec, solves


def scatter_assemble(d: int, elem_begin, elem_nodes, elem_active, n_nodes: int, book, n_free: int, Ae, fe):
    """RSolverFluid::buildSparseMatrixPattern + assemblyMatrix (src/rsolverfluid.cpp:2305-2419) restated:
    (CSR, b) of the active elements' blocks Ae / fe (concatenated in element order)."""
    eb = np.ascontiguousarray(elem_begin, np.uint32)
    en = np.ascontiguousarray(elem_nodes, np.uint32)
    act = None if elem_active is None else np.ascontiguousarray(elem_active, np.uint8)
    bk = np.ascontiguousarray(book, np.uint32)
    ae = np.ascontiguousarray(Ae, np.float64)
    fv = np.ascontiguousarray(fe, np.float64)
    args = (d, len(eb) - 1, _ptr(eb), _ptr(en), None if act is None else _ptr(act), n_nodes, _ptr(bk), n_free)
    nnz = lib().orc_scatter_assemble(*args, None, None, None, None, None, None)
    rp = np.empty(n_free + 1, np.uint32)
    ci = np.empty(nnz, np.uint32)
    val = np.empty(nnz, np.float64)
    b = np.empty(n_free, np.float64)
    lib().orc_scatter_assemble(*args, _ptr(ae), _ptr(fv), _ptr(rp), _ptr(ci), _ptr(val), _ptr(b))
    return CSR(n_free, rp, ci, val), b
