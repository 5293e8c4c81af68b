"""Python host layer over librsg.so (the B200 sparse linear-solve library).

Mirrors the reference's RMatrixSolver interface (include/rmatrixsolver.h):
`Solver(conf).solve(A, b, x, preconditioner, block_size)` with the same
argument meaning; the numerical work runs in the CUDA library through the C
ABI declared in include/rsg.h.  Host arrays are numpy; device arrays may be
passed as any object with `data_ptr()` (e.g. torch CUDA tensors).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (BREAKDOWN, ERR_INVALID_ARG, ERR_SINGULAR, ERR_UNSUPPORTED, MEM_DEVICE, MEM_HOST, NOT_CONVERGED,
                   OK, PREC_AMG, PREC_BLOCK_JACOBI, PREC_JACOBI, PREC_LEARNED, PREC_NONE, PRECISION_FP64,
                   PRECISION_MIXED, PRECISION_AUTO,
                   SOLVER_CG, SOLVER_GMRES, STOP_REFERENCE, STOP_TRUE_RELRES, RsgError, SolverConf, Stats, Time,
                   EIGEN_ARNOLDI, EIGEN_LANCZOS, EIGEN_RAYLEIGH)

__all__ = ["Context", "Matrix", "Assembly", "ScatterPlan", "Batch", "make_conf", "RsgError", "SolverConf", "Stats", "Solver"]


def _ptr(a) -> C.c_void_p:
    if a is None:
        return C.c_void_p(0)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _is_device(a) -> bool:
    return hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)


def make_conf(solver: str | int = "cg", n_outer: int = 1000, n_inner: int = 30, cvg: float = 1e-13,
              eps: float = 1e-14, stop_rule: str | int = "reference", rtol: float = 1e-10,
              precision: str | int = "fp64", scale_equations: bool = True, reliable_delta: float = 1e-3,
              flexible: bool = False, use_graph: bool = True, check_interval: int = 16,
              output_frequency: int = 0, output_file: str | None = None,
              l2_resident_f32: bool = False, autotune: bool = False, amg_sweeps: int = 1,
              persistent: int = 0) -> SolverConf:
    c = SolverConf()
    _lib.load().rsg_conf_default(C.byref(c))
    c.solver_type = solver if isinstance(solver, int) else {"cg": SOLVER_CG, "gmres": SOLVER_GMRES}[solver]
    c.n_outer = n_outer
    c.n_inner = n_inner
    c.cvg = cvg
    c.eps = eps
    c.stop_rule = stop_rule if isinstance(stop_rule, int) else {"reference": STOP_REFERENCE,
                                                                 "true": STOP_TRUE_RELRES}[stop_rule]
    c.rtol = rtol
    c.precision = precision if isinstance(precision, int) else {"fp64": PRECISION_FP64,
                                                                 "mixed": PRECISION_MIXED,
                                                                 "auto": PRECISION_AUTO}[precision]
    c.scale_equations = 1 if scale_equations else 0
    c.reliable_delta = reliable_delta
    c.flexible = 1 if flexible else 0
    c.use_graph = 1 if use_graph else 0
    c.check_interval = check_interval
    c.output_frequency = output_frequency
    c.output_file = output_file.encode() if output_file else None
    c.l2_resident_f32 = 1 if l2_resident_f32 else 0
    c.autotune = 1 if autotune else 0
    c.amg_sweeps = amg_sweeps
    c.persistent = persistent
    return c


class Context:
    """One GPU, one CUDA stream (rsg_context)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        s = self.lib.rsg_context_create(device, C.byref(h))
        if s != OK:
            raise RsgError(s, f"rsg_context_create({device}) failed: {self.lib.rsg_status_string(s).decode()}")
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            self.lib.rsg_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, s: int, what: str, allow=(OK,)):
        if s not in allow:
            raise RsgError(s, f"{what}: {self.lib.rsg_status_string(s).decode()}: "
                              f"{self.lib.rsg_last_error(self.h).decode()}")
        return s

    def sync(self):
        self.check(self.lib.rsg_synchronize(self.h), "synchronize")

    def set_stream(self, stream_ptr: int | None):
        self.check(self.lib.rsg_context_set_stream(self.h, C.c_void_p(stream_ptr or 0)), "set_stream")

    # ---- matrices ----
    def matrix(self, rp, ci, val) -> "Matrix":
        dev = _is_device(rp)
        if not dev:
            rp = np.ascontiguousarray(rp, np.uint32)
            ci = np.ascontiguousarray(ci, np.uint32)
            val = np.ascontiguousarray(val, np.float64)
        n = int(rp.shape[0]) - 1
        h = C.c_void_p()
        self.check(self.lib.rsg_csr_create(self.h, n, _ptr(rp), _ptr(ci), _ptr(val), MEM_DEVICE if dev else MEM_HOST,
                                           C.byref(h)), "csr_create")
        return Matrix(self, h)

    # ---- solve ----
    def solve(self, A: "Matrix", b, x=None, conf: SolverConf | None = None, prec: int = PREC_JACOBI,
              block_size: int = 1, allow=(OK, NOT_CONVERGED, BREAKDOWN), inplace: bool = False):
        """RMatrixSolver::solve: returns (x, Stats).  Device arrays are updated in place; a host x is
        copied first unless inplace=True (then a C-contiguous float64 x is the in/out array itself, as
        the C ABI's x is -- which keeps a pinned x pinned)."""
        conf = conf or make_conf()
        st = Stats()
        if _is_device(b):
            if x is None:
                raise ValueError("device solve needs an x array")
            s = self.lib.rsg_solve(self.h, A.h, C.byref(conf), prec, block_size, _ptr(b), _ptr(x), MEM_DEVICE,
                                   C.byref(st))
        else:
            b = np.ascontiguousarray(b, np.float64)
            if inplace and isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous:
                pass
            else:
                x = np.zeros(A.n) if x is None else np.array(x, np.float64, copy=True)
            s = self.lib.rsg_solve(self.h, A.h, C.byref(conf), prec, block_size, _ptr(b), _ptr(x), MEM_HOST,
                                   C.byref(st))
        self.check(s, "solve", allow)
        return x, st

    def solve_multi(self, A: "Matrix", B, X=None, conf: SolverConf | None = None, prec: int = PREC_JACOBI,
                    allow=(OK, NOT_CONVERGED, BREAKDOWN)):
        """k right-hand sides of one matrix (rsg_solve_multi).  B: (k, n) array, one
        right-hand side per row (numpy, or a contiguous CUDA tensor; then X must be one
        too and is updated in place).  Returns (X, [Stats per column], summary Stats)."""
        conf = conf or make_conf(stop_rule="true")
        k = int(B.shape[0])
        per = (Stats * k)()
        summ = Stats()
        if _is_device(B):
            if X is None:
                raise ValueError("device solve_multi needs an X array")
            s = self.lib.rsg_solve_multi(self.h, A.h, C.byref(conf), prec, k, _ptr(B), _ptr(X), MEM_DEVICE, per,
                                         C.byref(summ))
        else:
            B = np.ascontiguousarray(B, np.float64)
            X = np.zeros_like(B) if X is None else np.array(X, np.float64, copy=True)
            s = self.lib.rsg_solve_multi(self.h, A.h, C.byref(conf), prec, k, _ptr(B), _ptr(X), MEM_HOST, per,
                                         C.byref(summ))
        self.check(s, "solve_multi", allow)
        return X, list(per), summ

    # ---- multilevel aggregation preconditioner ----
    def amg_setup(self, A: "Matrix", conf: SolverConf | None = None) -> dict:
        """Build A's hierarchy from its current values (rsg_amg_setup, or rsg_amg_setup_conf: as a
        solve with conf builds it); returns its shape."""
        info = _lib.AmgInfo()
        if conf is None:
            self.check(self.lib.rsg_amg_setup(self.h, A.h, C.byref(info)), "amg_setup")
        else:
            self.check(self.lib.rsg_amg_setup_conf(self.h, A.h, C.byref(conf), C.byref(info)), "amg_setup")
        L = info.levels
        return {"levels": L, "dense_coarsest": bool(info.dense_coarsest), "rows": list(info.rows[:L]),
                "nnz": list(info.nnz[:L]), "mis_rounds": info.mis_rounds, "seconds_setup": info.seconds_setup,
                "setup_launches": info.setup_launches, "cycle_launches": list(info.cycle_launches),
                "persist_level": info.persist_level}

    def eigen_solve(self, M: "Matrix", K: "Matrix", start, method: int = _lib.EIGEN_LANCZOS, n_eigen: int = 4,
                    n_iterations: int = 100, cvg: float = 1e-8, mu0: float = 0.0, conf=None):
        """Eigenvalues of the pencil (M, K) by REigenValueSolver's methods (rsg_eigen_solve): returns
        (values, vectors or None, stats dict).  start: the n start values (the reference draws them
        with rand() / RAND_MAX); conf: the linear solves' configuration (default: CG, Jacobi,
        FP64 true relative residual 1e-12)."""
        start = np.ascontiguousarray(start, np.float64)
        ec = _lib.EigenConf(method=method, n_eigen=n_eigen, n_iterations=n_iterations, cvg=cvg, mu0=mu0)
        conf = conf if conf is not None else make_conf(n_outer=100000, stop_rule="true", rtol=1e-12)
        nv = 1 if method == _lib.EIGEN_RAYLEIGH else min(n_eigen, K.n)
        values = np.empty(nv, np.float64)
        vectors = None if method == _lib.EIGEN_LANCZOS else np.empty((nv, K.n), np.float64)
        st = _lib.EigenStats()
        self.check(self.lib.rsg_eigen_solve(self.h, M.h, K.h, C.byref(ec), C.byref(conf), _ptr(start), _ptr(values),
                                            None if vectors is None else _ptr(vectors), C.byref(st)), "eigen_solve")
        return values, vectors, {"n_values": st.n_values, "solves": st.solves, "iterations": st.iterations}

    def amg_level(self, A: "Matrix", level: int, n_rows: int, nnz: int, with_agg: bool = True):
        """(agg or None, row_ptr, col_idx, values) of one level of A's last hierarchy."""
        agg = np.empty(n_rows, np.uint32) if with_agg else None
        rp = np.empty(n_rows + 1, np.uint32)
        ci = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        self.check(self.lib.rsg_amg_level(self.h, A.h, level, _ptr(agg), _ptr(rp), _ptr(ci), _ptr(val)), "amg_level")
        return agg, rp, ci, val

    def amg_apply(self, A: "Matrix", r_dev, z_dev, sweeps: int = 2):
        """z = one V-cycle applied to r (device FP64 arrays)."""
        self.check(self.lib.rsg_amg_apply(self.h, A.h, _ptr(r_dev), _ptr(z_dev), sweeps), "amg_apply")

    def spmv(self, A: "Matrix", x_dev, y_dev):
        self.check(self.lib.rsg_spmv(self.h, A.h, _ptr(x_dev), _ptr(y_dev)), "spmv")

    def spmv_f32(self, A: "Matrix", x_dev, y_dev):
        self.check(self.lib.rsg_spmv_f32(self.h, A.h, _ptr(x_dev), _ptr(y_dev)), "spmv_f32")

    def jacobi(self, A: "Matrix", d_dev):
        self.check(self.lib.rsg_jacobi_build(self.h, A.h, _ptr(d_dev)), "jacobi_build")

    def block_jacobi(self, A: "Matrix", block_size: int, blocks_dev) -> int:
        w = C.c_uint32()
        self.check(self.lib.rsg_block_jacobi_build(self.h, A.h, block_size, _ptr(blocks_dev), C.byref(w)),
                   "block_jacobi_build")
        return w.value

    def profile_kernel(self, A: "Matrix", kernel: int, reps: int = 20, flush_l2: bool = True) -> float:
        """Average device seconds of one solver kernel (rsg_kernel_id) on A."""
        t = C.c_double()
        self.check(self.lib.rsg_profile_kernel(self.h, A.h, kernel, reps, 1 if flush_l2 else 0, C.byref(t)),
                   "profile_kernel")
        return t.value

    def autotune(self, A: "Matrix", cache_path: str | None = None) -> dict:
        """Pick A's layout and launch shapes by timing short solves of A (rsg_autotune)."""
        info = _lib.TuneInfo()
        self.check(self.lib.rsg_autotune(self.h, A.h, cache_path.encode() if cache_path else None, C.byref(info)),
                   "autotune")
        return info.as_dict()

    def tune_info(self, A: "Matrix") -> dict:
        info = _lib.TuneInfo()
        self.check(self.lib.rsg_tune_get(A.h, C.byref(info)), "tune_get")
        return info.as_dict()

    def save_matrix(self, A: "Matrix", path: str, b_dev=None):
        """CSR/RHS dump of A (and a device right-hand side) in the RSGCSR01 format (rsg_csr_save)."""
        self.check(self.lib.rsg_csr_save(self.h, A.h, _ptr(b_dev), path.encode()), "csr_save")

    def load_matrix(self, path: str, b_dev=None):
        """(Matrix, has_b) from an RSGCSR01 file; the right-hand side goes to b_dev when given."""
        h, n, nnz, hb = C.c_void_p(), C.c_uint32(), C.c_uint64(), C.c_int32()
        self.check(self.lib.rsg_csr_load(self.h, path.encode(), C.byref(h), _ptr(b_dev), C.byref(n), C.byref(nnz),
                                         C.byref(hb)), "csr_load")
        return Matrix(self, h), bool(hb.value)

    def selftest_wait_timeout(self, polls: int = 1024) -> int:
        """Status of the failure-detection self-test (RSG_ERR_TIMEOUT when detection works)."""
        return self.lib.rsg_selftest_wait_timeout(self.h, polls)

    def true_relres(self, A: "Matrix", b_dev, x_dev) -> float:
        r = C.c_double()
        self.check(self.lib.rsg_true_relres(self.h, A.h, _ptr(b_dev), _ptr(x_dev), C.byref(r)), "true_relres")
        return r.value


class Matrix:
    """Device CSR handle (rsg_csr)."""

    def __init__(self, ctx: Context, h: C.c_void_p):
        self.ctx = ctx
        self.h = h
        n = C.c_uint32()
        nnz = C.c_uint64()
        fro = C.c_double()
        ctx.check(ctx.lib.rsg_csr_info(h, C.byref(n), C.byref(nnz), C.byref(fro)), "csr_info")
        self.n, self.nnz, self.frobenius = n.value, nnz.value, fro.value

    def update_values(self, val):
        dev = _is_device(val)
        if not dev:
            val = np.ascontiguousarray(val, np.float64)
        self.ctx.check(self.ctx.lib.rsg_csr_update_values(self.ctx.h, self.h, _ptr(val),
                                                          MEM_DEVICE if dev else MEM_HOST), "csr_update_values")
        self.refresh_info()

    def refresh_info(self):
        fro = C.c_double()
        self.ctx.lib.rsg_csr_info(self.h, None, None, C.byref(fro))
        self.frobenius = fro.value

    def to_host(self):
        """(row_ptr, col_idx, values) copied back to numpy."""
        rp = np.empty(self.n + 1, np.uint32)
        ci = np.empty(self.nnz, np.uint32)
        val = np.empty(self.nnz, np.float64)
        self.ctx.check(self.ctx.lib.rsg_csr_copy_to_host(self.ctx.h, self.h, _ptr(rp), _ptr(ci), _ptr(val)),
                       "csr_copy_to_host")
        return rp, ci, val

    def device_arrays(self):
        rp, ci, val = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self.ctx.check(self.ctx.lib.rsg_csr_device_arrays(self.h, C.byref(rp), C.byref(ci), C.byref(val)),
                       "csr_device_arrays")
        return rp.value, ci.value, val.value

    def close(self):
        if self.h and self.ctx.h:
            self.ctx.lib.rsg_csr_destroy(self.ctx.h, self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Mirror of RMatrixSolver (include/rmatrixsolver.h:9-52) over a Context."""

    def __init__(self, ctx: Context, conf: SolverConf):
        self.ctx = ctx
        self.conf = conf
        self._cache: dict[int, tuple[Matrix, tuple]] = {}

    def solve(self, A_csr, b, x=None, prec: int = PREC_NONE, block_size: int = 1):
        """A_csr: (row_ptr, col_idx, values) host arrays.  The matrix is cached by
        identity of the row_ptr array; a same-pattern call only refreshes values
        (the reference's findSparseMatrixCache, src/rmatrixsolver.cpp:99-109)."""
        rp, ci, val = A_csr
        key = id(rp)
        hit = self._cache.get(key)
        if hit is not None and hit[1] == (len(rp), len(ci)) and np.array_equal(hit[2], ci):
            M = hit[0]
            M.update_values(val)
        else:
            M = self.ctx.matrix(rp, ci, val)
            self._cache[key] = (M, (len(rp), len(ci)), np.array(ci, copy=True))
        return self.ctx.solve(M, b, x, self.conf, prec, block_size)


class ModelGroups:
    """The model's elements and element groups as flat arrays for the node-book entry points.

    elements: list of node-id sequences (any element type), or a 2-D array (one element per row);
    groups: list of element-id sequences; computable: per-element flags or None (all computable).
    """

    def __init__(self, n_nodes: int, elements, groups, computable=None):
        if isinstance(elements, np.ndarray) and elements.ndim == 2:
            k = elements.shape[1]
            self.elem_nodes = np.ascontiguousarray(elements.reshape(-1), np.uint32)
            self.elem_begin = np.arange(0, k * elements.shape[0] + 1, k, dtype=np.uint32)
        else:
            lens = [len(e) for e in elements]
            self.elem_begin = np.zeros(len(lens) + 1, np.uint32)
            self.elem_begin[1:] = np.cumsum(lens)
            self.elem_nodes = np.ascontiguousarray(np.concatenate([np.asarray(e, np.uint32) for e in elements])
                                                   if elements else np.zeros(0, np.uint32))
        glens = [len(g) for g in groups]
        self.group_begin = np.zeros(len(glens) + 1, np.uint32)
        self.group_begin[1:] = np.cumsum(glens)
        self.group_elems = np.ascontiguousarray(np.concatenate([np.asarray(g, np.uint32) for g in groups])
                                                if groups else np.zeros(0, np.uint32))
        self.computable = None if computable is None else np.ascontiguousarray(computable, np.uint8)
        self.c = _lib.ModelGroups(n_nodes, len(self.elem_begin) - 1, _ptr(self.elem_begin).value,
                                  _ptr(self.elem_nodes).value, len(glens), _ptr(self.group_begin).value,
                                  _ptr(self.group_elems).value,
                                  None if self.computable is None else _ptr(self.computable).value)
        self.n_nodes = n_nodes


def node_book_generic(model: ModelGroups, explicit_bc) -> tuple[np.ndarray, int]:
    """RSolverGeneric::generateNodeBook (rsg_node_book_generic): (book, n_free)."""
    lib = _lib.load()
    flags = np.ascontiguousarray(explicit_bc, np.uint8)
    book = np.empty(model.n_nodes, np.uint32)
    n_free = C.c_uint32()
    s = lib.rsg_node_book_generic(C.byref(model.c), _ptr(flags), _ptr(book), C.byref(n_free))
    if s != OK:
        raise _lib.RsgError(s, "node_book_generic: " + lib.rsg_status_string(s).decode())
    return book, n_free.value


def node_book_stress(model: ModelGroups, group_bc, group_is_line) -> tuple[np.ndarray, int]:
    """RSolverStress::generateNodeBook (rsg_node_book_stress): (book of 3 n_nodes positions, n_free)."""
    lib = _lib.load()
    bc = np.ascontiguousarray(group_bc, np.uint8)
    line = np.ascontiguousarray(group_is_line, np.uint8)
    book = np.empty(3 * model.n_nodes, np.uint32)
    n_free = C.c_uint32()
    s = lib.rsg_node_book_stress(C.byref(model.c), _ptr(bc), _ptr(line), _ptr(book), C.byref(n_free))
    if s != OK:
        raise _lib.RsgError(s, "node_book_stress: " + lib.rsg_status_string(s).decode())
    return book, n_free.value


class Assembly:
    """Assembly plan (rsg_assembly): pattern + scatter map of one mesh and node book.

    heat: RSolverHeat::prepare/assemblyMatrix (src/rsolverheat.cpp:361-455, :755-820);
    stress: RSolverStress::prepare/assemblyMatrix (src/rsolverstress.cpp:384-715, :1654-1772);
    magnetostatics: RSolverMagnetostatics::prepare/assemblyMatrix (src/rsolvermagnetostatics.cpp:44-145,
    :234-287).
    """

    def __init__(self, ctx: Context, h: C.c_void_p, kind: str):
        self.ctx, self.h, self.kind = ctx, h, kind
        n = C.c_uint32()
        nnz = C.c_uint64()
        ctx.check(ctx.lib.rsg_assembly_info(h, C.byref(n), C.byref(nnz)), "assembly_info")
        self.n_free, self.nnz = n.value, nnz.value
        self.A: Matrix | None = None

    @classmethod
    def heat(cls, ctx: Context, p) -> "Assembly":
        m = p.mesh
        xyz = np.ascontiguousarray(m.xyz, np.float64)
        tets = np.ascontiguousarray(m.tets, np.uint32)
        book = np.ascontiguousarray(p.book, np.uint32)
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_assembly_create_heat(ctx.h, m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets), _ptr(book),
                                                   p.n_free, C.byref(h)), "assembly_create_heat")
        return cls(ctx, h, "heat")

    @classmethod
    def stress(cls, ctx: Context, p) -> "Assembly":
        m = p.mesh
        xyz = np.ascontiguousarray(m.xyz, np.float64)
        tets = np.ascontiguousarray(m.tets, np.uint32)
        tris = np.ascontiguousarray(p.tris, np.uint32)
        book = np.ascontiguousarray(p.book, np.uint32)
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_assembly_create_stress(ctx.h, m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets),
                                                     tris.shape[0], _ptr(tris), _ptr(book), p.n_free, C.byref(h)),
                  "assembly_create_stress")
        return cls(ctx, h, "stress")

    @classmethod
    def magnetostatics(cls, ctx: Context, p) -> "Assembly":
        m = p.mesh
        xyz = np.ascontiguousarray(m.xyz, np.float64)
        tets = np.ascontiguousarray(m.tets, np.uint32)
        book = np.ascontiguousarray(p.book, np.uint32)
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_assembly_create_magnetostatics(ctx.h, m.n_nodes, _ptr(xyz), m.n_tets, _ptr(tets),
                                                             _ptr(book), p.n_free, C.byref(h)),
                  "assembly_create_magnetostatics")
        return cls(ctx, h, "magnetostatics")

    def _time(self, p) -> Time:
        return Time(1 if getattr(p, "transient", False) else 0, getattr(p, "alpha", 1.0), getattr(p, "dt", 0.0))

    def assemble(self, p, b_dev, inputs_on_device: dict | None = None) -> Matrix:
        """Assemble problem p's values into the plan's matrix (created on first use) and b_dev (device)."""
        hA = C.c_void_p(self.A.h.value if self.A is not None else 0)
        tm = self._time(p)
        if self.kind == "heat":
            if inputs_on_device:
                d = inputs_on_device
                args = [d["k_e"], d["q_e"], d["rhoc_e"], d["node_t"]]
                mem = MEM_DEVICE
            else:
                args = [np.ascontiguousarray(a, np.float64) for a in (p.k_e, p.q_e, p.rhoc_e, p.node_t)]
                mem = MEM_HOST
            s = self.ctx.lib.rsg_assemble_heat(self.ctx.h, self.h, *[_ptr(a) for a in args], C.byref(tm), mem,
                                               C.byref(hA), _ptr(b_dev))
        elif self.kind == "magnetostatics":
            if inputs_on_device:
                args, mem = [inputs_on_device["node_j"], inputs_on_device["node_a"]], MEM_DEVICE
            else:
                args, mem = [np.ascontiguousarray(a, np.float64) for a in (p.node_j, p.node_a)], MEM_HOST
            s = self.ctx.lib.rsg_assemble_magnetostatics(self.ctx.h, self.h, *[_ptr(a) for a in args], mem,
                                                         C.byref(hA), _ptr(b_dev))
        else:
            keys = ("e_mod", "nu", "rho_e", "gravity", "texp_e", "dtemp_e", "traction", "node_u")
            if inputs_on_device:
                args, mem = [inputs_on_device[k] for k in keys], MEM_DEVICE
            else:
                args, mem = [np.ascontiguousarray(getattr(p, k), np.float64) for k in keys], MEM_HOST
            s = self.ctx.lib.rsg_assemble_stress(self.ctx.h, self.h, *[_ptr(a) for a in args], C.byref(tm), mem,
                                                 C.byref(hA), _ptr(b_dev))
        self.ctx.check(s, f"assemble_{self.kind}")
        if self.A is None:
            self.A = Matrix(self.ctx, hA)
        else:
            self.A.refresh_info()
        return self.A

    def close(self):
        if self.A is not None:
            self.A.close()
            self.A = None
        if self.h and self.ctx.h:
            self.ctx.lib.rsg_assembly_destroy(self.ctx.h, self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ScatterPlan:
    """Pattern-cached assembly of caller-computed element matrices (rsg_scatter_plan):
    RSolverFluid::buildSparseMatrixPattern / assemblyMatrix (src/rsolverfluid.cpp:2305-2419).  The plan
    holds the pattern of the active elements' enabled DOFs and, per entry, its contributions in
    element order; assemble() adds the element blocks on the GPU in that order."""

    def __init__(self, ctx: Context, dofs_per_node: int, elem_begin, elem_nodes, elem_active, n_nodes: int, book,
                 n_free: int):
        self.ctx = ctx
        eb = np.ascontiguousarray(elem_begin, np.uint32)
        en = np.ascontiguousarray(elem_nodes, np.uint32)
        act = None if elem_active is None else np.ascontiguousarray(elem_active, np.uint8)
        bk = np.ascontiguousarray(book, np.uint32)
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_scatter_plan_create(ctx.h, dofs_per_node, len(eb) - 1, _ptr(eb), _ptr(en),
                                                  None if act is None else _ptr(act), n_nodes, _ptr(bk), n_free,
                                                  C.byref(h)), "scatter_plan_create")
        self.h = h
        ae, fe, nnz = C.c_uint64(), C.c_uint64(), C.c_uint64()
        ctx.check(ctx.lib.rsg_scatter_plan_info(h, C.byref(ae), C.byref(fe), C.byref(nnz)), "scatter_plan_info")
        self.ae_values, self.fe_values, self.nnz, self.n_free = ae.value, fe.value, nnz.value, n_free
        self.A: Matrix | None = None

    def assemble(self, Ae, fe, b_dev=None) -> Matrix:
        """Element blocks (host numpy arrays, or device tensors) -> the plan's matrix (created on first
        use) and, when b_dev is given (device, n_free doubles), the right-hand side."""
        dev = _is_device(Ae)
        if not dev:
            Ae = np.ascontiguousarray(Ae, np.float64)
            fe = np.ascontiguousarray(fe, np.float64)
        hA = C.c_void_p(self.A.h.value if self.A is not None else 0)
        self.ctx.check(self.ctx.lib.rsg_scatter_assemble(self.ctx.h, self.h, _ptr(Ae), _ptr(fe),
                                                         MEM_DEVICE if dev else MEM_HOST, C.byref(hA),
                                                         _ptr(b_dev)), "scatter_assemble")
        if self.A is None:
            self.A = Matrix(self.ctx, hA)
        else:
            self.A.refresh_info()
        return self.A

    def close(self):
        if self.A is not None:
            self.A.close()
            self.A = None
        if self.h and self.ctx.h:
            self.ctx.lib.rsg_scatter_plan_destroy(self.ctx.h, self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent systems of uneven size solved together (rsg_batch).

    systems: list of (row_ptr, col_idx, values) host CSR arrays, one per system.
    """

    def __init__(self, ctx: Context, systems):
        self.ctx = ctx
        sizes = [len(rp) - 1 for rp, _, _ in systems]
        self.row_begin = np.zeros(len(systems) + 1, np.uint32)
        self.row_begin[1:] = np.cumsum(sizes)
        rps, cis, vals = [], [], []
        nnz_off = 0
        for (rp, ci, val), r0 in zip(systems, self.row_begin[:-1]):
            rp = np.asarray(rp, np.int64)
            rps.append(rp[:-1] + nnz_off)
            cis.append(np.asarray(ci, np.int64) + int(r0))
            vals.append(np.asarray(val, np.float64))
            nnz_off += int(rp[-1])
        self.rp = np.ascontiguousarray(np.concatenate(rps + [np.array([nnz_off])]).astype(np.uint32))
        self.ci = np.ascontiguousarray(np.concatenate(cis).astype(np.uint32))
        self.val = np.ascontiguousarray(np.concatenate(vals))
        self.sizes = sizes
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_batch_create(ctx.h, len(systems), _ptr(self.row_begin), _ptr(self.rp), _ptr(self.ci),
                                           _ptr(self.val), C.byref(h)), "batch_create")
        self.h = h
        ns, rows, prow, nnz = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        ctx.lib.rsg_batch_info(h, C.byref(ns), C.byref(rows), C.byref(prow), C.byref(nnz))
        self.n_systems, self.rows, self.padded_rows, self.nnz = ns.value, rows.value, prow.value, nnz.value

    def split(self, v):
        return [v[self.row_begin[i]:self.row_begin[i + 1]] for i in range(self.n_systems)]

    def solve(self, b, x=None, conf: SolverConf | None = None, prec: int = PREC_JACOBI,
              allow=(OK, NOT_CONVERGED, BREAKDOWN)):
        """Returns (x, per-system Stats list, summary Stats)."""
        conf = conf or make_conf(stop_rule="true")
        per = (Stats * self.n_systems)()
        summ = Stats()
        if _is_device(b):
            s = self.ctx.lib.rsg_batch_solve(self.ctx.h, self.h, C.byref(conf), prec, _ptr(b), _ptr(x), MEM_DEVICE,
                                             per, C.byref(summ))
        else:
            b = np.ascontiguousarray(b, np.float64)
            x = np.zeros(self.rows) if x is None else np.array(x, np.float64, copy=True)
            s = self.ctx.lib.rsg_batch_solve(self.ctx.h, self.h, C.byref(conf), prec, _ptr(b), _ptr(x), MEM_HOST,
                                             per, C.byref(summ))
        self.ctx.check(s, "batch_solve", allow)
        return x, list(per), summ

    def autotune(self) -> dict:
        """Pick the batch loop's grid per precision by timing short batch solves (rsg_batch_autotune)."""
        info = _lib.TuneInfo()
        self.ctx.check(self.ctx.lib.rsg_batch_autotune(self.ctx.h, self.h, C.byref(info)), "batch_autotune")
        return info.as_dict()

    def close(self):
        if self.h and self.ctx.h:
            self.ctx.lib.rsg_batch_destroy(self.ctx.h, self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def transient_heat(ctx: Context, problem, n_steps: int, conf: SolverConf | None = None, precision: str = "fp64",
                   stream_sync=None):
    """Backward-Euler (theta) time stepping of a heat problem on the GPU.

    The reference's time loop (src/rsolver.cpp:106-144) calls RSolverHeat::prepare
    every step, which rebuilds A and b from scratch (A.clear(), src/rsolverheat.cpp:85)
    with the theta scheme of assemblyMatrix (:768-779), then solves with x = 0 as
    the initial guess.  Here the assembly plan (pattern + scatter map) is built
    once; each step re-assembles values and right-hand side on the GPU from
    device-resident element fields and the previous temperatures, solves with the
    previous step's temperatures as the initial guess, and writes the solution back
    into the nodal field with rsg_assembly_scatter -- nothing leaves the GPU inside
    the loop.  Returns [(nodal temperatures after each step (host numpy), Stats)].
    """
    import copy
    import torch  # device buffers
    p = copy.copy(problem)
    p.transient = True
    asm = Assembly.heat(ctx, p)
    dev = f"cuda:{ctx.device}"
    fields = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k), np.float64)).to(dev)
              for k in ("k_e", "q_e", "rhoc_e", "node_t")}
    b = torch.empty(asm.n_free, dtype=torch.float64, device=dev)
    x = torch.zeros_like(b)
    conf = conf or make_conf(n_outer=50000, stop_rule="true", rtol=1e-10, precision=precision)
    free = p.book != 0xFFFFFFFF
    x.copy_(torch.from_numpy(np.ascontiguousarray(p.node_t[free][np.argsort(p.book[free])], np.float64)).to(dev))
    torch.cuda.synchronize()
    history, stats = [], []
    for _ in range(n_steps):
        A = asm.assemble(p, b, inputs_on_device=fields)
        _, st = ctx.solve(A, b, x, conf=conf)
        ctx.check(ctx.lib.rsg_assembly_scatter(ctx.h, asm.h, _ptr(x), _ptr(fields["node_t"])), "assembly_scatter")
        ctx.sync()  # the snapshot below runs on torch's stream, the scatter on the context's
        history.append(fields["node_t"].clone())
        stats.append(st)
    out = [(t.cpu().numpy(), st) for t, st in zip(history, stats)]
    asm.close()
    return out
