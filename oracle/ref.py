"""ctypes wrapper of the reference's own solver, compiled from its sources (TEST INFRASTRUCTURE ONLY).

`make -C oracle ref` compiles the reference project's src/rmatrixsolver.cpp,
src/rmatrixpreconditioner.cpp, src/riterationinfo.cpp, src/riterationinfovalue.cpp and
src/reigenvaluesolver.cpp unchanged
against the stand-in headers in oracle/ref_shim/ into oracle/_ref/libref_solver.so (see
oracle/ref_driver.cpp).  Only tests/ and bench.py's reference arm use it, as the checker of the
oracle's restatement and of the CUDA library, and as the timed CPU baseline.  It is built where the
reference sources are present; available() says whether the built library is here.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_solver.so")
_LIB = None

PREC_NONE, PREC_JACOBI, PREC_BLOCK_JACOBI = 0, 1, 2


class RefResult(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("lines", C.c_uint32), ("error", C.c_double), ("trend", C.c_double),
                ("seconds", C.c_double), ("message", C.c_char * 256)]


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} not built: run `make -C oracle ref` where the reference sources are")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.ref_matrix_create.restype = P
        L.ref_matrix_create.argtypes = [C.c_uint32, P, P, P]
        L.ref_matrix_update.argtypes = [P, P, P]
        L.ref_matrix_destroy.argtypes = [P]
        L.ref_solve.restype = C.c_int
        L.ref_solve.argtypes = [P, P, P, C.c_int, C.c_int, C.c_uint, C.c_uint, C.c_uint, C.c_double, C.c_char_p,
                                C.c_int, C.POINTER(RefResult)]
        L.ref_rand_start.argtypes = [C.c_uint, C.c_uint32, P, C.POINTER(C.c_double)]
        L.ref_eigen.restype = C.c_int
        L.ref_eigen.argtypes = [P, P, C.c_int, C.c_uint, C.c_uint, C.c_double, C.c_uint, C.c_uint, C.c_double,
                                C.c_int, C.c_uint32, P, P, C.POINTER(RefResult)]
        _LIB = L
    return _LIB


LANCZOS, ARNOLDI, RAYLEIGH = 0, 1, 2


def rand_start(seed: int, n: int):
    """The start vector and Rayleigh shift REigenValueSolver draws with rand() after srand(seed)."""
    start = np.empty(n, np.float64)
    mu = C.c_double()
    lib().ref_rand_start(seed, n, _p(start), C.byref(mu))
    return start, mu.value


def eigen(M: "RefMatrix", K: "RefMatrix", method: int, n_eigen: int, *, n_iterations: int = 100,
          cvg: float = 1e-8, seed: int = 1, n_outer: int = 100000, solver_cvg: float = 1e-13, threads: int = 1):
    """REigenValueSolver::solve(M, K, d, ev) after srand(seed) -> (d, ev or None, RefResult)."""
    nv = 1 if method == RAYLEIGH else min(n_eigen, K.n)
    d = np.empty(nv, np.float64)
    ev = np.zeros((nv, K.n), np.float64)
    res = RefResult()
    rc = lib().ref_eigen(M.h, K.h, method, n_eigen, n_iterations, cvg, seed, n_outer, solver_cvg, threads, nv,
                         _p(d), _p(ev), C.byref(res))
    if rc < 0:
        raise RuntimeError(f"reference eigen solve failed: {res.message.decode(errors='replace')}")
    return d[:rc], (None if method == LANCZOS else ev[:rc]), res


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class RefMatrix:
    """An RSparseMatrix built from CSR arrays.  The reference caches its CSR copy per matrix
    address for the life of the process (src/rmatrixsolver.cpp:99-109), as it does in a real
    application; keep one RefMatrix per system and update its values in place."""

    def __init__(self, rp, ci, val):
        self.rp = np.ascontiguousarray(rp, np.uint32)
        self.ci = np.ascontiguousarray(ci, np.uint32)
        val = np.ascontiguousarray(val, np.float64)
        self.n = len(self.rp) - 1
        self.h = lib().ref_matrix_create(self.n, _p(self.rp), _p(self.ci), _p(val))
        if not self.h:
            raise MemoryError("ref_matrix_create failed")

    def update_values(self, val):
        val = np.ascontiguousarray(val, np.float64)
        lib().ref_matrix_update(self.h, _p(self.rp), _p(val))

    def solve(self, b, x0=None, *, solver: str = "cg", prec: int = PREC_JACOBI, block_size: int = 1,
              n_outer: int = 1000, n_inner: int = 30, cvg: float = 1e-13, log_file: str | None = None,
              threads: int = 0):
        """RMatrixSolver::solve(A, b, x, prec, block_size) -> (x, RefResult).  threads > 0 sets the
        OpenMP team size (1 gives the serial, run-to-run reproducible result)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, np.float64, copy=True)
        res = RefResult()
        rc = lib().ref_solve(self.h, _p(b), _p(x), 1 if solver == "gmres" else 0, prec, block_size, n_outer, n_inner,
                             cvg, log_file.encode() if log_file else None, threads, C.byref(res))
        if rc != 0:
            raise RuntimeError(f"reference solve failed: {res.message.decode(errors='replace')}")
        return x, res

    def close(self):
        if self.h:
            lib().ref_matrix_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
