"""The oracle's restatement of REigenValueSolver against the reference's own eigenvalue source.

oracle/_ref/libref_solver.so includes the reference project's src/reigenvaluesolver.cpp, compiled
unchanged against the stand-in headers of oracle/ref_shim/.  The pencil is (M, K) with K a lognormal
heat matrix and M the uniform-conductivity heat matrix of the same mesh (one pattern, both SPD).  Start
values: the reference's own rand() draws after srand(seed), taken from the built library so both sides
start alike.  On one OpenMP thread the reference's solves and the oracle's are the same bit for bit,
and so are the eigenvalue recurrences on top of them: Lanczos, Arnoldi (with its QR iteration and
eigenvectors) and the Rayleigh quotient iteration agree to 1e-12.  Without the built library these
tests are skipped.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference sources absent)")


def pencil(n=8):
    K, _ = O.assemble_heat(W.heat_cube(n, sigma=1.5, seed=4, source="random"))
    M, _ = O.assemble_heat(W.heat_cube(n, sigma=0.0, seed=0, source="random"))
    assert np.array_equal(K.rp, M.rp) and np.array_equal(K.ci, M.ci)
    return M, K


SOLVE = dict(n_outer=100000, cvg=1e-13, threads=1)


@pytest.mark.parametrize("method", [O.EIGEN_LANCZOS, O.EIGEN_ARNOLDI, O.EIGEN_RAYLEIGH])
def test_oracle_matches_reference_build(method):
    M, K = pencil()
    start, mu0 = R.rand_start(7, K.n)
    ne, n_it, cvg = 5, 60, 1e-10
    d_r, ev_r, res = R.eigen(R.RefMatrix(M.rp, M.ci, M.val), R.RefMatrix(K.rp, K.ci, K.val), method, ne,
                             n_iterations=n_it, cvg=cvg, seed=7, n_outer=SOLVE["n_outer"], solver_cvg=SOLVE["cvg"])
    d_o, ev_o, solves = O.eigen_solve(M, K, method, ne, start, mu0=mu0, n_iterations=n_it, eig_cvg=cvg, **SOLVE)
    assert len(d_o) == len(d_r) == (1 if method == O.EIGEN_RAYLEIGH else ne)
    assert rel_err(d_o, d_r) <= 1e-12, (d_o, d_r)
    if method != O.EIGEN_LANCZOS:
        assert rel_err(ev_o, ev_r) <= 1e-10
    assert np.all(np.isfinite(d_o)) and solves >= 1


def test_lanczos_values_are_sorted_reciprocals():
    # solve()'s post-processing: |1/d| ascending; the QL step keeps the Lanczos diagonal
    M, K = pencil(6)
    start, _ = R.rand_start(3, K.n)
    d, _, _ = O.eigen_solve(M, K, O.EIGEN_LANCZOS, 4, start, **SOLVE)
    assert np.all(np.diff(d) >= 0) and np.all(d > 0)
