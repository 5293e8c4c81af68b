"""rsg_eigen_solve (REigenValueSolver's Lanczos, Arnoldi and Rayleigh methods on the GPU) against the
oracle's restatement, which the CPU tests pin to the reference's own src/reigenvaluesolver.cpp.

Both sides start from the same start values and run their linear solves with the reference's
stopping rule at cvg 1e-13 (CG + Jacobi); the GPU's dot products are reduced in a different (fixed)
order, so the bar is agreement to rounding amplified by the recurrences: eigenvalues to 1e-8,
eigenvectors (Arnoldi, Rayleigh) to 1e-6.
"""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu

SOLVE = dict(n_outer=100000, cvg=1e-13)


def pencil(n):
    K, _ = O.assemble_heat(W.heat_cube(n, sigma=1.5, seed=4, source="random"))
    M, _ = O.assemble_heat(W.heat_cube(n, sigma=0.0, seed=0, source="random"))
    return M, K


@pytest.mark.parametrize("method", [rsg.EIGEN_LANCZOS, rsg.EIGEN_ARNOLDI, rsg.EIGEN_RAYLEIGH])
@pytest.mark.parametrize("n", [8, 16])
def test_eigen_matches_oracle(ctx, method, n):
    M, K = pencil(n)
    start = np.random.default_rng(n).uniform(0.0, 1.0, K.n)
    mu0, ne, n_it, cvg = 3.7e8, 6, 80, 1e-10
    Md, Kd = ctx.matrix(M.rp, M.ci, M.val), ctx.matrix(K.rp, K.ci, K.val)
    conf = rsg.make_conf(**SOLVE)
    d_g, ev_g, st = ctx.eigen_solve(Md, Kd, start, method=method, n_eigen=ne, n_iterations=n_it, cvg=cvg, mu0=mu0,
                                    conf=conf)
    d_o, ev_o, solves = O.eigen_solve(M, K, method, ne, start, mu0=mu0, n_iterations=n_it, eig_cvg=cvg, **SOLVE)
    assert st["n_values"] == len(d_o) == len(d_g)
    assert rel_err(d_g, d_o) <= 1e-8, (d_g, d_o)
    if method != rsg.EIGEN_LANCZOS:
        assert rel_err(ev_g, ev_o) <= 1e-6
    assert st["solves"] == solves or method == rsg.EIGEN_RAYLEIGH  # Rayleigh may stop one step apart
    # the same call again gives the same bits
    d_2, ev_2, _ = ctx.eigen_solve(Md, Kd, start, method=method, n_eigen=ne, n_iterations=n_it, cvg=cvg, mu0=mu0,
                                   conf=conf)
    assert np.array_equal(d_g, d_2)


def test_eigen_argument_errors(ctx):
    M, K = pencil(6)
    Md, Kd = ctx.matrix(M.rp, M.ci, M.val), ctx.matrix(K.rp, K.ci, K.val)
    with pytest.raises(rsg.RsgError) as e:  # a zero start vector cannot be normalised
        ctx.eigen_solve(Md, Kd, np.zeros(K.n), method=rsg.EIGEN_LANCZOS)
    assert e.value.status == rsg._lib.ERR_INVALID_ARG
    D = O.csr_from_dense(np.eye(K.n) * 2.0)  # another pattern: Rayleigh needs one pattern
    Dd = ctx.matrix(D.rp, D.ci, D.val)
    with pytest.raises(rsg.RsgError) as e:
        ctx.eigen_solve(Dd, Kd, np.ones(K.n), method=rsg.EIGEN_RAYLEIGH, n_iterations=3)
    assert e.value.status == rsg._lib.ERR_UNSUPPORTED
    d, _, _ = ctx.eigen_solve(Md, Kd, np.ones(K.n), method=rsg.EIGEN_LANCZOS, n_eigen=3)
    assert len(d) == 3 and np.all(np.isfinite(d))  # the context is still usable
