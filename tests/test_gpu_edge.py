"""Edge sizes of the solve path against the CPU oracle, through the C ABI: systems smaller
than one 32-row SELL slice, sizes just around a slice boundary, and a row without a stored
diagonal (the reference's Jacobi then uses 0 for that row,
src/rmatrixpreconditioner.cpp:78-94).

Bar: the FP64 true relative residual reaches the requested 1e-10 and the solution agrees
with the oracle's tight solve to ||x-x_ref||/||x_ref|| <= 1e-8.
"""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from conftest import rel_err

pytestmark = pytest.mark.gpu


def spd_banded(n, seed):
    """Diagonally dominant SPD matrix with a few off-diagonal bands (dense for tiny n)."""
    rng = np.random.default_rng(seed)
    D = np.zeros((n, n))
    for k in (1, 3, 7):
        if k < n:
            v = rng.uniform(-1.0, 1.0, n - k)
            D += np.diag(v, k) + np.diag(v, -k)
    D += np.diag(np.abs(D).sum(axis=1) + rng.uniform(0.5, 2.0, n))
    return O.csr_from_dense(D), rng.uniform(-1.0, 1.0, n)


@pytest.mark.parametrize("n", [1, 5, 31, 32, 33, 95])
@pytest.mark.parametrize("solver,precision", [("cg", "fp64"), ("cg", "mixed"), ("gmres", "fp64"),
                                              ("gmres", "mixed")])
def test_small_and_ragged_sizes(ctx, n, solver, precision):
    A, b = spd_banded(n, seed=n)
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = rsg.make_conf(solver=solver, n_outer=5000, n_inner=30, stop_rule="true", rtol=1e-10,
                         precision=precision)
    x, st = ctx.solve(M, b, conf=conf, prec=rsg.PREC_JACOBI)
    assert st.converged == 1 and O.true_relres(A, b, x) <= 1e-10 * 1.01
    xo, _ = O.solve(A, b, prec=1, n_outer=5000, stop_rule="true", rtol=1e-13)
    assert rel_err(x, xo) < 1e-8


def test_missing_diagonal_row_gmres(ctx, torch_cuda):
    # row 3 stores no diagonal entry: Jacobi uses 0 there, as the reference does; GMRES still
    # solves the (nonsingular) system through the other rows' coupling
    n = 40
    A, b = spd_banded(n, seed=11)
    D = np.zeros((n, n))
    for i in range(n):
        D[i, A.ci[A.rp[i]:A.rp[i + 1]]] = A.val[A.rp[i]:A.rp[i + 1]]
    D[3, 3] = 0.0
    D[3, 4] = D[3, 4] + 5.0  # keep the system nonsingular
    Z = O.csr_from_dense(D)
    M = ctx.matrix(Z.rp, Z.ci, Z.val)
    d = torch_cuda.empty(n, dtype=torch_cuda.float64, device="cuda")
    torch_cuda.cuda.synchronize()
    ctx.jacobi(M, d)
    ctx.sync()
    assert np.array_equal(d.cpu().numpy(), O.jacobi(Z)) and d[3].item() == 0.0
    conf = rsg.make_conf(solver="gmres", n_outer=2000, n_inner=30, stop_rule="true", rtol=1e-10)
    x, st = ctx.solve(M, b, conf=conf, prec=rsg.PREC_NONE)
    assert st.converged == 1 and O.true_relres(Z, b, x) <= 1e-10 * 1.01
    xo = np.linalg.solve(D, b)
    assert rel_err(x, xo) < 1e-8


def test_block_jacobi_width_shrinks_to_a_divisor(ctx, torch_cuda):
    # BLOCK_JACOBI shrinks the block width until it divides n (5 on 12 rows -> 4), as the oracle
    # restating RMatrixPreconditioner does; the GPU build and a solve with it agree with the oracle
    A, b = spd_banded(12, seed=5)
    M = ctx.matrix(A.rp, A.ci, A.val)
    blocks = torch_cuda.empty(12 * 5, dtype=torch_cuda.float64, device="cuda")
    torch_cuda.cuda.synchronize()
    w = ctx.block_jacobi(M, 5, blocks)
    ctx.sync()
    B, w_ref = O.block_jacobi(A, 5)
    assert w == w_ref == 4
    assert np.allclose(blocks.cpu().numpy()[: 12 * w].reshape(12, w), B, rtol=1e-12,
                       atol=1e-16 * np.abs(B).max())
    A2, b2 = spd_banded(96, seed=6)
    M2 = ctx.matrix(A2.rp, A2.ci, A2.val)
    for precision in ("fp64", "mixed"):
        conf = rsg.make_conf(n_outer=5000, stop_rule="true", rtol=1e-10, precision=precision)
        x, st = ctx.solve(M2, b2, conf=conf, prec=rsg.PREC_BLOCK_JACOBI, block_size=5)
        assert st.converged == 1 and O.true_relres(A2, b2, x) <= 1e-10 * 1.01
        xo, _ = O.solve(A2, b2, prec=2, block_size=5, n_outer=5000, stop_rule="true", rtol=1e-13)
        assert rel_err(x, xo) < 1e-8


@pytest.mark.parametrize("solver,precision", [("cg", "fp64"), ("cg", "mixed"), ("gmres", "fp64")])
def test_incoming_x_is_the_initial_guess(ctx, solver, precision):
    # x is in/out and its incoming values are the initial guess (RMatrixSolver::solve scales it with
    # b, src/rmatrixsolver.cpp:164-198): a guess near the solution converges in fewer iterations to
    # the same answer, with the same count as the oracle started from the same guess (FP64 CG)
    A, b = spd_banded(600, seed=9)
    M = ctx.matrix(A.rp, A.ci, A.val)
    kw = dict(solver=solver, n_outer=5000, n_inner=30, stop_rule="true", rtol=1e-10)
    conf = rsg.make_conf(precision=precision, **kw)
    x_cold, st_cold = ctx.solve(M, b, conf=conf)
    xo, _ = O.solve(A, b, prec=1, **dict(kw, rtol=1e-13))
    guess = xo * (1.0 + 1e-6 * np.random.default_rng(1).standard_normal(A.n))
    x_warm, st_warm = ctx.solve(M, b, guess.copy(), conf=conf)
    assert st_warm.converged == 1 and O.true_relres(A, b, x_warm) <= 1e-10 * 1.01
    assert st_warm.iterations < st_cold.iterations
    assert rel_err(x_warm, xo) < 1e-8 and rel_err(x_cold, xo) < 1e-8
    if solver == "cg" and precision == "fp64":
        _, sto = O.solve(A, b, guess.copy(), prec=1, **kw)
        assert abs(int(st_warm.iterations) - int(sto.iterations)) <= 2
