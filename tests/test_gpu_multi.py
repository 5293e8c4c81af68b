"""GPU checks of the multi-right-hand-side solver (rsg_solve_multi) against
single-right-hand-side solves and the oracle.

Tolerances: every column reaches the FP64 true relative residual it was asked
for (1e-10), agrees with the oracle's tight solution to 1e-8 (relative
2-norm), and takes within 3 iterations of the single-column GPU solve."""
import numpy as np
import pytest

import rsg
from conftest import rel_err
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.fixture(scope="module")
def system():
    return O.assemble_heat(W.heat_cube(14, sigma=1.0, seed=21, source="random"))


def rhs(A, b, k, seed=0):
    rng = np.random.default_rng(seed)
    B = [b] + [rng.standard_normal(A.n) for _ in range(k - 1)]
    return np.stack(B[:k])


@pytest.mark.parametrize("k", [1, 3, 8, 16])
def test_multi_matches_single_and_oracle(ctx, system, k):
    A, b = system
    M = ctx.matrix(A.rp, A.ci, A.val)
    B = rhs(A, b, k, seed=k)
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=RTOL)
    X, per, summ = ctx.solve_multi(M, B, conf=conf)
    assert summ.converged == 1 and summ.status == 0 and summ.true_relres <= RTOL * 1.01
    for j in range(k):
        assert per[j].converged == 1
        assert O.true_relres(A, B[j], X[j]) <= RTOL * 1.01
        x1, st1 = ctx.solve(M, B[j], conf=conf)
        assert abs(int(per[j].iterations) - int(st1.iterations)) <= 3, (j, per[j].iterations, st1.iterations)
        xt, stt = O.solve(A, B[j], prec=1, n_outer=200000, stop_rule="true", rtol=1e-12)
        assert rel_err(X[j], xt) < 1e-8


def test_multi_zero_column_initial_guess_and_no_preconditioner(ctx, system):
    A, b = system
    M = ctx.matrix(A.rp, A.ci, A.val)
    B = rhs(A, b, 4, seed=7)
    B[2] = 0.0
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=RTOL)
    X0, _, _ = ctx.solve_multi(M, B, conf=conf)
    # restart from the solution: every column is already converged
    X1, per, summ = ctx.solve_multi(M, B, X0, conf=conf)
    assert all(p.iterations == 0 for p in per) and summ.converged == 1
    assert np.array_equal(X1, X0)
    assert np.all(X0[2] == 0.0) and per[2].converged == 1
    X2, per2, summ2 = ctx.solve_multi(M, B, conf=conf, prec=rsg.PREC_NONE)
    assert summ2.converged == 1
    for j in range(4):
        assert O.true_relres(A, B[j], X2[j]) <= RTOL * 1.01


def test_multi_device_arrays_and_iteration_cap(ctx, system, torch_cuda):
    torch = torch_cuda
    A, b = system
    M = ctx.matrix(A.rp, A.ci, A.val)
    B = rhs(A, b, 5, seed=3)
    Bd = torch.from_numpy(B).cuda()
    Xd = torch.zeros_like(Bd)
    torch.cuda.synchronize()
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=RTOL)
    _, per, summ = ctx.solve_multi(M, Bd, Xd, conf=conf)
    Xh, _, _ = ctx.solve_multi(M, B, conf=conf)
    assert np.array_equal(Xd.cpu().numpy(), Xh)  # same kernels, same bits
    capped = rsg.make_conf(n_outer=5, stop_rule="true", rtol=RTOL)
    Xc, perc, summc = ctx.solve_multi(M, B, conf=capped)
    assert summc.converged == 0 and all(p.iterations == 5 for p in perc)


def test_multi_argument_errors(ctx, system):
    A, b = system
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = rsg.make_conf(stop_rule="true", rtol=RTOL)
    with pytest.raises(rsg.RsgError):
        ctx.solve_multi(M, np.zeros((17, A.n)), conf=conf)
    with pytest.raises(rsg.RsgError):
        ctx.solve_multi(M, rhs(A, b, 2), conf=rsg.make_conf(rtol=RTOL))  # reference stop rule
    with pytest.raises(rsg.RsgError):
        ctx.solve_multi(M, rhs(A, b, 2), conf=rsg.make_conf(stop_rule="true", precision="mixed"))
    with pytest.raises(rsg.RsgError):
        ctx.solve_multi(M, rhs(A, b, 2), conf=conf, prec=rsg.PREC_BLOCK_JACOBI)
