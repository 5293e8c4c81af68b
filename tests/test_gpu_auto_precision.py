"""Precision AUTO: mixed precision that continues in FP64 when a residual refresh finds the FP32
recurrence more than 2x off the true residual.  On the heat systems it never switches and is the
mixed-precision solve bit for bit; on the stiff elasticity beam it switches at its first refresh
(measured: 624 FP64 iterations, 1600 mixed, 1005 auto of which ~600 in FP64), ends at the requested
FP64 true residual with the oracle's solution to 1e-8, in fewer iterations than mixed precision."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu


def conf(precision, **kw):
    return rsg.make_conf(n_outer=40000, stop_rule="true", rtol=1e-10, precision=precision, **kw)


@pytest.mark.parametrize("persistent", [-1, 1])
def test_auto_equals_mixed_without_drift(ctx, persistent):
    A, b = O.assemble_heat(W.heat_cube(24, sigma=1.5, seed=4, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    x_m, st_m = ctx.solve(M, b, conf=conf("mixed", persistent=persistent), prec=rsg.PREC_JACOBI)
    x_a, st_a = ctx.solve(M, b, conf=conf("auto", persistent=persistent), prec=rsg.PREC_JACOBI)
    assert st_a.fp64_iterations == 0
    assert np.array_equal(x_a, x_m) and st_a.iterations == st_m.iterations


@pytest.mark.parametrize("prec", [rsg.PREC_JACOBI, rsg.PREC_BLOCK_JACOBI])
def test_auto_switches_to_fp64_on_the_stiff_beam(ctx, prec):
    A, b = O.assemble_stress(W.stress_beam(32, 16, 16))
    M = ctx.matrix(A.rp, A.ci, A.val)
    _, st64 = ctx.solve(M, b, conf=conf("fp64"), prec=prec, block_size=3)
    _, st32 = ctx.solve(M, b, conf=conf("mixed"), prec=prec, block_size=3)
    x, st = ctx.solve(M, b, conf=conf("auto"), prec=prec, block_size=3)
    assert st.status == rsg.OK and st.converged == 1 and st.fp64_iterations > 0
    assert O.true_relres(A, b, x) <= 1e-10 * 1.01
    x_ref, _ = O.solve(A, b, prec=1, n_outer=40000, stop_rule="true", rtol=1e-11)
    assert rel_err(x, x_ref) <= 1e-8
    assert st.iterations < 0.75 * st32.iterations, (st.iterations, st32.iterations, st64.iterations)


def test_auto_rejected_where_it_does_not_apply(ctx):
    A, b = O.assemble_heat(W.heat_cube(6, sigma=1.0, seed=1, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    for c, prec in ((rsg.make_conf(solver="gmres", stop_rule="true", precision="auto"), rsg.PREC_JACOBI),
                    (rsg.make_conf(stop_rule="true", precision="auto"), rsg.PREC_AMG)):
        with pytest.raises(rsg.RsgError) as e:
            ctx.solve(M, b, conf=c, prec=prec)
        assert e.value.status == rsg._lib.ERR_UNSUPPORTED
