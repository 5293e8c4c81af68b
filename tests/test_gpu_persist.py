"""The CG loop as one persistent cooperative kernel (conf.persistent) against the graph-driven loop.

Both run the same grids: the persistent kernel executes each phase as the graph kernels' blocks
(virtual blocks), with their row assignment and reduction order, so the solution, the iteration
count and every reported statistic must be the same bit for bit -- FP64 and mixed precision,
with no preconditioner and with Jacobi, under both stopping rules.  Solutions also reach the
oracle-recomputed true residual.
"""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu


def systems():
    return {"heat12": O.assemble_heat(W.heat_cube(12, sigma=1.0, seed=2, source="random")),
            "heat33_lognormal": O.assemble_heat(W.heat_cube(33, sigma=1.5, seed=6, source="random")),
            "beam": O.assemble_stress(W.stress_beam(10, 5, 5))}


SYS = systems()


@pytest.mark.parametrize("name", list(SYS))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("prec", [rsg.PREC_JACOBI, rsg.PREC_NONE])
def test_persistent_loop_equals_graph_loop(ctx, name, precision, prec):
    A, b = SYS[name]
    M = ctx.matrix(A.rp, A.ci, A.val)
    base = dict(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision)
    x_g, st_g = ctx.solve(M, b, conf=rsg.make_conf(persistent=-1, **base), prec=prec)
    x_p, st_p = ctx.solve(M, b, conf=rsg.make_conf(persistent=1, **base), prec=prec)
    assert st_p.status == st_g.status == rsg.OK
    assert np.array_equal(x_p, x_g)
    assert (st_p.iterations, st_p.outer, st_p.true_relres) == (st_g.iterations, st_g.outer, st_g.true_relres)
    assert O.true_relres(A, b, x_p) <= 1e-10 * 1.01


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_loop_reference_rule_and_history(ctx, precision, tmp_path):
    A, b = SYS["heat12"]
    M = ctx.matrix(A.rp, A.ci, A.val)
    logs = []
    for mode in (-1, 1):
        path = str(tmp_path / f"log{mode}.txt")
        conf = rsg.make_conf(n_outer=5000, cvg=1e-12, persistent=mode, output_frequency=1, output_file=path,
                             precision=precision, stop_rule="reference" if precision == "fp64" else "true")
        x, st = ctx.solve(M, b, conf=conf, prec=rsg.PREC_JACOBI)
        logs.append((x, st.iterations, open(path).read()))
    assert np.array_equal(logs[0][0], logs[1][0]) and logs[0][1] == logs[1][1]
    assert logs[0][2] == logs[1][2]  # the convergence history, line for line
