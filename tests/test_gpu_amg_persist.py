"""The small coarse levels of each multilevel cycle as one persistent cooperative kernel
(k_amg_coarse_persist, conf.persistent > 0) against the same cycle launched kernel by kernel (the
default, conf.persistent <= 0): the same iteration count and the same solution bit for bit, with one and two
smoothing sweeps, from the graph-driven and the host-driven loop, where the persistent kernel takes
over at level 1 (30^3 heat: every coarse level) and at level 2 (72^3 heat: level 1 has more than
32768 rows and stays launched)."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu


def conf(persistent, sweeps, use_graph=True):
    return rsg.make_conf(n_outer=2000, stop_rule="true", rtol=1e-10, precision="mixed", persistent=persistent,
                         amg_sweeps=sweeps, use_graph=use_graph)


@pytest.mark.parametrize("n_hex,level", [(30, 1), (72, 2)])
@pytest.mark.parametrize("sweeps", [1, 2])
def test_persistent_coarse_levels_match_launched_bitwise(ctx, n_hex, level, sweeps):
    A, b = O.assemble_heat(W.heat_cube(n_hex, sigma=1.5, seed=3, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    x0, s0 = ctx.solve(M, b, conf=conf(0, sweeps), prec=rsg.PREC_AMG)
    x1, s1 = ctx.solve(M, b, conf=conf(1, sweeps), prec=rsg.PREC_AMG)
    assert ctx.amg_setup(M, conf=conf(1, sweeps))["persist_level"] == level
    assert ctx.amg_setup(M, conf=conf(0, sweeps))["persist_level"] == 0
    assert s1.status == rsg.OK and s1.converged == 1 and O.true_relres(A, b, x1) <= 1e-10 * 1.01
    assert s1.iterations == s0.iterations and np.array_equal(x1, x0)


def test_persistent_coarse_levels_host_loop(ctx):
    A, b = O.assemble_heat(W.heat_cube(24, sigma=1.0, seed=8, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    x0, s0 = ctx.solve(M, b, conf=conf(-1, 1, use_graph=False), prec=rsg.PREC_AMG)
    x1, s1 = ctx.solve(M, b, conf=conf(1, 1, use_graph=False), prec=rsg.PREC_AMG)
    x2, s2 = ctx.solve(M, b, conf=conf(1, 1), prec=rsg.PREC_AMG)
    assert s1.status == rsg.OK and s1.iterations == s0.iterations == s2.iterations
    assert np.array_equal(x1, x0) and np.array_equal(x2, x0)

