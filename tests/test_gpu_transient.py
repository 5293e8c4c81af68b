"""Transient heat (backward Euler) time stepping on the GPU against the oracle's
time loop: the reference rebuilds and solves every step (src/rsolver.cpp:106-144,
src/rsolverheat.cpp:768-779)."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_transient_heat_matches_oracle_time_loop(ctx, precision):
    p = W.heat_cube(8, sigma=1.0, seed=3, source="random", transient=True, dt=1e-3)
    steps = rsg.transient_heat(ctx, p, 4, precision=precision)
    # oracle time loop
    q = W.heat_cube(8, sigma=1.0, seed=3, source="random", transient=True, dt=1e-3)
    free = q.book != W.EOD
    idx = q.book[free].astype(np.int64)
    for k in range(4):
        A, b = O.assemble_heat(q)
        x0 = np.empty(A.n)
        x0[idx] = q.node_t[free]
        x, st = O.solve(A, b, x0, prec=1, n_outer=50000, stop_rule="true", rtol=1e-12)
        q.node_t[free] = x[idx]
        Tg, stg = steps[k]
        assert stg.true_relres <= 1e-10
        assert np.linalg.norm(Tg - q.node_t) / np.linalg.norm(q.node_t) < 1e-8
    # heat flows in from the T=1 face: the interior warms monotonically
    means = [T[free].mean() for T, _ in steps]
    assert all(b > a for a, b in zip(means, means[1:]))
