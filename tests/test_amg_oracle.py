"""The oracle's multilevel aggregation preconditioner (the checker of RSG_PREC_AMG), on the CPU.

Checks the properties the GPU's hierarchy is then compared against bit for bit: every row belongs
to exactly one aggregate and aggregates are numbered densely; roots are never strong neighbours
of each other; the coarse matrix equals P^T A P (scipy) with P the aggregate indicator; the dense
coarsest inverse inverts the last level; the cycle (a K-cycle: levels 1 and 2 solved by two
flexible-CG steps) is positive, and as a flexible-CG preconditioner it needs far fewer iterations
than Jacobi.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from rsg import workloads as W


def _sp(A):
    return sp.csr_matrix((A.val, A.ci.astype(np.int64), A.rp.astype(np.int64)), shape=(A.n, A.n))


@pytest.fixture(scope="module")
def heat24():
    A, b = O.assemble_heat(W.heat_cube(24, sigma=1.5, seed=2, source="random"))
    return A, b, O.Amg(A)


def test_hierarchy_shape_and_galerkin(heat24):
    A, _, H = heat24
    assert H.levels >= 3 and H.dense_coarsest and H.rows[-1] <= 128
    assert all(H.rows[l + 1] * 4 < H.rows[l] for l in range(H.levels - 1))
    M = _sp(A)
    for l in range(H.levels - 1):
        agg, F = H.level(l)
        _, C = H.level(l + 1)
        assert agg.max() == H.rows[l + 1] - 1 and np.all(np.bincount(agg) > 0)
        Fs = _sp(F)
        P = sp.csr_matrix((np.ones(F.n), (np.arange(F.n), agg.astype(np.int64))), shape=(F.n, C.n))
        G = (P.T @ Fs @ P).toarray()
        np.testing.assert_allclose(_sp(C).toarray(), G, rtol=0, atol=1e-13 * np.abs(G).max())
        assert all(np.all(np.diff(C.ci[C.rp[i]:C.rp[i + 1]].astype(np.int64)) > 0) for i in range(C.n))
    _, F0 = H.level(0)
    assert np.array_equal(F0.val, A.val)


def test_cycle_is_positive_and_accelerates_flexible_cg(heat24):
    """The cycle's K-cycle levels (two flexible-CG steps) make it a variable preconditioner: positive
    (u^T M(u) > 0) but not a fixed symmetric matrix, so the outer iteration is flexible CG (the
    Polak-Ribiere direction update, as the GPU's mixed-precision CG uses with this preconditioner)."""
    A, b, H = heat24
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal(A.n), rng.standard_normal(A.n)
    for sweeps in (1, 2):
        assert u @ H.apply(u, sweeps) > 0 and v @ H.apply(v, sweeps) > 0
    M = _sp(A)
    for sweeps, bound in ((1, 40), (2, 30)):
        x = np.zeros(A.n)
        r = b.copy()
        z = H.apply(r, sweeps)
        p = z.copy()
        rz = r @ z
        bn = np.linalg.norm(b)
        for it in range(1, 500):
            q = M @ p
            al = rz / (p @ q)
            x += al * p
            r -= al * q
            if np.linalg.norm(b - M @ x) / bn < 1e-10:
                break
            z = H.apply(r, sweeps)
            beta = -al * (q @ z) / rz
            rz = r @ z
            p = z + beta * p
        _, sj = O.solve(A, b, prec=1, n_outer=20000, stop_rule="true", rtol=1e-10)
        assert it <= bound and it * 8 < sj.iterations, (sweeps, it, sj.iterations)


def test_small_matrix_is_one_dense_level():
    A, b = O.assemble_heat(W.heat_cube(4, sigma=1.0, seed=1, source="random"))
    assert A.n <= 128
    H = O.Amg(A)
    assert H.levels == 1 and H.dense_coarsest
    z = H.apply(b)
    np.testing.assert_allclose(_sp(A) @ z, b, rtol=0, atol=1e-10 * np.abs(b).max())
