"""Batched solves of independent uneven systems (rsg_batch_*) against the oracle.

Each system must reach the FP64 true relative residual 1e-10 on its own and
agree with the oracle's tight solution to 1e-8, exactly as a single solve.
"""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu


def systems(specs):
    out = []
    for n, sigma, seed in specs:
        A, b = O.assemble_heat(W.heat_cube(n, sigma=sigma, seed=seed, source="random"))
        out.append((A, b))
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_uneven_heat_systems(ctx, precision, use_graph):
    sys_ = systems([(3, 1.0, 1), (9, 1.0, 2), (5, 0.5, 3), (14, 1.5, 4), (2, 1.0, 5), (11, 1.0, 6)])
    batch = rsg.Batch(ctx, [(A.rp, A.ci, A.val) for A, _ in sys_])
    assert batch.padded_rows % 32 == 0 and batch.rows == sum(A.n for A, _ in sys_)
    b = np.concatenate([bb for _, bb in sys_])
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision, use_graph=use_graph)
    x, per, summ = batch.solve(b, conf=conf)
    assert summ.status == rsg.OK
    for (A, bb), xs, st in zip(sys_, batch.split(x), per):
        assert st.status == rsg.OK and st.converged == 1
        assert st.true_relres <= 1e-10 and O.true_relres(A, bb, xs) <= 1e-10
        xr, sto = O.solve(A, bb, prec=1, n_outer=200000, stop_rule="true", rtol=1e-12)
        assert rel_err(xs, xr) <= 1e-8
        _, s1 = O.solve(A, bb, prec=1, n_outer=20000, stop_rule="true", rtol=1e-10)
        assert st.iterations <= 1.3 * s1.iterations + 5


def test_batch_matches_single_solves_fp64(ctx):
    sys_ = systems([(6, 1.0, 7), (10, 1.5, 8)])
    batch = rsg.Batch(ctx, [(A.rp, A.ci, A.val) for A, _ in sys_])
    b = np.concatenate([bb for _, bb in sys_])
    # single solves keep the reference's equation scaling (which keeps p^T A p far above the
    # reference's eps clamp); batch solves run unscaled with the clamp off
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10)
    x, per, _ = batch.solve(b, conf=conf)
    for (A, bb), xs, st in zip(sys_, batch.split(x), per):
        M = ctx.matrix(A.rp, A.ci, A.val)
        x1, s1 = ctx.solve(M, bb, conf=conf)
        assert abs(int(st.iterations) - int(s1.iterations)) <= 2
        assert rel_err(xs, x1) < 1e-9


def test_batch_zero_rhs_member_and_iteration_cap(ctx):
    sys_ = systems([(4, 1.0, 1), (7, 1.0, 2)])
    batch = rsg.Batch(ctx, [(A.rp, A.ci, A.val) for A, _ in sys_])
    b = np.concatenate([np.zeros(sys_[0][0].n), sys_[1][1]])
    x, per, _ = batch.solve(b, conf=rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10))
    assert per[0].status == rsg.OK and per[0].iterations == 0
    assert np.all(batch.split(x)[0] == 0.0)
    assert per[1].status == rsg.OK and per[1].true_relres <= 1e-10
    b2 = np.concatenate([bb for _, bb in sys_])
    x, per, summ = batch.solve(b2, conf=rsg.make_conf(n_outer=5, stop_rule="true", rtol=1e-10))
    assert summ.status == rsg.NOT_CONVERGED
    assert all(st.iterations == 5 and st.status == rsg.NOT_CONVERGED for st in per)


def test_batch_rejects_coupled_systems(ctx):
    (A1, _), (A2, _) = systems([(3, 1.0, 1), (3, 1.0, 2)])
    with pytest.raises(rsg.RsgError) as e:
        _coupled(ctx, A1, A2)
    assert e.value.status == rsg.ERR_INVALID_ARG


def _coupled(ctx, A1, A2):
    import ctypes as C
    rb = np.array([0, A1.n, A1.n + A2.n], np.uint32)
    rp = np.concatenate([A1.rp[:-1], A2.rp + A1.rp[-1]]).astype(np.uint32)
    ci = np.concatenate([A1.ci, A2.ci + A1.n]).astype(np.uint32)
    ci[A1.rp[-1]] = 0  # first entry of system 2 references system 1
    val = np.concatenate([A1.val, A2.val])
    h = C.c_void_p()
    ctx.check(ctx.lib.rsg_batch_create(ctx.h, 2, rb.ctypes.data_as(C.c_void_p), rp.ctypes.data_as(C.c_void_p),
                                       ci.ctypes.data_as(C.c_void_p), val.ctypes.data_as(C.c_void_p), C.byref(h)),
              "batch_create")


def test_batch_autotune_keeps_results(ctx):
    """The batch autotuner only changes launch shapes: every slice's partial sums and every
    system's sums of them are formed in the same order whatever the grid, so tuned solves give
    the untuned solutions bit for bit."""
    sys_ = systems([(6, 1.0, 11), (12, 1.2, 12), (4, 0.8, 13), (9, 1.0, 14)])
    batch = rsg.Batch(ctx, [(A.rp, A.ci, A.val) for A, _ in sys_])
    b = np.concatenate([bb for _, bb in sys_])
    results = {}
    for tag in ("default", "tuned"):
        if tag == "tuned":
            info = batch.autotune()
            assert info["tuned"] == 1 and info["candidates"] >= 2 * 8
            assert info["seconds_iter_fp64"] <= info["seconds_iter_fp64_default"]
            assert info["seconds_iter_fp32"] <= info["seconds_iter_fp32_default"]
        for precision in ("fp64", "mixed"):
            conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision)
            x, per, summ = batch.solve(b, conf=conf)
            assert summ.status == rsg.OK and summ.true_relres <= 1e-10
            results[(tag, precision)] = x
    for precision in ("fp64", "mixed"):
        assert np.array_equal(results[("tuned", precision)], results[("default", precision)])
