"""GPU checks of the autotuner (rsg_autotune): it picks valid layouts and
launch shapes, solves with them reach the same solution, and its cache file
round-trips."""
import pytest

import rsg
from conftest import rel_err
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    return O.assemble_heat(W.heat_cube(20, sigma=1.0, seed=4, source="random"))


def test_autotune_shapes_and_same_solution(ctx, system):
    A, b = system
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10)
    x0, _ = ctx.solve(M, b, conf=conf)
    assert ctx.tune_info(M)["tuned"] == 0
    info = ctx.autotune(M)
    assert info["tuned"] == 1 and info["from_cache"] == 0 and info["candidates"] > 8
    for k in ("grid_dir_fp64", "grid_dir_fp32", "grid_update_fp64", "grid_update_fp32"):
        assert 0 <= info[k] <= 16384, k
    assert info["format"] in (0, 1) and info["rows_per_warp"] in (4, 8, 16, 32)
    assert info["pdl_fp64"] in (0, 1) and info["pdl_fp32"] in (0, 1)
    # the built-in shapes are a candidate: the choice is never measured slower than them
    assert info["seconds_iter_fp64"] + info["seconds_iter_fp32"] <= \
        info["seconds_iter_fp64_default"] + info["seconds_iter_fp32_default"]
    for precision in ("fp64", "mixed"):
        conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision)
        x1, st1 = ctx.solve(M, b, conf=conf)
        assert st1.converged == 1 and O.true_relres(A, b, x1) <= 1e-10 * 1.01
        assert rel_err(x1, x0) < 1e-8


def test_autotune_cache_roundtrip(ctx, system, tmp_path):
    A, b = system
    path = str(tmp_path / "tune.txt")
    M1 = ctx.matrix(A.rp, A.ci, A.val)
    first = ctx.autotune(M1, path)
    assert first["from_cache"] == 0
    M2 = ctx.matrix(A.rp, A.ci, A.val)
    second = ctx.autotune(M2, path)
    assert second["from_cache"] == 1
    for k in ("format", "rows_per_warp", "grid_dir_fp64", "grid_dir_fp32", "grid_update_fp64", "grid_update_fp32",
              "pdl_fp64", "pdl_fp32"):
        assert first[k] == second[k], k
    assert open(path).read().startswith("rsg-tune-v2 ")
    x, st = ctx.solve(M2, b, conf=rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10))
    assert st.converged == 1


def test_conf_autotune_on_first_solve(ctx, system, monkeypatch):
    A, b = system
    monkeypatch.delenv("RSG_TUNE_CACHE", raising=False)
    M = ctx.matrix(A.rp, A.ci, A.val)
    x, st = ctx.solve(M, b, conf=rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, autotune=True))
    assert st.converged == 1 and ctx.tune_info(M)["tuned"] == 1
    assert O.true_relres(A, b, x) <= 1e-10 * 1.01


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("use_graph", [True, False])
def test_programmatic_launch_gives_identical_bits(ctx, system, monkeypatch, precision, use_graph):
    # programmatic dependent launch only changes when the loop's blocks are scheduled: every
    # kernel waits for its predecessor before touching its data, so the solve is bitwise the same
    A, b = system
    assert A.n <= 262144  # PDL is on by default at this size
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision, use_graph=use_graph)
    assert ctx.tune_info(M)["pdl_fp64"] == 1 and ctx.tune_info(M)["pdl_fp32"] == 1
    x_pdl, st_pdl = ctx.solve(M, b, conf=conf)
    monkeypatch.setenv("RSG_NO_PDL", "1")
    assert ctx.tune_info(M)["pdl_fp64"] == 0
    x_plain, st_plain = ctx.solve(M, b, conf=conf)
    assert st_pdl.iterations == st_plain.iterations and (x_pdl == x_plain).all()
    assert O.true_relres(A, b, x_pdl) <= 1e-10 * 1.01
