"""The golden fixtures (tests/golden/) through the C ABI on the GPU: the
reference's known-answer tests with the reference's own CG rule, and the small
fixture systems (GPU assembly and solve against the stored oracle results)."""
import json
import os

import numpy as np
import pytest

import rsg
from conftest import rel_err
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_known_answers_gpu(ctx):
    for case in json.load(open(os.path.join(GOLDEN, "golden_reference_kat.json")))["cases"]:
        D = np.zeros((case["n"], case["n"]))
        for i, j, v in case["entries"]:
            D[i, j] += v
        A = O.csr_from_dense(D)
        M = ctx.matrix(A.rp, A.ci, A.val)
        x, st = ctx.solve(M, np.array(case["b"]), conf=rsg.make_conf(n_outer=1000, n_inner=1000, cvg=1e-13),
                          prec=rsg.PREC_NONE)
        assert np.max(np.abs(x - np.array(case["x"]))) < case["tol"], case["name"]


@pytest.mark.parametrize("tag", ["heat4", "stress2"])
def test_fixture_systems_gpu(ctx, torch_cuda, tag):
    torch = torch_cuda
    z = np.load(os.path.join(GOLDEN, "golden_small_systems.npz"))
    rp, ci, val, b, x_ref = (z[f"{tag}_{k}"] for k in ("rp", "ci", "val", "b", "x"))
    p = W.heat_cube(4, sigma=1.5, seed=3, source="random") if tag == "heat4" else W.stress_beam(2, 2, 2)
    asm = rsg.Assembly.heat(ctx, p) if tag == "heat4" else rsg.Assembly.stress(ctx, p)
    bd = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
    M = asm.assemble(p, bd)
    ctx.sync()
    grp, gci, gval = M.to_host()
    assert np.array_equal(grp, rp) and np.array_equal(gci, ci)
    assert np.allclose(gval, val, rtol=1e-13, atol=1e-13 * np.abs(val).max())
    assert np.allclose(bd.cpu().numpy(), b, rtol=1e-13, atol=1e-13 * max(np.abs(b).max(), 1.0))
    for precision in ("fp64", "mixed"):
        x, st = ctx.solve(M, b, conf=rsg.make_conf(n_outer=100000, stop_rule="true", rtol=1e-12,
                                                   precision=precision))
        assert st.converged == 1 and rel_err(x, x_ref) < 1e-9
    asm.close()
