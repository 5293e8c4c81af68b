"""The committed golden fixtures (tests/golden/, written by make_golden.py)
against the CPU oracle: the reference's known-answer tests, and small
assembled systems with their tight solutions (regression pins)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def kat_cases():
    return json.load(open(os.path.join(GOLDEN, "golden_reference_kat.json")))["cases"]


def kat_matrix(case):
    D = np.zeros((case["n"], case["n"]))
    for i, j, v in case["entries"]:
        D[i, j] += v
    return O.csr_from_dense(D)


def fixture(tag):
    z = np.load(os.path.join(GOLDEN, "golden_small_systems.npz"))
    return O.CSR(len(z[f"{tag}_rp"]) - 1, z[f"{tag}_rp"], z[f"{tag}_ci"], z[f"{tag}_val"]), z[f"{tag}_b"], \
        z[f"{tag}_x"]


@pytest.mark.parametrize("case", kat_cases(), ids=lambda c: c["name"])
def test_reference_known_answers_on_oracle(case):
    x, st = O.solve(kat_matrix(case), np.array(case["b"]), prec=0, n_outer=1000, n_inner=1000, cvg=1e-13)
    assert np.max(np.abs(x - np.array(case["x"]))) < case["tol"]


@pytest.mark.parametrize("tag,problem", [("heat4", lambda: W.heat_cube(4, sigma=1.5, seed=3, source="random")),
                                         ("stress2", lambda: W.stress_beam(2, 2, 2))])
def test_small_systems_fixture(tag, problem):
    A, b, x = fixture(tag)
    Ao, bo = O.assemble_heat(problem()) if tag.startswith("heat") else O.assemble_stress(problem())
    assert np.array_equal(Ao.rp, A.rp) and np.array_equal(Ao.ci, A.ci)
    assert np.allclose(Ao.val, A.val, rtol=1e-13, atol=1e-13 * np.abs(A.val).max())
    assert np.allclose(bo, b, rtol=1e-13, atol=1e-13 * max(np.abs(b).max(), 1.0))
    xo, st = O.solve(A, b, prec=1, n_outer=100000, stop_rule="true", rtol=1e-13)
    assert rel_err(xo, x) < 1e-11
