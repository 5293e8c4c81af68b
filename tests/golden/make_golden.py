"""Writes the golden fixtures of tests/golden/ (run from the repository root).

1. golden_reference_kat.json: the known-answer tests of the reference's own
   test file tests/tst_matrix_solver.cpp (matrix entries, right-hand side and
   expected solution), parsed from that file when the reference tree is given
   (--reference DIR); the cases are small and the file cites the lines.
2. golden_small_systems.npz: small assembled systems (heat on a 4^3 lognormal
   cube, elasticity on a 2x2x2-hex beam) with the CPU oracle's assembly and
   tight FP64 solution -- regression pins for the oracle and the GPU path.
"""
import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "range-solver-lib_b200"))


def parse_kats(path):
    """Each test body: addValue(i, j, v) entries, b[i] = v assignments, and the
    expected x from `qAbs(x[i] - expr) < tol` checks (expr: a number or a/b)."""
    src = open(path).read()
    cases = []
    for m in re.finditer(r"void TestMatrixSolver::(\w+)\(\)\s*\{(.*?)\n\}", src, re.S):
        name, body = m.group(1), m.group(2)
        start = src[: m.start()].count("\n") + 1
        end = start + m.group(0).count("\n")
        n = int(re.search(r"setNRows\((\d+)\)", body).group(1))
        entries = [[int(i), int(j), float(v)] for i, j, v in
                   re.findall(r"addValue\((\d+),\s*(\d+),\s*([-\d.eE+]+)\)", body)]
        b = [0.0] * n
        for i, v in re.findall(r"\bb\[(\d+)\]\s*=\s*([-\d.eE+]+);", body):
            b[int(i)] = float(v)
        x = [None] * n
        for i, expr in re.findall(r"qAbs\(x\[(\d+)\]\s*-\s*([-\d.eE+ /]+)\)\s*<\s*tol", body):
            parts = [float(p) for p in expr.split("/")]
            x[int(i)] = parts[0] / parts[1] if len(parts) == 2 else parts[0]
        cases.append({"name": name, "source": f"tests/tst_matrix_solver.cpp:{start}-{end}", "n": n,
                      "entries": entries, "b": b, "x": x, "solver": "CG", "preconditioner": "NONE",
                      "tol": 1e-6})
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="reference project root (for the known-answer tests)")
    a = ap.parse_args()
    if a.reference:
        cases = parse_kats(os.path.join(a.reference, "tests", "tst_matrix_solver.cpp"))
        with open(os.path.join(HERE, "golden_reference_kat.json"), "w") as f:
            json.dump({"cases": cases}, f, indent=1)
        print(f"{len(cases)} known-answer tests")
    from oracle import oracle as O
    from rsg import workloads as W
    out = {}
    for tag, (A, b) in (("heat4", O.assemble_heat(W.heat_cube(4, sigma=1.5, seed=3, source="random"))),
                        ("stress2", O.assemble_stress(W.stress_beam(2, 2, 2)))):
        x, st = O.solve(A, b, prec=1, n_outer=100000, stop_rule="true", rtol=1e-13)
        assert st.converged == 1
        out[f"{tag}_rp"], out[f"{tag}_ci"], out[f"{tag}_val"] = A.rp, A.ci, A.val
        out[f"{tag}_b"], out[f"{tag}_x"] = b, x
    np.savez_compressed(os.path.join(HERE, "golden_small_systems.npz"), **out)
    print("small systems:", ", ".join(sorted({k.split("_")[0] for k in out})))


if __name__ == "__main__":
    main()
