"""The oracle's restatement against the reference's own solver, compiled from its sources.

oracle/_ref/libref_solver.so is the reference project's src/rmatrixsolver.cpp,
src/rmatrixpreconditioner.cpp, src/riterationinfo.cpp and src/riterationinfovalue.cpp built
unchanged against stand-in headers for range-base-lib, range-model-lib and Qt (oracle/ref_shim/).
These CPU tests pin the oracle to it: the reference's known-answer tests
(tests/tst_matrix_solver.cpp:33-77), and on the small heat and elasticity configurations, run on one
OpenMP thread each (the reference's multi-threaded reductions add in a run-dependent order), the
same iteration counts, the same errors and the same solutions bit for bit for CG with NONE, JACOBI
and BLOCK_JACOBI and for restarted GMRES (symmetric and nonsymmetric).  Multi-threaded runs agree
to rounding on a Jacobi-preconditioned system.  The built library exists where the reference
sources were present at build time; without it these tests are skipped.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference sources absent)")


def test_reference_known_answer_tests():
    # tests/tst_matrix_solver.cpp:33-54 and :56-77: CG without preconditioner, cvg 1e-13, tol 1e-6
    A = O.csr_from_dense(np.array([[4.0, 1.0], [1.0, 3.0]]))
    x, res = R.RefMatrix(A.rp, A.ci, A.val).solve(np.array([1.0, 2.0]), prec=R.PREC_NONE, n_outer=1000, cvg=1e-13)
    assert abs(x[0] - 1 / 11) < 1e-6 and abs(x[1] - 7 / 11) < 1e-6
    A = O.csr_from_dense(np.diag([2.0, 4.0, 5.0]))
    x, res = R.RefMatrix(A.rp, A.ci, A.val).solve(np.array([6.0, 8.0, 10.0]), prec=R.PREC_NONE, n_outer=1000,
                                                   cvg=1e-13)
    assert np.allclose(x, [3.0, 2.0, 2.0], atol=1e-6)


SYSTEMS = {"heat20": O.assemble_heat(W.heat_cube(20, sigma=0.0, seed=0, source="unit")),
           "heat12_lognormal": O.assemble_heat(W.heat_cube(12, sigma=1.5, seed=3, source="random")),
           "beam": O.assemble_stress(W.stress_beam(8, 4, 4))}


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("prec,block", [(0, 1), (1, 1), (1, 3), (2, 3)])
def test_cg_oracle_matches_reference_build_bitwise(name, prec, block):
    A, b = SYSTEMS[name]
    M = R.RefMatrix(A.rp, A.ci, A.val)
    x_ref, res = M.solve(b, prec=prec, block_size=block, n_outer=20000, cvg=1e-10, threads=1)
    x, st = O.solve(A, b, prec=prec, block_size=block, n_outer=20000, cvg=1e-10, threads=1)
    assert int(st.iterations) == int(res.iterations)
    assert st.error == res.error and st.trend == res.trend
    assert np.array_equal(x, x_ref)


@pytest.mark.parametrize("name", ["heat20", "heat12_lognormal"])
@pytest.mark.parametrize("prec", [0, 1])
def test_gmres_oracle_matches_reference_build_bitwise(name, prec):
    A, b = SYSTEMS[name]
    M = R.RefMatrix(A.rp, A.ci, A.val)
    x_ref, res = M.solve(b, solver="gmres", prec=prec, n_outer=500, n_inner=30, cvg=1e-10, threads=1)
    x, st = O.solve(A, b, prec=prec, solver="gmres", n_outer=500, n_inner=30, cvg=1e-10, threads=1)
    # the reference reports each restart's convergence check; the last one stops the loop
    assert int(st.outer) + 1 == int(res.iterations)
    assert st.error == res.error
    assert np.array_equal(x, x_ref)


def test_gmres_nonsymmetric_matches_reference_build():
    rng = np.random.default_rng(4)
    n = 300
    D = np.diag(np.full(n, 4.0)) + np.diag(np.full(n - 1, -1.4), 1) + np.diag(np.full(n - 1, -0.6), -1)
    D += np.diag(rng.uniform(-0.2, 0.2, n - 7), 7)
    A = O.csr_from_dense(D)
    b = rng.standard_normal(n)
    M = R.RefMatrix(A.rp, A.ci, A.val)
    for prec in (0, 1):
        x_ref, res = M.solve(b, solver="gmres", prec=prec, n_outer=200, n_inner=20, cvg=1e-12, threads=1)
        x, st = O.solve(A, b, prec=prec, solver="gmres", n_outer=200, n_inner=20, cvg=1e-12, threads=1)
        assert int(st.outer) + 1 == int(res.iterations)
        assert np.array_equal(x, x_ref)
        assert np.linalg.norm(D @ x_ref - b) / np.linalg.norm(b) < 1e-9


def test_multithreaded_runs_agree_to_rounding():
    A, b = SYSTEMS["heat12_lognormal"]
    M = R.RefMatrix(A.rp, A.ci, A.val)
    x_ref, res = M.solve(b, prec=1, n_outer=20000, cvg=1e-10, threads=4)
    x, st = O.solve(A, b, prec=1, n_outer=20000, cvg=1e-10, threads=4)
    assert abs(int(st.iterations) - int(res.iterations)) <= 2
    assert rel_err(x, x_ref) <= 1e-8


def test_reference_build_log_file_format(tmp_path):
    """RIterationInfo::writeToFile's convergence log, written by the reference's own code."""
    A, b = SYSTEMS["heat20"]
    f = tmp_path / "cvg.txt"
    _, res = R.RefMatrix(A.rp, A.ci, A.val).solve(b, prec=1, n_outer=5000, cvg=1e-10, log_file=str(f), threads=1)
    lines = f.read_text().splitlines()
    assert lines[0] == "Iteration number|Solver residual|Solver convergence"
    assert len(lines) == res.iterations + 1 and lines[-1].startswith(f"{res.iterations}|")
    assert float(lines[-1].split("|")[1]) == pytest.approx(res.error, rel=1e-6)
