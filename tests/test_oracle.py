"""CPU oracle pins: the reference's known-answer tests and textbook invariants.

The oracle is the checker for every GPU parity test, so it is pinned here
first: against the reference's only golden vectors
(tests/tst_matrix_solver.cpp:33-54 and :56-77 in the reference project), and
against properties the restated algorithms must have (dense solves, P1
patch tests, symmetry, rigid-body modes, load totals).
"""
import numpy as np
import pytest

from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err


def test_golden_spd_2x2():
    # tst_matrix_solver.cpp:33-54: A=[[4,1],[1,3]], b=[1,2] -> x=[1/11, 7/11], CG without preconditioner
    A = O.csr_from_dense(np.array([[4.0, 1.0], [1.0, 3.0]]))
    x, st = O.solve(A, np.array([1.0, 2.0]), prec=0, n_outer=1000, n_inner=1000, cvg=1e-13)
    assert x.shape == (2,)
    assert abs(x[0] - 1.0 / 11.0) < 1e-6 and abs(x[1] - 7.0 / 11.0) < 1e-6


def test_golden_diagonal_3x3():
    # tst_matrix_solver.cpp:56-77: diag(2,4,5) x = (6,8,10) -> x = (3,2,2)
    A = O.csr_from_dense(np.diag([2.0, 4.0, 5.0]))
    x, st = O.solve(A, np.array([6.0, 8.0, 10.0]), prec=0, n_outer=1000, cvg=1e-13)
    assert np.allclose(x, [3.0, 2.0, 2.0], atol=1e-6)


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return M @ M.T + n * np.eye(n)


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_cg_matches_dense_solve(prec):
    D = _spd(24, 1)
    A = O.csr_from_dense(D)
    b = np.arange(24, dtype=float) - 5.0
    x, st = O.solve(A, b, prec=prec, block_size=3, n_outer=500, stop_rule="true", rtol=1e-13)
    assert rel_err(x, np.linalg.solve(D, b)) < 1e-10
    assert st.true_relres <= 1e-13


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_gmres_matches_dense_solve_nonsymmetric(prec):
    rng = np.random.default_rng(3)
    D = _spd(30, 2) + 3.0 * rng.standard_normal((30, 30))
    A = O.csr_from_dense(D)
    b = rng.standard_normal(30)
    x, st = O.solve(A, b, prec=prec, block_size=3, solver="gmres", n_outer=200, n_inner=8, stop_rule="true",
                    rtol=1e-12)
    assert rel_err(x, np.linalg.solve(D, b)) < 1e-9


def test_jacobi_and_block_jacobi_builds():
    D = _spd(12, 4)
    D[5, 5] = 0.0  # zero diagonal -> 0 (src/rmatrixpreconditioner.cpp:88-91)
    A = O.csr_from_dense(D)
    d = O.jacobi(A)
    expect = np.where(np.diag(D) == 0.0, 0.0, 1.0 / np.where(np.diag(D) == 0.0, 1.0, np.diag(D)))
    assert np.allclose(d, expect, rtol=0, atol=0)
    D2 = _spd(12, 5)
    B, w = O.block_jacobi(O.csr_from_dense(D2), 5)  # 5 does not divide 12 -> width 4
    assert w == 4
    for k in range(3):
        inv = np.linalg.inv(D2[4 * k:4 * k + 4, 4 * k:4 * k + 4])
        assert np.allclose(B[4 * k:4 * k + 4], inv, rtol=1e-12, atol=1e-14)


def test_reference_stopping_rule_and_scaling():
    p = W.heat_cube(8)
    A, b = O.assemble_heat(p)
    x, st = O.solve(A, b, prec=1, n_outer=5000, cvg=1e-12)
    assert st.converged == 1
    # reference error measure is ||r||/(||A||_F ||x|| + ||b||) on the scaled system
    assert st.error < 1e-12
    assert st.equation_scale == pytest.approx(1e9 / (np.linalg.norm(b) / O.frobenius(A)))


def test_heat_patch_test_linear_field():
    # uniform k, no source, T=0 at x=0 and T=1 at x=1: P1 reproduces T=x exactly
    p = W.heat_cube(6, source="none")
    A, b = O.assemble_heat(p)
    x, st = O.solve(A, b, prec=1, n_outer=5000, stop_rule="true", rtol=1e-13)
    full = p.node_t.copy()
    free = p.book != W.EOD
    full[free] = x[p.book[free]]
    assert np.abs(full - p.mesh.xyz[:, 0]).max() < 1e-11


def test_heat_assembly_properties():
    p = W.heat_cube(5, sigma=1.0, seed=3, source="random")
    p.node_t[:] = 0.0  # homogeneous Dirichlet: no lifting, b only carries the source
    A, b = O.assemble_heat(p)
    D = A.to_dense()
    assert np.abs(D - D.T).max() <= 1e-14 * np.abs(D).max()
    assert np.all(np.linalg.eigvalsh(D) > 0)
    # total source = sum of element volume * Q; rows of Dirichlet nodes are dropped,
    # so the free rows carry a positive share of it, and exactly V Q / 4 per free tet node
    vol = 1.0 / (6 * 5 ** 3)
    total = (p.q_e * vol).sum()
    free_share = sum((p.book[p.mesh.tets[:, m]] != W.EOD) @ (p.q_e * vol / 4.0) for m in range(4))
    assert b.sum() == pytest.approx(free_share, rel=1e-13)
    assert 0 < b.sum() < total
    # transient: A = M + dt K is SPD and M's row sums equal the lumped volumes
    pt = W.heat_cube(4, transient=True, dt=1e-3)
    At, bt = O.assemble_heat(pt)
    Dt = At.to_dense()
    assert np.all(np.linalg.eigvalsh(Dt) > 0)


def test_stress_assembly_rigid_modes_and_load():
    # unconstrained beam: stiffness annihilates the 6 rigid-body modes
    p = W.stress_beam(4, 2, 2, traction=(0.0, 0.0, -1.0))
    free_all = np.zeros(3 * p.mesh.n_nodes, bool)
    book, n_free = W.node_book(free_all)
    p.book, p.n_free, p.disabled = book, n_free, free_all
    A, b = O.assemble_stress(p)
    D = A.to_dense()
    X = p.mesh.xyz
    modes = []
    for k in range(3):
        u = np.zeros((p.mesh.n_nodes, 3))
        u[:, k] = 1.0
        modes.append(u.ravel())
    for (i, j) in ((0, 1), (1, 2), (0, 2)):
        u = np.zeros((p.mesh.n_nodes, 3))
        u[:, i] = -X[:, j]
        u[:, j] = X[:, i]
        modes.append(u.ravel())
    for u in modes:
        assert np.abs(D @ u).max() <= 1e-9 * np.abs(D).max()
    assert np.abs(D - D.T).max() <= 1e-12 * np.abs(D).max()
    # total traction load = t * face area (1 x 1)
    assert b[2::3].sum() == pytest.approx(-1.0, rel=1e-12)
    assert abs(b[0::3].sum()) < 1e-14 and abs(b[1::3].sum()) < 1e-14


def test_stress_clamped_beam_solves():
    p = W.stress_beam(8, 4, 4)
    A, b = O.assemble_stress(p)
    assert A.n == p.n_free == 3 * (9 * 5 * 5 - 5 * 5)
    x, st = O.solve(A, b, prec=1, n_outer=20000, stop_rule="true", rtol=1e-10)
    assert st.true_relres <= 1e-10
    uz = x[2::3]
    assert uz.min() < 0  # the free end moves down under the -z traction


def test_magnetostatic_assembly_structure():
    # RSolverMagnetostatics (src/rsolvermagnetostatics.cpp:94-105, :256-286): each component carries
    # minus the unit-conductivity heat Laplacian; the zero blocks between components are in the pattern
    p = W.magnetostatic_cube(4, current="random", seed=2)
    A, b = O.assemble_magnetostatics(p)
    h = W.heat_cube(4, source="none")
    H, _ = O.assemble_heat(h)
    assert A.n == 3 * H.n and len(A.ci) == 9 * len(H.ci)
    D, DH = A.to_dense(), H.to_dense()
    for c in range(3):
        for d in range(3):
            blk = D[c::3, d::3]
            if c == d:
                assert np.array_equal(blk, -DH)  # bitwise: same products, negated
            else:
                assert not blk.any()
    # the source e0 V/4 (grad N_m x J_m) sums grad N_m over a node's tets: zero at interior nodes
    # for a uniform current, so only boundary rows carry it
    q = W.magnetostatic_cube(4, current="none")
    q.node_j = np.tile([1.0e6, -2.0e6, 0.5e6], q.mesh.n_nodes)
    _, bq = O.assemble_magnetostatics(q)
    xyz = q.mesh.xyz
    interior = np.all((xyz > 0.0) & (xyz < 1.0), axis=1)
    pos = q.book[3 * np.flatnonzero(interior)]
    scale = np.abs(bq).max()
    assert scale > 0 and np.abs(bq[pos[:, None] + np.arange(3)]).max() <= 1e-12 * scale


def test_magnetostatic_patch_test_linear_potential():
    # no current, A = 0 on x=0 and (1, -2, 3) on x=1: P1 reproduces the linear potential exactly
    p = W.magnetostatic_cube(5, current="none", a1=(1.0, -2.0, 3.0))
    A, b = O.assemble_magnetostatics(p)
    x, st = O.solve(A, b, prec=1, n_outer=5000, stop_rule="true", rtol=1e-13)
    full = p.node_a.copy()
    free = p.book != W.EOD
    full[free] = x[p.book[free]]
    expect = np.outer(p.mesh.xyz[:, 0], [1.0, -2.0, 3.0]).reshape(-1)
    assert np.abs(full - expect).max() < 1e-10


def test_rng_is_counter_based():
    a = W.uniform(7, 1, 1000)
    b = W.uniform(7, 1, 1000)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, W.uniform(8, 1, 1000))
    z = W.normal(0, 3, 200000)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01


def test_mesh_orientation_and_volume():
    m = W.box_tet_mesh(3, 2, 4, 1.5, 1.0, 2.0)
    X = m.xyz[m.tets.astype(np.int64)]
    a, b, c = X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))
    assert np.all(det > 0)
    assert det.sum() / 6.0 == pytest.approx(1.5 * 1.0 * 2.0, rel=1e-12)
