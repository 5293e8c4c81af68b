"""How far the transient answers move with the quadrature of the mass integral.

RSolverHeat integrates Me = N N^T rho c detJ w over the tetrahedron's integration points
(src/rsolverheat.cpp:424-431), whose rule comes from range-model-lib's RElement, absent here.  The
oracle and the GPU assembly use the exact P1 integral V (1 + d_mn) / 20 (any rule of degree >= 2); if
the library's rule for linear tetrahedra has a single centroid point the reference assembles V / 16
for every pair instead, and a lumped mass would put V / 4 on the diagonal.  All three give every element
row the same sum, so steady states and the long-time limit agree; the early steps do not.  Measured with the
oracle's time loop on the benchmark's transient (40^3 hexes, dt = 1e-3, backward Euler, 64 steps):
relative l2 change of T after the first step 1.1e-2 (centroid) / 4.2e-2 (lumped), after the 64th
1.1e-4 / 4.3e-4.  This test keeps those properties on a 12^3 mesh."""
import numpy as np

from oracle import oracle as O
from rsg import workloads as W


def _row_sums(A):
    return np.add.reduceat(A.val, A.rp[:-1].astype(np.int64))


def test_mass_rules_share_row_sums_and_leave_steady_states_alone():
    n = 6
    p = W.heat_cube(n, sigma=1.0, seed=2, source="random", transient=True, dt=1e-3)
    sums = {}
    for rule in (O.MASS_EXACT, O.MASS_CENTROID, O.MASS_LUMPED):
        A, _ = O.assemble_heat(p, rule)
        sums[rule] = _row_sums(A)
    # each rule's element mass rows sum to V/4: rows whose neighbours are all free (no Dirichlet
    # column eliminated: nodes away from the x = 0 and x = 1 faces) of A = M + dt K sum alike
    x = np.asarray(p.mesh.xyz).reshape(-1, 3)[:, 0]
    inner = (p.book != W.EOD) & (x > 1.5 / n) & (x < 1.0 - 1.5 / n)
    rows = p.book[inner].astype(np.int64)
    assert rows.size > 0
    for rule in (O.MASS_CENTROID, O.MASS_LUMPED):
        assert np.allclose(sums[rule][rows], sums[O.MASS_EXACT][rows], rtol=1e-12, atol=1e-15)
        # the rows next to the eliminated columns differ
        assert not np.allclose(sums[rule], sums[O.MASS_EXACT], rtol=1e-12, atol=1e-15)
    q = W.heat_cube(6, sigma=1.0, seed=2, source="random")
    A0, b0 = O.assemble_heat(q, O.MASS_EXACT)
    A1, b1 = O.assemble_heat(q, O.MASS_CENTROID)
    assert np.array_equal(A0.val, A1.val) and np.array_equal(b0, b1)


def test_transient_answers_move_with_the_mass_rule():
    p = W.heat_cube(12, sigma=1.0, seed=3, source="random", transient=True, dt=1e-3)
    free = p.book != W.EOD
    runs = {rule: O.transient_heat(p, 16, mass_rule=rule)
            for rule in (O.MASS_EXACT, O.MASS_CENTROID, O.MASS_LUMPED)}
    ex = runs[O.MASS_EXACT]

    def rel(rule, k):
        return np.linalg.norm(runs[rule][k][free] - ex[k][free]) / np.linalg.norm(ex[k][free])

    for rule in (O.MASS_CENTROID, O.MASS_LUMPED):
        first, last = rel(rule, 0), rel(rule, 15)
        assert first > 1e-2          # the early steps depend on the rule
        assert last < 0.3 * first    # and the difference decays towards the common steady state
    # lumping moves the answer further than the centroid rule
    assert rel(O.MASS_LUMPED, 0) > rel(O.MASS_CENTROID, 0)
