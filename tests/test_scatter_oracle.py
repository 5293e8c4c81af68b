"""The oracle's restatement of RSolverFluid's pattern-cached assembly (src/rsolverfluid.cpp:2305-2419)
against a dense assembly that adds the same element blocks in element order: same pattern, and the
same values bit for bit (both add each entry's contributions in element order starting from zero)."""
import numpy as np

from oracle import oracle as O


def mesh(seed=0):
    rng = np.random.default_rng(seed)
    n_nodes, d = 9, 4
    elems = [[0, 1, 2, 3], [1, 2, 3, 4], [4, 5, 6, 7], [2, 3, 4], [6, 7, 8], [5, 6, 7, 8], [0, 0, 1, 2]]
    active = np.array([1, 1, 0, 1, 1, 1, 1], np.uint8)
    begin = np.cumsum([0] + [len(e) for e in elems]).astype(np.uint32)
    nodes = np.concatenate(elems).astype(np.uint32)
    book = np.full(n_nodes * d, 0xFFFFFFFF, np.uint32)
    enabled = rng.uniform(size=n_nodes * d) > 0.2
    n_free = int(enabled.sum())
    book[enabled] = np.arange(n_free)
    blocks = [(len(e) * d) for e, a in zip(elems, active) if a]
    Ae = rng.standard_normal(sum(k * k for k in blocks))
    fe = rng.standard_normal(sum(blocks))
    return d, begin, nodes, active, n_nodes, book, n_free, Ae, fe, elems


def dense(d, elems, active, book, n_free, Ae, fe):
    A = np.zeros((n_free, n_free))
    pattern = np.zeros((n_free, n_free), bool)
    b = np.zeros(n_free)
    ao = fo = 0
    for e, a in zip(elems, active):
        if not a:
            continue
        nd = len(e) * d
        rows = [(m * d + i, book[e[m] * d + i]) for m in range(len(e)) for i in range(d)
                if book[e[m] * d + i] != 0xFFFFFFFF]
        blk = Ae[ao:ao + nd * nd].reshape(nd, nd)
        for la, ra in rows:
            b[ra] += fe[fo + la]
            for lc, rc in rows:
                A[ra, rc] += blk[la, lc]
                pattern[ra, rc] = True
        ao += nd * nd
        fo += nd
    return A, pattern, b


def test_pattern_and_values_match_dense_element_order_sum():
    d, begin, nodes, active, n_nodes, book, n_free, Ae, fe, elems = mesh()
    C, b = O.scatter_assemble(d, begin, nodes, active, n_nodes, book, n_free, Ae, fe)
    A, pattern, b_ref = dense(d, elems, active, book, n_free, Ae, fe)
    rows = np.repeat(np.arange(n_free), np.diff(C.rp.astype(np.int64)))
    assert C.rp[-1] == pattern.sum()
    assert np.all(pattern[rows, C.ci])
    for r in range(n_free):  # columns ascending within each row
        assert np.all(np.diff(C.ci[C.rp[r]:C.rp[r + 1]].astype(np.int64)) > 0)
    assert np.array_equal(C.val, A[rows, C.ci])
    assert np.array_equal(b, b_ref)
