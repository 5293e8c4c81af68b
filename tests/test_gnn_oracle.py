"""CPU checks of the learned-preconditioner oracle: its analytic gradient
against central finite differences of its own float64 loss."""
import numpy as np
import scipy.sparse as sp

from oracle import gnn_oracle as go


def _laplacian_2d(nx, ny, seed):
    """5-point diffusion matrix with lognormal edge conductances (SPD)."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    rows, cols, vals = [], [], []
    diag = np.full(n, 1e-2)
    idx = lambda i, j: i * ny + j  # noqa: E731
    for i in range(nx):
        for j in range(ny):
            for di, dj in ((1, 0), (0, 1)):
                if i + di < nx and j + dj < ny:
                    k = np.exp(rng.normal())
                    a, b = idx(i, j), idx(i + di, j + dj)
                    rows += [a, b]
                    cols += [b, a]
                    vals += [-k, -k]
                    diag[a] += k
                    diag[b] += k
    rows += list(range(n))
    cols += list(range(n))
    vals += list(diag)
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    A.sort_indices()
    return A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data


def test_gradient_matches_finite_differences():
    H, L = 8, 2
    rp, ci, val = _laplacian_2d(6, 5, 1)
    n = len(rp) - 1
    rng = np.random.default_rng(2)
    r = rng.normal(size=n)
    xyz = rng.uniform(size=(n, 3))
    p = rng.uniform(-0.5, 0.5, go.n_params(L, H))
    loss, g = go.loss_grad(p, L, rp, ci, val, r, xyz, H)
    assert np.isclose(loss, go.loss(p, L, rp, ci, val, r, xyz, H), rtol=1e-12)
    eps = 1e-6
    # every coordinate of the small network
    fd = np.empty_like(p)
    for k in range(p.size):
        e = np.zeros_like(p)
        e[k] = eps
        fd[k] = (go.loss(p + e, L, rp, ci, val, r, xyz, H) - go.loss(p - e, L, rp, ci, val, r, xyz, H)) / (2 * eps)
    err = np.linalg.norm(fd - g) / np.linalg.norm(fd)
    assert err < 1e-6, err


def test_positive_homogeneity_and_layout():
    H, L = 8, 3
    rp, ci, val = _laplacian_2d(5, 4, 3)
    n = len(rp) - 1
    p = go.glorot_params(L, 0, H)
    assert p.size == go.n_params(L, H)
    r = np.random.default_rng(0).normal(size=n)
    z1 = go.forward(p, L, rp, ci, val, r, None, H)
    z2 = go.forward(p, L, rp, ci, val, 3.5 * r, None, H)
    np.testing.assert_allclose(z2, 3.5 * z1, rtol=1e-12)
    # scaling A by c scales M(r) by 1/c (features are scale-free)
    z3 = go.forward(p, L, rp, ci, 4.0 * val, r, None, H)
    np.testing.assert_allclose(z3, z1 / 4.0, rtol=1e-12)
