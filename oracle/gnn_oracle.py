"""CPU oracle of the learned preconditioner (test infrastructure only).

Only tests/ and the smoke check import this file; the library never calls it.
The reference has no learned preconditioner (src/rmatrixpreconditioner.cpp has
Jacobi and block Jacobi only), so there is nothing of the reference's to pin
this against: it is pinned instead by central finite differences of its own
float64 loss (tests/test_gnn_oracle.py), and the CUDA forward/backward kernels
are checked against it.

Network (float64 throughout):
  d_i = a_ii (1 where a_ii <= 0), s_i = d_i^-1/2, logd_i = log d_i,
  rsum_i = sum_j a_ij / d_i, rms = sqrt(mean((s r)^2)) (1 when 0)
  f_i = [s_i r_i / rms, logd_i - mean(logd), rsum_i, x_i, y_i, z_i, 1, 0]
  h0 = relu(f W_in + b_in)
  m_l = G h_l with G_ij = -a_ij s_i s_j (i != j)
  h_{l+1} = h_l + relu([h_l, m_l] W_l + b_l)
  M(r)_i = (h_L w_out + b_out)_i * rms * s_i
Loss: ||r - A M(r)||^2 / ||r||^2 (s and rms are functions of A and r only).
Flat parameter layout: W_in [8][H], b_in [H], then per layer W_l [2H][H], b_l [H],
then w_out [H], b_out [1].
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

F = 8


def n_params(L: int, H: int = 64) -> int:
    return F * H + H + L * (2 * H * H + H) + H + 1


def unpack(p: np.ndarray, L: int, H: int = 64):
    p = np.asarray(p, np.float64)
    o = 0
    W_in = p[o:o + F * H].reshape(F, H); o += F * H
    b_in = p[o:o + H]; o += H
    layers = []
    for _ in range(L):
        W = p[o:o + 2 * H * H].reshape(2 * H, H); o += 2 * H * H
        b = p[o:o + H]; o += H
        layers.append((W, b))
    w_out = p[o:o + H]; o += H
    b_out = p[o]; o += 1
    assert o == p.size
    return W_in, b_in, layers, w_out, b_out


def _graph(rp, ci, val):
    n = len(rp) - 1
    A = sp.csr_matrix((np.asarray(val, np.float64), np.asarray(ci, np.int64), np.asarray(rp, np.int64)), shape=(n, n))
    d = A.diagonal().copy()
    d = np.where(d > 0.0, d, 1.0)
    s = 1.0 / np.sqrt(d)
    off = A - sp.diags(A.diagonal())
    G = -(sp.diags(s) @ off @ sp.diags(s))
    rsum = np.asarray(A.sum(axis=1)).ravel() / d
    logd = np.log(d)
    return A, G.tocsr(), s, logd - logd.mean(), rsum


def forward(p, L, rp, ci, val, r, xyz=None, H: int = 64, keep: bool = False):
    """z = M(r); with keep=True also returns the activations for backward()."""
    W_in, b_in, layers, w_out, b_out = unpack(p, L, H)
    A, G, s, logd_c, rsum = _graph(rp, ci, val)
    n = A.shape[0]
    r = np.asarray(r, np.float64)
    u = r * s
    rms = np.sqrt(np.sum(u * u) / n)
    rms = rms if rms > 0.0 else 1.0
    f = np.zeros((n, F))
    f[:, 0] = u / rms
    f[:, 1] = logd_c
    f[:, 2] = rsum
    if xyz is not None:
        f[:, 3:6] = np.asarray(xyz, np.float64).reshape(n, 3)
    f[:, 6] = 1.0
    pre0 = f @ W_in + b_in
    h = np.maximum(pre0, 0.0)
    hs, ms = [h], []
    for W, b in layers:
        m = G @ h
        z = np.concatenate([h, m], axis=1) @ W + b
        h = h + np.maximum(z, 0.0)
        hs.append(h)
        ms.append(m)
    y = h @ w_out + b_out
    out = y * rms * s
    if keep:
        return out, dict(A=A, G=G, s=s, rms=rms, f=f, pre0=pre0, hs=hs, ms=ms)
    return out


def loss_grad(p, L, rp, ci, val, r, xyz=None, H: int = 64):
    """(loss, flat gradient) of ||r - A M(r)||^2 / ||r||^2 (A symmetric)."""
    W_in, b_in, layers, w_out, b_out = unpack(p, L, H)
    z, c = forward(p, L, rp, ci, val, r, xyz, H, keep=True)
    A, G, s, rms = c["A"], c["G"], c["s"], c["rms"]
    r = np.asarray(r, np.float64)
    rr = float(r @ r)
    rr = rr if rr > 0.0 else 1.0
    e = r - A @ z
    loss = float(e @ e) / rr
    gz = -2.0 * (A.T @ e) / rr
    gy = gz * rms * s
    grads = []
    hL = c["hs"][-1]
    g_wout = hL.T @ gy
    g_bout = gy.sum()
    g = np.outer(gy, w_out)
    layer_grads = [None] * L
    for l in range(L - 1, -1, -1):
        W, b = layers[l]
        X = np.concatenate([c["hs"][l], c["ms"][l]], axis=1)
        zl = X @ W + b
        dz = g * (zl > 0.0)
        layer_grads[l] = (X.T @ dz, dz.sum(axis=0))
        gx = dz @ W.T
        g = g + gx[:, :H] + G.T @ gx[:, H:]
    dpre = g * (c["pre0"] > 0.0)
    grads.append((c["f"].T @ dpre).ravel())
    grads.append(dpre.sum(axis=0))
    for gW, gb in layer_grads:
        grads.append(gW.ravel())
        grads.append(gb)
    grads.append(g_wout)
    grads.append(np.array([g_bout]))
    return loss, np.concatenate(grads)


def loss(p, L, rp, ci, val, r, xyz=None, H: int = 64) -> float:
    z = forward(p, L, rp, ci, val, r, xyz, H)
    A = sp.csr_matrix((np.asarray(val, np.float64), np.asarray(ci, np.int64), np.asarray(rp, np.int64)),
                      shape=(len(rp) - 1, len(rp) - 1))
    r = np.asarray(r, np.float64)
    e = r - A @ z
    rr = float(r @ r)
    return float(e @ e) / (rr if rr > 0.0 else 1.0)


def glorot_params(L: int, seed: int, H: int = 64, gain_layer: float = 0.5, gain_out: float = 0.1) -> np.ndarray:
    """Random parameters with the library's initial scales (Glorot-uniform, zero biases)."""
    rng = np.random.default_rng(seed)
    parts = []
    a = np.sqrt(6.0 / (F + H))
    parts += [rng.uniform(-a, a, F * H), np.zeros(H)]
    for _ in range(L):
        a = gain_layer * np.sqrt(6.0 / (3 * H))
        parts += [rng.uniform(-a, a, 2 * H * H), np.zeros(H)]
    a = gain_out * np.sqrt(6.0 / (H + 1))
    parts += [rng.uniform(-a, a, H), np.zeros(1)]
    return np.concatenate(parts)
