"""rsg_true_relres_noalloc: the residual check for callers that cannot allocate.

Applications that give all device memory to their own pool allocator, or that
cannot take the device-wide synchronisation of cudaMalloc/cudaFree inside
their time loop, call this entry point with arrays they already own on the
device.  This file runs last (it is named to sort after the other test files)
so that a run stopping at its first failure has already run everything else.
It checks, through the C ABI, that two calls in a row agree with the
allocating rsg_true_relres within the FP64 reduction tolerance the other
tests use (1e-13 relative), that repeated calls give identical bits, that the
size limit is enforced before any work, and that no device memory is taken.
"""
import ctypes as C

import numpy as np
import pytest

import rsg
from rsg import _lib
from oracle import oracle as O
from rsg import workloads as W


def test_size_limit_is_rejected_before_any_work():
    lib = _lib.load()
    null = C.c_void_p(0)
    s = lib.rsg_true_relres_noalloc(_lib.NOALLOC_MAX_ROWS + 1, null, null, null, null, null, null, null)
    assert s == _lib.ERR_INVALID_ARG
    assert lib.rsg_true_relres_noalloc(0, null, null, null, null, null, null, null) == _lib.ERR_INVALID_ARG


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point():
    import torch
    assert torch.cuda.is_available()
    lib = _lib.load()
    p = W.heat_cube(24, sigma=1.5, seed=21, source="random")
    A, b = O.assemble_heat(p)
    x = np.random.default_rng(5).standard_normal(A.n)
    dev = {k: torch.tensor(v, device="cuda") for k, v in
           (("rp", A.rp.astype(np.int32)), ("ci", A.ci.astype(np.int32)), ("val", A.val), ("b", b), ("x", x))}
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    torch.cuda.synchronize()
    # reference value: the allocating entry point through a context and matrix handle
    with rsg.Context(0) as ctx:
        M = ctx.matrix(A.rp, A.ci, A.val)
        expect = ctx.true_relres(M, dev["b"], dev["x"])
        M.close()
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        s = lib.rsg_true_relres_noalloc(A.n, ptr(dev["rp"]), ptr(dev["ci"]), ptr(dev["val"]), ptr(dev["b"]),
                                        ptr(dev["x"]), ptr(out), C.c_void_p(stream))
        assert s == _lib.OK
        torch.cuda.synchronize()
        return out.cpu().numpy().copy()

    first = call()  # the first call on the device performs the one-time set-up
    free_before = torch.cuda.mem_get_info()[0]
    second = call()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    for got in (first, second):
        assert got[2] == pytest.approx(expect, rel=1e-13)
        r = O.spmv(A, x) - b
        assert got[0] == pytest.approx(np.linalg.norm(r), rel=1e-13)
        assert got[1] == pytest.approx(np.linalg.norm(b), rel=1e-13)
    assert np.array_equal(first, second)


def _tridiagonal(n: int, seed: int) -> O.CSR:
    """1-D Laplacian-like matrix with random positive couplings (CSR, sorted columns)."""
    rng = np.random.default_rng(seed)
    off = -rng.uniform(0.5, 1.5, n - 1)
    diag = np.zeros(n)
    diag[:-1] -= off
    diag[1:] -= off
    diag += 0.1
    cols = np.stack([np.arange(n) - 1, np.arange(n), np.arange(n) + 1], axis=1)
    vals = np.stack([np.r_[0.0, off], diag, np.r_[off, 0.0]], axis=1)
    keep = (cols >= 0) & (cols < n)
    rp = np.zeros(n + 1, np.uint32)
    rp[1:] = np.cumsum(keep.sum(axis=1))
    return O.CSR(n, rp, cols[keep].astype(np.uint32), vals[keep].astype(np.float64))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["tri33", "tri1", "heat22", "tri_max"])
def test_noalloc_ragged_and_maximum_sizes(case):
    """Sizes that leave the last 256-row block and the last 32-row chunk partly empty (33 rows, one
    row, a 22^3 heat cube with 11,109 rows) and the largest accepted size, RSG_NOALLOC_MAX_ROWS rows,
    which fills the last slot of the scratch array.  Two calls in a row, each against the oracle's
    residual to 1e-13 and against the allocating entry point."""
    import torch
    assert torch.cuda.is_available()
    lib = _lib.load()
    if case == "heat22":
        p = W.heat_cube(22, sigma=1.0, seed=3, source="random")
        A, b = O.assemble_heat(p)
    else:
        n = {"tri33": 33, "tri1": 1, "tri_max": _lib.NOALLOC_MAX_ROWS}[case]
        A = _tridiagonal(n, seed=n)
        b = np.random.default_rng(n + 1).standard_normal(n)
    if case != "tri_max":
        assert A.n % 32 != 0
    x = np.random.default_rng(7).standard_normal(A.n)
    r = O.spmv(A, x) - b
    want = np.array([np.linalg.norm(r), np.linalg.norm(b), np.linalg.norm(r) / np.linalg.norm(b)])
    dev = {k: torch.tensor(v, device="cuda") for k, v in
           (("rp", A.rp.astype(np.int32)), ("ci", A.ci.astype(np.int32)), ("val", A.val), ("b", b), ("x", x))}
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    with rsg.Context(0) as ctx:
        M = ctx.matrix(A.rp, A.ci, A.val)
        expect = ctx.true_relres(M, dev["b"], dev["x"])
        M.close()
    got = []
    for _ in range(2):
        s = lib.rsg_true_relres_noalloc(A.n, ptr(dev["rp"]), ptr(dev["ci"]), ptr(dev["val"]), ptr(dev["b"]),
                                        ptr(dev["x"]), ptr(out), C.c_void_p(stream))
        assert s == _lib.OK
        torch.cuda.synchronize()
        got.append(out.cpu().numpy().copy())
        out.fill_(float("nan"))
    for g in got:
        np.testing.assert_allclose(g, want, rtol=1e-13)
        assert g[2] == pytest.approx(expect, rel=1e-13)
    assert np.array_equal(got[0], got[1])
