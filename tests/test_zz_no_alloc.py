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
