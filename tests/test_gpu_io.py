"""File formats and the failure-detection self-test through the C ABI: the
RSGCSR01 CSR/RHS dump, the RSGGNN01 learned-preconditioner checkpoint, and a
bounded device wait that runs out without any fault."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import learned as RL
from rsg import workloads as W

pytestmark = pytest.mark.gpu


def parse_dump(path):
    """Independent reader of the documented layout."""
    raw = open(path, "rb").read()
    assert raw[:8] == b"RSGCSR01"
    n, has_b = np.frombuffer(raw, np.uint32, 2, 8)
    nnz = int(np.frombuffer(raw, np.uint64, 1, 16)[0])
    o = 64
    rp = np.frombuffer(raw, np.uint32, n + 1, o); o += 4 * (n + 1)
    ci = np.frombuffer(raw, np.uint32, nnz, o); o += 4 * nnz
    val = np.frombuffer(raw, np.float64, nnz, o); o += 8 * nnz
    b = np.frombuffer(raw, np.float64, n, o) if has_b else None
    if has_b:
        o += 8 * n
    assert o == len(raw)
    return rp, ci, val, b


def test_csr_dump_roundtrip(ctx, torch_cuda, tmp_path):
    torch = torch_cuda
    A, b = O.assemble_heat(W.heat_cube(6, sigma=1.0, seed=2, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    bd = torch.from_numpy(b).cuda()
    torch.cuda.synchronize()
    path = str(tmp_path / "sys.rsgcsr")
    ctx.save_matrix(M, path, bd)
    rp, ci, val, bb = parse_dump(path)
    assert np.array_equal(rp, A.rp) and np.array_equal(ci, A.ci) and np.array_equal(val, A.val)
    assert np.array_equal(bb, b)
    b2 = torch.zeros_like(bd)
    M2, has_b = ctx.load_matrix(path, b2)
    assert has_b and torch.equal(b2, bd)
    rp2, ci2, val2 = M2.to_host()
    assert np.array_equal(rp2, A.rp) and np.array_equal(ci2, A.ci) and np.array_equal(val2, A.val)
    ctx.save_matrix(M, str(tmp_path / "a_only.rsgcsr"))
    assert parse_dump(str(tmp_path / "a_only.rsgcsr"))[3] is None
    with pytest.raises(rsg.RsgError):
        ctx.load_matrix(str(tmp_path / "missing.rsgcsr"))
    (tmp_path / "bad.rsgcsr").write_bytes(b"NOTACSR0" + bytes(56))
    with pytest.raises(rsg.RsgError):
        ctx.load_matrix(str(tmp_path / "bad.rsgcsr"))


def _corrupt(raw: bytes, offset: int, value: np.ndarray) -> bytes:
    b = bytearray(raw)
    v = value.tobytes()
    b[offset:offset + len(v)] = v
    return bytes(b)


def test_corrupt_csr_dumps_are_rejected_before_any_copy(ctx, torch_cuda, tmp_path):
    """An untrusted header or row pointer never sizes a read past the file's arrays: a last row
    pointer above the stored nnz, a header nnz that does not match the payload, an absurd row
    count and a decreasing row pointer all return RSG_ERR_INVALID_ARG, and the context stays usable."""
    A, b = O.assemble_heat(W.heat_cube(4, sigma=1.0, seed=2, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    path = tmp_path / "ok.rsgcsr"
    ctx.save_matrix(M, str(path))
    raw = path.read_bytes()
    n = A.n
    cases = {
        "rp_end_above_nnz": _corrupt(raw, 64 + 4 * n, np.array([A.nnz + 1000], np.uint32)),
        "header_nnz_too_big": _corrupt(raw, 16, np.array([A.nnz + 7], np.uint64)),
        "header_n_huge": _corrupt(raw, 8, np.array([0xFFFFFFF0], np.uint32)),
        "rp_decreasing": _corrupt(raw, 64 + 4 * 3, np.array([0], np.uint32)),
        "truncated": raw[:-8],
    }
    for name, data in cases.items():
        f = tmp_path / f"{name}.rsgcsr"
        f.write_bytes(data)
        with pytest.raises(rsg.RsgError) as e:
            ctx.load_matrix(str(f))
        assert e.value.status == rsg._lib.ERR_INVALID_ARG, name
    M2, _ = ctx.load_matrix(str(path))
    assert np.array_equal(M2.to_host()[2], A.val)


def test_corrupt_checkpoint_is_rejected_before_allocating(ctx, tmp_path):
    m = RL.Learned(ctx, layers=2, seed=1)
    path = tmp_path / "m.rsggnn"
    m.save_binary(str(path))
    raw = path.read_bytes()
    for name, data in {"n_params_huge": _corrupt(raw, 24, np.array([1 << 60], np.uint64)),
                       "n_params_off_by_one": _corrupt(raw, 24, np.array([m.n_params + 1], np.uint64)),
                       "truncated": raw[:-4]}.items():
        f = tmp_path / f"{name}.rsggnn"
        f.write_bytes(data)
        with pytest.raises(rsg.RsgError) as e:
            RL.Learned.load_binary(ctx, str(f))
        assert e.value.status == rsg._lib.ERR_INVALID_ARG, name
    m.close()


def test_learned_binary_checkpoint(ctx, torch_cuda, tmp_path):
    torch = torch_cuda
    A, b = O.assemble_heat(W.heat_cube(6, sigma=1.0, seed=3, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    rd = torch.from_numpy(b).cuda()
    torch.cuda.synchronize()
    m = RL.Learned(ctx, layers=3, seed=9)
    for _ in range(4):
        m.train_step(M, rd, 1e-3)
    path = str(tmp_path / "model.rsggnn")
    m.save_binary(path)
    raw = open(path, "rb").read()
    assert raw[:8] == b"RSGGNN01" and len(raw) == 64 + 3 * 4 * m.n_params
    m2 = RL.Learned.load_binary(ctx, path)
    assert m2.layers == 3 and m2.step == 4
    for w in (RL.PARAMS, RL.ADAM_M, RL.ADAM_V):
        np.testing.assert_array_equal(m.get(w), m2.get(w))
    z1, z2 = torch.empty_like(rd), torch.empty_like(rd)
    m.apply(M, rd, z1)
    m2.apply(M, rd, z2)
    ctx.sync()
    assert torch.equal(z1, z2)
    m.close()
    m2.close()


def test_bounded_wait_timeout_is_reported_and_context_survives(ctx):
    assert ctx.selftest_wait_timeout(256) == rsg._lib.ERR_TIMEOUT
    assert "bounded wait" in ctx.lib.rsg_last_error(ctx.h).decode()
    ctx.sync()  # the error word was cleared: no second report
    A, b = O.assemble_heat(W.heat_cube(5, sigma=1.0, seed=1, source="random"))
    M = ctx.matrix(A.rp, A.ci, A.val)
    x, st = ctx.solve(M, b, conf=rsg.make_conf(n_outer=5000, stop_rule="true", rtol=1e-10))
    assert st.converged == 1 and O.true_relres(A, b, x) <= 1e-10 * 1.01
