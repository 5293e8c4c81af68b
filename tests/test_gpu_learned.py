"""GPU checks of the learned preconditioner through the C ABI.

Tolerances: the FP32 CUDA-core forward matches the float64 oracle to 1e-5
(relative 2-norm); the BF16 tensor-core forward to 3e-2; the FP32 gradient to
2e-3 (norm-wise, per parameter block); the tcgen05 (BF16) gradient to 3e-2 per
block and 5e-3 overall.  Solves with the learned preconditioner
reach the FP64 true relative residual they were asked for.
"""

import os

import numpy as np
import pytest

import rsg
from conftest import rel_err
from oracle import oracle as O
from oracle import gnn_oracle as GO
from rsg import learned as RL
from rsg import workloads as W

pytestmark = pytest.mark.gpu

_SYS = {}


def heat(n, sigma=1.0, seed=0, source="random"):
    key = (n, sigma, seed, source)
    if key not in _SYS:
        _SYS[key] = O.assemble_heat(W.heat_cube(n, sigma=sigma, seed=seed, source=source))
    return _SYS[key]


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


def _params(L, seed):
    """Library-scale random weights with small random biases (so every bias gradient is exercised)."""
    p = GO.glorot_params(L, seed)
    rng = np.random.default_rng(seed + 100)
    W_in, b_in, layers, w_out, _ = GO.unpack(p, L)
    b_in[:] = rng.uniform(-0.1, 0.1, b_in.size)
    for _, b in layers:
        b[:] = rng.uniform(-0.1, 0.1, b.size)
    p[-1] = 0.05
    return p


def _blocks(L, H=64):
    F = GO.F
    sizes = [F * H, H] + [2 * H * H, H] * L + [H, 1]
    names = ["W_in", "b_in"] + [f"{k}{l}" for l in range(L) for k in ("W", "b")] + ["w_out", "b_out"]
    offs = np.cumsum([0] + sizes)
    return [(nm, offs[i], offs[i + 1]) for i, nm in enumerate(names)]


@pytest.fixture(scope="module")
def model(ctx):
    m = RL.Learned(ctx, layers=3, seed=7)
    yield m
    m.close()


def test_create_info_layout(ctx, model):
    assert model.layers == 3 and model.hidden == 64
    assert model.n_params == GO.n_params(3)
    p = model.get()
    assert np.isfinite(p).all() and np.abs(p).max() > 0


def test_forward_matches_oracle(ctx, model, torch_cuda):
    torch = torch_cuda
    A, _ = heat(10, seed=3)
    M = ctx.matrix(A.rp, A.ci, A.val)
    p = _params(3, 1)
    model.set(p.astype(np.float32))
    p32 = p.astype(np.float32).astype(np.float64)
    r = np.random.default_rng(4).standard_normal(A.n)
    xyz = np.random.default_rng(5).uniform(size=(A.n, 3))
    want = GO.forward(p32, 3, A.rp, A.ci, A.val, r, xyz)
    rd, xd = _dev(torch, r), _dev(torch, xyz)
    z = torch.empty_like(rd)
    torch.cuda.synchronize()
    model.apply(M, rd, z, xd, tensor_cores=False)
    ctx.sync()
    assert rel_err(z.cpu().numpy(), want) < 1e-5
    model.apply(M, rd, z, xd, tensor_cores=True)
    ctx.sync()
    assert rel_err(z.cpu().numpy(), want) < 3e-2
    # without coordinates
    want0 = GO.forward(p32, 3, A.rp, A.ci, A.val, r, None)
    model.apply(M, rd, z, None, tensor_cores=False)
    ctx.sync()
    assert rel_err(z.cpu().numpy(), want0) < 1e-5


def test_gradient_matches_oracle(ctx, model, torch_cuda):
    torch = torch_cuda
    A, _ = heat(9, seed=5)
    M = ctx.matrix(A.rp, A.ci, A.val)
    p = _params(3, 2)
    model.set(p.astype(np.float32))
    p32 = p.astype(np.float32).astype(np.float64)
    r = np.random.default_rng(6).standard_normal(A.n)
    xyz = np.random.default_rng(7).uniform(size=(A.n, 3))
    want_loss, want_g = GO.loss_grad(p32, 3, A.rp, A.ci, A.val, r, xyz)
    rd, xd = _dev(torch, r), _dev(torch, xyz)
    torch.cuda.synchronize()
    loss, g = model.loss_grad(M, rd, xd, tensor_cores=False)
    assert abs(loss - want_loss) / want_loss < 1e-5
    for name, a, b in _blocks(3):
        assert rel_err(g[a:b], want_g[a:b]) < 2e-3, name
    assert rel_err(g, want_g) < 1e-3
    # the tcgen05 path: BF16 operands (8-bit mantissa) in the forward, data-backward and weight-gradient
    # products, FP32 accumulation.  Measured on B200: loss 7e-6, gradient 1.7e-3, worst block 1.2e-2.
    loss_t, g_t = model.loss_grad(M, rd, xd, tensor_cores=True)
    assert abs(loss_t - want_loss) / want_loss < 1e-4
    for name, a, b in _blocks(3):
        assert rel_err(g_t[a:b], want_g[a:b]) < 3e-2, name
    assert rel_err(g_t, want_g) < 5e-3


def test_train_step_reduces_loss(ctx, torch_cuda):
    torch = torch_cuda
    A, b = heat(10, seed=8)
    M = ctx.matrix(A.rp, A.ci, A.val)
    m = RL.Learned(ctx, layers=2, seed=3)
    rd = _dev(torch, b)
    torch.cuda.synchronize()
    losses = [m.train_step(M, rd, 2e-3) for _ in range(60)]
    assert m.step == 60
    assert losses[-1] < 0.7 * losses[0], (losses[0], losses[-1])
    m.close()


def test_checkpoint_roundtrip(ctx, torch_cuda, tmp_path):
    torch = torch_cuda
    A, b = heat(8, seed=9)
    M = ctx.matrix(A.rp, A.ci, A.val)
    m = RL.Learned(ctx, layers=2, seed=4)
    rd = _dev(torch, b)
    torch.cuda.synchronize()
    for _ in range(3):
        m.train_step(M, rd, 1e-3)
    path = str(tmp_path / "model.npz")
    m.save(path)
    m2 = RL.Learned.load(ctx, path)
    assert m2.step == 3 and m2.layers == 2
    for w in (RL.PARAMS, RL.ADAM_M, RL.ADAM_V):
        np.testing.assert_array_equal(m.get(w), m2.get(w))
    z1, z2 = torch.empty_like(rd), torch.empty_like(rd)
    m.apply(M, rd, z1)
    m2.apply(M, rd, z2)
    ctx.sync()
    assert torch.equal(z1, z2)
    # an inference-only checkpoint carries the parameters alone and applies the same network
    path2 = str(tmp_path / "params.npz")
    m.save(path2, with_adam=False)
    assert "adam_m" not in np.load(path2).files
    m3 = RL.Learned.load(ctx, path2)
    np.testing.assert_array_equal(m3.get(RL.PARAMS), m.get(RL.PARAMS))
    z3 = torch.empty_like(rd)
    m3.apply(M, rd, z3)
    ctx.sync()
    assert torch.equal(z1, z3)
    m.close()
    m2.close()
    m3.close()


@pytest.mark.parametrize("solver", ["cg", "gmres"])
def test_learned_solve_converges(ctx, model, solver):
    A, b = heat(12, seed=11)
    M = ctx.matrix(A.rp, A.ci, A.val)
    model.set(_params(3, 3).astype(np.float32))
    conf = RL.learned_conf(model, rsg.make_conf(solver=solver, n_outer=3000, n_inner=30, stop_rule="true",
                                                rtol=1e-10))
    x, st = ctx.solve(M, b, conf=conf, prec=rsg.PREC_LEARNED)
    assert st.converged == 1 and st.status == 0
    assert st.true_relres <= 1e-10 * 1.01
    assert O.true_relres(A, b, x) <= 1e-10 * 1.01


def test_learned_initial_guess(ctx, model):
    A, b = heat(12, seed=12)
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = RL.learned_conf(model, rsg.make_conf(n_outer=3000, stop_rule="true", rtol=1e-10), initial_guess=True)
    x, st = ctx.solve(M, b, conf=conf, prec=rsg.PREC_JACOBI)
    assert st.converged == 1 and st.true_relres <= 1e-10 * 1.01


def test_learned_argument_errors(ctx, model):
    A, b = heat(6, seed=1)
    M = ctx.matrix(A.rp, A.ci, A.val)
    with pytest.raises(rsg.RsgError):  # learned requested without a model
        ctx.solve(M, b, conf=rsg.make_conf(stop_rule="true"), prec=rsg.PREC_LEARNED)
    with pytest.raises(rsg.RsgError):  # flexible CG needs the true-residual stop rule
        ctx.solve(M, b, conf=RL.learned_conf(model, rsg.make_conf()), prec=rsg.PREC_LEARNED)
    with pytest.raises(rsg.RsgError):  # FP32 inner vectors are not offered with the learned preconditioner
        ctx.solve(M, b, conf=RL.learned_conf(model, rsg.make_conf(stop_rule="true", precision="mixed")),
                  prec=rsg.PREC_LEARNED)


def test_ablation_trained_network_cuts_iterations(ctx, torch_cuda):
    """What the trained network gains over the method without it: a model trained
    on the GPU (own forward/backward/Adam kernels) on plain-PCG trajectory
    residuals of seeded lognormal heat problems, evaluated on a held-out seed.
    Measured on B200: FCG 158 -> 51 iterations (Jacobi-PCG -> learned), flexible
    GMRES(30) 240 -> 43; the bars below leave room for run-to-run differences."""
    torch = torch_cuda
    rng = np.random.default_rng(0)
    samples, keep = [], []
    for i, n in enumerate([10, 12, 14, 16, 18, 20, 12, 16]):
        p = W.heat_cube(n, sigma=float(rng.uniform(0.5, 2.0)), seed=100 + i, source="random")
        asm = rsg.Assembly.heat(ctx, p)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        A = asm.assemble(p, b)
        ctx.sync()
        keep.append((asm, b))
        samples += [(A, r, None) for r in RL.trajectory_residuals(ctx, A, b, seed=i)]
    model = RL.Learned(ctx, layers=6, seed=1)
    losses = RL.train(ctx, model, samples, 3000, lr=1e-3)
    assert np.mean(losses[-200:]) < 0.25 * np.mean(losses[:50])

    A, b = heat(20, sigma=1.0, seed=999)
    M = ctx.matrix(A.rp, A.ci, A.val)
    its = {}
    for name, prec, conf in [
        ("pcg", rsg.PREC_JACOBI, rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10)),
        ("fcg", rsg.PREC_LEARNED, RL.learned_conf(model, rsg.make_conf(n_outer=20000, stop_rule="true",
                                                                        rtol=1e-10))),
        ("gmres", rsg.PREC_JACOBI, rsg.make_conf(solver="gmres", n_outer=20000, stop_rule="true", rtol=1e-10)),
        ("fgmres", rsg.PREC_LEARNED, RL.learned_conf(model, rsg.make_conf(solver="gmres", n_outer=20000,
                                                                           stop_rule="true", rtol=1e-10))),
    ]:
        x, st = ctx.solve(M, b, conf=conf, prec=prec)
        assert st.converged == 1 and O.true_relres(A, b, x) <= 1e-10 * 1.01, name
        its[name] = st.iterations
    assert its["fcg"] <= 0.6 * its["pcg"], its
    assert its["fgmres"] <= 0.4 * its["gmres"], its
    model.close()
    for asm, _ in keep:
        asm.close()


def test_committed_model_cuts_iterations(ctx):
    """The parameters shipped in rsg/models (trained by `bench.py --workload learned --train-seeds
    1000 --save-model ...` on the 60^3 heat family) load, and flexible CG with them needs fewer
    iterations than Jacobi-PCG on a held-out seed of the family at its own mesh size (2.7x fewer
    on eight held-out seeds when measured), at the same FP64 true residual."""
    path = os.path.join(os.path.dirname(RL.__file__), "models", "heat_family_60.npz")
    model = RL.Learned.load(ctx, path)
    assert model.layers == 6 and model.step > 0
    base = W.heat_cube(60, sigma=1.0, seed=0, source="random")
    p = W.reseed_heat(base, sigma=RL.family_sigma(7), seed=7)
    A, b = O.assemble_heat(p)
    M = ctx.matrix(A.rp, A.ci, A.val)
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10)
    x_l, st_l = ctx.solve(M, b, conf=RL.learned_conf(model, conf), prec=rsg.PREC_LEARNED)
    x_j, st_j = ctx.solve(M, b, conf=conf, prec=rsg.PREC_JACOBI)
    assert st_l.converged == 1 and O.true_relres(A, b, x_l) <= 1e-10 * 1.01
    assert st_j.converged == 1
    assert st_l.iterations * 2 < st_j.iterations, (st_l.iterations, st_j.iterations)
    model.close()
