"""Learned preconditioner (rsg_learned): a message-passing network over the
matrix graph, trained on the GPU with the library's own forward, backward and
Adam kernels.

No counterpart in the reference, whose preconditioners are Jacobi and block
Jacobi (src/rmatrixpreconditioner.cpp:24-101).  The network is used as
`PREC_LEARNED` (flexible CG, or GMRES with a stored Z) with Jacobi as the
fallback, and as an initial guess (`learned_initial_guess`).

Training data are residuals of plain Jacobi-PCG trajectories on assembled heat
problems: r_k = b - A x_k after k iterations, for k spread over the trajectory,
plus random right-hand sides.  The loss is ||r - A M(r)||^2 / ||r||^2.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import OK, PREC_JACOBI, SolverConf

PARAMS, GRAD, ADAM_M, ADAM_V = 0, 1, 2, 3


def _ptr(a) -> C.c_void_p:
    if a is None:
        return C.c_void_p(0)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


class Learned:
    """A learned preconditioner model on one Context's device."""

    def __init__(self, ctx, layers: int = 6, seed: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_learned_create(ctx.h, layers, seed, C.byref(h)), "learned_create")
        self.h = h
        self._info()

    def _info(self):
        L, H, npar, step = C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint64()
        self.ctx.check(self.ctx.lib.rsg_learned_info(self.h, C.byref(L), C.byref(H), C.byref(npar), C.byref(step)),
                       "learned_info")
        self.layers, self.hidden, self.n_params, self.step = L.value, H.value, npar.value, step.value

    # ---- parameters ----
    def get(self, which: int = PARAMS) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self.ctx.check(self.ctx.lib.rsg_learned_get_params(self.ctx.h, self.h, _ptr(out), which), "learned_get")
        return out

    def set(self, values, which: int = PARAMS):
        v = np.ascontiguousarray(values, np.float32)
        if v.size != self.n_params:
            raise ValueError(f"expected {self.n_params} values, got {v.size}")
        self.ctx.check(self.ctx.lib.rsg_learned_set_params(self.ctx.h, self.h, _ptr(v), which), "learned_set")

    def save(self, path: str, with_adam: bool = True):
        """Parameters (and, with_adam, the Adam moments to resume training) as a compressed .npz."""
        self._info()
        extra = {"adam_m": self.get(ADAM_M), "adam_v": self.get(ADAM_V)} if with_adam else {}
        np.savez_compressed(path, layers=self.layers, hidden=self.hidden, step=self.step, params=self.get(PARAMS),
                            **extra)

    @classmethod
    def load(cls, ctx, path: str) -> "Learned":
        d = np.load(path)
        m = cls(ctx, int(d["layers"]))
        if int(d["hidden"]) != m.hidden:
            raise ValueError(f"checkpoint hidden width {int(d['hidden'])} != library width {m.hidden}")
        m.set(d["params"], PARAMS)
        if "adam_m" in d.files:  # inference-only checkpoints carry the parameters alone
            m.set(d["adam_m"], ADAM_M)
            m.set(d["adam_v"], ADAM_V)
        ctx.check(ctx.lib.rsg_learned_set_step(m.h, int(d["step"])), "learned_set_step")
        m._info()
        return m

    def save_binary(self, path: str):
        """Checkpoint in the library's RSGGNN01 format (rsg_learned_save)."""
        self.ctx.check(self.ctx.lib.rsg_learned_save(self.ctx.h, self.h, path.encode()), "learned_save")

    @classmethod
    def load_binary(cls, ctx, path: str) -> "Learned":
        h = C.c_void_p()
        ctx.check(ctx.lib.rsg_learned_load(ctx.h, path.encode(), C.byref(h)), "learned_load")
        m = cls.__new__(cls)
        m.ctx, m.h = ctx, h
        m._info()
        return m

    # ---- compute ----
    def apply(self, A, r_dev, z_dev, xyz_dev=None, tensor_cores: bool = True):
        """z = M(r) on the device (r, z: n doubles; xyz: 3n doubles or None)."""
        self.ctx.check(self.ctx.lib.rsg_learned_apply(self.ctx.h, self.h, A.h, _ptr(r_dev), _ptr(z_dev),
                                                      _ptr(xyz_dev), 1 if tensor_cores else 0), "learned_apply")

    def loss_grad(self, A, r_dev, xyz_dev=None, tensor_cores: bool = False):
        """(loss, gradient) of ||r - A M(r)||^2/||r||^2 without updating the parameters."""
        loss = C.c_double()
        self.ctx.check(self.ctx.lib.rsg_learned_loss_grad(self.ctx.h, self.h, A.h, _ptr(r_dev), _ptr(xyz_dev),
                                                          1 if tensor_cores else 0, C.byref(loss)),
                       "learned_loss_grad")
        return loss.value, self.get(GRAD)

    def train_step(self, A, r_dev, lr: float = 1e-3, xyz_dev=None) -> float:
        """One Adam step on one residual; returns the loss before the step."""
        loss = C.c_double()
        self.ctx.check(self.ctx.lib.rsg_learned_train_step(self.ctx.h, self.h, A.h, _ptr(r_dev), _ptr(xyz_dev),
                                                           C.c_float(lr), C.byref(loss)), "learned_train_step")
        self.step += 1
        return loss.value

    def close(self):
        if self.h and self.ctx.h:
            self.ctx.lib.rsg_learned_destroy(self.ctx.h, self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def trajectory_residuals(ctx, A, b_dev, checkpoints=(0, 1, 2, 4, 8, 16, 32, 64, 128, 256), n_random: int = 2,
                         seed: int = 0):
    """Residuals of a plain Jacobi-PCG run on A x = b (x0 = 0) after k iterations,
    k in checkpoints, plus those of n_random random right-hand sides.  Returns a
    list of device tensors (the residuals a preconditioner meets in a solve)."""
    import torch
    from . import make_conf
    dev = b_dev.device
    g = torch.Generator(device="cpu").manual_seed(seed)
    rhs = [b_dev] + [torch.randn(A.n, generator=g, dtype=torch.float64).to(dev) for _ in range(n_random)]
    out = []
    ax = torch.empty_like(b_dev)
    for b in rhs:
        for k in checkpoints:
            x = torch.zeros_like(b)
            if k > 0:
                conf = make_conf(n_outer=k, stop_rule="true", rtol=1e-14, use_graph=False)
                torch.cuda.synchronize()
                ctx.solve(A, b, x, conf=conf, prec=PREC_JACOBI)
                ctx.sync()
            ctx.spmv(A, x, ax)
            ctx.sync()
            r = b - ax
            if float(torch.linalg.vector_norm(r)) > 0.0:
                out.append(r)
    return out


def train(ctx, model: Learned, samples, steps: int, lr: float = 1e-3, seed: int = 0, lr_final: float | None = None,
          log_every: int = 0):
    """Adam over (matrix, residual[, xyz]) samples drawn uniformly at random.
    Cosine decay from lr to lr_final.  Returns the per-step losses."""
    rng = np.random.default_rng(seed)
    lr_final = lr * 0.1 if lr_final is None else lr_final
    losses = []
    for t in range(steps):
        A, r, xyz = samples[int(rng.integers(len(samples)))]
        cur = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * t / max(steps - 1, 1)))
        loss = model.train_step(A, r, float(cur), xyz)
        losses.append(loss)
        if log_every and (t % log_every == 0 or t == steps - 1):
            print(f"step {t:5d}  lr {cur:.2e}  loss {loss:.4f}", flush=True)
    return losses


def family_sigma(seed: int, lo: float = 0.5, hi: float = 2.0) -> float:
    """Per-seed conductivity spread sigma ~ U(lo, hi) of the learned-preconditioner heat family."""
    from . import workloads as W
    return float(lo + (hi - lo) * W.uniform(seed, 3, 1)[0])


def train_heat_family(ctx, model: Learned, n_hex: int, seeds, lr: float = 1e-3, lr_final: float = 1e-4,
                      checkpoints=(0, 1, 2, 4, 8, 16, 32, 64, 128, 256), n_random: int = 1, log_every: int = 0,
                      base=None):
    """Online training over seeded lognormal heat problems on one n_hex^3 mesh: for each seed
    the GPU assembles the system (one plan, new values), the plain Jacobi-PCG trajectory
    gives residuals, and each residual is one Adam step.  Returns per-step losses."""
    import torch
    from . import Assembly
    from . import workloads as W
    base = base or W.heat_cube(n_hex, sigma=1.0, seed=0, source="random")
    asm = Assembly.heat(ctx, base)
    b = torch.empty(asm.n_free, dtype=torch.float64, device=f"cuda:{ctx.device}")
    seeds = list(seeds)
    per = len(checkpoints) * (1 + n_random)
    total = max(len(seeds) * per, 1)
    rng = np.random.default_rng(12345)
    losses, t = [], 0
    for seed in seeds:
        p = W.reseed_heat(base, sigma=family_sigma(seed), seed=seed)
        A = asm.assemble(p, b)
        ctx.sync()
        rs = trajectory_residuals(ctx, A, b, checkpoints, n_random, seed)
        for i in rng.permutation(len(rs)):
            cur = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * min(t, total - 1) / max(total - 1, 1)))
            losses.append(model.train_step(A, rs[i], float(cur)))
            t += 1
        if log_every and (len(losses) // per) % log_every == 0:
            print(f"seed {seed}  steps {t}  loss {np.mean(losses[-per:]):.4f}", flush=True)
    asm.close()
    return losses


def evaluate_heat_family(ctx, model: Learned, n_hex: int, seeds, rtol: float = 1e-10, base=None,
                         methods=("pcg", "fcg", "gmres", "fgmres"), max_it: int = 100000):
    """Solve each held-out seed with plain Jacobi-PCG / GMRES(30) and their learned (flexible)
    counterparts; returns one dict per seed with iterations, device seconds, true residual."""
    import torch
    from . import Assembly, make_conf, PREC_LEARNED
    from . import workloads as W
    base = base or W.heat_cube(n_hex, sigma=1.0, seed=0, source="random")
    asm = Assembly.heat(ctx, base)
    b = torch.empty(asm.n_free, dtype=torch.float64, device=f"cuda:{ctx.device}")
    x = torch.zeros_like(b)
    confs = {
        "pcg": (PREC_JACOBI, make_conf(n_outer=max_it, stop_rule="true", rtol=rtol)),
        "fcg": (PREC_LEARNED, learned_conf(model, make_conf(n_outer=max_it, stop_rule="true", rtol=rtol))),
        "gmres": (PREC_JACOBI, make_conf(solver="gmres", n_outer=max_it, n_inner=30, stop_rule="true", rtol=rtol)),
        "fgmres": (PREC_LEARNED, learned_conf(model, make_conf(solver="gmres", n_outer=max_it, n_inner=30,
                                                               stop_rule="true", rtol=rtol))),
        "pcg_x0": (PREC_JACOBI, learned_conf(model, make_conf(n_outer=max_it, stop_rule="true", rtol=rtol),
                                             initial_guess=True)),
    }
    out = []
    for seed in seeds:
        p = W.reseed_heat(base, sigma=family_sigma(seed), seed=seed)
        A = asm.assemble(p, b)
        ctx.sync()
        row = {"seed": int(seed), "sigma": family_sigma(seed)}
        for name in methods:
            prec, conf = confs[name]
            x.zero_()
            torch.cuda.synchronize()
            _, st = ctx.solve(A, b, x, conf=conf, prec=prec)
            row[name] = {"iterations": int(st.iterations), "seconds": float(st.seconds_solve),
                         "true_relres": float(st.true_relres), "fallbacks": int(st.fallbacks),
                         "converged": int(st.converged)}
        out.append(row)
    asm.close()
    return out


def learned_conf(model: Learned, base: SolverConf | None = None, initial_guess: bool = False) -> SolverConf:
    """A copy of base (default: TRUE_RELRES CG) that points at model."""
    from . import make_conf
    c = make_conf(stop_rule="true") if base is None else SolverConf.from_buffer_copy(base)
    c.learned = model.h.value
    c.learned_initial_guess = 1 if initial_guess else 0
    return c


__all__ = ["Learned", "trajectory_residuals", "train", "learned_conf", "train_heat_family", "evaluate_heat_family",
           "family_sigma", "PARAMS", "GRAD", "ADAM_M", "ADAM_V", "OK"]
