"""Benchmark: time-to-solve of the heterogeneous-heat system on B200.

Workload ("heat_lognormal_100"): unit cube, 100^3 hexes -> 6,000,000 linear
tets, 1,030,301 nodes (1,009,899 free DOFs), per-tet conductivity
lognormal(0, 1.5), per-node source U(0,1) averaged per tet, T=0 / T=1 on
x=0 / x=1; target FP64 true relative residual 1e-10.  Inputs are generated
from seeds (synthetic data of the stated shape; no dataset is involved).

One step = one solve of that system to 1e-10 with the library's fastest
solver -- mixed-precision CG with reliable updates, preconditioned either by
Jacobi or by the multilevel aggregation preconditioner (whose hierarchy is
rebuilt on the GPU inside every timed solve) -- matrix and right-hand side
resident in HBM, x zeroed in the step.  The plain FP64 Jacobi-PCG drop-in and
the other solver are timed the same way and reported beside it.  Steps are
timed with CUDA events on the library's stream, L2 is flushed (256 MB write)
between steps, and the max over ranks is taken.  With --gpus N each rank
solves its own replica (different seed): the path does not shard, so this is
weak scaling of independent replicas, no collective on the data path.

`--impl reference` times the reference's own CPU implementation -- its
RMatrixSolver::solve with CG + JACOBI compiled from its sources into oracle/_ref
(the oracle's restatement where that build is absent) -- on all host cores on
the same system, one full solve per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "range-solver-lib_b200"))
sys.path.insert(0, REPO)

METRIC = "time-to-solve (s) at FP64 rel. residual 1e-10: learned/mixed vs plain GPU PCG"
UNIT = "s"
N_HEX = int(os.environ.get("RSG_BENCH_N", "100"))
SIGMA = 1.5
RTOL = 1e-10
# DRAM bytes of one launch of the headline solver's dominant kernel on heat_lognormal_100, and where
# each figure comes from (an ncu capture; None where none was taken of the current kernel)
TRAFFIC = {"mixed_jacobi": 113.65e6, "mixed_amg": 120.06e6}
# trained parameters of the learned preconditioner (bench.py --workload learned --save-model ...)
LEARNED_MODEL = os.path.join(REPO, "range-solver-lib_b200", "rsg", "models", "heat_family_60.npz")
TRAFFIC_SOURCE = {
    "mixed_jacobi": ("ncu --set full capture of k_mx_dir on heat_lognormal_100, dram__bytes_read.sum + "
                     "dram__bytes_write.sum of one launch (profiles/k_mx_dir_heat_lognormal_100.md)"),
    "mixed_amg": ("ncu --set full capture of k_amg_fine (the cycle's last finest-level sweep) on "
                  "heat_lognormal_100, dram__bytes_read.sum + dram__bytes_write.sum of one launch "
                  "(profiles/k_amg_fine_heat_lognormal_100.md)")}


def evict_l2(buf):
    """Evicts L2 before a timed step by reading a buffer larger than it (256 MB against 126 MB).  A
    read leaves clean lines; writing the buffer would leave dirty ones whose write-back then runs
    during the timed step."""
    buf.max()


def load_peaks() -> tuple[float, str]:
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = [r.split(",") for r in getattr(self, "out", "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_problem(seed: int):
    from rsg import workloads as W
    return W.heat_cube(N_HEX, sigma=SIGMA, seed=seed, source="random")


def spmv_bytes(n: int, nnz: int, val_bytes: int, idx_bytes: int, vec_bytes: int) -> int:
    """Algorithmic bytes of the fused CG direction kernel: matrix values + column
    indexes + row pointer, gathered z and p_old read once, p_new and q written once."""
    return nnz * (val_bytes + idx_bytes) + 4 * (n + 1) + 4 * n * vec_bytes


def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch
    import rsg

    torch.cuda.set_device(local_rank)
    ctx = rsg.Context(local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # torch ops and the library share one stream
    ctx.set_stream(stream.cuda_stream)
    p = build_problem(seed=rank)
    asm = rsg.Assembly.heat(ctx, p)
    n = asm.n_free
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    A = asm.assemble(p, b)
    # assembly timing (numeric phase, plan already built): element fields resident on the
    # device (kernel + CSR refresh), and from host arrays (adds their pageable copies)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    dev_in = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k), np.float64)).cuda()
              for k in ("k_e", "q_e", "rhoc_e", "node_t")}
    torch.cuda.synchronize()
    asm_ms, asm_host_ms = [], []
    for _ in range(4):
        ev[0].record(stream)
        asm.assemble(p, b, inputs_on_device=dev_in)
        ev[1].record(stream)
        ev[1].synchronize()
        asm_ms.append(ev[0].elapsed_time(ev[1]))
        ev[0].record(stream)
        asm.assemble(p, b)
        ev[1].record(stream)
        ev[1].synchronize()
        asm_host_ms.append(ev[0].elapsed_time(ev[1]))

    # launch shapes of the CG loop picked by the library's autotuner (set-up, not timed)
    tune = ctx.autotune(A) if not args.no_autotune else ctx.tune_info(A)
    conf_mixed = rsg.make_conf(n_outer=50000, stop_rule="true", rtol=RTOL, precision="mixed",
                               reliable_delta=args.delta, use_graph=not args.host_loop)
    conf_fp64 = rsg.make_conf(n_outer=50000, stop_rule="true", rtol=RTOL, precision="fp64",
                              use_graph=not args.host_loop)
    conf_amg = rsg.make_conf(n_outer=50000, stop_rule="true", rtol=RTOL, precision="mixed",
                             reliable_delta=args.delta, use_graph=not args.host_loop, amg_sweeps=args.amg_sweeps)
    # the solvers timed: the plain FP64 Jacobi-PCG drop-in, mixed-precision Jacobi-PCG, and mixed-precision
    # CG with the multilevel aggregation preconditioner (its hierarchy rebuilt inside every timed solve)
    solvers = {"fp64_jacobi": (conf_fp64, rsg.PREC_JACOBI), "mixed_jacobi": (conf_mixed, rsg.PREC_JACOBI),
               "mixed_amg": (conf_amg, rsg.PREC_AMG)}

    def step(key):
        conf, prec = solvers[key]
        evict_l2(flush)  # evict L2 between steps (not timed)
        x.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, st = ctx.solve(A, b, x, conf=conf, prec=prec)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, st

    for _ in range(args.warmup):
        step("mixed_amg")
        step("mixed_jacobi")
    step("fp64_jacobi")

    def timed(key, k):
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        tot, stats = 0.0, None
        for _ in range(k):
            t, stats = step(key)
            tot += t
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            tt = torch.tensor([tot], dtype=torch.float64, device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            tot = float(tt.item())
        return tot / k, stats

    sampler = ClockSampler(local_rank)
    times, stats = {}, {}
    with sampler:  # clocks over every timed region
        for key in ("mixed_amg", "mixed_jacobi", "fp64_jacobi"):
            times[key], stats[key] = timed(key, args.steps)
    best = min(("mixed_amg", "mixed_jacobi"), key=lambda k: times[k])

    # accuracy of each solution against the FP64 Jacobi-PCG one (all at 1e-10)
    xs_host = {}
    for key in solvers:
        conf, prec = solvers[key]
        _, stats[key] = ctx.solve(A, b, x.zero_(), conf=conf, prec=prec)
        xs_host[key] = x.cpu().numpy()
    x64 = xs_host["fp64_jacobi"]
    err_vs_fp64 = {k: float(np.linalg.norm(v - x64) / np.linalg.norm(x64)) for k, v in xs_host.items()}

    # the learned preconditioner on the same system: flexible CG in FP64 with the trained network as
    # M (Jacobi fallback), parameters from the committed checkpoint; two solves, L2 flushed, the
    # faster one reported (not part of the headline choice, which is between the timed solvers)
    learned = None
    if args.learned_model and os.path.exists(args.learned_model):
        from rsg import learned as RL
        model = RL.Learned.load(ctx, args.learned_model)
        conf_l = RL.learned_conf(model, rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL))
        tl = []
        for _ in range(2):
            evict_l2(flush)
            x.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, st_l = ctx.solve(A, b, x, conf=conf_l, prec=rsg.PREC_LEARNED)
            e1.record(stream)
            e1.synchronize()
            tl.append(e0.elapsed_time(e1) / 1e3)
        xs_host["learned_fcg"] = x.cpu().numpy()
        learned = {"s": min(tl), "iterations": st_l.iterations, "true_relres": st_l.true_relres,
                   "fallbacks": st_l.fallbacks,
                   "err_vs_fp64_solution": float(np.linalg.norm(xs_host["learned_fcg"] - x64) / np.linalg.norm(x64)),
                   "speedup_vs_plain_fp64": times["fp64_jacobi"] / min(tl),
                   "solver": "flexible CG (FP64) with the learned message-passing preconditioner applied every "
                             "iteration, Jacobi fallback",
                   "model": os.path.relpath(args.learned_model, REPO), "model_train_steps": model.step}
        model.close()
    amg_info = ctx.amg_setup(A)

    # dominant kernels, timed live (HBM-bound: L2 flushed before each launch)
    kd = {}
    for name, kid in (("cg_dir_fp64", 0), ("cg_dir_mixed", 1), ("cg_update_fp64", 2),
                      ("cg_update_mixed", 3), ("spmv_fp64", 4), ("spmv_fp32", 5), ("amg_sweep_fine", 6)):
        kd[name] = {"cold_s": ctx.profile_kernel(A, kid, reps=10, flush_l2=True),
                    "warm_s": ctx.profile_kernel(A, kid, reps=20, flush_l2=False)}
    nnz = A.nnz
    peak, peak_kind = load_peaks()
    by64 = spmv_bytes(n, nnz, 8, 2, 8)
    by32 = spmv_bytes(n, nnz, 4, 2, 4)
    # finest-level V-cycle smoothing sweep: FP32 values + 16-bit offsets, row pointers, the iterate
    # (gathered once), r and dw read once, the smoothed iterate written once
    by_amg = nnz * 6 + 4 * (n + 1) + 4 * n * 4
    achieved64 = by64 / kd["cg_dir_fp64"]["cold_s"] / 1e9
    achieved32 = by32 / kd["cg_dir_mixed"]["cold_s"] / 1e9
    achieved_amg = by_amg / kd["amg_sweep_fine"]["cold_s"] / 1e9
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the dominant kernel on
    # this workload: not measurable inside this run (ncu replays kernels), so it is the figure of the
    # ncu capture named in TRAFFIC_SOURCE, taken of the same kernel on the same workload
    traffic = TRAFFIC.get(best) if N_HEX == 100 else None

    # launches per solve: setup (norm, 2 scalings, Jacobi, FP32 copy, init residual + z, fold,
    # unscale, true residual) + per 2-iteration graph body (3 kernels per iteration + tail); the
    # multilevel preconditioner adds one cycle per application (once at the start and once per
    # iteration) and its set-up, both as counted by the library (rsg_amg_info)
    def launches(key):
        st = stats[key]
        bodies = (st.iterations + 1) // 2
        base = 10 + bodies * 7 + (0 if key == "fp64_jacobi" else 1)
        if key != "mixed_amg":
            return base
        per_cycle = amg_info["cycle_launches"][args.amg_sweeps - 1]
        return base + per_cycle * (st.iterations + 1) + amg_info["setup_launches"]

    # end to end through the reference-facing API with pinned host buffers
    rp_h, ci_h, val_h = A.to_host()
    val_pin = torch.from_numpy(val_h).pin_memory().numpy()
    b_pin = torch.empty(n, dtype=torch.float64).pin_memory()
    b_pin.copy_(b.cpu())
    b_pin = b_pin.numpy()
    x_pin = torch.zeros(n, dtype=torch.float64).pin_memory().numpy()
    e2e = []
    for i in range(max(2, min(args.steps, 5))):
        x_pin[:] = 0.0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        A.update_values(val_pin)  # the reference re-reads A's values on every solve (src/rmatrixsolver.cpp:56-97)
        xs, st_e = ctx.solve(A, b_pin, x_pin, conf=solvers[best][0], prec=solvers[best][1], inplace=True)
        t1 = time.perf_counter()
        if i > 0:
            e2e.append(t1 - t0)
    e2e_s = float(np.mean(e2e))

    out = {
        "times": times, "stats": stats, "best": best, "err_vs_fp64": err_vs_fp64, "kd": kd,
        "achieved64": achieved64, "achieved32": achieved32, "achieved_amg": achieved_amg, "peak": peak,
        "peak_kind": peak_kind, "by64": by64, "by32": by32, "by_amg": by_amg,
        "by_spmv64": nnz * 10 + 4 * (n + 1) + 2 * n * 8, "traffic": traffic, "n": n, "nnz": nnz,
        "asm_ms": float(np.median(asm_ms[1:])), "asm_host_ms": float(np.median(asm_host_ms[1:])),
        "clocks": sampler.summary(), "e2e_s": e2e_s, "tune": tune, "amg_info": amg_info,
        "h2d": int(nnz * 8 + 2 * n * 8), "d2h": int(n * 8), "launches": launches(best), "learned": learned,
        "ctx": ctx, "A": A, "b": b, "rp": rp_h, "ci": ci_h, "val": val_h, "xs": xs_host, "problem": p,
    }
    return out


class ReferenceCG:
    """The reference's own RMatrixSolver::solve (CG + JACOBI), compiled from its sources into
    oracle/_ref when they were present at build time, else the oracle's restatement of it.

    The reference stops on its own error ||r|| / (||A||_F ||x|| + ||b||) < cvg
    (src/rmatrixsolver.cpp:335-345); the metric is the FP64 true relative residual 1e-10.  So the
    iteration count is fixed (cvg 0) to the count at which the oracle's Jacobi-PCG first reaches
    1e-10, raised by 2% until the reference's own solution, checked by the oracle, reaches it too."""

    def __init__(self, A, b, threads: int):
        from oracle import oracle as O
        from oracle import ref as R
        self.O, self.A, self.b, self.threads = O, A, b, threads
        self.kind = "reference" if R.available() else "port"
        _, st = O.solve(A, b, prec=1, n_outer=50000, stop_rule="true", rtol=RTOL, threads=threads)
        self.iterations = int(st.iterations)
        self.M = R.RefMatrix(A.rp, A.ci, A.val) if self.kind == "reference" else None
        if self.M is not None:
            for _ in range(8):
                x, _ = self.M.solve(b, prec=1, n_outer=self.iterations, cvg=0.0, threads=threads)
                if O.true_relres(A, b, x) <= RTOL:
                    break
                self.iterations = int(self.iterations * 1.02) + 1

    def solve(self):
        """One timed solve: (seconds, iterations, FP64 true relative residual, x)."""
        if self.M is not None:
            x, res = self.M.solve(self.b, prec=1, n_outer=self.iterations, cvg=0.0, threads=self.threads)
            return res.seconds, int(res.iterations), self.O.true_relres(self.A, self.b, x), x
        x, st = self.O.solve(self.A, self.b, prec=1, n_outer=50000, stop_rule="true", rtol=RTOL, threads=self.threads)
        return st.seconds, int(st.iterations), st.true_relres, x

    def describe(self) -> str:
        if self.kind == "reference":
            return ("the reference's RMatrixSolver::solve (CG + JACOBI; src/rmatrixsolver.cpp, "
                    "src/rmatrixpreconditioner.cpp, src/riterationinfo.cpp compiled unchanged, OpenMP), "
                    f"{self.iterations} iterations (the count that reaches FP64 true relative residual 1e-10), "
                    "Jacobi build and CSR-cache refresh included")
        return "the oracle's OpenMP restatement of RMatrixSolver::solveCG + Jacobi, to FP64 true relative residual 1e-10"


def cpu_baseline(rp, ci, val, b, threads: int) -> dict:
    from oracle import oracle as O
    ref = ReferenceCG(O.CSR(len(rp) - 1, rp, ci, val), b, threads)
    ref.solve()  # the reference's first call builds its CSR cache
    t, its, relres, _ = ref.solve()
    return {"value": t, "iterations": its, "relres": relres, "kind": ref.kind, "sample": ref.describe()}


def oracle_check(r: dict, threads: int) -> dict:
    """Parity of the timed GPU results with the oracle (untimed): the oracle assembles the same
    problem on the host and solves it to a tight FP64 true residual (1e-12); the GPU matrix is
    compared entry by entry and both GPU solutions by ||x - x_ref|| / ||x_ref|| and by the true
    residual the oracle recomputes on its own system."""
    from oracle import oracle as O
    Ao, bo = O.assemble_heat(r["problem"])
    same_pattern = bool(np.array_equal(Ao.rp, r["rp"]) and np.array_equal(Ao.ci, r["ci"]))
    rowmax = np.maximum.reduceat(np.abs(Ao.val), Ao.rp[:-1].astype(np.int64))
    scale = np.repeat(rowmax, np.diff(Ao.rp.astype(np.int64)))
    entry_err = float(np.max(np.abs(r["val"] - Ao.val) / np.maximum(np.abs(Ao.val), scale))) if same_pattern else None
    rhs_err = float(np.max(np.abs(r["b"].cpu().numpy() - bo)) / np.max(np.abs(bo)))
    x_ref, st = O.solve(Ao, bo, prec=1, n_outer=50000, stop_rule="true", rtol=1e-12, threads=threads)
    nref = np.linalg.norm(x_ref)
    out = {"assembly_same_pattern": same_pattern, "assembly_max_rel_entry_err": entry_err,
           "rhs_max_rel_err": rhs_err, "oracle_tight_relres": st.true_relres}
    for key, xv in r["xs"].items():
        out[f"err_vs_oracle_{key}"] = float(np.linalg.norm(xv - x_ref) / nref)
        out[f"oracle_relres_{key}"] = O.true_relres(Ao, bo, xv)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--delta", type=float, default=1e-3)
    ap.add_argument("--batch-mode", default="shard", choices=["shard", "replicas"],
                    help="batch256: shard one batch of 256 systems across the ranks (default), or solve 256 "
                         "systems on every rank")
    ap.add_argument("--amg-sweeps", type=int, default=1, choices=[1, 2],
                    help="damped-Jacobi sweeps per side of the multilevel preconditioner's cycle (1: fewer "
                         "launches per iteration, measured faster than 2 at 100^3)")
    ap.add_argument("--learned-model", default=LEARNED_MODEL,
                    help="heat100: trained learned-preconditioner parameters (.npz) for the learned FCG row; "
                         "'' skips it")
    ap.add_argument("--save-model", default="", help="learned: write the trained parameters (.npz) here")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="heat100, batch256: keep the built-in launch shapes")
    ap.add_argument("--batch-systems", type=int, default=256,
                    help="batch256: solve the first K systems of the draw (a smaller case for profiling)")
    ap.add_argument("--batch-precisions", default="fp64,mixed",
                    help="batch256: the precisions to time (comma-separated; the fastest gives the value)")
    ap.add_argument("--workload", default="heat100",
                    choices=["heat100", "stress", "batch256", "transient40", "learned", "gmres100", "multi100",
                             "magneto64"],
                    help="heat100 (default, the headline); stress: 64x32x32 elasticity beam; batch256: 256 "
                         "independent heat cubes with 8..60 hexes per side; transient40: 64 backward-Euler steps "
                         "on a 40^3 mesh; learned: train the learned preconditioner on the GPU on seeded "
                         "60^3 lognormal heat problems, evaluate on held-out seeds and on the 100^3 system; "
                         "gmres100: restarted GMRES(30) + Jacobi on the 100^3 system, FP64 and mixed; "
                         "multi100: k = 4, 8, 16 right-hand sides of the 100^3 matrix against single solves; "
                         "magneto64: magnetostatic assembly + Jacobi-PCG on a 64^3 coil problem")
    ap.add_argument("--train-seeds", type=int, default=100, help="learned: training problems (seeds)")
    ap.add_argument("--eval-seeds", type=int, default=8, help="learned: held-out evaluation seeds")
    ap.add_argument("--learned-hex", type=int, default=60, help="learned: hexes per side of the family mesh")
    ap.add_argument("--no-headline-eval", action="store_true",
                    help="learned: skip the evaluation on the 100^3 system (small profiling runs)")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the CG loop from the host (same kernels, launched one by one) so that "
                         "profilers which cannot see kernels inside conditional CUDA graphs list them")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1

    if args.workload != "heat100":
        return run_other(args, rank, world, local_rank, threads)

    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as O
        p = build_problem(seed=0)
        t0 = time.perf_counter()
        Ah, bh = O.assemble_heat(p)
        t_asm = time.perf_counter() - t0
        ref = ReferenceCG(Ah, bh, threads)
        times = []
        its = relres = None
        for i in range(args.warmup + args.steps):
            t, its, relres, _ = ref.solve()
            if i >= args.warmup:
                times.append(t)
        v = float(np.mean(times))
        print(json.dumps({
            "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"heat_lognormal_{N_HEX}", "n_free": Ah.n, "nnz": Ah.nnz, "sigma": SIGMA,
                       "rtol": RTOL, "solver": "Jacobi-PCG FP64 (" + ref.describe() + ")",
                       "iterations": its, "true_relres": relres, "oracle_assembly_s_serial": t_asm},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": ref.kind,
                             "sample": f"one full Jacobi-PCG solve of the {N_HEX}^3 system per step: " + ref.describe()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    r = run_ours(args, rank, world, local_rank)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
        return

    cpu = None
    parity = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(r["rp"], r["ci"], r["val"], r["b"].cpu().numpy(), threads)
        parity = oracle_check(r, threads)
    kd = r["kd"]
    best, times, stats = r["best"], r["times"], r["stats"]
    st_b, st_f = stats[best], stats["fp64_jacobi"]
    names = {"mixed_amg": "mixed-precision CG (FP32 inner, FP64 reliable updates) with the multilevel aggregation "
                          "preconditioner (FP32 V-cycle, hierarchy rebuilt on the GPU in every solve)",
             "mixed_jacobi": "mixed-precision Jacobi-PCG (FP32 inner, FP64 reliable updates)",
             "fp64_jacobi": "plain FP64 Jacobi-PCG (the drop-in)"}
    per_solver = {k: {"s": times[k], "iterations": stats[k].iterations, "residual_refreshes": stats[k].outer,
                      "true_relres": stats[k].true_relres, "setup_s": stats[k].seconds_setup,
                      "loop_s": stats[k].seconds_solve, "ms_per_iteration": times[k] / max(stats[k].iterations, 1) * 1e3,
                      "err_vs_fp64_solution": r["err_vs_fp64"][k],
                      "err_vs_oracle": parity[f"err_vs_oracle_{k}"] if parity else None,
                      "speedup_vs_plain_fp64": times["fp64_jacobi"] / times[k], "solver": names[k]}
                  for k in times}
    if best == "mixed_amg":
        roof = {"bound": "hbm", "kernel": "k_amg_fine (finest-level V-cycle smoothing sweep, FP32 SELL-32)",
                "achieved": r["achieved_amg"], "algorithmic_bytes": r["by_amg"],
                "avg_launch_s": kd["amg_sweep_fine"]["cold_s"],
                "bytes": "nnz*(4+2) + 4*(n+1) + 4*n*4 (values, 16-bit offsets, row pointers, iterate, r, dw, "
                         "smoothed iterate)"}
    else:
        roof = {"bound": "hbm", "kernel": "k_mx_dir (fused FP32 CG direction + SpMV)", "achieved": r["achieved32"],
                "algorithmic_bytes": r["by32"], "avg_launch_s": kd["cg_dir_mixed"]["cold_s"]}
    roof.update({"peak": r["peak"], "unit": "GB/s", "frac": roof["achieved"] / r["peak"], "traffic": r["traffic"],
                 "traffic_source": TRAFFIC_SOURCE.get(best) if r["traffic"] is not None else None,
                 "peak_source": r["peak_kind"]})
    line = {
        "metric": METRIC, "value": times[best], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": times[best] * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32-inner/f64-outer", "data": "synthetic (seeded lognormal heat, 100^3 hexes)",
        "config": {"workload": f"heat_lognormal_{N_HEX}", "n_free": r["n"], "nnz": r["nnz"], "sigma": SIGMA,
                   "rtol": RTOL, "solver": names[best], "headline_solver": best,
                   "l2": "evicted between steps (a 256 MB buffer read)", "parallelism": f"replicas x{world}",
                   "iterations": st_b.iterations, "residual_refreshes": st_b.outer,
                   "true_relres": st_b.true_relres, "err_vs_fp64_solution": r["err_vs_fp64"][best],
                   "err_vs_oracle": parity[f"err_vs_oracle_{best}"] if parity else None,
                   "oracle_parity": parity,
                   "plain_fp64_pcg_s": times["fp64_jacobi"], "plain_fp64_iterations": st_f.iterations,
                   "plain_fp64_true_relres": st_f.true_relres,
                   "speedup_vs_plain_fp64": times["fp64_jacobi"] / times[best],
                   "target_3x_over_plain_fp64_met": times["fp64_jacobi"] / times[best] >= 3.0,
                   "solvers": per_solver, "amg_hierarchy": r["amg_info"], "amg_sweeps": args.amg_sweeps,
                   "learned_fcg": (dict(r["learned"], err_vs_oracle=parity.get("err_vs_oracle_learned_fcg")
                                        if parity else None) if r["learned"] else None),
                   "assembly_numeric_s": r["asm_ms"] / 1e3,
                   "assembly_numeric_from_host_arrays_s": r["asm_host_ms"] / 1e3,
                   "autotune": r["tune"]},
        "roofline": roof,
        "roofline_mixed_jacobi": {"bound": "hbm", "kernel": "k_mx_dir (fused FP32 CG direction + SpMV)",
                                  "achieved": r["achieved32"], "peak": r["peak"], "unit": "GB/s",
                                  "frac": r["achieved32"] / r["peak"], "algorithmic_bytes": r["by32"],
                                  "avg_launch_s": kd["cg_dir_mixed"]["cold_s"], "peak_source": r["peak_kind"]},
        "roofline_fp64": {"bound": "hbm", "kernel": "k_cg_dir (fused FP64 CG direction + SpMV)",
                          "achieved": r["achieved64"], "peak": r["peak"], "unit": "GB/s",
                          "frac": r["achieved64"] / r["peak"], "algorithmic_bytes": r["by64"],
                          "avg_launch_s": kd["cg_dir_fp64"]["cold_s"], "peak_source": r["peak_kind"]},
        "roofline_spmv_fp64": {"bound": "hbm", "kernel": "k_spmv (FP64 SpMV alone, rsg_spmv)",
                               "achieved": r["by_spmv64"] / kd["spmv_fp64"]["cold_s"] / 1e9, "peak": r["peak"],
                               "unit": "GB/s", "frac": r["by_spmv64"] / kd["spmv_fp64"]["cold_s"] / 1e9 / r["peak"],
                               "algorithmic_bytes": r["by_spmv64"], "avg_launch_s": kd["spmv_fp64"]["cold_s"],
                               "peak_source": r["peak_kind"],
                               "bytes": "nnz*(8+2) + 4*(n+1) + 2*n*8 (values, 16-bit offsets, row pointers, x, y)"},
        "kernels": kd,
        "e2e": {"value": r["e2e_s"], "unit": UNIT, "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"],
                "api": "rsg_csr_update_values + rsg_solve with pinned host buffers (headline solver)"},
        "gpu_launches": r["launches"] * args.steps,
        "clocks": r["clocks"],
    }
    if cpu:
        line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": threads, "kind": cpu["kind"],
                                "sample": "one full FP64 Jacobi-PCG solve of the same system: " + cpu["sample"],
                                "iterations": cpu["iterations"], "true_relres": cpu["relres"]}
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def _events_time(fn, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, out


def run_other(args, rank, world, local_rank, threads):
    """Secondary workloads (one JSON line each); the driver's default is heat100."""
    import torch
    import rsg
    from rsg import workloads as W
    from oracle import oracle as O
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=900))
    torch.cuda.set_device(local_rank)
    ctx = rsg.Context(local_rank)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    line = {"n_gpus": world, "steps": args.steps, "warmup": args.warmup, "vs_baseline": None, "data": "synthetic",
            "scaling": "weak"}

    def max_over_ranks(v):
        if world == 1:
            return v
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.workload in ("gmres100", "multi100"):
        p = build_problem(seed=rank)
        asm = rsg.Assembly.heat(ctx, p)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        x = torch.zeros_like(b)
        A = asm.assemble(p, b)

    if args.workload == "gmres100":
        res = {}
        for precision in ("fp64", "mixed"):
            conf = rsg.make_conf(solver="gmres", n_outer=100000, n_inner=30, stop_rule="true", rtol=RTOL,
                                 precision=precision)
            for _ in range(args.warmup):
                x.zero_()
                ctx.solve(A, b, x, conf=conf)
            tot = 0.0
            for _ in range(args.steps):
                evict_l2(flush)
                x.zero_()
                t, (_, st) = _events_time(lambda: ctx.solve(A, b, x, conf=conf), stream)
                tot += t
            res[precision] = {"s": max_over_ranks(tot / args.steps), "inner_iterations": st.iterations,
                              "restarts": st.outer, "true_relres": st.true_relres}
        best = min(res, key=lambda k: res[k]["s"])
        line.update({"metric": f"time-to-solve (s) at FP64 rel. residual 1e-10, GMRES(30) + Jacobi, {N_HEX}^3 heat",
                     "value": res[best]["s"], "unit": "s", "ms_per_step": res[best]["s"] * 1e3,
                     "higher_is_better": False, "dtype": "f64 / f32-Arnoldi",
                     "config": {"workload": f"gmres30_heat_lognormal_{N_HEX}", "n_free": A.n, "nnz": A.nnz,
                                "best": best, "variants": res}})
        if world == 1 and not args.no_cpu_baseline:
            rp, ci, val = A.to_host()
            cycles = 3
            xo, sto = O.solve(O.CSR(A.n, rp, ci, val), b.cpu().numpy(), prec=1, solver="gmres", n_outer=cycles,
                              n_inner=30, stop_rule="true", rtol=RTOL, threads=threads)
            per_inner = sto.seconds / max(sto.iterations, 1)
            line["cpu_baseline"] = {"value": per_inner * res["fp64"]["inner_iterations"], "unit": "s",
                                    "cores": threads, "kind": "port",
                                    "sample": f"{cycles} restart cycles ({sto.iterations} inner steps) of the "
                                              "oracle's FP64 GMRES(30), scaled to the GPU run's inner-step count"}

    elif args.workload == "multi100":
        conf = rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL)
        rng = np.random.default_rng(rank)
        res = {}
        for _ in range(args.warmup):
            x.zero_()
            ctx.solve(A, b, x, conf=conf)
        tot = 0.0
        for _ in range(args.steps):
            evict_l2(flush)
            x.zero_()
            t, (_, st) = _events_time(lambda: ctx.solve(A, b, x, conf=conf), stream)
            tot += t
        res["k1_single_solve"] = {"s_per_rhs": max_over_ranks(tot / args.steps), "iterations": st.iterations}
        for k in (4, 8, 16):
            B = torch.from_numpy(np.stack([b.cpu().numpy() * rng.uniform(0.5, 1.5, A.n) for _ in range(k)])).cuda()
            X = torch.zeros_like(B)
            for _ in range(args.warmup):
                X.zero_()
                ctx.solve_multi(A, B, X, conf=conf)
            tot = 0.0
            for _ in range(args.steps):
                evict_l2(flush)
                X.zero_()
                t, (_, per, summ) = _events_time(lambda: ctx.solve_multi(A, B, X, conf=conf), stream)
                tot += t
            res[f"k{k}"] = {"s_per_rhs": max_over_ranks(tot / args.steps) / k, "max_iterations": summ.iterations,
                            "worst_true_relres": max(q.true_relres for q in per)}
        best = min(res, key=lambda q: res[q]["s_per_rhs"])
        line.update({"metric": f"seconds per right-hand side at FP64 rel. residual 1e-10, FP64 Jacobi-PCG, "
                               f"{N_HEX}^3 heat matrix",
                     "value": res[best]["s_per_rhs"], "unit": "s", "ms_per_step": res[best]["s_per_rhs"] * 1e3,
                     "higher_is_better": False, "dtype": "f64",
                     "config": {"workload": f"multi_rhs_heat_lognormal_{N_HEX}", "n_free": A.n, "nnz": A.nnz,
                                "best": best, "variants": res}})

    elif args.workload == "magneto64":
        p = W.magnetostatic_cube(64, current="coil")
        asm = rsg.Assembly.magnetostatics(ctx, p)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        x = torch.zeros_like(b)
        dev_in = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k), np.float64)).cuda()
                  for k in ("node_j", "node_a")}
        A = asm.assemble(p, b, inputs_on_device=dev_in)
        asm_t = []
        for i in range(args.warmup + args.steps):
            evict_l2(flush)
            t, _ = _events_time(lambda: asm.assemble(p, b, inputs_on_device=dev_in), stream)
            if i >= args.warmup:
                asm_t.append(t)
        res = {}
        for precision in ("fp64", "mixed"):
            conf = rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL, precision=precision)
            for _ in range(args.warmup):
                x.zero_()
                ctx.solve(A, b, x, conf=conf)
            tot = 0.0
            for _ in range(args.steps):
                evict_l2(flush)
                x.zero_()
                t, (_, st) = _events_time(lambda: ctx.solve(A, b, x, conf=conf), stream)
                tot += t
            res[precision] = {"s": max_over_ranks(tot / args.steps), "iterations": st.iterations,
                              "true_relres": st.true_relres}
        best = min(res, key=lambda k: res[k]["s"])
        asm_s = max_over_ranks(float(np.median(asm_t)))
        line.update({"metric": "time-to-solve (s) at FP64 rel. residual 1e-10, 64^3 magnetostatic coil "
                               "(GPU assembly + Jacobi-PCG)",
                     "value": res[best]["s"] + asm_s, "unit": "s", "ms_per_step": (res[best]["s"] + asm_s) * 1e3,
                     "higher_is_better": False, "dtype": "f64 / f32-inner",
                     "config": {"workload": "magnetostatic_coil_64", "n_free": A.n, "nnz": A.nnz,
                                "assembly_numeric_s": asm_s, "best": best, "variants": res}})
        if world == 1 and not args.no_cpu_baseline:
            t0 = time.perf_counter()
            Ao, bo = O.assemble_magnetostatics(p)
            t_asm = time.perf_counter() - t0
            xo, sto = O.solve(Ao, bo, prec=1, n_outer=100000, stop_rule="true", rtol=RTOL, threads=threads)
            line["cpu_baseline"] = {"value": t_asm + sto.seconds, "unit": "s", "cores": threads, "kind": "port",
                                    "sample": "serial oracle assembly plus one FP64 Jacobi-PCG solve (OpenMP) "
                                              "of the same problem",
                                    "assembly_s": t_asm, "solve_s": sto.seconds, "iterations": sto.iterations}

    elif args.workload == "stress":
        p = W.stress_beam(64, 32, 32)
        asm = rsg.Assembly.stress(ctx, p)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        x = torch.zeros_like(b)
        A = asm.assemble(p, b)
        dev_in = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k), np.float64).reshape(-1)).cuda()
                  for k in ("e_mod", "nu", "rho_e", "gravity", "texp_e", "dtemp_e", "traction", "node_u")}
        asm_t = []
        for i in range(args.warmup + args.steps):
            evict_l2(flush)
            t, _ = _events_time(lambda: asm.assemble(p, b, inputs_on_device=dev_in), stream)
            if i >= args.warmup:
                asm_t.append(t)
        asm_s = max_over_ranks(float(np.median(asm_t)))
        res = {}
        for name, prec, blk, precision in (("jacobi_fp64", rsg.PREC_JACOBI, 1, "fp64"),
                                           ("jacobi_mixed", rsg.PREC_JACOBI, 1, "mixed"),
                                           ("block3_fp64", rsg.PREC_BLOCK_JACOBI, 3, "fp64"),
                                           ("block3_mixed", rsg.PREC_BLOCK_JACOBI, 3, "mixed")):
            conf = rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL, precision=precision)
            for _ in range(args.warmup):
                x.zero_()
                ctx.solve(A, b, x, conf=conf, prec=prec, block_size=blk)
            tot = 0.0
            for _ in range(args.steps):
                evict_l2(flush)
                x.zero_()
                t, (_, st) = _events_time(lambda: ctx.solve(A, b, x, conf=conf, prec=prec, block_size=blk), stream)
                tot += t
            res[name] = {"s": max_over_ranks(tot / args.steps), "iterations": st.iterations,
                         "true_relres": st.true_relres}
        best = min(res, key=lambda k: res[k]["s"])
        line.update({"metric": "time-to-solve (s) at FP64 rel. residual 1e-10, 64x32x32 elasticity beam",
                     "value": res[best]["s"], "unit": "s", "ms_per_step": res[best]["s"] * 1e3,
                     "higher_is_better": False, "dtype": "f64 / f32-inner",
                     "config": {"workload": "stress_beam_64x32x32", "n_free": A.n, "nnz": A.nnz, "best": best,
                                "assembly_numeric_s": asm_s, "variants": res}})
        if world == 1 and not args.no_cpu_baseline:
            rp, ci, val = A.to_host()
            xo, sto = O.solve(O.CSR(A.n, rp, ci, val), b.cpu().numpy(), prec=1, n_outer=100000, stop_rule="true",
                              rtol=RTOL, threads=threads)
            line["cpu_baseline"] = {"value": sto.seconds, "unit": "s", "cores": threads, "kind": "port",
                                    "sample": "one full FP64 Jacobi-PCG solve of the same system",
                                    "iterations": sto.iterations}
    elif args.workload == "batch256":
        from rsg import distributed as D
        # one batch of 256 independent heat systems (hexes per side drawn from 8..60, the same draw on
        # every rank); with --batch-mode shard the systems are partitioned across ranks by estimated
        # work (strong scaling: the same 256 systems whatever N), with replicas every rank solves its
        # own 256 (weak scaling)
        ns = max(1, min(256, args.batch_systems))
        sizes = np.random.default_rng(1000 + (rank if args.batch_mode == "replicas" else 0)).integers(8, 61, 256)[:ns]
        seeds = [(10000 * rank if args.batch_mode == "replicas" else 0) + i for i in range(ns)]
        costs = [D.estimated_cost(15 * (int(nh) + 1) ** 3, (int(nh) + 1) ** 3) for nh in sizes]
        mine = D.shard_systems(costs, world)[rank] if args.batch_mode == "shard" else list(range(ns))
        systems, rhs = [], []
        for i in mine:
            p = W.heat_cube(int(sizes[i]), sigma=1.0, seed=seeds[i], source="random")
            asm = rsg.Assembly.heat(ctx, p)
            bb = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
            A = asm.assemble(p, bb)
            systems.append(A.to_host())
            rhs.append(bb.cpu().numpy())
            asm.close()
        batch = rsg.Batch(ctx, systems)
        tune = batch.autotune() if not args.no_autotune else None  # launch shapes of the batch loop (set-up)
        b_all = torch.from_numpy(np.concatenate(rhs)).cuda()
        x_all = torch.zeros_like(b_all)
        res = {}
        worst = 0.0
        for precision in args.batch_precisions.split(","):
            conf = rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL, precision=precision,
                                 use_graph=not args.host_loop)
            for _ in range(args.warmup):
                x_all.zero_()
                batch.solve(b_all, x_all, conf=conf)
            if world > 1:
                dist.barrier()
            tot = 0.0
            for _ in range(args.steps):
                evict_l2(flush)
                x_all.zero_()
                t, (_, per, summ) = _events_time(lambda: batch.solve(b_all, x_all, conf=conf), stream)
                tot += t
            worst = max(worst, max(q.true_relres for q in per))
            res[precision] = {"s": max_over_ranks(tot / args.steps), "max_iterations_this_rank": summ.iterations,
                              "worst_true_relres_this_rank": summ.true_relres}
        # every system converged on every rank (one reduction, after the timed regions)
        worst_all = max_over_ranks(worst)
        t_best = min(r["s"] for r in res.values())
        total = ns * (world if args.batch_mode == "replicas" else 1)
        line.update({"metric": f"systems solved per second to FP64 rel. residual 1e-10 ({ns} uneven heat systems"
                               + (" per GPU)" if args.batch_mode == "replicas" else ", sharded across the GPUs)"),
                     "value": total / t_best, "unit": "systems/s", "ms_per_step": t_best * 1e3,
                     "higher_is_better": True, "dtype": "f64 / f32-inner",
                     "scaling": "weak" if args.batch_mode == "replicas" else "strong",
                     "config": {"workload": f"batch{ns}_heat_8to60", "rows_this_rank": batch.rows,
                                "nnz_this_rank": batch.nnz, "systems_this_rank": len(mine), "autotune": tune,
                                "worst_true_relres_all_ranks": worst_all,
                                "parallelism": (f"independent replicas x{world}" if args.batch_mode == "replicas"
                                                else f"{ns} systems sharded over {world} ranks by estimated work "
                                                     "(rsg.distributed.shard_systems), no collective in the solve"),
                                "variants": res}})
        if world == 1 and not args.no_cpu_baseline:
            t0 = time.perf_counter()
            for (rp, ci, val), bb in list(zip(systems, rhs))[:16]:
                O.solve(O.CSR(len(rp) - 1, rp, ci, val), bb, prec=1, n_outer=100000, stop_rule="true", rtol=RTOL,
                        threads=threads)
            t16 = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": 16 / t16, "unit": "systems/s", "cores": threads, "kind": "port",
                                    "sample": "the first 16 systems of the batch, solved one after another"}
    elif args.workload == "learned":
        from rsg import learned as RL
        model = RL.Learned(ctx, layers=6, seed=1 + rank)
        base = W.heat_cube(args.learned_hex, sigma=1.0, seed=0, source="random")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        losses = RL.train_heat_family(ctx, model, args.learned_hex, range(100000, 100000 + args.train_seeds),
                                      base=base)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - t0
        if args.save_model:
            os.makedirs(os.path.dirname(os.path.abspath(args.save_model)), exist_ok=True)
            model.save(args.save_model, with_adam=False)
        methods = ("pcg", "fcg", "gmres", "fgmres", "pcg_x0")
        ev = RL.evaluate_heat_family(ctx, model, args.learned_hex, range(args.eval_seeds), rtol=RTOL, base=base,
                                     methods=methods)

        def mean(meth, key):
            return float(np.mean([row[meth][key] for row in ev]))
        summary = {m: {"iterations": mean(m, "iterations"), "seconds": mean(m, "seconds"),
                       "worst_true_relres": max(row[m]["true_relres"] for row in ev),
                       "fallbacks": int(sum(row[m]["fallbacks"] for row in ev)),
                       "converged": int(sum(row[m]["converged"] for row in ev))} for m in methods}
        # the 100^3 headline system with the same model
        p100 = W.heat_cube(N_HEX if not args.no_headline_eval else args.learned_hex, sigma=SIGMA, seed=0,
                           source="random")
        asm = rsg.Assembly.heat(ctx, p100)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        x = torch.zeros_like(b)
        A = asm.assemble(p100, b)
        big = {}
        for name, prec, conf in (
                ("pcg", rsg.PREC_JACOBI, rsg.make_conf(n_outer=100000, stop_rule="true", rtol=RTOL)),
                ("fcg", rsg.PREC_LEARNED, RL.learned_conf(model, rsg.make_conf(n_outer=100000, stop_rule="true",
                                                                                rtol=RTOL))),
                ("gmres", rsg.PREC_JACOBI, rsg.make_conf(solver="gmres", n_outer=100000, n_inner=30,
                                                         stop_rule="true", rtol=RTOL)),
                ("fgmres", rsg.PREC_LEARNED, RL.learned_conf(model, rsg.make_conf(
                    solver="gmres", n_outer=100000, n_inner=30, stop_rule="true", rtol=RTOL)))):
            x.zero_()
            torch.cuda.synchronize()
            _, st = ctx.solve(A, b, x, conf=conf, prec=prec)
            big[name] = {"iterations": st.iterations, "seconds": st.seconds_solve, "true_relres": st.true_relres,
                         "fallbacks": st.fallbacks}
        r_apply = b.clone()
        z = torch.empty_like(b)
        model.apply(A, r_apply, z)
        ctx.sync()
        t_apply, _ = _events_time(lambda: [model.apply(A, r_apply, z) for _ in range(10)], stream)
        asm.close()
        line.update({
            "metric": f"time-to-solve (s) at FP64 rel. residual 1e-10, learned-preconditioned FCG(16), "
                      f"held-out {args.learned_hex}^3 lognormal heat seeds",
            "value": max_over_ranks(summary["fcg"]["seconds"]), "unit": "s",
            "ms_per_step": summary["fcg"]["seconds"] * 1e3, "higher_is_better": False,
            "dtype": "f64 Krylov / bf16 network (fp32 accumulate)",
            "config": {"workload": f"learned_heat_{args.learned_hex}", "train_seeds": args.train_seeds,
                       "train_steps": len(losses), "train_seconds": t_train,
                       "train_loss_first100": float(np.mean(losses[:100])),
                       "train_loss_last100": float(np.mean(losses[-100:])),
                       "eval_seeds": args.eval_seeds, "summary": summary,
                       "iteration_ratio_pcg_over_fcg": summary["pcg"]["iterations"] / summary["fcg"]["iterations"],
                       "iteration_ratio_gmres_over_fgmres":
                           summary["gmres"]["iterations"] / summary["fgmres"]["iterations"],
                       "time_ratio_fcg_over_pcg": summary["fcg"]["seconds"] / summary["pcg"]["seconds"],
                       "time_ratio_fgmres_over_gmres": summary["fgmres"]["seconds"] / summary["gmres"]["seconds"],
                       f"heat_lognormal_{N_HEX}": big,
                       f"network_apply_s_{N_HEX}": t_apply / 10,
                       "network": "6 message-passing layers, 64 wide, BF16 tcgen05 MMA with FP32 accumulation"}})
    else:  # transient40
        p = W.heat_cube(40, sigma=1.0, seed=rank, source="random", transient=True, dt=1e-3)
        per_step = {}
        for precision in ("fp64", "mixed"):
            rsg.transient_heat(ctx, p, 4, precision=precision)  # warm-up: plan build and graph paths
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            steps = rsg.transient_heat(ctx, p, 64, precision=precision)
            per_step[precision] = (max_over_ranks((time.perf_counter() - t0) / 64), steps)
        t, steps = per_step["mixed"]
        T64 = per_step["fp64"][1][-1][0]
        err = float(np.linalg.norm(steps[-1][0] - T64) / np.linalg.norm(T64))
        line.update({"metric": "seconds per backward-Euler step (GPU re-assembly + solve to 1e-10), 40^3 heat",
                     "value": t, "unit": "s", "ms_per_step": t * 1e3, "higher_is_better": False, "dtype": "f32/f64",
                     "config": {"workload": "transient_heat_40_64steps", "steps": 64,
                                "solver": "mixed-precision Jacobi-PCG (FP32 inner, FP64 refreshes)",
                                "fp64_s_per_step": per_step["fp64"][0],
                                "err_final_T_vs_fp64": err,
                                "iterations_per_step": [int(st.iterations) for _, st in steps[:8]],
                                "note": "wall clock per step; includes the plan build, the field upload and the read-back of every step's T once at the end; assembly, solve and the solution scatter stay on the GPU"}})
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
