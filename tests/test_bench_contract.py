"""The JSON line of bench.py's reference arm (CPU only): one line, the keys the benchmark contract
requires, and a CPU baseline that describes the same run.  Runs on a 10^3 system so that it takes a
second."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    env = dict(os.environ, RSG_BENCH_N="10")
    out = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "3"], capture_output=True, text=True, env=env, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3 and d["higher_is_better"] is False
    assert d["value"] > 0 and d["unit"] == "s" and abs(d["ms_per_step"] - 1e3 * d["value"]) < 1e-9
    from oracle import ref as R
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == ("reference" if R.available() else "port")
    assert d["e2e"] == {"value": d["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "heat_lognormal_10" and d["config"]["true_relres"] <= 1e-10


def test_reference_arm_under_torchrun_prints_once():
    """Launched like the driver launches N > 1 (torchrun, one process per GPU): rank 0 alone runs the
    reference arm and prints its line; the other rank exits 0 without work."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, RSG_BENCH_N="8")
    out = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                          "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
                          "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3"],
                         capture_output=True, text=True, env=env, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.strip().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["config"]["workload"] == "heat_lognormal_8"
