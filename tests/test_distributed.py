"""Multi-process sharding of batched solves, on CPU with the gloo backend.

Each rank solves its shard with the oracle (standing in for the GPU batch
solver, which these CPU tests cannot run), and rank 0 gathers everything; the
same host logic drives rsg.Batch on GPUs.  Also checks the load balance of the
work-based partition."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from rsg import distributed as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_balance_and_coverage():
    rng = np.random.default_rng(0)
    sizes = rng.integers(8, 61, 256)
    costs = [D.estimated_cost(15 * (n + 1) ** 3, (n + 1) ** 3) for n in sizes]
    for world in (1, 2, 4, 8):
        shards = D.shard_systems(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) <= 1.05 * (sum(costs) / world) + max(costs)
        assert max(loads) / min(loads) < 1.1
    assert D.shard_systems(costs, 4) == D.shard_systems(costs, 4)  # deterministic


def _worker(rank, world, port, out_path):
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [repo, os.path.join(repo, "range-solver-lib_b200")]
    from oracle import oracle as O
    from rsg import workloads as W
    from rsg import distributed as D2
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    probs = [W.heat_cube(n, sigma=1.0, seed=s, source="random") for n, s in ((3, 1), (5, 2), (4, 3), (6, 4), (2, 5))]
    sys_ = [O.assemble_heat(p) for p in probs]
    systems = [(A.rp, A.ci, A.val) for A, _ in sys_]
    rhs = [b for _, b in sys_]

    def oracle_local(ss, bs):
        xs, sts = [], []
        for (rp, ci, val), b in zip(ss, bs):
            x, st = O.solve(O.CSR(len(rp) - 1, rp, ci, val), b, prec=1, n_outer=20000, stop_rule="true",
                            rtol=1e-10, threads=1)
            xs.append(x)
            sts.append({"iterations": st.iterations, "true_relres": st.true_relres, "rank": rank})
        return xs, sts

    x_all, s_all = D2.solve_sharded(systems, rhs, rank, world, oracle_local)
    if rank == 0:
        ok = all(O.true_relres(A, b, x) <= 1e-10 for (A, b), x in zip(sys_, x_all))
        ranks = sorted({s["rank"] for s in s_all})
        with open(out_path, "w") as f:
            f.write(f"{int(ok)} {len(x_all)} {','.join(map(str, ranks))}")
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_solve_gloo(tmp_path):
    out = str(tmp_path / "result.txt")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    ok, count, ranks = open(out).read().split()
    assert ok == "1" and int(count) == 5 and ranks == "0,1"
