"""The sharded batch path on a GPU: rsg.distributed.solve_sharded driving rsg.Batch through
gpu_batch_solver (one rank, gloo process group), every system checked against the oracle.

The multi-rank host logic (partition, gather) is covered on the CPU by tests/test_distributed.py;
this test runs the same call with the real GPU batch solver as the local solver."""
import os
import socket

import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import distributed as D
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_sharded_with_gpu_batch_solver(ctx, precision):
    import torch.distributed as dist
    specs = [(3, 1.0, 1), (9, 1.0, 2), (5, 0.5, 3), (14, 1.5, 4), (2, 1.0, 5), (11, 1.0, 6), (20, 1.0, 7)]
    sys_ = [O.assemble_heat(W.heat_cube(n, sigma=s, seed=seed, source="random")) for n, s, seed in specs]
    systems = [(A.rp, A.ci, A.val) for A, _ in sys_]
    rhs = [b for _, b in sys_]
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10, precision=precision)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        x_all, s_all = D.solve_sharded(systems, rhs, 0, 1, D.gpu_batch_solver(ctx, conf))
    finally:
        dist.destroy_process_group()
    assert len(x_all) == len(specs)
    for (A, b), x, st in zip(sys_, x_all, s_all):
        assert st["converged"] == 1 and O.true_relres(A, b, x) <= 1e-10 * 1.01
        xr, _ = O.solve(A, b, prec=1, n_outer=200000, stop_rule="true", rtol=1e-12)
        assert rel_err(x, xr) <= 1e-8
