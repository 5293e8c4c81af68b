"""GPU assembly (rsg_assembly_* / rsg_assemble_*) against the CPU oracle.

Bar: the sparsity pattern is identical; every assembled entry and RHS value
matches the oracle within 1e-13 relative (absolute floor 1e-13 of the row's
largest entry, for entries that cancel to rounding noise); repeated assemblies
are bitwise identical.
"""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W

pytestmark = pytest.mark.gpu


def device_csr(ctx, torch, M):
    rp, ci, val = M.to_host()
    return O.CSR(M.n, rp, ci, val)


def compare(Ag, bg, Ao, bo, rtol=1e-13):
    assert np.array_equal(Ag.rp, Ao.rp)
    assert np.array_equal(Ag.ci, Ao.ci)
    rowmax = np.maximum.reduceat(np.abs(Ao.val), Ao.rp[:-1].astype(np.int64))
    scale = np.repeat(rowmax, np.diff(Ao.rp.astype(np.int64)))
    diff = np.abs(Ag.val - Ao.val)
    assert np.all(diff <= rtol * np.abs(Ao.val) + 1e-13 * scale), diff.max()
    bscale = np.abs(bo).max() if bo.size else 1.0
    assert np.all(np.abs(bg - bo) <= rtol * np.abs(bo) + 1e-13 * bscale)


def run_heat(ctx, torch, p):
    asm = rsg.Assembly.heat(ctx, p)
    b = torch.empty(p.n_free, dtype=torch.float64, device="cuda")
    M = asm.assemble(p, b)
    ctx.sync()
    return asm, M, b


@pytest.mark.parametrize("transient,alpha", [(False, 1.0), (True, 1.0), (True, 0.5)])
def test_heat_assembly_matches_oracle(ctx, torch_cuda, transient, alpha):
    torch = torch_cuda
    p = W.heat_cube(7, sigma=1.5, seed=4, source="random", transient=transient, dt=1e-3)
    p.alpha = alpha
    if transient:
        p.node_t = W.uniform(4, 9, p.mesh.n_nodes)
        p.node_t[p.mesh.xyz[:, 0] == 1.0] = 1.0
        p.node_t[p.mesh.xyz[:, 0] == 0.0] = 0.0
    asm, M, b = run_heat(ctx, torch, p)
    Ao, bo = O.assemble_heat(p)
    assert asm.n_free == Ao.n and asm.nnz == Ao.nnz
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)
    assert M.frobenius == pytest.approx(O.frobenius(Ao), rel=1e-13)


def test_heat_assembly_deterministic_and_reassembly(ctx, torch_cuda):
    torch = torch_cuda
    p = W.heat_cube(9, sigma=1.0, seed=1, source="random")
    asm, M, b = run_heat(ctx, torch, p)
    v1 = device_csr(ctx, torch, M).val.copy()
    b1 = b.clone()
    asm.assemble(p, b)
    ctx.sync()
    assert np.array_equal(device_csr(ctx, torch, M).val, v1) and torch.equal(b, b1)
    p2 = W.heat_cube(9, sigma=1.0, seed=2, source="random")
    asm.assemble(p2, b)  # same pattern, new conductivities: written in place
    ctx.sync()
    Ao, bo = O.assemble_heat(p2)
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)


def test_heat_assembly_device_inputs(ctx, torch_cuda):
    torch = torch_cuda
    p = W.heat_cube(6, sigma=1.0, seed=3, source="random")
    asm = rsg.Assembly.heat(ctx, p)
    b = torch.empty(p.n_free, dtype=torch.float64, device="cuda")
    d = {k: torch.tensor(getattr(p, k), device="cuda") for k in ("k_e", "q_e", "rhoc_e", "node_t")}
    torch.cuda.synchronize()  # the library runs on its own stream
    M = asm.assemble(p, b, inputs_on_device=d)
    ctx.sync()
    Ao, bo = O.assemble_heat(p)
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)


@pytest.mark.parametrize("variant", ["plain", "body_loads", "transient"])
def test_stress_assembly_matches_oracle(ctx, torch_cuda, variant):
    torch = torch_cuda
    p = W.stress_beam(6, 3, 3)
    if variant == "body_loads":
        p.gravity = np.array([0.0, -9.81, 1.5])
        p.texp_e = np.full(p.mesh.n_tets, 1.2e-5)
        p.dtemp_e = W.uniform(3, 4, p.mesh.n_tets, -20.0, 40.0)
        p.e_mod = W.lognormal(5, 6, p.mesh.n_tets, np.log(210e9), 0.3)
    if variant == "transient":
        p.transient, p.alpha, p.dt = True, 1.0, 1e-4
        p.node_u = 1e-5 * W.normal(1, 2, 3 * p.mesh.n_nodes)
        p.node_u[p.disabled] = 0.0
    asm = rsg.Assembly.stress(ctx, p)
    b = torch.empty(p.n_free, dtype=torch.float64, device="cuda")
    M = asm.assemble(p, b)
    ctx.sync()
    Ao, bo = O.assemble_stress(p)
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)


def test_gpu_assembly_then_solve_patch_test(ctx, torch_cuda):
    torch = torch_cuda
    p = W.heat_cube(10, source="none")
    asm, M, b = run_heat(ctx, torch, p)
    x = torch.zeros_like(b)
    torch.cuda.synchronize()
    _, st = ctx.solve(M, b, x, conf=rsg.make_conf(n_outer=10000, stop_rule="true", rtol=1e-13))
    full = p.node_t.copy()
    free = p.book != W.EOD
    full[free] = x.cpu().numpy()[p.book[free]]
    assert np.abs(full - p.mesh.xyz[:, 0]).max() < 1e-10


def test_assembly_rejects_bad_inputs(ctx):
    p = W.heat_cube(3)
    bad = p.book.copy()
    free = np.nonzero(bad != W.EOD)[0]
    bad[free[0]], bad[free[1]] = bad[free[1]], bad[free[0]]  # not increasing
    p2 = W.heat_cube(3)
    p2.book = bad
    with pytest.raises(rsg.RsgError) as e:
        rsg.Assembly.heat(ctx, p2)
    assert e.value.status == rsg.ERR_INVALID_ARG
    p3 = W.heat_cube(3)
    p3.mesh.tets = p3.mesh.tets.copy()
    p3.mesh.tets[5, 2] = p3.mesh.n_nodes + 3
    with pytest.raises(rsg.RsgError):
        rsg.Assembly.heat(ctx, p3)


@pytest.mark.parametrize("kind", ["heat", "heat_transient", "stress", "stress_transient"])
def test_warp_and_thread_row_kernels_bitwise_equal(ctx, torch_cuda, monkeypatch, kind):
    """The warp-per-row kernels apply every element contribution to an entry in the
    same order as the one-thread-per-row kernels: identical bits."""
    torch = torch_cuda
    if kind.startswith("heat"):
        p = W.heat_cube(8, sigma=1.2, seed=6, source="random", transient=kind.endswith("transient"), dt=1e-3)
        if p.transient:
            p.node_t = W.uniform(6, 9, p.mesh.n_nodes)
    else:
        p = W.stress_beam(6, 4, 4)
        if kind.endswith("transient"):
            p.transient, p.dt, p.alpha = True, 1e-4, 0.5
            p.node_u = W.uniform(2, 3, 3 * p.mesh.n_nodes) * 1e-4
    out = []
    for forced in ("0", "1"):
        monkeypatch.setenv("RSG_ASM_ROW_THREADS", forced)
        asm = rsg.Assembly.heat(ctx, p) if kind.startswith("heat") else rsg.Assembly.stress(ctx, p)
        b = torch.empty(asm.n_free, dtype=torch.float64, device="cuda")
        M = asm.assemble(p, b)
        ctx.sync()
        out.append((M.to_host()[2], b.cpu().numpy()))
        asm.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_electrostatics_through_the_heat_plan(ctx, torch_cuda):
    """RSolverElectrostatics' volume integrals are the heat ones with k = eps_r e0 and
    source -rho: a parallel-plate capacitor (uniform eps_r, no charge) gives the exact
    linear potential, and a charged lognormal case matches the oracle assembly."""
    torch = torch_cuda
    p = W.electrostatic_cube(6, eps_r=4.0, v0=0.0, v1=10.0)
    asm, M, b = run_heat(ctx, torch, p)
    x, st = ctx.solve(M, b.cpu().numpy(), conf=rsg.make_conf(n_outer=10000, stop_rule="true", rtol=1e-13))
    free = p.book != 0xFFFFFFFF
    order = np.argsort(p.book[free])
    expect = 10.0 * p.mesh.xyz[free, 0][order]
    assert np.max(np.abs(x - expect)) < 1e-8
    asm.close()
    q = W.electrostatic_cube(7, eps_r=3.0, charge=2e-9, sigma=0.8, seed=5)
    asm, M, b = run_heat(ctx, torch, q)
    Ao, bo = O.assemble_heat(q)
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)
    asm.close()


def run_magneto(ctx, torch, p):
    asm = rsg.Assembly.magnetostatics(ctx, p)
    b = torch.empty(p.n_free, dtype=torch.float64, device="cuda")
    M = asm.assemble(p, b)
    ctx.sync()
    return asm, M, b


@pytest.mark.parametrize("current", ["coil", "random"])
def test_magnetostatics_matches_oracle(ctx, torch_cuda, current):
    # RSolverMagnetostatics::prepare + assemblyMatrix (src/rsolvermagnetostatics.cpp:44-145, :234-287)
    torch = torch_cuda
    p = W.magnetostatic_cube(7, current=current, seed=3, a1=(0.2, -0.1, 0.4))
    asm, M, b = run_magneto(ctx, torch, p)
    Ao, bo = O.assemble_magnetostatics(p)
    assert asm.n_free == Ao.n and asm.nnz == Ao.nnz
    Ag = device_csr(ctx, torch, M)
    compare(Ag, b.cpu().numpy(), Ao, bo)
    # entries coupling different components are exact zeros (rows and columns are 3 * position + component)
    rows = np.repeat(np.arange(Ag.n), np.diff(Ag.rp.astype(np.int64)))
    cross = rows % 3 != Ag.ci.astype(np.int64) % 3
    assert cross.sum() == 2 * (~cross).sum() and not Ag.val[cross].any()
    # the solve the reference runs on it (CG + Jacobi, :151-153); the matrix is negative definite
    conf = rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10)
    x, st = ctx.solve(M, b.cpu().numpy(), conf=conf, prec=rsg.PREC_JACOBI)
    assert st.true_relres <= 1e-10
    xo, _ = O.solve(Ao, bo, prec=1, n_outer=20000, stop_rule="true", rtol=1e-12)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8


def test_magnetostatics_thread_local_rows_match_global(ctx, torch_cuda, monkeypatch):
    torch = torch_cuda
    p = W.magnetostatic_cube(6, current="random", seed=5, a0=(0.1, 0.2, 0.3))
    _, M, b = run_magneto(ctx, torch, p)
    v_local, b_local = device_csr(ctx, torch, M).val.copy(), b.cpu().numpy()
    monkeypatch.setenv("RSG_ASM_ROW_THREADS", "1")
    _, M2, b2 = run_magneto(ctx, torch, p)
    assert np.array_equal(device_csr(ctx, torch, M2).val, v_local)
    assert np.array_equal(b2.cpu().numpy(), b_local)


def test_magnetostatics_patch_test_and_book_check(ctx, torch_cuda):
    torch = torch_cuda
    p = W.magnetostatic_cube(6, current="none", a1=(1.0, -2.0, 3.0))
    asm, M, b = run_magneto(ctx, torch, p)
    x, st = ctx.solve(M, b.cpu().numpy(), conf=rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-13),
                      prec=rsg.PREC_JACOBI)
    full = p.node_a.copy()
    free = p.book != W.EOD
    full[free] = x[p.book[free]]
    assert np.abs(full - np.outer(p.mesh.xyz[:, 0], [1.0, -2.0, 3.0]).reshape(-1)).max() < 1e-9
    # the solution back into the nodal field on the device
    xd = torch.tensor(x, device="cuda")
    nodal = torch.tensor(p.node_a, device="cuda")
    torch.cuda.synchronize()
    ctx.check(ctx.lib.rsg_assembly_scatter(ctx.h, asm.h, rsg._ptr(xd), rsg._ptr(nodal)), "assembly_scatter")
    ctx.sync()
    assert np.array_equal(nodal.cpu().numpy(), full)
    # one node book position per node: a node with one component disabled is rejected
    q = W.magnetostatic_cube(3, current="none")
    good = q.book.copy()
    bad = q.book.copy()
    inner = int(np.flatnonzero(~q.disabled)[0])
    bad[3 * inner + 1] = W.EOD
    with pytest.raises(rsg.RsgError):
        q.book = bad
        rsg.Assembly.magnetostatics(ctx, q)
    # and its three components sit at 3 * position + c
    swapped = good.copy()
    swapped[3 * inner], swapped[3 * inner + 1] = good[3 * inner + 1], good[3 * inner]
    with pytest.raises(rsg.RsgError):
        q.book = swapped
        rsg.Assembly.magnetostatics(ctx, q)


@pytest.mark.parametrize("forced", ["0", "1"])
def test_stress_rollers_match_oracle(ctx, torch_cuda, monkeypatch, forced):
    # rollers disable a subset of a node's components (RSolverStress::generateNodeBook,
    # src/rsolverstress.cpp:1564-1652): u_y on the y=0 face and u_z on the z=0 face, clamped at x=0;
    # the pattern then holds 1-3 columns per neighbour node, on both row kernels
    torch = torch_cuda
    monkeypatch.setenv("RSG_ASM_ROW_THREADS", forced)
    p = W.stress_beam(6, 3, 3)
    xyz = p.mesh.xyz
    dis = p.disabled.reshape(-1, 3).copy()
    dis[xyz[:, 1] == 0.0, 1] = True
    dis[xyz[:, 2] == 0.0, 2] = True
    p.disabled = dis.reshape(-1)
    p.book, p.n_free = W.node_book(p.disabled)
    p.node_u = np.zeros(3 * p.mesh.n_nodes)
    p.gravity = np.array([0.0, 0.0, -9.81])
    asm = rsg.Assembly.stress(ctx, p)
    b = torch.empty(p.n_free, dtype=torch.float64, device="cuda")
    M = asm.assemble(p, b)
    ctx.sync()
    Ao, bo = O.assemble_stress(p)
    assert asm.n_free == Ao.n and asm.nnz == Ao.nnz
    compare(device_csr(ctx, torch, M), b.cpu().numpy(), Ao, bo)
    x, st = ctx.solve(M, b.cpu().numpy(), conf=rsg.make_conf(n_outer=20000, stop_rule="true", rtol=1e-10),
                      prec=rsg.PREC_JACOBI)
    assert st.true_relres <= 1e-10
    xo, _ = O.solve(Ao, bo, prec=1, n_outer=20000, stop_rule="true", rtol=1e-12)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-8
