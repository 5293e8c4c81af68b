"""rsg_scatter_plan (RSolverFluid's pattern-cached assembly, src/rsolverfluid.cpp:2305-2419, on the GPU)
against the oracle's restatement: the same pattern and the same values and right-hand side bit for
bit (each entry adds its element contributions in element order), from host and from device element
blocks, on re-assembly into the same matrix; then restarted GMRES with Jacobi -- the solve
RSolverFluid::solve makes (src/rsolverfluid.cpp:510-511) -- on the assembled nonsymmetric system
agrees with the oracle's GMRES solution to 1e-8."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import workloads as W
from conftest import rel_err

pytestmark = pytest.mark.gpu

D = 4  # velocity x, y, z and pressure per node, as the fluid solver


def fluid_like(n_hex, seed):
    """A tet mesh with some of its faces as surface elements, a 4-DOF node book with the velocity
    fixed on the x = 0 face and one pressure fixed, and random element blocks made diagonally
    dominant (nonsymmetric)."""
    rng = np.random.default_rng(seed)
    m = W.heat_cube(n_hex, sigma=0.0, seed=0, source="random").mesh
    tets = np.asarray(m.tets, np.uint32).reshape(-1, 4)
    tris = tets[rng.choice(len(tets), size=len(tets) // 10, replace=False), :3]
    elems = [list(t) for t in tets] + [list(t) for t in tris]
    active = (rng.uniform(size=len(elems)) > 0.05).astype(np.uint8)
    begin = np.cumsum([0] + [len(e) for e in elems]).astype(np.uint32)
    nodes = np.concatenate(elems).astype(np.uint32)
    xyz = np.asarray(m.xyz).reshape(-1, 3)
    book = np.zeros(m.n_nodes * D, np.uint32)
    fixed = np.zeros(m.n_nodes * D, bool)
    on_x0 = np.where(np.isclose(xyz[:, 0], xyz[:, 0].min()))[0]
    for c in range(3):
        fixed[on_x0 * D + c] = True
    fixed[D * (m.n_nodes - 1) + 3] = True
    n_free = int((~fixed).sum())
    book[fixed] = 0xFFFFFFFF
    book[~fixed] = np.arange(n_free)
    sizes = [len(e) * D for e, a in zip(elems, active) if a]
    blocks, rhs = [], []
    for nd in sizes:
        blk = rng.standard_normal((nd, nd)) * 0.1
        blk[np.arange(nd), np.arange(nd)] += nd
        blocks.append(blk.ravel())
        rhs.append(rng.standard_normal(nd))
    return (begin, nodes, active, m.n_nodes, book, n_free), np.concatenate(blocks), np.concatenate(rhs)


@pytest.mark.parametrize("n_hex", [3, 10])
def test_scatter_assembly_matches_oracle_bitwise(ctx, torch_cuda, n_hex):
    torch = torch_cuda
    mesh, Ae, fe = fluid_like(n_hex, seed=n_hex)
    C, b_o = O.scatter_assemble(D, *mesh[:5], mesh[5], Ae, fe)
    plan = rsg.ScatterPlan(ctx, D, *mesh)
    assert plan.ae_values == Ae.size and plan.fe_values == fe.size and plan.nnz == C.rp[-1]
    b = torch.empty(plan.n_free, dtype=torch.float64, device="cuda")
    A = plan.assemble(Ae, fe, b)
    rp, ci, val = A.to_host()
    assert np.array_equal(rp, C.rp) and np.array_equal(ci, C.ci) and np.array_equal(val, C.val)
    assert np.array_equal(b.cpu().numpy(), b_o)
    # new values into the same matrix, from device arrays
    Ae2, fe2 = Ae * 1.5 - 0.25, fe * -2.0
    C2, b2_o = O.scatter_assemble(D, *mesh[:5], mesh[5], Ae2, fe2)
    A2 = plan.assemble(torch.tensor(Ae2, device="cuda"), torch.tensor(fe2, device="cuda"), b)
    assert A2 is A
    assert np.array_equal(A2.to_host()[2], C2.val) and np.array_equal(b.cpu().numpy(), b2_o)
    plan.close()


def test_scatter_assembly_then_gmres(ctx, torch_cuda):
    torch = torch_cuda
    mesh, Ae, fe = fluid_like(6, seed=11)
    C, b_o = O.scatter_assemble(D, *mesh[:5], mesh[5], Ae, fe)
    plan = rsg.ScatterPlan(ctx, D, *mesh)
    b = torch.empty(plan.n_free, dtype=torch.float64, device="cuda")
    A = plan.assemble(Ae, fe, b)
    conf = rsg.make_conf(solver="gmres", n_outer=2000, n_inner=30, stop_rule="true", rtol=1e-11)
    x, st = ctx.solve(A, b.cpu().numpy(), conf=conf, prec=rsg.PREC_JACOBI)
    assert st.status == rsg.OK and O.true_relres(C, b_o, x) <= 1e-11 * 1.01
    x_o, st_o = O.solve(C, b_o, prec=1, solver="gmres", n_outer=2000, n_inner=30, stop_rule="true", rtol=1e-13)
    assert rel_err(x, x_o) <= 1e-8
    plan.close()


def test_scatter_plan_rejects_bad_input(ctx):
    mesh, Ae, fe = fluid_like(2, seed=1)
    begin, nodes, active, n_nodes, book, n_free = mesh
    bad = book.copy()
    bad[bad != 0xFFFFFFFF] += n_free  # equation numbers past n_free
    with pytest.raises(rsg.RsgError):
        rsg.ScatterPlan(ctx, D, begin, nodes, active, n_nodes, bad, n_free)
    bad_nodes = nodes.copy()
    bad_nodes[0] = n_nodes + 5
    with pytest.raises(rsg.RsgError):
        rsg.ScatterPlan(ctx, D, begin, bad_nodes, active, n_nodes, book, n_free)
