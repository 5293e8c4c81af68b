"""Seeded synthetic workloads: structured tetrahedral meshes, random fields and
the boundary-value problems that the solver path is measured on.

Everything here is input generation.  The same arrays feed the CUDA library
and the CPU oracle, so parity is checked on identical inputs.

Meshes are unit-spaced boxes of hexahedra, each split into 6 tetrahedra that
share the hex's main diagonal (Kuhn/Freudenthal split), all positively
oriented.  Node ids run x-fastest: id = i + (nx+1) * (j + (ny+1) * k).

Random numbers use a counter-based SplitMix64 stream (Steele, Lea & Flood,
"Fast splittable pseudorandom number generators", OOPSLA 2014) so that value i
of a stream depends only on (seed, stream, i); normals come from the
Box-Muller transform.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

EOD = np.uint32(0xFFFFFFFF)

_M64 = (1 << 64) - 1


def splitmix64(seed: int, stream: int, n: int, offset: int = 0) -> np.ndarray:
    """n uint64 outputs of SplitMix64 at counters offset..offset+n-1 of (seed, stream)."""
    gamma = np.uint64(0x9E3779B97F4A7C15)
    base = np.uint64((seed * 0xD1B54A32D192ED03 + stream * 0x8CB92BA72F3D8DD7) & _M64)
    with np.errstate(over="ignore"):
        z = base + (np.arange(offset, offset + n, dtype=np.uint64) + np.uint64(1)) * gamma
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, stream: int, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
    """Uniform doubles in [lo, hi) from the top 53 bits."""
    u = (splitmix64(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    return lo + (hi - lo) * u


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """Standard normals by Box-Muller on pairs of uniforms (cosine branch only)."""
    u = (splitmix64(seed, stream, 2 * n) >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def lognormal(seed: int, stream: int, n: int, mu: float, sigma: float) -> np.ndarray:
    return np.exp(mu + sigma * normal(seed, stream, n))


@dataclass
class TetMesh:
    nx: int
    ny: int
    nz: int
    xyz: np.ndarray  # (n_nodes, 3) float64
    tets: np.ndarray  # (n_tets, 4) uint32

    @property
    def n_nodes(self) -> int:
        return self.xyz.shape[0]

    @property
    def n_tets(self) -> int:
        return self.tets.shape[0]

    def node_id(self, i, j, k):
        return i + (self.nx + 1) * (j + (self.ny + 1) * k)


def box_tet_mesh(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0) -> TetMesh:
    """Structured box of nx*ny*nz hexes, 6 tets each (ordered hex by hex, x fastest)."""
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # node order x fastest: transpose to (k, j, i) flattening
    xs = (np.arange(nx + 1) * (lx / nx))
    ys = (np.arange(ny + 1) * (ly / ny))
    zs = (np.arange(nz + 1) * (lz / nz))
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    xyz = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1).astype(np.float64)

    hk, hj, hi = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    base = (hi + (nx + 1) * (hj + (ny + 1) * hk)).ravel().astype(np.int64)
    step = {0: 1, 1: nx + 1, 2: (nx + 1) * (ny + 1)}
    tets = []
    for perm in itertools.permutations(range(3)):
        a, b, c = perm
        v0 = base
        v1 = v0 + step[a]
        v2 = v1 + step[b]
        v3 = v2 + step[c]
        # orientation of (e_a, e_b, e_c) is the permutation's sign
        inversions = sum(1 for p in range(3) for q in range(p + 1, 3) if perm[p] > perm[q])
        if inversions % 2 == 0:
            tets.append(np.stack([v0, v1, v2, v3], axis=1))
        else:
            tets.append(np.stack([v0, v2, v1, v3], axis=1))
    # interleave so that the 6 tets of one hex are consecutive
    tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.uint32)
    return TetMesh(nx, ny, nz, xyz, tets)


def face_triangles_x_max(mesh: TetMesh) -> np.ndarray:
    """Triangles of the x = max face, split along the diagonal the Kuhn tets use."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    kk, jj = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
    jj = jj.ravel()
    kk = kk.ravel()
    n = lambda j, k: nx + (nx + 1) * (j + (ny + 1) * k)  # noqa: E731
    v00, v10, v01, v11 = n(jj, kk), n(jj + 1, kk), n(jj, kk + 1), n(jj + 1, kk + 1)
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v01, v11], axis=1)
    return np.stack([t1, t2], axis=1).reshape(-1, 3).astype(np.uint32)


def node_book(disabled: np.ndarray) -> tuple[np.ndarray, int]:
    """Consecutive numbering of enabled positions; disabled -> EOD."""
    disabled = np.asarray(disabled, dtype=bool)
    book = np.full(disabled.shape[0], EOD, dtype=np.uint32)
    free = ~disabled
    n_free = int(free.sum())
    book[free] = np.arange(n_free, dtype=np.uint32)
    return book, n_free


@dataclass
class HeatProblem:
    """Steady or transient heat conduction on a tet mesh (RSolverHeat inputs)."""

    mesh: TetMesh
    k_e: np.ndarray  # conductivity per tet
    q_e: np.ndarray  # volumetric heat source per tet
    rhoc_e: np.ndarray  # density * capacity per tet
    node_t: np.ndarray  # prescribed T at Dirichlet nodes / previous T for transient
    disabled: np.ndarray  # bool per node
    book: np.ndarray
    n_free: int
    transient: bool = False
    alpha: float = 1.0
    dt: float = 0.0
    name: str = ""
    meta: dict = field(default_factory=dict)


def heat_cube(n: int, *, sigma: float = 0.0, seed: int = 0, source: str = "unit", transient: bool = False,
              dt: float = 1.0e-3, rhoc: float = 1.0, mu: float = 0.0) -> HeatProblem:
    """Unit cube, n^3 hexes -> 6 n^3 tets; T=0 on x=0, T=1 on x=1, other faces insulated.

    sigma == 0 gives uniform k=1.  Otherwise k_e ~ lognormal(mu, sigma) per tet.
    source "unit": Q=1 per tet; "random": nodal s_i ~ U(0,1), Q_e = mean of its 4 nodes.
    """
    mesh = box_tet_mesh(n, n, n)
    nt = mesh.n_tets
    k_e = np.ones(nt) if sigma == 0.0 else lognormal(seed, 1, nt, mu, sigma)
    if source == "unit":
        q_e = np.ones(nt)
    elif source == "random":
        s = uniform(seed, 2, mesh.n_nodes)
        q_e = s[mesh.tets].mean(axis=1)
    elif source == "none":
        q_e = np.zeros(nt)
    else:
        raise ValueError(source)
    x = mesh.xyz[:, 0]
    disabled = (x == 0.0) | (x == 1.0)
    node_t = np.where(x == 1.0, 1.0, 0.0)
    book, n_free = node_book(disabled)
    return HeatProblem(mesh, k_e, q_e, np.full(nt, rhoc), node_t, disabled, book, n_free,
                       transient=transient, alpha=1.0, dt=dt if transient else 0.0,
                       name=f"heat_cube_{n}", meta=dict(n=n, sigma=sigma, seed=seed, source=source))


# vacuum permittivity [F/m] as RSolverGeneric::e0 (src/rsolvergeneric.cpp:13)
E0 = 8.854187817e-12


def electrostatic_cube(n: int, *, eps_r: float = 1.0, charge: float = 0.0, v0: float = 0.0, v1: float = 1.0,
                       sigma: float = 0.0, seed: int = 0) -> HeatProblem:
    """Electrostatics on the unit cube (potential v0 on x=0, v1 on x=1, other faces insulated).

    RSolverElectrostatics' 3-D volume integrals (src/rsolverelectrostatics.cpp:322-344) are the heat
    conduction ones with k = eps_r * e0 and a volumetric source of -rho (fe -= rho N detJ w), and its
    Dirichlet lifting (:800-812) is the heat one, so the heat assembly plan serves them: the returned
    problem carries k_e = eps_r e0 (lognormal spread sigma when > 0) and q_e = -charge per tet.
    """
    p = heat_cube(n, sigma=sigma, seed=seed, source="none")
    nt = p.mesh.n_tets
    p.k_e = (np.full(nt, eps_r) if sigma == 0.0 else lognormal(seed, 1, nt, np.log(eps_r), sigma)) * E0
    p.q_e = np.full(nt, -charge)
    x = p.mesh.xyz[:, 0]
    p.node_t = np.where(x == 1.0, v1, np.where(x == 0.0, v0, 0.0))
    p.name = f"electrostatic_cube_{n}"
    return p


@dataclass
class MagnetostaticProblem:
    """Magnetostatics on a tet mesh (RSolverMagnetostatics inputs): vector potential, 3 dofs per node
    interleaved (3 * position + component), a node's three dofs enabled or disabled together."""

    mesh: TetMesh
    node_j: np.ndarray  # (3 n_nodes,) nodal current density
    node_a: np.ndarray  # (3 n_nodes,) prescribed potential at disabled nodes
    disabled: np.ndarray  # (n_nodes,) bool
    book: np.ndarray  # (3 n_nodes,)
    n_free: int
    name: str = ""


def magnetostatic_cube(n: int, *, current: str = "coil", a0=(0.0, 0.0, 0.0), a1=(0.0, 0.0, 0.0), j0: float = 1.0e6,
                       seed: int = 0) -> MagnetostaticProblem:
    """Unit cube (n^3 hexes, 6 tets each); potential a0 on x=0 and a1 on x=1 (all components).

    current "coil": J = j0 (-(y - 1/2), x - 1/2, 0) inside the cylinder (x-1/2)^2 + (y-1/2)^2 < 1/16
    (a circulating current about the z axis), zero outside; "random": J ~ j0 U(-1, 1) per node and
    component; "none": J = 0.  The reference converts element current densities to nodes with
    range-model-lib's convertElementToNodeVector (src/rsolvermagnetostatics.cpp:38-40); the nodal
    field is the input here.
    """
    mesh = box_tet_mesh(n, n, n)
    nn = mesh.n_nodes
    x, y = mesh.xyz[:, 0], mesh.xyz[:, 1]
    if current == "coil":
        inside = (x - 0.5) ** 2 + (y - 0.5) ** 2 < 1.0 / 16.0
        J = np.stack([-(y - 0.5), x - 0.5, np.zeros(nn)], axis=1) * j0 * inside[:, None]
    elif current == "random":
        J = (uniform(seed, 5, 3 * nn, -1.0, 1.0) * j0).reshape(nn, 3)
    elif current == "none":
        J = np.zeros((nn, 3))
    else:
        raise ValueError(current)
    disabled = (x == 0.0) | (x == 1.0)
    A = np.zeros((nn, 3))
    A[x == 0.0] = np.asarray(a0, float)
    A[x == 1.0] = np.asarray(a1, float)
    book, n_free = node_book(np.repeat(disabled, 3))
    return MagnetostaticProblem(mesh, J.reshape(-1).copy(), A.reshape(-1).copy(), disabled, book, n_free,
                                name=f"magnetostatic_cube_{n}")


def reseed_heat(p: HeatProblem, *, sigma: float, seed: int, mu: float = 0.0) -> HeatProblem:
    """p with a new lognormal(mu, sigma) conductivity field and random source drawn from seed
    (same mesh, node book and boundary values; the streams heat_cube uses for that seed)."""
    import copy
    q = copy.copy(p)
    m = p.mesh
    q.k_e = lognormal(seed, 1, m.n_tets, mu, sigma)
    q.q_e = uniform(seed, 2, m.n_nodes)[m.tets].mean(axis=1)
    q.meta = dict(p.meta, sigma=sigma, seed=seed, source="random")
    return q


@dataclass
class StressProblem:
    """Linear elasticity on a tet mesh (RSolverStress inputs), 3 dofs per node interleaved."""

    mesh: TetMesh
    e_mod: np.ndarray
    nu: np.ndarray
    rho_e: np.ndarray
    gravity: np.ndarray  # (3,)
    texp_e: np.ndarray
    dtemp_e: np.ndarray
    tris: np.ndarray  # traction triangles
    traction: np.ndarray  # (n_tris, 3)
    node_u: np.ndarray  # (3 n_nodes,)
    disabled: np.ndarray  # (3 n_nodes,)
    book: np.ndarray
    n_free: int
    transient: bool = False
    alpha: float = 1.0
    dt: float = 0.0
    name: str = ""


def stress_beam(nx: int = 64, ny: int = 32, nz: int = 32, *, length: float = 2.0, e_mod: float = 210e9,
                nu: float = 0.3, traction=(0.0, 0.0, -1.0e6), rho: float = 7850.0) -> StressProblem:
    """Beam length x 1 x 1 (nx x ny x nz hexes, 6 tets each), clamped at x=0, traction on x=L."""
    mesh = box_tet_mesh(nx, ny, nz, length, 1.0, 1.0)
    nt = mesh.n_tets
    tris = face_triangles_x_max(mesh)
    x = mesh.xyz[:, 0]
    clamped = x == 0.0
    disabled = np.repeat(clamped, 3)
    book, n_free = node_book(disabled)
    return StressProblem(mesh, np.full(nt, e_mod), np.full(nt, nu), np.full(nt, rho), np.zeros(3),
                         np.zeros(nt), np.zeros(nt), tris, np.tile(np.asarray(traction, float), (tris.shape[0], 1)),
                         np.zeros(3 * mesh.n_nodes), disabled, book, n_free, name=f"stress_beam_{nx}x{ny}x{nz}")
