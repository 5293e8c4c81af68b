"""Native DOF numbering (rsg_node_book_generic / rsg_node_book_stress) against the oracle's
restatement of RSolverGeneric::generateNodeBook (src/rsolvergeneric.cpp:498-582) and
RSolverStress::generateNodeBook (src/rsolverstress.cpp:1564-1652), and against the numbering the
Python problem generators use.  Host-only entry points: these run without a GPU.  Books must be
identical (integer work: bit-exact)."""
import numpy as np
import pytest

import rsg
from oracle import oracle as O
from rsg import _lib
from rsg import workloads as W

EOD = 0xFFFFFFFF


def boundary_triangles(mesh, axis, value):
    """Tet faces lying in the plane xyz[:, axis] == value (each once)."""
    faces = np.concatenate([mesh.tets[:, [0, 1, 2]], mesh.tets[:, [0, 1, 3]], mesh.tets[:, [0, 2, 3]],
                            mesh.tets[:, [1, 2, 3]]])
    on = np.all(mesh.xyz[faces, axis] == value, axis=1)
    return np.unique(np.sort(faces[on], axis=1), axis=0).astype(np.uint32)


def boundary_line(mesh, y, z):
    """Edges along x on the line (y, z)."""
    nodes = np.flatnonzero((mesh.xyz[:, 1] == y) & (mesh.xyz[:, 2] == z))
    nodes = nodes[np.argsort(mesh.xyz[nodes, 0])]
    return np.stack([nodes[:-1], nodes[1:]], axis=1).astype(np.uint32)


def model_from(mesh, groups_of_elements, computable_tets=None):
    """Element list = tets, then every boundary group's elements; one group per entry (the tets first)."""
    elements = [list(t) for t in mesh.tets]
    groups = [list(range(mesh.n_tets))]
    for els in groups_of_elements:
        first = len(elements)
        elements += [list(e) for e in els]
        groups.append(list(range(first, len(elements))))
    computable = None
    if computable_tets is not None:
        computable = np.ones(len(elements), np.uint8)
        computable[:mesh.n_tets] = computable_tets
    return rsg.ModelGroups(mesh.n_nodes, elements, groups, computable), elements, groups, computable


def flat(elements, groups):
    eb = np.zeros(len(elements) + 1, np.uint32)
    eb[1:] = np.cumsum([len(e) for e in elements])
    gb = np.zeros(len(groups) + 1, np.uint32)
    gb[1:] = np.cumsum([len(g) for g in groups])
    return eb, np.concatenate(elements).astype(np.uint32), gb, np.concatenate(groups).astype(np.uint32)


def test_heat_book_matches_oracle_and_generator():
    p = W.heat_cube(6, sigma=1.0, seed=1, source="random")
    mesh = p.mesh
    x0, x1, y0 = boundary_triangles(mesh, 0, 0.0), boundary_triangles(mesh, 0, 1.0), boundary_triangles(mesh, 1, 0.0)
    model, elements, groups, _ = model_from(mesh, [x0, x1, y0])
    explicit = np.array([0, 1, 1, 0], np.uint8)  # T prescribed on x=0 and x=1; y=0 carries a flux (not explicit)
    book, n_free = rsg.node_book_generic(model, explicit)
    ob, on = O.node_book_generic(mesh.n_nodes, *flat(elements, groups), explicit)
    assert n_free == on == p.n_free
    assert np.array_equal(book, ob) and np.array_equal(book, p.book)


def test_heat_book_non_computable_elements():
    """Nodes touched only by non-computable elements are disabled; a shared node stays free."""
    p = W.heat_cube(5, sigma=1.0, seed=2, source="random")
    mesh = p.mesh
    cen = mesh.xyz[mesh.tets].mean(axis=1)
    computable = ~((cen[:, 0] > 0.6) & (cen[:, 1] > 0.6))  # a corner column of elements is not computed
    model, elements, groups, comp = model_from(mesh, [boundary_triangles(mesh, 0, 0.0)], computable.astype(np.uint8))
    explicit = np.array([0, 1], np.uint8)
    book, n_free = rsg.node_book_generic(model, explicit)
    ob, on = O.node_book_generic(mesh.n_nodes, *flat(elements, groups), explicit, comp)
    assert np.array_equal(book, ob) and n_free == on
    touched = np.zeros(mesh.n_nodes, bool)
    touched[mesh.tets[computable].ravel()] = True
    expect = (mesh.xyz[:, 0] == 0.0) | ~touched
    wb, wn = W.node_book(expect)
    assert np.array_equal(book, wb) and n_free == wn
    assert 0 < (~touched).sum() < mesh.n_nodes


def test_stress_book_rollers_match_oracle_and_generator():
    """Clamped face (all three components), a roller face (x only), a roller line (y and z), a
    normal-displacement face (all three), and a group with no displacement condition."""
    p = W.stress_beam(8, 4, 4)
    mesh = p.mesh
    clamp = boundary_triangles(mesh, 0, 0.0)
    roller_face = boundary_triangles(mesh, 0, 2.0)
    roller_line = boundary_line(mesh, 1.0, 1.0)
    normal_face = boundary_triangles(mesh, 2, 0.0)
    free_face = boundary_triangles(mesh, 1, 0.0)
    model, elements, groups, _ = model_from(mesh, [clamp, roller_face, roller_line, normal_face, free_face])
    B = _lib
    bc = np.array([0, B.BC_DISPLACEMENT, B.BC_DISPLACEMENT_ROLLER, B.BC_DISPLACEMENT_ROLLER,
                   B.BC_DISPLACEMENT_NORMAL, 0], np.uint8)
    line = np.array([0, 0, 0, 1, 0, 0], np.uint8)
    book, n_free = rsg.node_book_stress(model, bc, line)
    ob, on = O.node_book_stress(mesh.n_nodes, *flat(elements, groups), bc, line)
    assert np.array_equal(book, ob) and n_free == on
    x, y, z = mesh.xyz.T
    dis = np.zeros((mesh.n_nodes, 3), bool)
    dis[x == 0.0] = True
    dis[z == 0.0] = True
    dis[x == 2.0, 0] = True
    dis[(y == 1.0) & (z == 1.0), 1:] = True
    wb, wn = W.node_book(dis.reshape(-1))
    assert np.array_equal(book, wb) and n_free == wn
    # the clamped beam of the elasticity benchmark
    model2, el2, gr2, _ = model_from(mesh, [clamp])
    book2, n2 = rsg.node_book_stress(model2, np.array([0, B.BC_DISPLACEMENT], np.uint8), np.zeros(2, np.uint8))
    assert np.array_equal(book2, p.book) and n2 == p.n_free


def test_books_at_benchmark_size():
    """100^3 heat cube (1,030,301 nodes, 6M tets): the blocked parallel numbering equals the oracle's."""
    mesh = W.box_tet_mesh(100, 100, 100)
    faces = [boundary_triangles(mesh, 0, 0.0), boundary_triangles(mesh, 0, 1.0)]
    n_t = mesh.n_tets
    elem_nodes = np.concatenate([mesh.tets.reshape(-1)] + [f.reshape(-1) for f in faces]).astype(np.uint32)
    sizes = np.r_[np.full(n_t, 4), np.full(sum(len(f) for f in faces), 3)]
    eb = np.zeros(len(sizes) + 1, np.uint32)
    eb[1:] = np.cumsum(sizes)
    gb = np.array([0, n_t, n_t + len(faces[0]), n_t + len(faces[0]) + len(faces[1])], np.uint32)
    ge = np.arange(gb[-1], dtype=np.uint32)
    model = rsg.ModelGroups.__new__(rsg.ModelGroups)
    model.elem_begin, model.elem_nodes, model.group_begin, model.group_elems, model.computable = eb, elem_nodes, gb, ge, None
    model.n_nodes = mesh.n_nodes
    P = lambda a: a.ctypes.data  # noqa: E731
    model.c = _lib.ModelGroups(mesh.n_nodes, len(sizes), P(eb), P(elem_nodes), 3, P(gb), P(ge), None)
    explicit = np.array([0, 1, 1], np.uint8)
    book, n_free = rsg.node_book_generic(model, explicit)
    ob, on = O.node_book_generic(mesh.n_nodes, eb, elem_nodes, gb, ge, explicit)
    assert n_free == on == 1009899 and np.array_equal(book, ob)


def test_invalid_models_are_rejected():
    mesh = W.box_tet_mesh(2, 2, 2)
    bad = mesh.tets.copy()
    bad[3, 2] = mesh.n_nodes  # node id out of range
    with pytest.raises(rsg.RsgError) as e:
        rsg.node_book_generic(rsg.ModelGroups(mesh.n_nodes, bad, [[0, 1]]), [1])
    assert e.value.status == _lib.ERR_INVALID_ARG
    with pytest.raises(rsg.RsgError):  # element id out of range in a group
        rsg.node_book_generic(rsg.ModelGroups(mesh.n_nodes, mesh.tets, [[0, mesh.n_tets]]), [1])
    with pytest.raises(rsg.RsgError):
        rsg.node_book_stress(rsg.ModelGroups(mesh.n_nodes, bad, [[0]]), [1], [0])
    # no groups at all: every node touched by an element is free
    book, n = rsg.node_book_generic(rsg.ModelGroups(mesh.n_nodes, mesh.tets, []), [])
    assert n == mesh.n_nodes and np.array_equal(book, np.arange(mesh.n_nodes))
