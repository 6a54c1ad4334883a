"""Meshes, edge numbering, orientations and reference-element tables (what gmsh supplies
to the reference), checked against their defining properties."""

import numpy as np
import pytest

from snoopy_b200 import finite_element as FE
from snoopy_b200 import mesh as M


@pytest.fixture(scope="module")
def msh():
    return M.window_frame_mesh(4000, jitter=0.2, seed=4)


def test_positive_orientation_and_euler(msh):
    assert (M.tet_volumes6(msh.nodes, msh.cells) > 0).all()
    faces = msh.boundary_faces()
    c = np.sort(msh.cells.astype(np.int64), axis=1)
    allf = np.concatenate([c[:, [0, 1, 2]], c[:, [0, 1, 3]], c[:, [0, 2, 3]], c[:, [1, 2, 3]]])
    n_faces = len(np.unique(allf, axis=0))
    # Euler characteristic of a ball: V - E + F - T = 1
    assert msh.num_nodes - msh.num_dofs + n_faces - msh.num_elements == 1
    assert len(faces) > 0


def test_total_volume(msh):
    vol = M.tet_volumes6(msh.nodes, msh.cells).sum() / 6.0
    assert abs(vol - 1.0 * 1.0 * 1.2) < 1e-12


def test_edge_ids_and_orientation_signs(msh):
    c = msh.cells.astype(np.int64)
    for j, (a, b) in enumerate(FE.TET_EDGES):
        lo, hi = msh.edges[msh.elem_edges[:, j]].T
        na, nb = c[:, a], c[:, b]
        assert np.array_equal(np.minimum(na, nb), lo) and np.array_equal(np.maximum(na, nb), hi)
        sign = FE.orientation_signs(msh.orientations)[:, j]
        assert np.array_equal(sign > 0, na < nb)


def test_whitney_dofs_are_edge_integrals():
    """int_edge_k w_j . t_k = delta_jk on the reference element (Gauss-Legendre on each edge)."""
    verts = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    s, ws = np.polynomial.legendre.leggauss(4)
    s = 0.5 * (s + 1)
    ws = 0.5 * ws
    for k, (a, b) in enumerate(FE.TET_EDGES):
        t = verts[b] - verts[a]
        pts = verts[a][None] + s[:, None] * t[None]
        w = FE.edge_basis_functions(pts.reshape(-1))  # [P, 6, 3]
        integ = np.einsum("p,pjd,d->j", ws, w, t)
        expect = np.zeros(6)
        expect[k] = 1.0
        np.testing.assert_allclose(integ, expect, atol=1e-14)


def test_curls_match_finite_differences():
    c = FE.reference_curls()
    p = np.array([0.2, 0.3, 0.1])
    h = 1e-6
    for j in range(6):
        J = np.zeros((3, 3))
        for d in range(3):
            e = np.zeros(3)
            e[d] = h
            J[:, d] = (FE.edge_basis_functions(p + e)[0, j] - FE.edge_basis_functions(p - e)[0, j]) / (2 * h)
        curl = np.array([J[2, 1] - J[1, 2], J[0, 2] - J[2, 0], J[1, 0] - J[0, 1]])
        np.testing.assert_allclose(curl, c[j], atol=1e-8)


@pytest.mark.parametrize("order", [1, 2, 3, 4, 5, 6, 8])
def test_quadrature_exactness(order):
    from math import factorial

    w, q = FE.quadrature_rule(order)
    p = q.reshape(-1, 3)
    assert abs(w.sum() - 1.0 / 6.0) < 1e-15
    for a in range(order + 1):
        for b in range(order + 1 - a):
            for c in range(order + 1 - a - b):
                exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
                got = np.sum(w * p[:, 0] ** a * p[:, 1] ** b * p[:, 2] ** c)
                assert abs(got - exact) < 1e-14, (a, b, c)


def test_dirichlet_edges_on_box_surface(msh):
    ids = msh.get_edge_boundary_dofs(["Dirichlet Boundary"]) - 1
    xyz = msh.nodes[msh.edges[ids]]  # [m, 2, 3]
    half = np.array([0.5, 0.5, 0.6])
    on = np.zeros(len(ids), bool)
    for d in range(3):
        for s in (-1, 1):
            on |= np.all(np.abs(xyz[:, :, d] - s * half[d]) < 1e-12, axis=1)
    assert on.all()
    assert len(ids) > 0


def test_locate_points(msh, oracle_mod):
    """The oracle's bucket search (the checker of the device mesh index)."""
    rng = np.random.default_rng(0)
    pts = rng.uniform([-0.5, -0.5, -0.6], [0.5, 0.5, 0.6], (200, 3))
    el, bary = oracle_mod.locate_points(msh.nodes, msh.cells, pts)
    assert (el >= 0).all()
    rec = np.einsum("pi,pid->pd", bary, msh.nodes[msh.cells[el]])
    np.testing.assert_allclose(rec, pts, atol=1e-12)


def test_microbench_mesh_counts():
    m = M.kuhn_microbench_mesh(4, 5, 3, seed=1)
    assert m.num_elements == 6 * 4 * 5 * 3
    assert m.num_nodes == 5 * 6 * 4
    frac = (m.elem_domain == M.TAG_IRON).mean()
    assert 0.2 < frac < 0.6


def test_coil_terminals_split_ring():
    m = M.window_frame_mesh(6000, jitter=0.1, seed=2, coils=True)
    for tag in (M.TAG_COIL_1, M.TAG_COIL_2):
        t1, t2 = m.coil_terminals[tag]
        assert len(t1) > 0 and len(t2) > 0
        assert not np.intersect1d(t1, t2).size


def test_cotree_split_is_a_spanning_tree(msh):
    tree, cotree = msh.get_cotree_dofs()
    assert len(tree) == msh.num_nodes - 1 and len(tree) + len(cotree) == msh.num_dofs
    assert not np.intersect1d(tree, cotree).size
    parent = np.arange(msh.num_nodes)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for e in tree:  # acyclic with N - 1 edges: spanning
        a, b = find(msh.edges[e, 0]), find(msh.edges[e, 1])
        assert a != b
        parent[a] = b
    # the tree spans the outer boundary's nodes through boundary edges first
    bnd = msh.boundary_edge_ids()
    n_bnodes = len(np.unique(msh.edges[bnd].ravel()))
    assert np.isin(tree, bnd).sum() == n_bnodes - 1


def test_block_jacobi_partition():
    """dof_blocks: runs of equal keys among free DoFs, at most 8 long, never across a multiple of
    256, constrained DoFs alone; offsets and sizes encoded per DoF."""
    from snoopy_b200.newton import dof_blocks

    rng = np.random.default_rng(4)
    for n in (1, 7, 255, 256, 257, 3001):
        keys = np.sort(rng.integers(0, max(1, n // 5), n))
        free = rng.random(n) > 0.1
        meta = dof_blocks(keys, free)
        off, size = meta & 0xFF, meta >> 8
        i = 0
        while i < n:
            s = int(size[i])
            assert off[i] == 0 and 1 <= s <= 8 and i + s <= n
            assert i // 256 == (i + s - 1) // 256
            assert np.array_equal(off[i:i + s], np.arange(s)) and np.all(size[i:i + s] == s)
            if s > 1:
                assert np.all(free[i:i + s]) and np.all(keys[i:i + s] == keys[i])
            if not free[i]:
                assert s == 1
            # maximal: the next DoF would have fit (same key, free, same tile, room) only if cut by the cap
            j = i + s
            if j < n and s < 8 and j % 256 != 0 and free[i] and free[j] and keys[j] == keys[i]:
                raise AssertionError(f"block at {i} not maximal")
            i = j
