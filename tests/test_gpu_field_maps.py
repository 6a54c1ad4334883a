"""Field-map output on the device: point location, nodal averaging and interpolation
(``snoopy/evaluators.py``, ``CurlCurlAssembler.compute_nodal_fields``) against the oracle."""

import numpy as np
import pytest

import snoopy_b200 as S
from helpers import rel_max
from snoopy_b200 import evaluators as EV
from snoopy_b200 import finite_element as FE
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def msh():
    return M.window_frame_mesh(30000, jitter=0.2, seed=21)


def _contains(msh, el, pts, tol=1e-10):
    """Barycentric coordinates of pts in elements el (numpy) are all >= -tol."""
    P = msh.nodes[msh.cells[el]]
    T = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)
    lam = np.linalg.solve(T, (pts - P[:, 0])[:, :, None])[:, :, 0]
    lam = np.concatenate([1.0 - lam.sum(1, keepdims=True), lam], axis=1)
    return lam.min(axis=1) >= -tol


def test_locate_matches_oracle(msh, oracle_mod):
    rng = np.random.default_rng(3)
    inside = rng.uniform([-0.5, -0.5, -0.6], [0.5, 0.5, 0.6], (4000, 3))
    outside = np.array([[0.7, 0.0, 0.0], [0.0, -0.8, 0.1], [0.1, 0.2, 5.0], [np.nan, 0.0, 0.0], [1e300, 0, 0]])
    at_nodes = msh.nodes[rng.choice(msh.num_nodes, 300, replace=False)]
    pts = np.concatenate([inside, outside, at_nodes])
    el, bary = msh.locate(pts)
    elo, baryo = oracle_mod.locate_points(msh.nodes, msh.cells, pts)
    n_in = len(inside)
    # generic interior points: the same element and coordinates
    assert (el[:n_in] >= 0).all()
    assert np.array_equal(el[:n_in], elo[:n_in])
    assert np.abs(bary[:n_in] - baryo[:n_in]).max() < 1e-12
    # outside, NaN and huge coordinates: not located
    assert (el[n_in:n_in + 5] == -1).all() and not bary[n_in:n_in + 5].any()
    # mesh nodes belong to several elements: any one holding the point is right
    e3 = el[n_in + 5:]
    assert (e3 >= 0).all() and _contains(msh, e3, at_nodes).all()
    rec = np.einsum("pi,pid->pd", bary[:n_in], msh.nodes[msh.cells[el[:n_in]]])
    assert np.abs(rec - inside).max() < 1e-12
    info = msh.index().info()
    assert info["max_bucket"] > 0 and min(info["h"]) > 0


def test_locate_empty_and_repeat(msh):
    el, bary = msh.locate(np.zeros((0, 3)))
    assert el.shape == (0,) and bary.shape == (0, 4)
    pts = np.random.default_rng(1).uniform(-0.4, 0.4, (500, 3))
    a = msh.locate(pts)
    b = msh.locate(pts)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_nodal_fields_match_oracle(msh, oracle_mod):
    rel = MAT.atan_reluctance()
    A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [rel, S.ConstantReluctance(0.25e7 / np.pi)])
    x = np.random.default_rng(2).normal(0, 1e-3, msh.num_dofs)
    w, q = FE.quadrature_rule(1)
    curls, n_orient = FE.curl_edge_basis_functions(q)
    dphi = FE.evaluate_basis_derivative(q)
    Be = oracle_mod.element_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, curls, n_orient, dphi, x)
    for tags in ([M.TAG_IRON], [M.TAG_AIR], [M.TAG_IRON, M.TAG_AIR]):
        got = A.compute_nodal_fields(x, tags)
        sel = np.isin(msh.elem_domain, tags)
        ref = oracle_mod.nodal_fields(msh.num_nodes, msh.cells[sel], Be[sel])
        assert rel_max(got, ref) < 1e-12
        # nodes that touch none of the materials stay 0
        touched = np.zeros(msh.num_nodes, dtype=bool)
        touched[msh.cells[sel].ravel()] = True
        assert not got[~touched].any()
    # deterministic: node sums run in element order
    assert np.array_equal(A.compute_nodal_fields(x, [M.TAG_IRON]), A.compute_nodal_fields(x, [M.TAG_IRON]))


def test_evaluators_match_oracle(msh, oracle_mod):
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1e-3, msh.num_dofs)
    pts = np.concatenate([rng.uniform(-0.5, 0.5, (2000, 3)) * [1, 1, 1.2], [[0.9, 0.9, 0.9]]])
    elo, baryo = oracle_mod.locate_points(msh.nodes, msh.cells, pts)
    vol = [M.TAG_IRON]
    # B at points inside the iron only
    B = EV.evaluate_curl_curl_solution(pts, msh, vol, x, msh.elem_edges + 1)
    w, q = FE.quadrature_rule(1)
    curls, n_orient = FE.curl_edge_basis_functions(q)
    dphi = FE.evaluate_basis_derivative(q)
    Be = oracle_mod.element_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, curls, n_orient, dphi, x)
    in_iron = (elo >= 0) & (msh.elem_domain[np.maximum(elo, 0)] == M.TAG_IRON)
    ref = np.where(in_iron[:, None], Be[np.maximum(elo, 0)], 0.0)
    assert in_iron.sum() > 100 and rel_max(B, ref) < 1e-12
    # interpolation of two domains' nodal sets, scalar and vector values
    vol2 = [M.TAG_IRON, M.TAG_AIR]
    sets = [rng.normal(size=(msh.num_nodes, 3)), rng.normal(size=(msh.num_nodes, 3))]
    got = EV.evaluate_interpolation(pts, msh, vol2, sets)
    dom = np.array([vol2.index(t) if e >= 0 else -1 for e, t in zip(elo, msh.elem_domain[np.maximum(elo, 0)])])
    ref = oracle_mod.interpolate_nodal(msh.cells, elo, baryo, sets, dom)
    assert got.shape == (len(pts), 3) and rel_max(got, ref) < 1e-12
    sc = [rng.normal(size=msh.num_nodes)]
    got1 = EV.evaluate_interpolation(pts, msh, [M.TAG_AIR], sc)
    dom1 = np.where((elo >= 0) & (msh.elem_domain[np.maximum(elo, 0)] == M.TAG_AIR), 0, -1)
    ref1 = oracle_mod.interpolate_nodal(msh.cells, elo, baryo, sc, dom1)
    assert got1.shape == (len(pts), 1) and rel_max(got1, ref1) < 1e-12
    assert got1[-1, 0] == 0.0  # outside the mesh


def test_node_interpolation_of_a_solved_field(oracle_mod):
    """evaluate_fem_solution_node_interpolation on a solved reduced problem against the oracle's
    restatement of the same chain (element fields averaged at the nodes, the coils' field at
    the nodes, barycentric interpolation)."""
    msh = M.window_frame_mesh(20000, jitter=0.15, seed=7)
    g = msh.geometry
    coils = g.coils()
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [MAT.atan_reluctance()], quad_order=2)
    solver.verbose = False
    x, st = solver.solve_to_residual(1e-8)
    probes = np.concatenate([g.aperture_probes(300), np.random.default_rng(9).uniform(-0.45, 0.45, (300, 3))])
    doms = [M.TAG_AIR, M.TAG_IRON]
    Bn = EV.evaluate_fem_solution_node_interpolation(msh, probes, solver, coils, x, doms)
    w, q = FE.quadrature_rule(1)
    curls, n_orient = FE.curl_edge_basis_functions(q)
    dphi = FE.evaluate_basis_derivative(q)
    Be = oracle_mod.element_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, curls, n_orient, dphi, x)
    b_coil = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), msh.nodes, c.current, c.rad) for c in coils)
    sets = [oracle_mod.nodal_fields(msh.num_nodes, msh.cells[msh.elem_domain == t], Be[msh.elem_domain == t]) + b_coil
            for t in doms]
    elo, baryo = oracle_mod.locate_points(msh.nodes, msh.cells, probes)
    dom = np.array([doms.index(t) if e >= 0 else -1 for e, t in zip(elo, msh.elem_domain[np.maximum(elo, 0)])])
    ref = oracle_mod.interpolate_nodal(msh.cells, elo, baryo, sets, dom)
    assert np.isfinite(Bn).all() and (dom >= 0).all()
    assert rel_max(Bn, ref) < 1e-12
