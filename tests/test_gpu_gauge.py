"""Tree-cotree gauged solves (``apply_gauge=True``, ``mesh_tools.py:468-566``): the spanning
tree's edges are fixed, the field is the ungauged one."""

import numpy as np
import pytest

import snoopy_b200 as S
from helpers import rel_max
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M
from test_gpu_parity import _oracle_red, _red_setup

pytestmark = pytest.mark.gpu


def test_reduced_gauged_matches_oracle_and_ungauged(oracle_mod):
    msh, g, coils, rel, solver = _red_setup(6000)
    O, sf, mask = _oracle_red(oracle_mod, msh, coils, rel, solver)
    tree, cotree = msh.get_cotree_dofs()
    gmask = solver.gauge_mask()
    assert not gmask[tree].any() and np.array_equal(gmask, mask & np.isin(np.arange(msh.num_dofs), cotree))
    solver.max_newton_iterations = 25
    xg = solver.solve(tolerance=1e-4, apply_gauge=True)
    assert not xg[tree].any()
    xr, st = oracle_mod.newton_reference(O, gmask, sf, tolerance=1e-4)
    assert abs(solver.last_stats["newton_iterations"] - st["newton"]) <= 1
    probes = g.aperture_probes(200)
    el, _ = msh.locate(probes)
    A = solver.curl_curl_factory
    assert rel_max(A.compute_B_at_points(xg, probes, el), A.compute_B_at_points(xr, probes, el)) < 1e-2
    # the gauge removes only the gradient null space: driven to a 1e-10 residual, the gauged
    # answer carries the ungauged field (the reference-mode solves stop at CG rtol 1e-5, and the
    # tree gauge worsens the conditioning, so those agree only to that level)
    xg10, sg = solver.newton_engine(apply_gauge=True).solve(None, tol=1e-10, max_newton=50)
    x, _ = solver.solve_to_residual(1e-10)
    assert sg["rel_res"] <= 1e-10 and not xg10.cpu().numpy()[tree].any()
    Bg = A.compute_B_at_points(xg10.cpu().numpy(), probes, el)
    assert rel_max(Bg, A.compute_B_at_points(x, probes, el)) < 1e-7


def test_total_potential_gauged():
    msh = M.bar_conductor_mesh(12000)
    t1, t2 = msh.coil_terminals[M.TAG_COIL_1]
    Phi = 3e6 * 0.8
    solver = S.MVPSolver(msh, [M.TAG_COIL_1], [M.TAG_IRON], [M.TAG_AIR], [(t1, t2)], [MAT.atan_reluctance()],
                         quad_order=2, max_newton_iterations=60)
    solver.verbose = False
    xg = solver.solve_nonlin([Phi], tolerance=1e-6, apply_gauge=True)
    tree, _ = msh.get_cotree_dofs()
    assert not xg[tree].any()
    cen = msh.element_centroids()
    probe = msh.domain_elements(M.TAG_IRON)[::5]
    A = solver.curl_curl_factory
    xg10, sg = solver._engine([Phi], apply_gauge=True).solve(None, tol=1e-10, max_newton=60)
    assert sg["rel_res"] <= 1e-10 and not xg10.cpu().numpy()[tree].any()
    Bg = A.compute_B_at_points(xg10.cpu().numpy(), cen[probe], probe)
    x, st = solver.solve_to_residual([Phi], rtol=1e-10, max_newton=60)
    B = A.compute_B_at_points(x, cen[probe], probe)
    assert rel_max(Bg, B) < 1e-7
    assert rel_max(A.compute_B_at_points(xg, cen[probe], probe), B) < 5e-2


def test_total_potential_linear_solve(oracle_mod):
    """MVPSolver.solve_lin: K(0) x = rhs by device Jacobi-PCG to scipy's default relative
    tolerance (1e-5), with and without the gauge; residual measured with the oracle's K."""
    from scipy.sparse import csr_array

    from snoopy_b200 import finite_element as FE

    msh = M.bar_conductor_mesh(12000)
    t1, t2 = msh.coil_terminals[M.TAG_COIL_1]
    solver = S.MVPSolver(msh, [M.TAG_COIL_1], [M.TAG_IRON], [M.TAG_AIR], [(t1, t2)], [MAT.atan_reluctance()],
                         quad_order=2)
    solver.verbose = False
    rhs = solver.compute_source_rhs([3e6 * 0.8])
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    mats = []
    for tag, rel in ((M.TAG_COIL_1, S.ConstantReluctance(0.25e7 / np.pi)), (M.TAG_IRON, MAT.atan_reluctance()),
                     (M.TAG_AIR, S.ConstantReluctance(0.25e7 / np.pi))):
        e = msh.domain_elements(tag)
        mats.append(dict(cells=msh.cells[e], glob_ids=msh.elem_edges[e], orientations=msh.orientations[e],
                         reluctance=rel))
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, w, q, dphi, curls)
    K, _, _ = O.compute_stiffness_and_jacobi_matrix_c(np.zeros(msh.num_dofs))
    K = csr_array(K)
    for gauge in (False, True):
        x = solver.solve_lin([3e6 * 0.8], apply_gauge=gauge)
        mask = solver.make_boundary_mask()
        if gauge:
            mask[msh.get_cotree_dofs()[0]] = False
        Kf = K[mask, :][:, mask]
        r = Kf @ x[mask] - rhs[mask]
        assert solver.last_exit_code == 0 and not x[~mask].any()
        assert np.linalg.norm(r) <= 1.01e-5 * np.linalg.norm(rhs[mask])
