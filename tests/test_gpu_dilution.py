"""Diluted steel on the device (``compute_K_dK_Hcurl_red_dil`` path) against the reference's
golden vectors and the CPU oracle, and the diluted reduced solver end to end.

Bars as for the plain kernels: CSR structure identical, float64 values within 1e-12 of the
per-entry term-magnitude scale, vectors within 1e-12 of their max, converged fields at
probes within 1e-8."""

import numpy as np
import pytest
from scipy.sparse import csr_array

import snoopy_b200 as S
from helpers import assert_csr_close, csr_from, golden_materials, rel_max, scale_csr
from snoopy_b200 import finite_element as FE
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu

NU0 = 0.25 / np.pi * 1e7


def _dilution_from(coef):
    d = MAT.Dilution(0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0)
    d.c_num, d.m_num, d.c_den, d.m_den = (float(v) for v in coef)
    return d


def _iron_dilution(mag_type=1):
    """Iron fraction varying over the window-frame yoke's z extent [-0.25, 0.25]."""
    return MAT.Dilution(0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, z_pos=-0.25, z_len=0.5, mag_type=mag_type)


def test_diluted_curlcurl_golden(golden, oracle_mod):
    from snoopy_b200 import fem_c

    g = golden
    n = int(g["num_dofs"])
    el = g["iron"]
    rel = golden_materials(g)[0]
    dil = _dilution_from(g["dil_coef"])
    geo = (g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"])
    K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(
        *geo, g["phi"], g["d_phi"], g["orientations"][el], g["x"], g["B_s"], rel, dil, g["q"], g["w"], n, 6)
    sc = {}
    ti, tj, _, _, _ = oracle_mod.curl_curl_triplets(*geo, g["d_phi"], g["orientations"][el], g["x"], g["B_s"], rel,
                                                   g["q"], g["w"], n, 6, scales=sc, phi=g["phi"], dilution=dil)
    assert_csr_close(K, csr_from(g, "cc_iron_dil_K", n), 1e-12, scale_csr(ti, tj, sc["K"], n))
    assert_csr_close(dK, csr_from(g, "cc_iron_dil_dK", n), 1e-12, scale_csr(ti, tj, sc["dK"], n))
    assert rel_max(rhs, g["cc_iron_dil_rhs"]) < 1e-12
    # without a source field the plain kernel runs (the reference's air branch)
    K2, dK2, rhs2 = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(
        *geo, g["phi"], g["d_phi"], g["orientations"][el], g["x"], np.zeros((0, 3)), rel, dil, g["q"], g["w"], n, 6)
    sc2 = {}
    ti, tj, _, _, _ = oracle_mod.curl_curl_triplets(*geo, g["d_phi"], g["orientations"][el], g["x"], np.zeros((0, 3)),
                                                   rel, g["q"], g["w"], n, 6, scales=sc2)
    assert_csr_close(K2, csr_from(g, "cc_iron_plain_K", n), 1e-12, scale_csr(ti, tj, sc2["K"], n))
    assert_csr_close(dK2, csr_from(g, "cc_iron_plain_dK", n), 1e-12, scale_csr(ti, tj, sc2["dK"], n))
    assert not rhs2.any()


@pytest.mark.parametrize("order,mag_type", [(2, 1), (3, 3), (1, 1)])
def test_diluted_curlcurl_orders(oracle_mod, order, mag_type):
    """4-, 5- and 1-point rules (compile-time and runtime point counts), both magnet types."""
    from snoopy_b200 import fem_c

    msh = M.window_frame_mesh(40000 if order == 2 else 8000, jitter=0.2, seed=10 + order)
    w, q = FE.quadrature_rule(order)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    rng = np.random.default_rng(order)
    x = rng.normal(0, 3e-3, msh.num_dofs)
    n = msh.num_dofs
    el = msh.domain_elements(M.TAG_IRON)
    bs = rng.normal(0, 1.0, (len(el) * len(w), 3))
    rel = MAT.atan_reluctance()
    dil = _iron_dilution(mag_type)
    geo = (msh.nodes, msh.cells[el], msh.elem_edges[el], curls)
    K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(*geo, phi, dphi, msh.orientations[el], x,
                                                                             bs, rel, dil, q, w, n, 6)
    sc = {}
    ti, tj, vK, vdK, rr = oracle_mod.curl_curl_triplets(*geo, dphi, msh.orientations[el], x, bs, rel, q, w, n, 6,
                                                        scales=sc, phi=phi, dilution=dil)
    assert_csr_close(K, csr_array((vK, (ti, tj)), shape=(n, n)), 1e-12, scale_csr(ti, tj, sc["K"], n))
    assert_csr_close(dK, csr_array((vdK, (ti, tj)), shape=(n, n)), 1e-12, scale_csr(ti, tj, sc["dK"], n))
    assert rel_max(rhs, rr) < 1e-12


def _diluted_problem(ntet=6000, seed=7, mag_type=1):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    g = msh.geometry
    coils = g.coils()
    rel = MAT.atan_reluctance()
    dil = _iron_dilution(mag_type)
    solver = S.RedMVPSolverDiluted(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], [dil], max_newton_iterations=50,
                                   quad_order=2)
    solver.verbose = False
    return msh, g, coils, rel, dil, solver


def _oracle_assembler(oracle_mod, msh, coils, rel, dil, solver):
    tb = solver.curl_curl_factory.tables(solver.quad_order)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    P = np.einsum("qi,eid->eqd", tb.phi.reshape(tb.nq, 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad) for c in coils)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel, dilution=dil),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(NU0))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls, phi=tb.phi)
    return O, [Bs, np.zeros((0, 3))], solver.make_boundary_mask()


def test_diluted_assembler_vs_oracle(oracle_mod):
    msh, g, coils, rel, dil, solver = _diluted_problem(20000, seed=3)
    A = solver.curl_curl_factory
    O, sf, mask = _oracle_assembler(oracle_mod, msh, coils, rel, dil, solver)
    x = np.random.default_rng(0).normal(0, 2e-3, msh.num_dofs)
    Kr, Jr, rr = O.compute_stiffness_and_jacobi_matrix_c(x, sf)
    K, J, r = A.compute_stiffness_and_jacobi_matrix_c(x, quad_order=2, source_fields=sf)
    sK, sJ = O.scales(x, sf)
    nd = assert_csr_close(K, Kr, 1e-12, sK, zero_pattern_diff=True)
    nd += assert_csr_close(J, Jr, 1e-12, sJ, zero_pattern_diff=True)
    assert nd <= 1e-4 * Kr.nnz
    assert rel_max(r, rr) < 1e-12


@pytest.mark.parametrize("layout", ["elem", "csr"])
def test_diluted_solver_converges_to_the_oracle_root(oracle_mod, monkeypatch, layout):
    """Device Newton to 1e-10 with the matrix-free and the CSR Jacobian: the answer is a root
    of the oracle's diluted residual, and the dilution changes the field."""
    monkeypatch.setenv("SNP_JACOBIAN", layout)
    msh, g, coils, rel, dil, solver = _diluted_problem()
    assert solver.newton_engine().jacobian_layout == layout
    O, sf, mask = _oracle_assembler(oracle_mod, msh, coils, rel, dil, solver)
    x, stats = solver.solve_to_residual(1e-10)
    assert stats["rel_res"] <= 1e-10
    K, J, rhs = O.compute_stiffness_and_jacobi_matrix_c(np.zeros(msh.num_dofs), sf)
    F0 = np.linalg.norm((-rhs)[mask])
    K, J, rhs = O.compute_stiffness_and_jacobi_matrix_c(x, sf)
    F = K @ x - rhs
    assert np.linalg.norm(F[mask]) <= 2e-10 * F0
    probes = g.aperture_probes(500)
    el, _ = msh.locate(probes)
    B = solver.evaluate_B(x, probes, el)
    plain = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=50, quad_order=2)
    plain.verbose = False
    xp, sp = plain.solve_to_residual(1e-10)
    Bp = plain.evaluate_B(xp, probes, el)
    assert rel_max(B, Bp) > 1e-4  # the dilution is applied inside the Newton loop
    # reference stopping rule (increment test) on the same problem
    xr = solver.solve(tolerance=1e-4)
    Br = solver.evaluate_B(xr, probes, el)
    assert rel_max(Br, B) < 1e-2


def test_diluted_layouts_agree():
    """Matrix-free (elem) and CSR Jacobians give the same converged field."""
    out = {}
    import os

    for layout in ("elem", "csr"):
        os.environ["SNP_JACOBIAN"] = layout
        try:
            msh, g, coils, rel, dil, solver = _diluted_problem(mag_type=3)
            x, st = solver.solve_to_residual(1e-10)
        finally:
            del os.environ["SNP_JACOBIAN"]
        probes = g.aperture_probes(500)
        el, _ = msh.locate(probes)
        out[layout] = solver.evaluate_B(x, probes, el)
    assert rel_max(out["elem"], out["csr"]) < 1e-8
