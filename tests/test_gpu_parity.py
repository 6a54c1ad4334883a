"""GPU kernels (through the C ABI) against the CPU oracle and the reference's golden vectors.

Bars: CSR structure identical (row pointers and column indices); float64 values within
1e-12 relative to the entry, or to the sum of absolute element contributions where those
cancel (tests/helpers.py); vectors within 1e-12 relative to their max.
"""

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


@pytest.fixture(scope="module")
def rel(golden):
    return golden_materials(golden)[0]


@pytest.fixture(scope="module")
def perm(golden):
    return golden_materials(golden)[1]


@pytest.fixture(scope="module")
def fem_c():
    from snoopy_b200 import fem_c as F

    return F


@pytest.mark.parametrize("name", ["air", "iron_red", "iron_plain"])
def test_curlcurl_golden(golden, fem_c, oracle_mod, rel, name):
    g = golden
    n = int(g["num_dofs"])
    el = g["air"] if name == "air" else g["iron"]
    mat = S.ConstantReluctance(NU0) if name == "air" else rel
    bs = g["B_s"] if name == "iron_red" else np.zeros((0, 3))
    args = (g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["d_phi"], g["orientations"][el], g["x"], bs, mat,
            g["q"], g["w"], n, 6)
    K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(*args)
    sc = {}
    ti, tj, vK, vdK, _ = oracle_mod.curl_curl_triplets(*args, scales=sc)
    assert_csr_close(K, csr_from(g, f"cc_{name}_K", n), 1e-12, scale_csr(ti, tj, sc["K"], n))
    assert_csr_close(dK, csr_from(g, f"cc_{name}_dK", n), 1e-12, scale_csr(ti, tj, sc["dK"], n))
    if name == "iron_red":
        assert rel_max(rhs, g[f"cc_{name}_rhs"]) < 1e-12
    else:
        assert not rhs.any()


@pytest.mark.parametrize("name", ["bspline", "const"])
def test_gradgrad_golden(golden, fem_c, oracle_mod, perm, name):
    g = golden
    pm = perm if name == "bspline" else S.ConstantPermeability(1.0)
    nn = g["nodes"].shape[0]
    K, dK = fem_c.compute_stiffness_and_jacobi_matrix(g["nodes"], g["cells"], g["d_phi"], g["x_nodal"], pm, g["q"], g["w"])
    sc = {}
    ti, tj, vK, vdK = oracle_mod.grad_grad_triplets(g["nodes"], g["cells"], g["d_phi"], g["x_nodal"], pm, g["q"], g["w"],
                                                    scales=sc)
    assert_csr_close(K, csr_from(g, f"gg_{name}_K", nn), 1e-12, scale_csr(ti, tj, sc["K"], nn))
    assert_csr_close(dK, csr_from(g, f"gg_{name}_dK", nn), 1e-12, scale_csr(ti, tj, sc["dK"], nn))


def test_rhs_red_golden(golden, fem_c, rel):
    g = golden
    el = g["iron"]
    rhs = fem_c.compute_rhs_Hcurl_red_c(g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["d_phi"],
                                        g["orientations"][el], g["B_s"], rel, g["x"], g["q"], g["w"], int(g["num_dofs"]), 6)
    assert rel_max(rhs, g["rhs_red"]) < 1e-12


def test_b_hcurl_golden(golden, fem_c):
    g = golden
    pts, B = fem_c.compute_B_Hcurl(g["nodes"], g["cells"], g["glob_ids"], g["curls"], g["phi"], g["d_phi"],
                                   g["orientations"], g["x"], g["q"], g["w"], int(g["num_dofs"]), 6)
    assert rel_max(pts, g["bq_points"]) < 1e-14
    assert rel_max(B, g["bq_B"]) < 1e-12


def test_biot_savart_golden(golden, fem_c):
    g = golden
    B = fem_c.compute_B_line_segs_cpp(g["bs_src"], g["bs_tar"], float(g["bs_current"]), float(g["bs_rad"]))
    nan = np.isnan(g["bs_B"])
    assert np.array_equal(np.isnan(B), nan)
    assert rel_max(B[~nan], g["bs_B"][~nan]) < 1e-13
    assert fem_c.compute_B_line_segs_cpp(np.zeros((3, 5)), g["bs_tar"], 1.0, 0.1) == -1


@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_curlcurl_orders_and_sizes(fem_c, oracle_mod, rel, order):
    """Quadrature orders 1-4 (1, 4, 5 and 27 points), reduced and plain, on a 40k-tet mesh."""
    msh = M.window_frame_mesh(40000 if order == 2 else 8000, jitter=0.2, seed=order)
    w, q = FE.quadrature_rule(order)
    dphi = FE.evaluate_basis_derivative(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    rng = np.random.default_rng(order)
    x = rng.normal(0, 3e-3, msh.num_dofs)
    n = msh.num_dofs
    for tag, bs_on in ((M.TAG_IRON, True), (M.TAG_AIR, False)):
        el = msh.domain_elements(tag)
        bs = rng.normal(0, 1.0, (len(el) * len(w), 3)) if bs_on else np.zeros((0, 3))
        mat = rel if tag == M.TAG_IRON else S.ConstantReluctance(NU0)
        args = (msh.nodes, msh.cells[el], msh.elem_edges[el], curls, dphi, msh.orientations[el], x, bs, mat, q, w, n, 6)
        K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(*args)
        sc = {}
        ti, tj, vK, vdK, rr = oracle_mod.curl_curl_triplets(*args, scales=sc)
        assert_csr_close(K, csr_array((vK, (ti, tj)), shape=(n, n)), 1e-12, scale_csr(ti, tj, sc["K"], n))
        assert_csr_close(dK, csr_array((vdK, (ti, tj)), shape=(n, n)), 1e-12, scale_csr(ti, tj, sc["dK"], n))
        if bs_on:
            assert rel_max(rhs, rr) < 1e-12


def test_curlcurl_zero_state_and_empty(fem_c, oracle_mod, rel):
    """x = 0: no dK without a source field (|B| < 1e-14 branch); an empty element list."""
    msh = M.window_frame_mesh(3000, jitter=0.1, seed=1)
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    el = msh.domain_elements(M.TAG_IRON)
    n = msh.num_dofs
    K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(msh.nodes, msh.cells[el], msh.elem_edges[el], curls,
                                                                     dphi, msh.orientations[el], np.zeros(n),
                                                                     np.zeros((0, 3)), rel, q, w, n, 6)
    assert K.nnz > 0 and dK.nnz == K.nnz and not dK.data.any()
    K0, dK0, rhs0 = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(msh.nodes, msh.cells[:0], msh.elem_edges[:0],
                                                                        curls, dphi, msh.orientations[:0], np.zeros(n),
                                                                        np.zeros((0, 3)), rel, q, w, n, 6)
    assert K0.nnz == 0 and dK0.nnz == 0 and not rhs0.any()


def _two_material_problem(ntet=20000, seed=3):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    rel = MAT.atan_reluctance()
    return msh, rel


def test_assembler_vs_oracle_assembler(oracle_mod):
    msh, rel = _two_material_problem()
    A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [rel, S.ConstantReluctance(NU0)])
    tb = A.tables(2)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    rng = np.random.default_rng(0)
    x = rng.normal(0, 2e-3, msh.num_dofs)
    Bs = rng.normal(0, 0.5, (len(iron) * tb.nq, 3))
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron], reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(NU0))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls)
    Kr, Jr, rr = O.compute_stiffness_and_jacobi_matrix_c(x, [Bs, np.zeros((0, 3))])
    K, J, r = A.compute_stiffness_and_jacobi_matrix_c(x, quad_order=2, source_fields=[Bs, np.zeros((0, 3))])
    sK, sJ = O.scales(x, [Bs, np.zeros((0, 3))])
    # exact zeros are dropped on both sides: entries that one side computes as an exact 0 and
    # the other as a rounding residue may differ in presence (jittered nodes keep this rare)
    nd = assert_csr_close(K, Kr, 1e-12, sK, zero_pattern_diff=True)
    nd += assert_csr_close(J, Jr, 1e-12, sJ, zero_pattern_diff=True)
    assert nd <= 1e-4 * Kr.nnz
    assert rel_max(r, rr) < 1e-12
    assert np.array_equal(A.global_ids[0], msh.elem_edges[iron] + 1)


def test_spmv_and_pcg_match_scipy(oracle_mod):
    """Masked SpMV and Jacobi-PCG with scipy cg's stopping rule against scipy on the same J."""
    import ctypes

    from scipy.sparse import diags
    from scipy.sparse.linalg import cg

    from snoopy_b200 import _lib
    from snoopy_b200.device import upload, zeros

    msh, rel = _two_material_problem(8000, seed=5)
    A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [rel, S.ConstantReluctance(NU0)])
    rng = np.random.default_rng(1)
    x = rng.normal(0, 1e-3, msh.num_dofs)
    out = A.assemble_device(x, 2, (), K=False, J=True, rhs=False)
    pat = out["pattern"]
    J = pat.to_scipy(out["J"])
    mask = np.ones(msh.num_dofs, bool)
    mask[msh.get_edge_boundary_dofs() - 1] = False
    fm = upload(mask.astype(np.uint8), np.uint8)
    y = zeros(msh.num_dofs)
    xv = upload(x, np.float64)
    _lib.call("snp_spmv", msh.num_dofs, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["J"]), _lib.ptr(fm),
              _lib.ptr(xv), _lib.ptr(y), _lib.stream_ptr())
    Jc = J[mask, :][:, mask]
    ref = np.zeros(msh.num_dofs)
    ref[mask] = Jc @ x[mask]
    assert rel_max(y.cpu().numpy()[: msh.num_dofs], ref) < 1e-13
    # a consistent right-hand side (J is singular: gradients lie in its kernel)
    b = np.zeros(msh.num_dofs)
    b[mask] = Jc @ rng.normal(0, 1.0, int(mask.sum()))
    its = ctypes.c_int64()
    res = ctypes.c_double()
    xs = zeros(msh.num_dofs)
    b_d = upload(b, np.float64)
    _lib.call("snp_pcg", msh.num_dofs, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["J"]), _lib.ptr(fm),
              _lib.ptr(b_d), _lib.ptr(xs), 1e-8, 0.0, -1, ctypes.byref(its), ctypes.byref(res),
              _lib.stream_ptr())
    count = [0]

    def cb(_):
        count[0] += 1

    xr, info = cg(Jc, b[mask], rtol=1e-8, atol=0.0, M=diags(1.0 / Jc.diagonal()), callback=cb)
    assert info == 0
    assert abs(its.value - count[0]) <= max(2, count[0] // 50)
    got = xs.cpu().numpy()[: msh.num_dofs]
    assert not got[~mask].any()
    r_gpu = np.linalg.norm(b[mask] - Jc @ got[mask])
    assert r_gpu <= 1e-8 * np.linalg.norm(b[mask]) * 1.01
    assert res.value <= 1e-8 * np.linalg.norm(b[mask])


def _red_setup(ntet, seed=7, quad_order=2):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    g = msh.geometry
    coils = g.coils()
    rel = MAT.atan_reluctance()
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=50,
                            quad_order=quad_order)
    solver.verbose = False
    return msh, g, coils, rel, solver


def _oracle_red(oracle_mod, msh, coils, rel, solver):
    tb = solver.curl_curl_factory.tables(solver.quad_order)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    P = np.einsum("qi,eid->eqd", tb.phi.reshape(tb.nq, 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad) for c in coils)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron], reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(NU0))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls)
    return O, [Bs, np.zeros((0, 3))], solver.make_boundary_mask()


def test_source_fields_match_oracle(oracle_mod):
    msh, g, coils, rel, solver = _red_setup(6000)
    O, sf, mask = _oracle_red(oracle_mod, msh, coils, rel, solver)
    got = solver.compute_source_fields()[0].cpu().numpy().reshape(-1, 3)
    assert rel_max(got, sf[0]) < 1e-12


def test_red_mvp_reference_semantics(oracle_mod):
    """RedMVPSolver.solve (increment test, CG atol=tol) vs the oracle's restatement of it."""
    msh, g, coils, rel, solver = _red_setup(6000)
    O, sf, mask = _oracle_red(oracle_mod, msh, coils, rel, solver)
    solver.max_newton_iterations = 25
    x = solver.solve(tolerance=1e-4)
    xr, st = oracle_mod.newton_reference(O, mask, sf, tolerance=1e-4)
    assert abs(solver.last_stats["newton_iterations"] - st["newton"]) <= 1
    probes = g.aperture_probes(200)
    el, _ = msh.locate(probes)
    Bg = solver.curl_curl_factory.compute_B_at_points(x, probes, el)
    Bo = solver.curl_curl_factory.compute_B_at_points(xr, probes, el)
    # both stop on the loose reference tolerances, so they agree to that level
    assert rel_max(Bg, Bo) < 1e-2


def test_red_mvp_residual_parity_at_probes(oracle_mod):
    """Newton to a relative residual of 1e-10 on both sides; B at probes within 1e-8."""
    msh, g, coils, rel, solver = _red_setup(6000)
    O, sf, mask = _oracle_red(oracle_mod, msh, coils, rel, solver)
    x, stats = solver.solve_to_residual(1e-10)
    xr, st = oracle_mod.newton_residual(O, mask, sf, rtol=1e-10, cg_rtol=1e-10)
    assert stats["rel_res"] <= 1e-10 and st["rel_res"] <= 1e-10
    # residual of the GPU answer measured by the oracle
    K, J, rhs = O.compute_stiffness_and_jacobi_matrix_c(x, sf)
    F = K @ x - rhs
    assert np.linalg.norm(F[mask]) <= 2e-10 * st["res"][0]
    probes = g.aperture_probes(1000)
    el, _ = msh.locate(probes)
    A = solver.curl_curl_factory
    Bg = solver.evaluate_B(x, probes, el)
    Bo = A.compute_B_at_points(xr, probes, el) + sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), probes, c.current, c.rad) for c in coils)
    err = np.linalg.norm(Bg - Bo, axis=1) / np.linalg.norm(Bo, axis=1).max()
    assert err.max() < 1e-8, err.max()


def test_mixed_precision_reaches_fp64_answer(oracle_mod):
    msh, g, coils, rel, solver = _red_setup(6000)
    x64, s64 = solver.solve_to_residual(1e-8)
    x32, s32 = solver.solve_to_residual(1e-8, precision="mixed")
    assert s32["rel_res"] <= 1e-8
    probes = g.aperture_probes(300)
    el, _ = msh.locate(probes)
    A = solver.curl_curl_factory
    B64 = A.compute_B_at_points(x64, probes, el)
    B32 = A.compute_B_at_points(x32, probes, el)
    assert rel_max(B32, B64) < 1e-5


def test_gradgrad_assembler_and_laplace(oracle_mod):
    msh = M.window_frame_mesh(8000, jitter=0.1, seed=2, coils=True)
    perm = MAT.atan_permeability()
    tags = [M.TAG_COIL_1, M.TAG_IRON]
    G = S.GradGradAssembler(msh, tags)
    rng = np.random.default_rng(3)
    xn = rng.normal(0, 30.0, msh.num_nodes)
    K, J = G.compute_stiffness_and_jacobi_matrix_c(xn, [S.ConstantPermeability(1.0), perm], quad_order=2)
    w, q = FE.quadrature_rule(2)
    O = oracle_mod.OracleGradGradAssembler(msh.nodes, [msh.cells[msh.domain_elements(t)] for t in tags], w, q,
                                           FE.evaluate_basis_derivative(q))
    Kr, Jr = O.compute_stiffness_and_jacobi_matrix_c(xn, [S.ConstantPermeability(1.0), perm])
    sK, sJ = O.scales(xn, [S.ConstantPermeability(1.0), perm])
    # axis-aligned tets on the unjittered material planes give gradients that are exactly
    # orthogonal: exact zeros on one side may be rounding residues on the other
    nd = assert_csr_close(K, Kr, 1e-12, sK, zero_pattern_diff=True)
    nd += assert_csr_close(J, Jr, 1e-12, sJ, zero_pattern_diff=True)
    assert nd <= 0.01 * Kr.nnz
    t1, t2 = msh.coil_terminals[M.TAG_COIL_1]
    L = S.LaplaceSubdomainSolver(msh, M.TAG_COIL_1, (t1, t2), quad_order=2)
    phi = L.solve(1.0)
    term = np.concatenate([t1, t2])
    ref = oracle_mod.laplace_subdomain_solve(msh.nodes, msh.cells[msh.domain_elements(M.TAG_COIL_1)], term,
                                             msh.domain_nodes_mask(M.TAG_COIL_1), 1.0, t1, t2, w, q,
                                             FE.evaluate_basis_derivative(q))
    assert rel_max(phi, ref) < 1e-9


def test_mvp_solver_total_potential(oracle_mod):
    """MVPSolver: Laplace coil potential -> source rhs -> Newton, against the oracle chain.

    A conductor bar through the whole box in an iron ring: the terminals lie on the Dirichlet
    boundary, so the source current closes through it and the problem is consistent (with
    terminal faces inside the domain the current is open and the rhs has a component in the
    curl-curl null space that no solve removes).  Checked in the reference's increment mode and
    to a 1e-9 relative residual.
    """
    msh = M.bar_conductor_mesh(12000)
    rel = MAT.atan_reluctance()
    t1, t2 = msh.coil_terminals[M.TAG_COIL_1]
    Phi = 3e6 * 0.8  # grad phi = 3e6 along the 0.8 m bar: J = 3 A/mm^2 in the reference's convention
    solver = S.MVPSolver(msh, [M.TAG_COIL_1], [M.TAG_IRON], [M.TAG_AIR], [(t1, t2)], [rel], quad_order=2,
                         max_newton_iterations=60)
    solver.verbose = False
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    # oracle chain: Laplace solve, rhs by a numpy statement of compute_rhs_electric_potential
    el = msh.domain_elements(M.TAG_COIL_1)
    phi = oracle_mod.laplace_subdomain_solve(msh.nodes, msh.cells[el], np.concatenate([t1, t2]),
                                             msh.domain_nodes_mask(M.TAG_COIL_1), Phi, t1, t2, w, q, dphi)
    X = msh.nodes[msh.cells[el]]
    Jm = np.einsum("eid,il->edl", X, dphi[0])
    Ji = np.linalg.inv(Jm)
    det = np.linalg.det(Jm)
    G = np.einsum("eld,el->ed", Ji, np.einsum("il,ei->el", dphi[0], phi[msh.cells[el]]))
    s = FE.orientation_signs(msh.orientations[el])
    wq = np.einsum("eld,qjl->eqjd", Ji, FE.edge_basis_functions(q)) * s[:, None, :, None]
    rhs = np.zeros(msh.num_dofs)
    np.add.at(rhs, msh.elem_edges[el].reshape(-1), np.einsum("eqjd,ed,q,e->ej", wq, G, w, det).reshape(-1))
    assert rel_max(solver.compute_source_rhs([Phi]), rhs) < 1e-9
    mats = []
    for tag in (M.TAG_COIL_1, M.TAG_IRON, M.TAG_AIR):
        e = msh.domain_elements(tag)
        mats.append(dict(cells=msh.cells[e], glob_ids=msh.elem_edges[e], orientations=msh.orientations[e],
                         reluctance=rel if tag == M.TAG_IRON else S.ConstantReluctance(NU0)))

    class WithRhs(oracle_mod.OracleCurlCurlAssembler):
        def compute_stiffness_and_jacobi_matrix_c(self, x, source_fields=()):
            K, J, r = super().compute_stiffness_and_jacobi_matrix_c(x, source_fields)
            return K, J, r + rhs

    O = WithRhs(msh.nodes, mats, msh.num_dofs, w, q, dphi, curls)
    mask = solver.make_boundary_mask()
    cen = msh.element_centroids()
    probe = msh.domain_elements(M.TAG_IRON)[::5]
    A = solver.curl_curl_factory
    # reference semantics (increment test 1e-4, inexact CG): both stop at that level
    x0 = solver.solve_nonlin([Phi], tolerance=1e-4)
    xr0, st0 = oracle_mod.newton_reference(O, mask, (), tolerance=1e-4, max_newton_iterations=60)
    assert abs(solver.last_stats["newton_iterations"] - st0["newton"]) <= 2
    B0 = A.compute_B_at_points(xr0, cen[probe], probe)
    assert rel_max(A.compute_B_at_points(x0, cen[probe], probe), B0) < 1e-3
    # residual criterion on both sides
    x, stats = solver.solve_to_residual([Phi], rtol=1e-9, max_newton=60)
    assert stats["rel_res"] <= 1e-9
    xr, st = oracle_mod.newton_residual(O, mask, (), rtol=1e-9, cg_rtol=1e-10, max_newton_iterations=60)
    Bo = A.compute_B_at_points(xr, cen[probe], probe)
    assert 0.5 < np.linalg.norm(Bo, axis=1).max() < 3.0  # tesla, saturating iron
    assert rel_max(A.compute_B_at_points(x, cen[probe], probe), Bo) < 1e-7


def test_error_statuses():
    """Failures come back as statuses with messages; nothing faults the device."""
    import ctypes

    from snoopy_b200 import _lib
    from snoopy_b200.device import Pattern, upload, zeros

    bad = upload(np.array([[0, 1, 2, 3, 4, 99]]), np.int32)
    with pytest.raises(_lib.SnpError) as e:
        Pattern(bad, 1, 6, 10)
    assert e.value.status == 1 and "outside" in str(e.value)
    msh, g, coils, rel, solver = _red_setup(3000)
    eng = solver.newton_engine()
    x0 = np.zeros(msh.num_dofs)
    x0[int(np.flatnonzero(solver.make_boundary_mask())[0])] = np.nan
    with pytest.raises(_lib.SnpError) as e:
        eng.solve(x0, mode=1, tol=1e-8)
    assert e.value.status in (4, 5)
    # maxiter = 1 on a real system: NOT_CONVERGED from snp_pcg
    out = solver.curl_curl_factory.assemble_device(np.zeros(msh.num_dofs), 2, solver.compute_source_fields(), K=False,
                                                   J=True, rhs=True)
    pat = out["pattern"]
    fm = upload(solver.make_boundary_mask().astype(np.uint8), np.uint8)
    its = ctypes.c_int64()
    res = ctypes.c_double()
    x1 = zeros(msh.num_dofs)
    rc = _lib.load().snp_pcg(msh.num_dofs, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["J"]),
                             _lib.ptr(fm), _lib.ptr(out["rhs"]), _lib.ptr(x1), 1e-12, 0.0, 1,
                             ctypes.byref(its), ctypes.byref(res), _lib.stream_ptr())
    assert rc == 3 and its.value == 1
    # a zero Jacobian diagonal on a free row
    Jz = out["J"].clone()
    Jz[pat.diag_pos[int(np.flatnonzero(solver.make_boundary_mask())[0])].long()] = 0.0
    x2 = zeros(msh.num_dofs)
    rc = _lib.load().snp_pcg(msh.num_dofs, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(Jz), _lib.ptr(fm),
                             _lib.ptr(out["rhs"]), _lib.ptr(x2), 1e-8, 0.0, 10, ctypes.byref(its),
                             ctypes.byref(res), _lib.stream_ptr())
    assert rc == 5
