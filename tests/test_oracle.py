"""The CPU oracle (oracle/restated.c + oracle/oracle.py) against the reference.

Pins the restatement to golden vectors produced by the reference's own C kernels
(tests/golden/make_golden.py), and, where the reference library was compiled here
(oracle/_ref), to live calls on fresh inputs.
"""

import numpy as np
import pytest

import snoopy_b200 as S
from helpers import abs_contrib, assert_csr_close, assert_same_pattern, csr_from, golden_materials, rel_max
from snoopy_b200 import finite_element as FE
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M


@pytest.fixture(scope="module")
def rel(golden):
    return golden_materials(golden)[0]


@pytest.fixture(scope="module")
def perm(golden):
    return golden_materials(golden)[1]


def test_golden_inputs_regenerate(golden):
    from golden.make_golden import golden_inputs

    msh, w, q, dphi, phi, curls, x, iron, air, Bs, xn = golden_inputs()
    assert np.array_equal(msh.cells, golden["cells"])
    assert np.array_equal(msh.elem_edges, golden["glob_ids"])
    assert np.allclose(msh.nodes, golden["nodes"], rtol=0, atol=1e-15)
    assert np.array_equal(msh.orientations, golden["orientations"])


def test_pchip_matches_reference(golden, oracle_mod, rel):
    nu, dnu = oracle_mod.pchip_eval(rel, golden["pchip_B"], backend="oracle")
    assert rel_max(nu, golden["pchip_nu"]) < 1e-14
    assert rel_max(dnu, golden["pchip_dnu"]) < 1e-13
    # below the first knot (and NaN-free negative input) the law gives 0, as the reference
    assert nu[-2] == 0.0 and dnu[-2] == 0.0


def test_bspline_mu_matches_reference(golden, oracle_mod, perm):
    mu, dmu = oracle_mod.mu_eval(perm, golden["mu_H"], backend="oracle")
    np.testing.assert_array_equal(mu, golden["mu_mu"])
    np.testing.assert_allclose(dmu, golden["mu_dmu"], rtol=1e-14, atol=0)


def test_bspline_mu_agrees_with_scipy(oracle_mod):
    from scipy.interpolate import splev

    perm = MAT.atan_permeability()
    H = np.logspace(0, 6, 200)
    H = H[H > perm.H_min]
    mu, dmu = oracle_mod.mu_eval(perm, H)
    np.testing.assert_allclose(mu, splev(np.log10(H), perm.spl), rtol=1e-12)
    np.testing.assert_allclose(dmu, splev(np.log10(H), perm.spl, der=1) / H / np.log(10), rtol=1e-10, atol=1e-30)


@pytest.mark.parametrize("name", ["air", "iron_red", "iron_plain"])
def test_curlcurl_matches_reference(golden, oracle_mod, rel, name):
    g = golden
    n = int(g["num_dofs"])
    el = g["air"] if name == "air" else g["iron"]
    mat = S.ConstantReluctance(0.25 / np.pi * 1e7) if name == "air" else rel
    bs = g["B_s"] if name == "iron_red" else np.zeros((0, 3))
    ti, tj, vK, vdK, rhs = oracle_mod.curl_curl_triplets(g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"],
                                                         g["d_phi"], g["orientations"][el], g["x"], bs, mat, g["q"],
                                                         g["w"], n, 6)
    from scipy.sparse import csr_array

    K = csr_array((vK, (ti, tj)), shape=(n, n))
    dK = csr_array((vdK, (ti, tj)), shape=(n, n))
    assert_csr_close(K, csr_from(g, f"cc_{name}_K", n), 1e-13, abs_contrib(ti, tj, vK, n))
    assert_csr_close(dK, csr_from(g, f"cc_{name}_dK", n), 1e-13, abs_contrib(ti, tj, vdK, n))
    ref_rhs = g[f"cc_{name}_rhs"]
    if name == "iron_red":
        assert rel_max(rhs, ref_rhs) < 1e-13
    else:
        assert not ref_rhs.any() and not rhs.any()


def test_dilution_coefficients_match_reference(golden):
    for case, ref in zip(golden["dil_cases"], golden["dil_cases_ref"]):
        d = MAT.Dilution(*case[:10], mag_type=int(case[10]))
        np.testing.assert_allclose(d.coefficients(), ref, rtol=1e-15, atol=0)
    with pytest.raises(ValueError):
        MAT.Dilution(*golden["dil_cases"][0][:10], mag_type=2)


def test_curlcurl_diluted_matches_reference(golden, oracle_mod, rel):
    g = golden
    n = int(g["num_dofs"])
    el = g["iron"]
    dil = MAT.Dilution(0, 0, 0, 0, 0, 0, 0, 0, 0.0, 1.0)
    dil.c_num, dil.m_num, dil.c_den, dil.m_den = g["dil_coef"]
    K, dK, rhs = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(
        g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["phi"], g["d_phi"], g["orientations"][el], g["x"],
        g["B_s"], rel, dil, g["q"], g["w"], n, 6)
    assert_same_pattern(K, csr_from(g, "cc_iron_dil_K", n))
    # same operation order as the reference: bitwise apart from summation of duplicates
    assert_csr_close(K, csr_from(g, "cc_iron_dil_K", n), 1e-14, atol_rel=1e-16)
    assert_csr_close(dK, csr_from(g, "cc_iron_dil_dK", n), 1e-14, atol_rel=1e-16)
    assert rel_max(rhs, g["cc_iron_dil_rhs"]) < 1e-14
    # the dilution changes the answer (s runs from 4/3 to 35/38 over the iron)
    K0, _, _ = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl(
        g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["d_phi"], g["orientations"][el], g["x"],
        g["B_s"], rel, g["q"], g["w"], n, 6)
    assert rel_max(K.data, K0.data) > 1e-3
    # without a source field the plain kernel runs, as in the reference's air branch
    Ka, _, ra = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(
        g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["phi"], g["d_phi"], g["orientations"][el], g["x"],
        np.zeros((0, 3)), rel, dil, g["q"], g["w"], n, 6)
    assert_csr_close(Ka, csr_from(g, "cc_iron_plain_K", n), 1e-13, atol_rel=1e-15)
    assert not ra.any()


def test_rhs_red_matches_reference(golden, oracle_mod, rel):
    g = golden
    el = g["iron"]
    rhs = oracle_mod.compute_rhs_Hcurl_red_c(g["nodes"], g["cells"][el], g["glob_ids"][el], g["curls"], g["d_phi"],
                                             g["orientations"][el], g["B_s"], rel, g["x"], g["q"], g["w"],
                                             int(g["num_dofs"]), 6)
    assert rel_max(rhs, g["rhs_red"]) < 1e-13


@pytest.mark.parametrize("name", ["bspline", "const"])
def test_gradgrad_matches_reference(golden, oracle_mod, perm, name):
    g = golden
    pm = perm if name == "bspline" else S.ConstantPermeability(1.0)
    n = g["nodes"].shape[0]
    ti, tj, vK, vdK = oracle_mod.grad_grad_triplets(g["nodes"], g["cells"], g["d_phi"], g["x_nodal"], pm, g["q"], g["w"])
    from scipy.sparse import csr_array

    assert_csr_close(csr_array((vK, (ti, tj)), shape=(n, n)), csr_from(g, f"gg_{name}_K", n), 1e-13,
                     abs_contrib(ti, tj, vK, n))
    assert_csr_close(csr_array((vdK, (ti, tj)), shape=(n, n)), csr_from(g, f"gg_{name}_dK", n), 1e-12,
                     abs_contrib(ti, tj, vdK, n))


def test_b_hcurl_matches_reference(golden, oracle_mod):
    g = golden
    pts, B = oracle_mod.compute_B_Hcurl(g["nodes"], g["cells"], g["glob_ids"], g["curls"], g["phi"], g["d_phi"],
                                        g["orientations"], g["x"], g["q"], g["w"], int(g["num_dofs"]), 6)
    assert rel_max(pts, g["bq_points"]) < 1e-15
    assert rel_max(B, g["bq_B"]) < 1e-13


def test_biot_savart_matches_reference(golden, oracle_mod):
    g = golden
    B = oracle_mod.compute_B_line_segs_cpp(g["bs_src"], g["bs_tar"], float(g["bs_current"]), float(g["bs_rad"]))
    ref = g["bs_B"]
    # a target exactly on a filament gives 0/0 in the reference's inner-conductor branch
    nan = np.isnan(ref)
    assert nan.any() and np.array_equal(np.isnan(B), nan)
    assert rel_max(B[~nan], ref[~nan]) < 1e-14


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference C not compiled here")
def test_restatement_vs_live_reference(oracle_mod, rel):
    """Fresh seeded inputs through both backends (reduced kernel, 5-point rule with a negative weight)."""
    msh = M.window_frame_mesh(3000, jitter=0.2, seed=99)
    w, q = FE.quadrature_rule(3)
    dphi = FE.evaluate_basis_derivative(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    rng = np.random.default_rng(5)
    x = rng.normal(0, 5e-3, msh.num_dofs)
    el = msh.domain_elements(M.TAG_IRON)
    Bs = rng.normal(0, 1.0, (len(el) * len(w), 3))
    n = msh.num_dofs
    a = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl(msh.nodes, msh.cells[el], msh.elem_edges[el], curls,
                                                                 dphi, msh.orientations[el], x, Bs, rel, q, w, n, 6)
    b = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl(msh.nodes, msh.cells[el], msh.elem_edges[el], curls,
                                                                 dphi, msh.orientations[el], x, Bs, rel, q, w, n, 6,
                                                                 backend="ref")
    assert_same_pattern(a[0], b[0])
    assert_csr_close(a[0], b[0], 1e-12, atol_rel=1e-15)
    assert_csr_close(a[1], b[1], 1e-12, atol_rel=1e-15)
    assert rel_max(a[2], b[2]) < 1e-13


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference C not compiled here")
def test_diluted_restatement_vs_live_reference(oracle_mod, rel):
    """Diluted reduced kernel on fresh inputs, magnet type 3, 5-point rule."""
    msh = M.window_frame_mesh(3000, jitter=0.2, seed=98)
    w, q = FE.quadrature_rule(3)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    rng = np.random.default_rng(6)
    x = rng.normal(0, 5e-3, msh.num_dofs)
    el = msh.domain_elements(M.TAG_IRON)
    Bs = rng.normal(0, 1.0, (len(el) * len(w), 3))
    dil = MAT.Dilution(0.01, 0.28, 0.33, 0.70, 0.03, 0.42, 0.47, 0.85, -0.3, 0.6, mag_type=3)
    n = msh.num_dofs
    args = (msh.nodes, msh.cells[el], msh.elem_edges[el], curls, phi, dphi, msh.orientations[el], x, Bs, rel, dil, q,
            w, n, 6)
    a = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(*args)
    b = oracle_mod.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(*args, backend="ref")
    assert_same_pattern(a[0], b[0])
    assert_csr_close(a[0], b[0], 1e-14, atol_rel=1e-16)
    assert_csr_close(a[1], b[1], 1e-14, atol_rel=1e-16)
    assert rel_max(a[2], b[2]) < 1e-14


def test_mlp_oracle_backward_matches_finite_differences():
    """The MLP oracle's own backward pass against central differences of its forward pass
    (float64, no BF16 rounding): the oracle that checks the device gradients is itself pinned."""
    import mlp_oracle as MO

    rng = np.random.default_rng(0)
    sizes = [9, 8, 8, 4]
    W = [rng.normal(0, 0.5, (sizes[i + 1], sizes[i])) for i in range(3)]
    b = [rng.normal(0, 0.1, sizes[i + 1]) for i in range(3)]
    X = rng.normal(0, 1, (5, 9))
    T = rng.normal(0, 1, (5, 4))
    grads, _ = MO.backward(W, b, X, T)

    def loss():
        Y, _ = MO.forward(W, b, X)
        return float(np.mean((Y - T) ** 2))

    h = 1e-6
    for l in range(3):
        for (i, j) in [(0, 0), (1, 3), (sizes[l + 1] - 1, sizes[l] - 1)]:
            W[l][i, j] += h
            lp = loss()
            W[l][i, j] -= 2 * h
            lm = loss()
            W[l][i, j] += h
            assert abs((lp - lm) / (2 * h) - grads[l][0][i, j]) < 1e-7
        b[l][0] += h
        lp = loss()
        b[l][0] -= 2 * h
        lm = loss()
        b[l][0] += h
        assert abs((lp - lm) / (2 * h) - grads[l][1][0]) < 1e-7


def test_bf16_rounding_is_nearest_even():
    import mlp_oracle as MO

    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159265], dtype=np.float32)
    r = MO.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie between 1 and 1 + 2^-7 goes to even (1.0)
    assert r[2] == 1.0 + 2 ** -7        # above the tie rounds up
    assert r[3] == -2.5
    assert abs(r[4] - 3.140625) < 1e-12


def test_block_jacobi_newton_on_the_oracle(oracle_mod):
    """The oracle's residual Newton with the product's block partition (edges sharing their
    lower node) reaches the point-Jacobi field in far fewer CG iterations: the preconditioner
    the device's residual mode runs, restated on scipy's CG."""
    import snoopy_b200 as S
    from snoopy_b200 import finite_element as fe
    from snoopy_b200 import materials as MAT
    from snoopy_b200 import mesh as M
    from snoopy_b200.newton import dof_blocks

    msh = M.window_frame_mesh(6000, jitter=0.15, seed=7)
    n = msh.num_dofs
    rel = MAT.atan_reluctance()
    w, q = fe.quadrature_rule(2)
    dphi = fe.evaluate_basis_derivative(q)
    curls, n_orient = fe.curl_edge_basis_functions(q)
    phi = fe.evaluate_basis(q)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    P = np.einsum("qi,eid->eqd", phi.reshape(len(w), 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad) for c in msh.geometry.coils())
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(0.25 / np.pi * 1e7))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, n, w, q, dphi, curls)
    mask = np.ones(n, dtype=bool)
    mask[np.asarray(msh.get_edge_boundary_dofs()) - 1] = False
    sf = [Bs, np.zeros((0, 3))]
    kw = dict(rtol=1e-8, cg_rtol=0.1, forcing="ew", line_search="energy", max_newton_iterations=40)
    xj, sj = oracle_mod.newton_residual(O, mask, sf, **kw)
    xb, sb = oracle_mod.newton_residual(O, mask, sf, blocks=dof_blocks(msh.edges[:, 0], mask), **kw)
    assert sj["rel_res"] <= 1e-8 and sb["rel_res"] <= 1e-8
    assert sum(sb["cg"]) < 0.75 * sum(sj["cg"]), (sum(sb["cg"]), sum(sj["cg"]))
    Bj = oracle_mod.element_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, curls, n_orient, dphi, xj)
    Bb = oracle_mod.element_B(msh.nodes, msh.cells, msh.elem_edges, msh.orientations, curls, n_orient, dphi, xb)
    assert np.abs(Bb - Bj).max() <= 1e-6 * np.abs(Bj).max()
