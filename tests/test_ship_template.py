"""SHiP template 1 meshed without gmsh: the quarter model's geometry, materials, boundary and
coils (CPU), checked against their definitions."""

import json

import numpy as np
import pytest

from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M
from snoopy_b200 import ship


def template_parameters(X_mgap=(0.0, 0.0)):
    """One design of the template (its own numbers, in the SHiP table's columns)."""
    return {"yoke_type": ["Mag1"], "coil_material": ["cu_test.json"], "max_turns": [10], "J_tar(A/mm2)": [3.0],
            "NI(A)": [4000.0], "coil_diam(mm)": [9.0], "insulation(mm)": [0.5], "yoke_spacer(mm)": [5.0],
            "material": ["iron_test.json"], "field_density": [4], "delta_x(m)": [0.4], "delta_y(m)": [0.4],
            "delta_z(m)": [0.5], "Z_pos(m)": [-2.0], "Z_len(m)": [4.0], "Xmgap1(m)": [X_mgap[0]],
            "Xcore1(m)": [0.25], "Xvoid1(m)": [0.31], "Xyoke1(m)": [1.2], "Xmgap2(m)": [X_mgap[1]],
            "Xcore2(m)": [0.28], "Xvoid2(m)": [0.34], "Xyoke2(m)": [1.3], "Ycore1(m)": [0.2], "Yvoid1(m)": [0.2],
            "Yyoke1(m)": [0.5], "Ycore2(m)": [0.3], "Yvoid2(m)": [0.3], "Yyoke2(m)": [0.6]}


def _iron_area(g, t, diluted):
    """Cross-section area of the quarter model's iron (and wing) at fraction t of the length."""
    v = {k: g[k + "_1"] + t * (g[k + "_2"] - g[k + "_1"]) for k in ("X_mgap", "X_core", "X_void", "X_yoke",
                                                                     "Y_core", "Y_void", "Y_yoke")}
    outer = (v["X_yoke"] - v["X_mgap"]) * v["Y_yoke"]
    void = (v["X_void"] - v["X_core"]) * v["Y_core"]
    return outer - void, (v["X_yoke"] - v["X_void"]) * v["Y_void"] if diluted else 0.0


@pytest.mark.parametrize("diluted", [False, True])
@pytest.mark.parametrize("X_mgap", [(0.0, 0.0), (0.05, 0.08)])
def test_template_mesh_volumes_and_boundary(diluted, X_mgap):
    g = ship.mag_1_parameters(template_parameters(X_mgap))
    msh = ship.mag_1_mesh(g, lc=0.5, use_diluted_steel=diluted)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    assert (vol > 0).all()
    box = (g["lim_x"] * g["lim_y"] * (g["z_max"] - g["z_min"]))
    assert abs(vol.sum() - box) < 1e-9 * box
    # planar boundaries: the tetrahedra fill the iron exactly; the area is quadratic in z (Simpson)
    a = [_iron_area(g, t, diluted) for t in (0.0, 0.5, 1.0)]
    iron = g["Z_len"] * (a[0][0] + 4 * a[1][0] + a[2][0]) / 6.0
    wing = g["Z_len"] * (a[0][1] + 4 * a[1][1] + a[2][1]) / 6.0
    if diluted:
        iron -= wing  # the wing is cut out of the outer leg
    got_iron = vol[msh.elem_domain == M.TAG_IRON].sum()
    got_wing = vol[msh.elem_domain == ship.TAG_WING].sum()
    assert abs(got_iron - iron) < 1e-9 * iron and abs(got_wing - wing) < 1e-9 * max(wing, 1.0)
    # y = 0 is the symmetry plane: no Dirichlet edge lies in it unless it also bounds another face
    d = msh.dirichlet_edge_ids()
    b = msh.boundary_edge_ids()
    on_plane = np.all(np.abs(msh.nodes[msh.edges[:, :]][:, :, 1]) < 1e-12, axis=1)
    inner_plane = np.setdiff1d(np.flatnonzero(on_plane), np.flatnonzero(np.any(
        (np.abs(msh.nodes[msh.edges][:, :, 0]) < 1e-12) | (np.abs(msh.nodes[msh.edges][:, :, 0] - g["lim_x"]) < 1e-12) |
        (np.abs(msh.nodes[msh.edges][:, :, 2] - g["z_min"]) < 1e-12) |
        (np.abs(msh.nodes[msh.edges][:, :, 2] - g["z_max"]) < 1e-12), axis=1) & on_plane))
    assert len(inner_plane) > 0 and not np.isin(inner_plane, d).any() and np.isin(inner_plane, b).all()
    assert len(d) < len(b)


def test_template_2_mesh():
    P = template_parameters()
    for k in ("Xmgap1(m)", "Xmgap2(m)"):
        del P[k]
    P["Yvoid1(m)"], P["Yvoid2(m)"] = [0.25], [0.35]
    g = ship.mag_1_parameters(P)
    assert g["X_mgap_1"] == 0.0 and g["X_mgap_2"] == 0.0
    msh = ship.template_mesh(g, 2, lc=0.5, inner=0.3)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    assert (vol > 0).all()

    def area(t):
        v = {k: g[k + "_1"] + t * (g[k + "_2"] - g[k + "_1"]) for k in ("X_core", "X_void", "X_yoke", "Y_core",
                                                                         "Y_void", "Y_yoke")}
        return (v["X_core"] * v["Y_core"] + v["X_yoke"] * (v["Y_yoke"] - v["Y_void"])
                + (v["X_yoke"] - v["X_void"]) * v["Y_void"])

    iron = g["Z_len"] * (area(0.0) + 4 * area(0.5) + area(1.0)) / 6.0
    got = vol[msh.elem_domain == M.TAG_IRON].sum()
    assert abs(got - iron) < 1e-9 * iron


def template_4_parameters():
    """Two table rows: X_A, X_B, X_C from the first, X_D, X_E, X_F from the second."""
    P = template_parameters()
    two = {k: v * 2 for k, v in P.items()}
    for e, (a, b, c, d_, e_, f) in ((1, (0.0, 0.1, 0.16, 0.46, 0.52, 0.9)), (2, (0.0, 0.12, 0.18, 0.5, 0.56, 1.0))):
        two[f"Xmgap{e}(m)"] = [a, 0.0]
        two[f"Xcore{e}(m)"] = [b, d_]
        two[f"Xvoid{e}(m)"] = [c, e_]
        two[f"Xyoke{e}(m)"] = [0.0, f]
    return two


def test_template_4_mesh():
    g = ship.mag_4_parameters(template_4_parameters())
    msh = ship.template_mesh(g, 4, lc=0.5, inner=1.0)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    assert (vol > 0).all()

    def areas(t):
        v = {k: g[k + "_1"] + t * (g[k + "_2"] - g[k + "_1"]) for k in ("X_A", "X_B", "X_C", "X_D", "X_E", "X_F",
                                                                         "Y_core", "Y_yoke")}
        core = (v["X_D"] - v["X_C"]) * v["Y_core"]
        yoke = (v["X_F"] - v["X_A"]) * v["Y_yoke"] - (v["X_E"] - v["X_B"]) * v["Y_core"]
        return core, yoke

    a = [areas(t) for t in (0.0, 0.5, 1.0)]
    core = g["Z_len"] * (a[0][0] + 4 * a[1][0] + a[2][0]) / 6.0
    yoke = g["Z_len"] * (a[0][1] + 4 * a[1][1] + a[2][1]) / 6.0
    assert abs(vol[msh.elem_domain == M.TAG_IRON].sum() - core) < 1e-9 * core
    assert abs(vol[msh.elem_domain == ship.TAG_YOKE].sum() - yoke) < 1e-9 * yoke
    coils, _, _, _, _ = ship._coils(g, 3e6, 0.6, template=4)
    assert len(coils) == 2


def test_template_coils():
    for X_mgap, n_coils in (((0.0, 0.0), 1), ((0.05, 0.08), 2)):
        g = ship.mag_1_parameters(template_parameters(X_mgap))
        coils, A_cu, A_coil, perimeter, J = ship._coils(g, 3e6, 0.6)
        assert len(coils) == n_coils
        assert abs(A_cu - 4000.0 / 3e6) < 1e-15 and abs(A_coil - A_cu / 0.6) < 1e-15
        slot = 2 * 0.2
        n = min(int(slot / 2 / (4.5e-3 + 0.5e-3)), 10)
        assert all(len(c.y) == n for c in coils)
        assert abs(perimeter - sum(c.get_length() for c in coils)) < 1e-12
        # the turns wrap the core: straight parts just outside the core's z ends
        seg = coils[0].get_segments()
        assert seg[:, 2].min() < g["Z_pos"] and seg[:, 2].max() > g["Z_pos"] + g["Z_len"]


def test_template_3_coils_wrap_the_legs():
    g = ship.mag_1_parameters(template_parameters())
    coils, _, _, perimeter, _ = ship._coils(g, 3e6, 0.6, template=3)
    assert len(coils) == 2
    d = 5e-3 + 0.5e-3 + 4.5e-3
    seg = coils[0].get_segments()
    xs = np.concatenate([seg[:, 0], seg[:, 3]])
    assert xs.min() >= min(g["X_void_1"], g["X_void_2"]) - d - 1e-12
    assert xs.max() <= max(g["X_yoke_1"], g["X_yoke_2"]) + d + 1e-12
    seg2 = coils[1].get_segments()
    assert np.allclose(seg2[:, [0, 3]], -seg[:, [0, 3]]) and np.allclose(seg2[:, [1, 2, 4, 5]], seg[:, [1, 2, 4, 5]])


def test_compute_J_opt():
    d = {"material_cost(CHF/kg)": 20.0, "manufacturing_cost(CHF/kg)": 80.0, "density(g/m3)": 8.9e6,
         "resistivity(Ohm.m)": 1.7e-8}
    J = ship.compute_J_opt(d, 5.0)
    assert abs(J - np.sqrt(100.0 * 8.9e3 / 5.0 / 1.7e-8) * 1e-6) < 1e-12 * J


def ncsc_parameters():
    """An NC magnet (row 0, template-1 yoke) followed by an SC magnet (row 1, template-2 core and yoke)."""
    P = {k: v * 2 for k, v in template_parameters().items()}
    P["Z_pos(m)"] = [-3.0, 1.2]
    P["Z_len(m)"] = [3.5, 2.5]
    for e, (c, v, y, yc, yv, yy) in ((1, (0.2, 0.26, 0.9, 0.15, 0.2, 0.45)), (2, (0.22, 0.28, 1.0, 0.18, 0.24, 0.5))):
        P[f"Xmgap{e}(m)"] = [0.0, 0.0]
        P[f"Xcore{e}(m)"] = [P[f"Xcore{e}(m)"][0], c]
        P[f"Xvoid{e}(m)"] = [P[f"Xvoid{e}(m)"][0], v]
        P[f"Xyoke{e}(m)"] = [P[f"Xyoke{e}(m)"][0], y]
        P[f"Ycore{e}(m)"] = [P[f"Ycore{e}(m)"][0], yc]
        P[f"Yvoid{e}(m)"] = [P[f"Yvoid{e}(m)"][0], yv]
        P[f"Yyoke{e}(m)"] = [P[f"Yyoke{e}(m)"][0], yy]
    return P


def test_multi_magnet_mesher():
    """One magnet: the same grid as the single-magnet mesher.  Two magnets along z: each
    magnet's iron volume is exact, and the box is filled."""
    g = ship.mag_1_parameters(template_parameters())
    m = ship.Magnet(g["Z_pos"], g["Z_pos"] + g["Z_len"], ["gap", "core", "void", "leg", "out"],
                    [g["X_mgap_1"], g["X_core_1"], g["X_void_1"], g["X_yoke_1"]],
                    [g["X_mgap_2"], g["X_core_2"], g["X_void_2"], g["X_yoke_2"]], ["low", "top", "out"],
                    [g["Y_core_1"], g["Y_yoke_1"]], [g["Y_core_2"], g["Y_yoke_2"]],
                    lambda X, Y: np.where(ship._tag_type_1(X, Y), M.TAG_IRON, 0), 0.1)
    a = ship.magnets_mesh([m], g["lim_x"], g["lim_y"], g["z_min"], g["z_max"], 0.5)
    b = ship.mag_1_mesh(g, lc=0.5)
    assert np.array_equal(a.cells, b.cells) and np.array_equal(a.elem_domain, b.elem_domain)
    assert np.abs(a.nodes - b.nodes).max() < 1e-14
    P = ncsc_parameters()
    g1, g2 = ship.mag_1_parameters(P, 0), ship.mag_1_parameters(P, 1)

    def simpson(area, L):
        return L * (area(0.0) + 4 * area(0.5) + area(1.0)) / 6.0

    def lerp(g, k, t):
        return g[k + "_1"] + t * (g[k + "_2"] - g[k + "_1"])

    def area1(t):
        return ((lerp(g1, "X_yoke", t) - lerp(g1, "X_mgap", t)) * lerp(g1, "Y_yoke", t)
                - (lerp(g1, "X_void", t) - lerp(g1, "X_core", t)) * lerp(g1, "Y_core", t))

    def area2(t):
        return (lerp(g2, "X_core", t) * lerp(g2, "Y_core", t)
                + lerp(g2, "X_yoke", t) * (lerp(g2, "Y_yoke", t) - lerp(g2, "Y_void", t))
                + (lerp(g2, "X_yoke", t) - lerp(g2, "X_void", t)) * lerp(g2, "Y_void", t))

    e = lambda g, keys: ([g[f"{k}_1"] for k in keys], [g[f"{k}_2"] for k in keys])
    nc = ship.Magnet(g1["Z_pos"], g1["Z_pos"] + g1["Z_len"], ["gap", "core", "void", "leg", "out"],
                     *e(g1, ["X_mgap", "X_core", "X_void", "X_yoke"]), ["low", "top", "out"],
                     *e(g1, ["Y_core", "Y_yoke"]), lambda X, Y: np.where(ship._tag_type_1(X, Y), ship.TAG_NC, 0), 0.2)
    sc = ship.Magnet(g2["Z_pos"], g2["Z_pos"] + g2["Z_len"], ["core", "void", "leg", "out"],
                     *e(g2, ["X_core", "X_void", "X_yoke"]), ["low", "mid", "top", "out"],
                     *e(g2, ["Y_core", "Y_void", "Y_yoke"]),
                     lambda X, Y: np.where(ship._tag_type_2(X, Y), M.TAG_IRON, 0), 0.2)
    lim_x, lim_y = max(g1["lim_x"], g2["lim_x"]), max(g1["lim_y"], g2["lim_y"])
    msh = ship.magnets_mesh([nc, sc], lim_x, lim_y, g1["z_min"], g2["z_max"], 0.5)
    vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
    assert (vol > 0).all()
    box = lim_x * lim_y * (g2["z_max"] - g1["z_min"])
    assert abs(vol.sum() - box) < 1e-9 * box
    v1 = simpson(area1, g1["Z_len"])
    v2 = simpson(area2, g2["Z_len"])
    assert abs(vol[msh.elem_domain == ship.TAG_NC].sum() - v1) < 1e-9 * v1
    assert abs(vol[msh.elem_domain == M.TAG_IRON].sum() - v2) < 1e-9 * v2


def test_polygon_area():
    sq = np.array([[0, 0], [1, 0], [1, 1], [0, 1], [0, 0]], dtype=float)
    assert ship.compute_area_polygon(sq) == 1.0
    assert ship.compute_area_polygon(sq[:-1], isclosed=False) == 1.0
    assert ship.compute_area_polygon(sq[::-1]) == -1.0


def test_get_NI_and_prices(tmp_path):
    B, H = MAT.atan_bh_table(mu_r=2500.0, Js=2.0)
    (tmp_path / "iron_test.json").write_text(json.dumps({"density(g/m3)": 7.8e6, "material_cost(CHF/kg)": 1.5,
                                                         "manufacturing_cost(CHF/kg)": 2.5,
                                                         "BH_data": {"B(T)": list(B), "H(A/m)": list(H)}}))
    (tmp_path / "cu_test.json").write_text(json.dumps({"material_cost(CHF/kg)": 20.0,
                                                       "manufacturing_cost(CHF/kg)": 80.0}))
    P = template_parameters()
    rel = MAT.Reluctance(str(tmp_path / "iron_test.json"))
    g = ship.mag_1_parameters(P)
    Zl = g["Z_len"]
    # the side-view areas of the reference's polygons (first point at the origin)
    A1 = ship.compute_area_polygon(np.array([[0, 0], [g["X_core_1"], 0], [g["X_core_2"], Zl], [g["X_mgap_2"], Zl],
                                             [g["X_mgap_1"], 0]]))
    A2 = ship.compute_area_polygon(np.array([[0, 0], [g["Y_yoke_1"], 0], [g["Y_yoke_2"], Zl], [g["Y_void_2"], Zl],
                                             [g["Y_void_1"], 0]]))
    A3 = ship.compute_area_polygon(np.array([[0, 0], [g["X_yoke_1"], 0], [g["X_yoke_2"], Zl], [g["X_void_2"], Zl],
                                             [g["X_void_1"], 0]]))
    l1 = 0.25 * (g["Y_core_1"] + g["Y_core_2"] + g["Y_yoke_1"] + g["Y_yoke_2"])
    l2 = (0.5 * (g["X_yoke_1"] + g["X_yoke_2"]) + 0.5 * (g["X_void_1"] + g["X_void_2"])
          - 0.5 * (g["X_core_1"] + g["X_core_2"]) - 0.5 * (g["X_mgap_1"] + g["X_mgap_2"]))
    for kind, Bg in (("Mag1", 1.2), ("Mag1", -1.2), ("Mag3", 0.8)):
        P["yoke_type"] = [kind]
        NI, valid = ship.get_NI(Bg, P, 0, materials_directory=str(tmp_path))
        Phi = abs(Bg) * (A1 if kind == "Mag1" else A3)
        Bs = ([Bg] if kind == "Mag1" else [Phi / A1]) + [Phi / A2, Phi / A3]
        want = sum(float(rel.evaluate_nu(b)) * b * l for b, l in zip(Bs, (l1, l2, l1)))
        want = -want if Bg < 0 and kind == "Mag1" else want
        assert abs(NI - want) <= 1e-12 * abs(want) and valid == ((A1 < A3) if kind == "Mag1" else (A1 > A3))
    C_iron, C_coil, C_edf = ship.compute_prices(P, 0, 2e6, 1e5, 3e4, materials_directory=str(tmp_path))
    assert abs(C_iron - 1e-3 * 2e6 * 4.0 * 0.5) < 1e-9 and abs(C_coil - 1e-3 * 1e5 * 100.0 * 0.5) < 1e-9
    assert abs(C_edf - 3e4 * 5.0 / 72000.0 * 72000 * 0.5) < 1e-6

