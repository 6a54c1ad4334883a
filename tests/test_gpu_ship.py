"""The SHiP template-1 driver end to end on the GPU: meshing, coils, the reduced Newton solve
(plain and with the diluted wing), the field map and the design figures."""

import json

import numpy as np
import pytest

from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M
from snoopy_b200 import ship
from test_ship_template import ncsc_parameters, template_4_parameters, template_parameters

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def materials_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("materials")
    B, H = MAT.atan_bh_table(mu_r=2500.0, Js=2.0)
    (d / "iron_test.json").write_text(json.dumps({"density(g/m3)": 7.8e6, "material_cost(CHF/kg)": 1.0,
                                                  "manufacturing_cost(CHF/kg)": 1.0,
                                                  "BH_data": {"B(T)": list(B), "H(A/m)": list(H)}}))
    (d / "cu_test.json").write_text(json.dumps({"density(g/m3)": 8.9e6, "resistivity(Ohm.m)": 1.7e-8,
                                                "material_cost(CHF/kg)": 20.0, "manufacturing_cost(CHF/kg)": 80.0,
                                                "filling_factor": 0.6}))
    return str(d)


def test_template_1_plain_and_diluted(materials_dir, tmp_path):
    P = template_parameters()
    g = ship.mag_1_parameters(P)
    probes = np.array([[0.12, 0.1, 0.0], [0.12, 0.05, 1.0], [0.8, 0.3, 0.0], [0.3, 0.7, 0.0]])
    out = {}
    for diluted in (False, True):
        spec = "_dil" if diluted else ""
        pts, B, M_iron, M_coil, Q, J = ship.get_vector_field_mag_1(
            P, lc=0.4, eval_pos=probes, materials_directory=materials_dir, result_directory=str(tmp_path),
            result_spec=spec, use_diluted_steel=diluted, quad_order=2)
        assert pts.shape == B.shape and np.isfinite(B).all()
        msh = ship.mag_1_mesh(g, lc=0.4, use_diluted_steel=diluted)
        vol = M.tet_volumes6(msh.nodes, msh.cells) / 6.0
        tags = [M.TAG_IRON, ship.TAG_WING] if diluted else [M.TAG_IRON]
        assert abs(M_iron - 4 * vol[np.isin(msh.elem_domain, tags)].sum() * 7.8e6) < 1e-9 * M_iron
        assert M_coil > 0 and Q > 0 and J > 0
        Be = np.loadtxt(tmp_path / f"B{spec}.csv", delimiter=",", skiprows=1)
        assert Be.shape == (4, 6) and np.array_equal(Be[:, :3], probes)
        # the coil loops lie in x-z planes around the core: the core field runs along y
        assert abs(Be[0, 4]) > 5 * max(abs(Be[0, 3]), abs(Be[0, 5])) and 0.05 < abs(Be[0, 4]) < 2.5
        out[diluted] = Be[:, 3:]
    # the diluted wing changes the field
    assert np.abs(out[True] - out[False]).max() > 1e-3 * np.abs(out[False]).max()


def test_template_3(materials_dir, tmp_path):
    P = template_parameters()
    probes = np.array([[0.12, 0.1, 0.0], [0.8, 0.1, 0.0]])
    pts, B, M_iron, M_coil, Q, J = ship.get_vector_field_mag_3(P, lc=0.4, eval_pos=probes, quad_order=2,
                                                               materials_directory=materials_dir,
                                                               result_directory=str(tmp_path), result_spec="_m3")
    assert np.isfinite(B).all() and M_coil > 0 and Q > 0
    Be = np.loadtxt(tmp_path / "B_m3.csv", delimiter=",", skiprows=1)[:, 3:]
    # the coils sit around the legs: both the core and the leg carry flux along y
    assert abs(Be[0, 1]) > 0.05 and abs(Be[1, 1]) > 0.05


def test_template_2(materials_dir, tmp_path):
    P = template_parameters()
    for k in ("Xmgap1(m)", "Xmgap2(m)"):
        del P[k]
    P["Yvoid1(m)"], P["Yvoid2(m)"] = [0.25], [0.35]
    probes = np.array([[0.12, 0.1, 0.0]])
    pts, B, M_iron, M_coil, Q, J = ship.get_vector_field_mag_2(P, lc=0.4, eval_pos=probes, quad_order=2,
                                                               materials_directory=materials_dir,
                                                               result_directory=str(tmp_path), result_spec="_m2")
    assert np.isfinite(B).all() and M_iron > 0 and M_coil > 0
    Be = np.atleast_2d(np.loadtxt(tmp_path / "B_m2.csv", delimiter=",", skiprows=1))[0, 3:]
    assert abs(Be[1]) > 5 * max(abs(Be[0]), abs(Be[2]))  # core field along y
    assert (tmp_path / "parameters_m2.csv").exists()


def test_template_4(materials_dir, tmp_path):
    P = template_4_parameters()
    probes = np.array([[0.3, 0.1, 0.0]])
    out = {}
    for diluted in (False, True):
        pts, B, M_iron, M_coil, Q, J = ship.get_vector_field_mag_4(P, lc=0.4, eval_pos=probes, quad_order=2,
                                                                   materials_directory=materials_dir,
                                                                   result_directory=str(tmp_path),
                                                                   result_spec=f"_m4{int(diluted)}",
                                                                   use_diluted_steel=diluted)
        assert np.isfinite(B).all() and M_iron > 0
        Be = np.atleast_2d(np.loadtxt(tmp_path / f"B_m4{int(diluted)}.csv", delimiter=",", skiprows=1))[0, 3:]
        assert abs(Be[1]) > 5 * max(abs(Be[0]), abs(Be[2]))  # core field along y
        out[diluted] = Be
    assert np.abs(out[True] - out[False]).max() > 1e-3 * np.abs(out[False]).max()


def test_ncsc(materials_dir, tmp_path):
    P = ncsc_parameters()
    probes = np.array([[0.1, 0.08, -1.0], [0.1, 0.08, 2.4]])  # NC core, SC core
    pts, B, M_iron, M_coil, Q, J = ship.get_vector_field_ncsc(P, lc=0.4, eval_pos=probes, quad_order=2,
                                                              materials_directory=materials_dir,
                                                              result_directory=str(tmp_path), result_spec="_ncsc")
    assert np.isfinite(B).all() and M_iron > 0 and M_coil > 0 and J == 3e6
    Be = np.loadtxt(tmp_path / "B_ncsc.csv", delimiter=",", skiprows=1)[:, 3:]
    # both cores carry flux along y (the superconducting core's is weaker and less uniform: an
    # air gap separates it from its yoke)
    for b in Be:
        assert abs(b[1]) > 2 * max(abs(b[0]), abs(b[2])) and abs(b[1]) > 0.02

