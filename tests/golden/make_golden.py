"""Generate the golden fixtures in this directory from the reference's own C kernels.

Runs the reference ``fem_c/ctools.c`` (compiled from its sources by ``oracle/build_oracle.py``
into ``oracle/_ref/``) with the Cython layer's marshalling (``oracle/oracle.py``, backend
"ref") on small seeded inputs, and stores inputs and outputs in ``golden_small.npz``:

* curl-curl K, dK (CSR with explicit zeros, as ``csr_array((v,(i,j)))`` returns them) and rhs,
  plain kernel (air) and reduced kernel (iron with a source field), 4-point rule; the
  diluted-steel reduced kernel (``compute_K_dK_Hcurl_red_dil``) on the iron;
* grad-grad K, dK with a B-spline permeability and with a constant one;
* B at quadrature points; Biot-Savart of a racetrack coil's segments;
* PCHIP nu, nu' and B-spline mu, mu' at sample points.

Usage: ``python tests/golden/make_golden.py`` (needs the reference checkout).
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
import snoopy_b200 as S  # noqa: E402
from snoopy_b200 import finite_element as FE  # noqa: E402
from snoopy_b200 import mesh as M  # noqa: E402
from snoopy_b200 import materials as MAT  # noqa: E402


def golden_inputs(seed=3):
    """Deterministic inputs of the fixtures (also rebuilt by the tests to check the inputs match)."""
    msh = M.window_frame_mesh(800, jitter=0.15, seed=seed)
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    rng = np.random.default_rng(seed)
    x = rng.normal(0.0, 2e-3, msh.num_dofs)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    Bs = rng.normal(0.0, 0.8, (len(iron) * len(w), 3))
    xn = rng.normal(0.0, 50.0, msh.num_nodes)
    return msh, w, q, dphi, phi, curls, x, iron, air, Bs, xn


DILUTION_CASES = [(0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, -0.25, 0.5, 1),
                  (0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, -0.25, 0.5, 3),
                  (0.05, 0.62, 0.70, 1.45, 0.11, 0.93, 1.02, 2.10, 3.0, 4.5, 1),
                  (0.05, 0.62, 0.70, 1.45, 0.11, 0.93, 1.02, 2.10, 3.0, 4.5, 3)]


def reference_dilution_coefficients():
    """(c_num, m_num, c_den, m_den) of the reference's own ``snoopy/materials.py`` Dilution for
    every case of DILUTION_CASES (its plotting import is stubbed: nothing plots here)."""
    import importlib.util
    import types

    for name in ("matplotlib", "matplotlib.pyplot"):
        sys.modules.setdefault(name, types.ModuleType(name))
    ref = os.environ.get("SNOOPY_REFERENCE", "/root/reference")
    spec = importlib.util.spec_from_file_location("_ref_materials", os.path.join(ref, "snoopy", "materials.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = []
    for c in DILUTION_CASES:
        d = mod.Dilution(*c)
        out.append([d.c_num, d.m_num, d.c_den, d.m_den])
    return np.array(out)


def golden_dilution():
    """Magnet type 1 with an iron fraction changing over z in [-0.25, 0.25]: s = 4/3 at the
    entrance, 35/38 at the exit."""
    return MAT.Dilution(0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, z_pos=-0.25, z_len=0.5, mag_type=1)


def main():
    O.lib("ref")
    msh, w, q, dphi, phi, curls, x, iron, air, Bs, xn = golden_inputs()
    rel = MAT.atan_reluctance()
    perm = MAT.atan_permeability()
    out = {"nodes": msh.nodes, "cells": msh.cells, "glob_ids": msh.elem_edges, "orientations": msh.orientations,
           "iron": iron, "air": air, "w": w, "q": q, "d_phi": dphi, "phi": phi, "curls": curls, "x": x, "B_s": Bs,
           "x_nodal": xn, "num_dofs": msh.num_dofs}
    # the material tables themselves, so the fixtures do not depend on how they were fitted
    out["rel_c"], out["rel_x"] = rel.get_spline_information()
    t, c, k, hmin, muh = perm.get_spline_information()
    out["perm_t"], out["perm_c"], out["perm_k"], out["perm_hmin"], out["perm_muhmin"] = t, c, k, hmin, muh
    n = msh.num_dofs
    for name, el, bs, mat in (("air", air, np.zeros((0, 3)), S.ConstantReluctance(0.25 / np.pi * 1e7)),
                              ("iron_red", iron, Bs, rel), ("iron_plain", iron, np.zeros((0, 3)), rel)):
        K, dK, rhs = O.compute_stiffness_and_jacobi_matrix_curl_curl(
            msh.nodes, msh.cells[el], msh.elem_edges[el], curls, dphi, msh.orientations[el], x, bs, mat, q, w, n, 6,
            backend="ref")
        for tag, A in (("K", K), ("dK", dK)):
            out[f"cc_{name}_{tag}_indptr"] = A.indptr
            out[f"cc_{name}_{tag}_indices"] = A.indices
            out[f"cc_{name}_{tag}_data"] = A.data
        out[f"cc_{name}_rhs"] = rhs
    # diluted steel (type 1): iron fraction running linearly over the iron's z extent
    dil = golden_dilution()
    out["dil_coef"] = np.array(dil.coefficients())
    out["dil_cases"] = np.array(DILUTION_CASES, dtype=np.float64)
    out["dil_cases_ref"] = reference_dilution_coefficients()
    K, dK, rhs = O.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(
        msh.nodes, msh.cells[iron], msh.elem_edges[iron], curls, phi, dphi, msh.orientations[iron], x, Bs, rel, dil, q,
        w, n, 6, backend="ref")
    for tag, A in (("K", K), ("dK", dK)):
        out[f"cc_iron_dil_{tag}_indptr"] = A.indptr
        out[f"cc_iron_dil_{tag}_indices"] = A.indices
        out[f"cc_iron_dil_{tag}_data"] = A.data
    out["cc_iron_dil_rhs"] = rhs
    out["rhs_red"] = O.compute_rhs_Hcurl_red_c(msh.nodes, msh.cells[iron], msh.elem_edges[iron], curls, dphi,
                                               msh.orientations[iron], Bs, rel, x, q, w, n, 6, backend="ref")
    for name, pm in (("bspline", perm), ("const", S.ConstantPermeability(1.0))):
        K, dK = O.compute_stiffness_and_jacobi_matrix(msh.nodes, msh.cells, dphi, xn, pm, q, w, backend="ref")
        for tag, A in (("K", K), ("dK", dK)):
            out[f"gg_{name}_{tag}_indptr"] = A.indptr
            out[f"gg_{name}_{tag}_indices"] = A.indices
            out[f"gg_{name}_{tag}_data"] = A.data
    pts, B = O.compute_B_Hcurl(msh.nodes, msh.cells, msh.elem_edges, curls, phi, dphi, msh.orientations, x, q, w, n, 6,
                               backend="ref")
    out["bq_points"], out["bq_B"] = pts, B
    g = msh.geometry
    coil = g.coils(n_turns=2)[0]
    segs = coil.get_segments()
    tar = np.concatenate([pts[::7], np.array([[segs[0, 0], segs[0, 1], segs[0, 2]]]),
                          0.5 * (segs[3, :3] + segs[3, 3:])[None] + 1e-3])
    out["bs_src"], out["bs_tar"], out["bs_current"], out["bs_rad"] = segs, tar, coil.current, coil.rad
    out["bs_B"] = O.compute_B_line_segs_cpp(segs, tar, coil.current, coil.rad, backend="ref")
    bsamp = np.concatenate([np.linspace(0, 7.0, 301), rel.get_spline_information()[1], [-1.0, 1e-300]])
    out["pchip_B"] = bsamp
    out["pchip_nu"], out["pchip_dnu"] = O.pchip_eval(rel, bsamp, backend="ref")
    hs = np.concatenate([np.logspace(-3, 8, 301), [0.0, perm.H_min, 1e7]])
    out["mu_H"] = hs
    out["mu_mu"], out["mu_dmu"] = O.mu_eval(perm, hs, backend="ref")
    path = os.path.join(HERE, "golden_small.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes;", msh.num_elements, "tets,", n, "edges")


if __name__ == "__main__":
    main()
