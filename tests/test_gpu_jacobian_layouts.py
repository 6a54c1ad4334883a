"""The residual-mode Newton loop's Jacobian layouts against the CSR export of the same assembly.

The solver keeps the Jacobian of its Krylov loop as element tensors (matrix-free, the
default), as an assembled CSR, or as a SELL-C-sigma copy of that CSR, chosen by the
environment variable SNP_JACOBIAN when the solver is finalized.  Each layout's product
J x is checked against the CSR that ``snp_solver_assemble`` exports at the same iterate,
and solves in every layout must reach the same answer.
"""

import contextlib
import os

import numpy as np
import pytest
import torch

import snoopy_b200 as S
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M
from snoopy_b200._lib import SnpError
from snoopy_b200.device import upload

pytestmark = pytest.mark.gpu

LAYOUTS = ["elem", "csr", "sell"]


@contextlib.contextmanager
def jacobian_layout(name):
    old = os.environ.get("SNP_JACOBIAN")
    os.environ["SNP_JACOBIAN"] = name
    try:
        yield
    finally:
        if old is None:
            del os.environ["SNP_JACOBIAN"]
        else:
            os.environ["SNP_JACOBIAN"] = old


def _solver(layout, ntet=6000, seed=7):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    solver = S.RedMVPSolver(msh, msh.geometry.coils(), [M.TAG_IRON], [M.TAG_AIR], [MAT.atan_reluctance()],
                            max_newton_iterations=50, quad_order=2)
    solver.verbose = False
    with jacobian_layout(layout):
        eng = solver.newton_engine()
    assert eng.jacobian_layout == layout
    return msh, solver, eng


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("layout", LAYOUTS)
def test_jacobian_apply_matches_csr_export(layout, precision):
    msh, solver, eng = _solver(layout)
    x, st = solver.solve_to_residual(1e-8, precision=precision, return_device=True)
    assert st["rel_res"] <= 1e-8
    n = msh.num_dofs
    Jc = eng.pattern.to_scipy(eng.assemble(x, J=True, F=False)["J"], drop_zeros=False)
    mask = solver.make_boundary_mask()
    z = np.random.default_rng(5).standard_normal(n)
    zf = np.where(mask, z, 0.0)
    want = np.where(mask, Jc @ zf, 0.0)
    dt = torch.float64 if precision == "fp64" else torch.float32
    zd = upload(z, np.float64).to(dt)
    yd = torch.full_like(zd, 7.0)
    eng.jacobian_apply(zd, yd, precision)
    got = yd.double().cpu().numpy()
    scale = np.abs(Jc) @ np.abs(zf)
    # float64: rounding of differently ordered sums; float32: values and vectors in float32
    tol = 1e-12 if precision == "fp64" else 2e-6
    err = np.abs(got - want) / (scale + 1e-300)
    assert err[mask].max() <= tol, err[mask].max()
    assert np.all(got[~mask] == 0.0)


def test_jacobian_apply_without_solve_is_an_error():
    msh, solver, eng = _solver("elem", ntet=2000)
    z = upload(np.ones(msh.num_dofs), np.float64)
    y = torch.empty_like(z)
    with pytest.raises(SnpError):
        eng.jacobian_apply(z, y, "fp64")


def test_layouts_reach_the_same_solution():
    out = {}
    for layout in LAYOUTS:
        msh, solver, eng = _solver(layout)
        if layout == "elem":
            eng.set_preconditioner("jacobi")  # the layouts compared under the same preconditioner
        x, st = solver.solve_to_residual(1e-10)
        assert st["rel_res"] <= 1e-10, (layout, st)
        probes = msh.geometry.aperture_probes(300)
        el, _ = msh.locate(probes)
        # curl-curl has gradients in its null space (air and iron alike): compare B = curl A
        out[layout] = (solver.curl_curl_factory.compute_B_at_points(x, probes, el), st)
    B0, s0 = out["csr"]
    for layout in ("elem", "sell"):
        B1, s1 = out[layout]
        assert abs(s1["newton_iterations"] - s0["newton_iterations"]) <= 1
        err = np.linalg.norm(B1 - B0, axis=1).max() / np.linalg.norm(B0, axis=1).max()
        assert err < 1e-8, (layout, err)


def test_element_layout_is_deterministic():
    """The element layout has no atomics in its assembly sums or its products: two solves
    from the same start take the same iterations and give the same bits."""
    msh, solver, eng = _solver("elem")
    x1, s1 = solver.solve_to_residual(1e-8)
    x2, s2 = solver.solve_to_residual(1e-8)
    assert s1["cg_iterations"] == s2["cg_iterations"]
    assert np.array_equal(x1, x2)


def test_total_potential_solve_in_element_and_csr_layouts():
    """MVPSolver (plain curl-curl, conductor source rhs) gives the same answer in both layouts."""
    msh = M.bar_conductor_mesh(8000)
    t1, t2 = msh.coil_terminals[M.TAG_COIL_1]
    Phi = 3e6 * 0.8
    cen = msh.element_centroids()
    probe = msh.domain_elements(M.TAG_IRON)[::5]
    out = {}
    for layout in ("elem", "csr"):
        sol = S.MVPSolver(msh, [M.TAG_COIL_1], [M.TAG_IRON], [M.TAG_AIR], [(t1, t2)], [MAT.atan_reluctance()],
                          quad_order=2, max_newton_iterations=60)
        sol.verbose = False
        with jacobian_layout(layout):
            x, st = sol.solve_to_residual([Phi], rtol=1e-9, max_newton=60)
        assert sol._engine([Phi]).jacobian_layout == layout
        assert st["rel_res"] <= 1e-9
        # the total-potential curl-curl has gradients in its null space: compare B = curl A
        out[layout] = sol.curl_curl_factory.compute_B_at_points(x, cen[probe], probe)
    err = np.linalg.norm(out["elem"] - out["csr"], axis=1).max() / np.linalg.norm(out["csr"], axis=1).max()
    assert err < 1e-7, err


def test_element_layout_multi_pass_grid():
    """A mesh large enough that every warp of the element and DoF passes loops several times
    (the grid is one wave of resident blocks), against the CSR layout."""
    out = {}
    for layout in ("elem", "csr"):
        msh, solver, eng = _solver(layout, ntet=300000)
        x, st = solver.solve_to_residual(1e-8)
        assert st["rel_res"] <= 1e-8, (layout, st)
        probes = msh.geometry.aperture_probes(200)
        el, _ = msh.locate(probes)
        out[layout] = solver.curl_curl_factory.compute_B_at_points(x, probes, el)
    err = np.linalg.norm(out["elem"] - out["csr"], axis=1).max() / np.linalg.norm(out["csr"], axis=1).max()
    assert err < 1e-6, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_assemble_tensors_at_any_iterate(precision):
    """snp_solver_assemble_tensors at a random iterate: J(x) z and F(x) against the CSR
    assembly of the same x (the reduced formulation with a source field)."""
    msh, solver, eng = _solver("elem")
    n = msh.num_dofs
    rng = np.random.default_rng(9)
    x = upload(rng.normal(0.0, 2e-3, n), np.float64)
    F = torch.zeros(n, dtype=torch.float64, device="cuda")
    eng.assemble_tensors(x, precision, F)
    ref = eng.assemble(x, J=True, F=True, rhs=True)
    Jc = eng.pattern.to_scipy(ref["J"], drop_zeros=False)
    mask = solver.make_boundary_mask()
    z = rng.standard_normal(n)
    zf = np.where(mask, z, 0.0)
    want = np.where(mask, Jc @ zf, 0.0)
    dt = torch.float64 if precision == "fp64" else torch.float32
    yd = torch.zeros(n, dtype=dt, device="cuda")
    eng.jacobian_apply(upload(z, np.float64).to(dt), yd, precision)
    got = yd.double().cpu().numpy()
    scale = np.abs(Jc) @ np.abs(zf)
    tol = 1e-12 if precision == "fp64" else 2e-6
    assert (np.abs(got - want) / (scale + 1e-300))[mask].max() <= tol
    # F: same float64 terms summed in another order; bound by the terms' magnitudes
    Fg, Fr = F.cpu().numpy(), ref["F"].cpu().numpy()
    Kabs = np.abs(Jc) @ np.abs(x.cpu().numpy())
    rhs = np.abs(ref["rhs"].cpu().numpy())
    assert np.all(np.abs(Fg - Fr) <= 1e-12 * (Kabs + rhs) + 1e-13 * np.abs(Fr).max())
