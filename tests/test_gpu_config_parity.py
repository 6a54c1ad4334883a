"""Parity at the benchmark's own configurations, against the CPU oracle run on the reference's
C kernels (``oracle/_ref``).

* ~1.2M tets, assembly: ``CurlCurlAssembler.compute_stiffness_and_jacobi_matrix_c`` (the drop-in
  of ``curl_curl_assembler.py:815-932``) returns the same CSR structure as the reference's
  kernels through scipy (``interface_c.pyx:365-368``, ``K += this_K``, ``dK + K``), values within
  1e-12 of the entry's term-magnitude scale, rhs within 1e-12.
* ~40k, ~1.2M and ~4M tets, solves: the device Newton (float64, and float32 Jacobian and CG
  inside the float64 Newton loop) to the benchmark's 1e-8 relative residual; the total field B
  at 1000 seeded aperture probes within 1e-8 (relative to max |B|) of the oracle's float64
  solve to 1e-10, stored by ``tests/golden/make_config_golden.py`` (``red_mvp_solver.py:178-222``
  semantics: reference kernels, scipy's Jacobi ``cg``).
* Batched instances (``snp_solver_solve_many``): one reduced-potential and one total-potential
  variant of the batched family, their device solutions checked by the oracle's own residual.
"""

import os

import numpy as np
import pytest

import snoopy_b200 as S
from helpers import assert_csr_close, oracle_relative_residual, rel_max
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu

NU0 = 0.25 / np.pi * 1e7
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_B = 1e-8


def _fixture(name):
    path = os.path.join(GOLDEN, f"config_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"{path} not generated (tests/golden/make_config_golden.py)")
    return dict(np.load(path))


def _solver(tets):
    import bench

    msh, coils, rel = bench.workload(tets)
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=60, quad_order=2)
    solver.verbose = False
    return msh, coils, rel, solver


def _field_error(msh, solver, x, fx):
    """max |B_gpu - B_oracle| / max |B_oracle| at the fixture's probes (located on the device:
    the same elements as the oracle's CPU search)."""
    el, _ = msh.locate(fx["probes"])
    assert np.array_equal(el, fx["elements"]), "device and oracle point location disagree"
    B = solver.evaluate_B(x, fx["probes"], el)
    return float(np.abs(B - fx["B"]).max() / np.linalg.norm(fx["B"], axis=1).max())


@pytest.mark.parametrize("name,tets", [("c1", 40_000), ("c2", 1_200_000), ("c3", 4_000_000)])
def test_solves_match_fp64_oracle_at_probes(name, tets):
    fx = _fixture(name)
    msh, coils, rel, solver = _solver(tets)
    assert msh.num_elements == int(fx["tets"]) and msh.num_dofs == int(fx["dofs"])
    errs = {}
    for prec in ("fp64", "mixed"):
        x, st = solver.solve_to_residual(1e-8, precision=prec, max_newton=60)
        assert st["rel_res"] <= 1e-8, (prec, st)
        errs[prec] = _field_error(msh, solver, x, fx)
    assert errs["fp64"] < TOL_B and errs["mixed"] < TOL_B, errs


def test_c2_assembly_matches_reference_kernels(oracle_mod):
    """~1.2M tets: K, J = dK + K and rhs of the drop-in assembler against the oracle driving the
    reference's compute_K_dK_Hcurl[_red] through scipy's CSR conversion and sparse adds."""
    msh, coils, rel, solver = _solver(1_200_000)
    A = solver.curl_curl_factory
    tb = A.tables(2)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    rng = np.random.default_rng(11)
    x = rng.normal(0, 2e-3, msh.num_dofs)
    x[~solver.make_boundary_mask()] = 0.0
    P = np.einsum("qi,eid->eqd", tb.phi.reshape(tb.nq, 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad, backend="ref") for c in coils)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(NU0))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls, backend="ref")
    Kr, Jr, rr = O.compute_stiffness_and_jacobi_matrix_c(x, [Bs, np.zeros((0, 3))])
    K, J, r = A.compute_stiffness_and_jacobi_matrix_c(x, quad_order=2, source_fields=[Bs, np.zeros((0, 3))])
    sK, sJ = O.scales(x, [Bs, np.zeros((0, 3))])
    # structure: identical up to entries that one side sums to an exact 0 (dropped by the
    # reference's K += this_K) and the other to a rounding residue within the value bar
    nd = assert_csr_close(K, Kr, 1e-12, sK, zero_pattern_diff=True)
    nd += assert_csr_close(J, Jr, 1e-12, sJ, zero_pattern_diff=True)
    assert nd <= 1e-5 * Kr.nnz, nd
    assert rel_max(r, rr) < 1e-12
    assert Kr.nnz > 2e7  # the ~1.2M-tet system (about 22.5M stored entries)


def test_batched_instances_match_oracle_residual(oracle_mod):
    """A reduced-potential and a total-potential variant solved together by snp_solver_solve_many:
    the oracle (reference kernels) finds each device solution at the 1e-8 relative residual."""
    from snoopy_b200 import batch as B

    V = B.sample_variants(4, seed=5)[:2]
    for v in V:
        v["tets"] = min(v["tets"], 60000)
    inst = [B.Instance(v) for v in V]
    st = B.solve_many(inst, rtol=1e-8)
    assert {i.v["kind"] for i in inst} == {"reduced", "total"}
    for ins, s in zip(inst, st):
        assert s["status"] == 0 and s["rel_res"] <= 1e-8, s
        assert oracle_relative_residual(oracle_mod, ins, ins.x.cpu().numpy()) <= 1.5e-8
