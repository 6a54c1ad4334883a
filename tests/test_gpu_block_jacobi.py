"""Block-Jacobi preconditioner of the matrix-free Newton Jacobian: its blocks against the
oracle's assembled Jacobian, and Newton with it against Newton with point Jacobi."""

import numpy as np
import pytest
import torch

import snoopy_b200 as S
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M
from snoopy_b200.device import upload

pytestmark = pytest.mark.gpu

NU0 = 0.25 / np.pi * 1e7


def _setup(ntet, seed=7):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    coils = msh.geometry.coils()
    rel = MAT.atan_reluctance()
    solver = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=50, quad_order=2)
    solver.verbose = False
    return msh, coils, rel, solver


def _oracle(oracle_mod, msh, coils, rel, solver):
    tb = solver.curl_curl_factory.tables(solver.quad_order)
    iron = msh.domain_elements(M.TAG_IRON)
    air = msh.domain_elements(M.TAG_AIR)
    P = np.einsum("qi,eid->eqd", tb.phi.reshape(tb.nq, 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
    Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad) for c in coils)
    mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                 reluctance=rel),
            dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                 reluctance=S.ConstantReluctance(NU0))]
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls)
    return O, [Bs, np.zeros((0, 3))]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_block_inverse_matches_oracle_blocks(oracle_mod, precision):
    """z = M r from the device blocks against the inverses of the same diagonal blocks of the
    oracle's assembled Jacobian (float32 storage of the inverse: 1e-5 of max |z|)."""
    msh, coils, rel, solver = _setup(6000)
    eng = solver.newton_engine()
    assert eng.block_jacobi
    x, st = solver.solve_to_residual(1e-6, return_device=True)  # a state with saturated iron
    O, sf = _oracle(oracle_mod, msh, coils, rel, solver)
    _, J, _ = O.compute_stiffness_and_jacobi_matrix_c(x.cpu().numpy(), sf)
    J = J.tocsr()
    mask = solver.make_boundary_mask()
    from snoopy_b200.newton import dof_blocks

    meta = dof_blocks(msh.edges[:, 0], mask)
    r = np.random.default_rng(2).standard_normal(msh.num_dofs)
    want = np.zeros_like(r)
    i, n = 0, msh.num_dofs
    sizes = []
    while i < n:
        s = int(meta[i] >> 8)
        if mask[i]:
            idx = np.arange(i, i + s)
            want[idx] = np.linalg.solve(J[idx][:, idx].toarray(), r[idx])
        sizes.append(s)
        i += s
    assert np.mean(sizes) > 2  # edges sharing their lower node (many boundary DoFs at this size)
    eng.assemble_tensors(x, precision)
    z, fallbacks = eng.precond_apply(upload(r, np.float64), precision)
    z = z.cpu().numpy()
    assert fallbacks == 0
    assert np.all(z[~mask] == 0.0)
    err = np.abs(z - want).max() / np.abs(want).max()
    assert err < (1e-5 if precision == "fp64" else 1e-4), err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_block_jacobi_newton_matches_point_jacobi(precision):
    """Newton to 1e-10 with block Jacobi and with point Jacobi: the same field, fewer CG
    iterations with the blocks, and bitwise repeatable."""
    msh, coils, rel, solver = _setup(20000)
    eng = solver.newton_engine()
    probes = msh.geometry.aperture_probes(300)
    el, _ = msh.locate(probes)
    tol = 1e-10 if precision == "fp64" else 1e-8
    xb, sb = solver.solve_to_residual(tol, precision=precision, return_device=True)
    xb2, sb2 = solver.solve_to_residual(tol, precision=precision, return_device=True)
    eng.set_preconditioner("jacobi")
    try:
        xj, sj = solver.solve_to_residual(tol, precision=precision, return_device=True)
    finally:
        eng.set_preconditioner("block")
    assert sb["rel_res"] <= tol and sj["rel_res"] <= tol
    assert sb["cg_iterations"] < 0.75 * sj["cg_iterations"], (sb["cg_iterations"], sj["cg_iterations"])
    assert sb2["cg_iterations"] == sb["cg_iterations"] and torch.equal(xb, xb2)
    A = solver.curl_curl_factory
    Bb = A.compute_B_at_points(xb, probes, el)
    Bj = A.compute_B_at_points(xj, probes, el)
    err = np.linalg.norm(Bb - Bj, axis=1).max() / np.linalg.norm(Bj, axis=1).max()
    assert err < (1e-8 if precision == "fp64" else 1e-6), err


def test_block_partition_is_checked():
    msh, coils, rel, solver = _setup(2000)
    eng = solver.newton_engine()
    meta = np.full(msh.num_dofs, 1 << 8, dtype=np.uint16)
    meta[0] = (2 << 8)  # claims a block of two that the next entry does not continue
    from snoopy_b200._lib import SnpError

    with pytest.raises(SnpError):
        eng._set_blocks(meta)
    eng.set_preconditioner("block")
    assert eng.block_jacobi


def test_exported_blocks_and_inverses(oracle_mod):
    """The device block rows (snp_solver_block_jacobi_export) equal the oracle's Jacobian on
    each block, and the stored inverses are the symmetric inverses of those blocks (float32)."""
    from snoopy_b200 import _lib
    from snoopy_b200.newton import dof_blocks

    msh, coils, rel, solver = _setup(6000)
    eng = solver.newton_engine()
    x, _ = solver.solve_to_residual(1e-4, return_device=True)
    O, sf = _oracle(oracle_mod, msh, coils, rel, solver)
    _, J, _ = O.compute_stiffness_and_jacobi_matrix_c(x.cpu().numpy(), sf)
    J = J.tocsr()
    mask = solver.make_boundary_mask()
    meta = dof_blocks(msh.edges[:, 0], mask)
    n = msh.num_dofs
    eng.assemble_tensors(x, "fp64")
    bm = torch.zeros(n * 8, dtype=torch.float64, device="cuda")
    bi = torch.zeros(n * 8, dtype=torch.float32, device="cuda")
    _lib.call("snp_solver_block_jacobi_export", eng.handle, 0, _lib.ptr(bm), _lib.ptr(bi), _lib.stream_ptr(None))
    torch.cuda.synchronize()
    bm = bm.cpu().numpy().reshape(n, 8)
    bi = bi.cpu().numpy().reshape(n, 8).astype(np.float64)
    i = 0
    worst_rows = worst_inv = 0.0
    while i < n:
        s = int(meta[i] >> 8)
        assert not bm[i:i + s, s:].any() and not bi[i:i + s, s:].any()
        if mask[i]:
            B = J[i:i + s, i:i + s].toarray()
            worst_rows = max(worst_rows, np.abs(bm[i:i + s, :s] - B).max() / np.abs(B).max())
            X = np.linalg.inv(B)
            assert np.array_equal(bi[i:i + s, :s], bi[i:i + s, :s].T)
            worst_inv = max(worst_inv, np.abs(bi[i:i + s, :s] - X).max() / np.abs(X).max())
        else:
            assert s == 1 and not bi[i].any()
        i += s
    assert worst_rows < 1e-12, worst_rows
    # float32 rounding of entries up to cond(block) ~ 1e4 times 6e-8
    assert worst_inv < 2e-3, worst_inv


@pytest.mark.parametrize("precond", ["block", "jacobi"])
def test_one_launch_pcg_reaches_the_graph_loops_answer(precond):
    """The Krylov loop as one cooperative launch (SNP_PCG_COOP=1: grid barriers between the
    element and DoF passes, every block summing the partials itself) solves the same Newton
    problem as the graph-captured loop: both reach 1e-8 and the fields agree to that level."""
    import os

    msh, coils, rel, solver = _setup(20000, seed=9)
    eng = solver.newton_engine()
    eng.set_preconditioner(precond)
    x_graph, st_g = solver.solve_to_residual(1e-8)
    os.environ["SNP_PCG_COOP"] = "1"
    try:
        x_coop, st_c = solver.solve_to_residual(1e-8)
        x_coop2, _ = solver.solve_to_residual(1e-8)
    finally:
        del os.environ["SNP_PCG_COOP"]
    eng.set_preconditioner("block")
    assert st_g["rel_res"] <= 1e-8 and st_c["rel_res"] <= 1e-8
    assert abs(st_c["newton_iterations"] - st_g["newton_iterations"]) <= 1
    assert np.array_equal(x_coop, x_coop2)  # deterministic run to run
    probes = msh.geometry.aperture_probes(300)
    el, _ = msh.locate(probes)
    Bg = solver.evaluate_B(x_graph, probes, el)
    Bc = solver.evaluate_B(x_coop, probes, el)
    assert float(np.abs(Bc - Bg).max() / np.abs(Bg).max()) < 1e-7


@pytest.mark.parametrize("precond", ["block", "jacobi"])
def test_gmres_newton_reaches_the_cg_answer(precond):
    """Newton steps solved by restarted GMRES (snp_solver_set_krylov, right-preconditioned by the
    same block or point Jacobi) reach the 1e-8 residual and the CG solve's field: B at 300
    aperture probes within 1e-7 of the CG answer (both stop at 1e-8), bitwise repeatable; a
    mixed-precision solve with GMRES is refused."""
    from snoopy_b200._lib import SnpError

    msh, coils, rel, solver = _setup(20000, seed=11)
    eng = solver.newton_engine()
    eng.set_preconditioner(precond)
    x_cg, st_cg = solver.solve_to_residual(1e-8)
    eng.set_krylov("gmres", restart=40)
    try:
        x_gm, st_gm = solver.solve_to_residual(1e-8)
        x_gm2, _ = solver.solve_to_residual(1e-8)
        with pytest.raises(SnpError):
            solver.solve_to_residual(1e-8, precision="mixed")
    finally:
        eng.set_krylov("cg")
        eng.set_preconditioner("block")
    assert st_gm["rel_res"] <= 1e-8 and st_cg["rel_res"] <= 1e-8
    assert st_gm["cg_iterations"] > 0
    assert np.array_equal(x_gm, x_gm2)
    probes = msh.geometry.aperture_probes(300)
    el, _ = msh.locate(probes)
    Bc = solver.evaluate_B(x_cg, probes, el)
    Bg = solver.evaluate_B(x_gm, probes, el)
    assert float(np.abs(Bg - Bc).max() / np.abs(Bc).max()) < 1e-7


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_iterations_per_graph_body_do_not_change_the_answer(precision):
    """The Krylov graph's loop body holds SNP_PCG_UNROLL CG iterations (read when the graph is
    built); the passes of a finished solve return at once, so one and four iterations per body
    give bitwise the same Newton solve, CG count and residual."""
    import os

    out = {}
    for unroll in ("1", "4"):
        os.environ["SNP_PCG_UNROLL"] = unroll
        try:
            msh, coils, rel, solver = _setup(15000, seed=11)
            x, st = solver.solve_to_residual(1e-8, precision=precision)
        finally:
            del os.environ["SNP_PCG_UNROLL"]
        out[unroll] = (x, st)
    (x1, s1), (x4, s4) = out["1"], out["4"]
    assert s1["rel_res"] <= 1e-8
    assert np.array_equal(x1, x4)
    assert (s1["newton_iterations"], s1["cg_iterations"], s1["res"]) == (s4["newton_iterations"], s4["cg_iterations"],
                                                                         s4["res"])
