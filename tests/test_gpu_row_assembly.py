"""Two-phase CSR assembly (element records, then one gather per CSR row) against the element
kernels that add into the CSR with atomics, its determinism, and the solver's use of it.

Bars: every entry within 1e-12 of the largest entry of its row (both sides sum the same element
contributions in float64, in different orders and groupings); vectors within 1e-12 of their
max; the row gather bitwise repeatable, J bitwise K + dK.  The oracle comparisons of the same
path are the golden and assembler tests of tests/test_gpu_parity.py, which now run on it.
"""

import os

import numpy as np
import pytest
import torch

import snoopy_b200 as S
from snoopy_b200 import _lib
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu

NU0 = 0.25 / np.pi * 1e7


def _row_close(a, b, row_ptr, tol=1e-12):
    a = a.double().cpu().numpy()
    b = b.double().cpu().numpy()
    rp = row_ptr.cpu().numpy()
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    rmax = np.zeros(len(rp) - 1)
    np.maximum.at(rmax, rows, np.abs(b))
    err = np.abs(a - b) / np.maximum(rmax[rows], 1e-300)
    return float(err.max()) if err.size else 0.0


def _vec_close(a, b):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _problem(ntet=30000, seed=4, diluted=False):
    msh = M.window_frame_mesh(ntet, jitter=0.15, seed=seed)
    rel = MAT.atan_reluctance()
    mats = [rel, S.ConstantReluctance(NU0)]
    if diluted:
        dil = MAT.Dilution(0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, z_pos=-0.25, z_len=0.5)
        A = S.CurlCurlAssemblerDiluted(msh, [M.TAG_IRON, M.TAG_AIR], mats, [dil, None])
    else:
        A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], mats)
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 2e-3, msh.num_dofs)
    tb = A.tables(2)
    Bs = rng.normal(0, 0.5, (len(msh.domain_elements(M.TAG_IRON)) * tb.nq, 3))
    return msh, A, x, [Bs, np.zeros((0, 3))]


@pytest.mark.parametrize("diluted", [False, True])
def test_rows_match_atomic_kernels(diluted):
    msh, A, x, sf = _problem(diluted=diluted)
    pat = A.pattern
    assert pat.rows_supported
    kw = dict(K=True, J=True, dK=True, rhs=True, F=True)
    R = A.assemble_device(x, 2, sf, method="rows", **kw)
    R2 = A.assemble_device(x, 2, sf, method="rows", **kw)
    T = A.assemble_device(x, 2, sf, method="atomic", **kw)
    torch.cuda.synchronize()
    for key in ("K", "dK", "J"):
        assert torch.equal(R[key], R2[key]), key  # bitwise repeatable
        err = _row_close(R[key], T[key], pat.row_ptr)
        assert err < 1e-12, (key, err)
    assert torch.equal(R["J"], R["K"] + R["dK"])  # J = K + dK entry by entry, as the reference's dK + K
    for key in ("rhs", "F"):
        assert torch.equal(R[key], R2[key]), key
        assert _vec_close(R[key], T[key]) < 1e-12, key
    assert R["rhs"].abs().max() > 0 and R["dK"].abs().max() > 0


def test_rows_subsets_of_outputs():
    """Requesting fewer outputs writes the same values for those requested (the records differ)."""
    msh, A, x, sf = _problem(12000, seed=8)
    full = A.assemble_device(x, 2, sf, method="rows", K=True, J=True, dK=True, rhs=True, F=True)
    jf = A.assemble_device(x, 2, sf, method="rows", K=False, J=True, rhs=False, F=True)
    k_only = A.assemble_device(x, 2, sf, method="rows", K=True, J=False, rhs=False)
    f_only = A.assemble_device(x, 2, sf, method="rows", K=False, J=False, rhs=False, F=True)
    d_only = A.assemble_device(x, 2, sf, method="rows", K=False, J=False, dK=True, rhs=False)
    torch.cuda.synchronize()
    assert torch.equal(k_only["K"], full["K"])
    assert torch.equal(d_only["dK"], full["dK"])
    assert torch.equal(f_only["F"], full["F"])
    assert torch.equal(jf["F"], full["F"])
    assert torch.equal(jf["J"], full["J"])


def test_solver_assembly_rows_vs_atomic():
    """snp_solver_assemble (the solver's CSR assembly: reference-semantics Newton, the drop-in
    export) on the row gather by default and on the atomic kernels with SNP_ASSEMBLY=atomic."""
    msh = M.window_frame_mesh(20000, jitter=0.15, seed=5)
    coils = msh.geometry.coils()
    rel = MAT.atan_reluctance()

    def make():
        s = S.RedMVPSolver(msh, coils, [M.TAG_IRON], [M.TAG_AIR], [rel], max_newton_iterations=20, quad_order=2)
        s.verbose = False
        return s

    rows = make()
    os.environ["SNP_ASSEMBLY"] = "atomic"
    try:
        atomic = make()
        eng_a = atomic.newton_engine()
    finally:
        del os.environ["SNP_ASSEMBLY"]
    eng_r = rows.newton_engine()
    x = torch.as_tensor(np.random.default_rng(1).normal(0, 2e-3, msh.num_dofs), device="cuda")
    nnz, n = eng_r.pattern.nnz, msh.num_dofs
    out = {}
    for name, eng in (("rows", eng_r), ("rows2", eng_r), ("atomic", eng_a)):
        K = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        J = torch.zeros(nnz, dtype=torch.float64, device="cuda")
        F = torch.zeros(n, dtype=torch.float64, device="cuda")
        rhs = torch.zeros(n, dtype=torch.float64, device="cuda")
        _lib.call("snp_solver_assemble", eng.handle, _lib.ptr(x), _lib.ptr(K), _lib.ptr(J), _lib.ptr(rhs), _lib.ptr(F),
                  _lib.stream_ptr())
        out[name] = (K, J, rhs, F)
    torch.cuda.synchronize()
    for a, b in zip(out["rows"], out["rows2"]):
        assert torch.equal(a, b)
    rp = eng_r.pattern.row_ptr
    assert _row_close(out["rows"][0], out["atomic"][0], rp) < 1e-12
    assert _row_close(out["rows"][1], out["atomic"][1], rp) < 1e-12
    assert _vec_close(out["rows"][2], out["atomic"][2]) < 1e-12
    assert _vec_close(out["rows"][3], out["atomic"][3]) < 1e-12
    # the reference-semantics Newton solve (CSR assembly + point-Jacobi PCG) on both assemblies
    x1 = rows.solve(1e-8)
    x2 = atomic.solve(1e-8)
    d = float(np.abs(x1 - x2).max() / np.abs(x2).max())
    assert d < 1e-6, d


def test_gradgrad_assembly_is_repeatable_and_matches_atomic():
    """Grad-grad (P1) assembly: each CSR entry gets the sum of the call's contributions in
    element order, so two assemblies agree bit for bit; SNP_ASSEMBLY=atomic (float64 atomics per
    contribution) agrees to rounding (1e-12 of the row's largest entry)."""
    msh = M.window_frame_mesh(8000, jitter=0.1, seed=2, coils=True)
    perm = MAT.atan_permeability()
    tags = [M.TAG_COIL_1, M.TAG_IRON]
    x = np.random.default_rng(3).normal(0, 30.0, msh.num_nodes)
    mus = [S.ConstantPermeability(1.0), perm]

    def run():
        G = S.GradGradAssembler(msh, tags)
        K, J = G.compute_stiffness_and_jacobi_matrix_c(x, mus, quad_order=2, device=True)
        torch.cuda.synchronize()
        return K.values().clone(), J.values().clone(), K.crow_indices()

    K1, J1, rp = run()
    K2, J2, _ = run()
    assert torch.equal(K1, K2) and torch.equal(J1, J2)
    os.environ["SNP_ASSEMBLY"] = "atomic"
    try:
        Ka, Ja, _ = run()
    finally:
        del os.environ["SNP_ASSEMBLY"]
    assert _row_close(K1, Ka, rp) < 1e-12
    assert _row_close(J1, Ja, rp) < 1e-12
    assert K1.abs().max() > 0
