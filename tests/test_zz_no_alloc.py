"""snp_pcg_noalloc: the CG solve for callers that cannot allocate device memory while they
solve (their device memory belongs to a pool set up at start-up, or cudaFree's device-wide
synchronisation is not acceptable where they solve).  Its work vectors come from a static
device array instead of cudaMalloc.

Checked through the C ABI against snp_pcg, the allocating entry point, on the same system
twice in a row (the second call reuses the array the first one left behind).  This file is
collected last so that a run stopping at the first failure has run every other test.
"""

import ctypes

import numpy as np
import pytest

import snoopy_b200 as S
from helpers import rel_max
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu


def _system():
    from snoopy_b200.device import upload

    msh = M.window_frame_mesh(30000, jitter=0.15, seed=21)
    rel = MAT.atan_reluctance()
    A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [rel, S.ConstantReluctance(0.25 / np.pi * 1e7)])
    rng = np.random.default_rng(2)
    out = A.assemble_device(rng.normal(0, 1e-3, msh.num_dofs), 2, (), K=False, J=True, rhs=False)
    pat = out["pattern"]
    J = pat.to_scipy(out["J"])
    mask = np.ones(msh.num_dofs, bool)
    mask[msh.get_edge_boundary_dofs() - 1] = False
    b = np.zeros(msh.num_dofs)
    b[mask] = J[mask, :][:, mask] @ rng.normal(0, 1.0, int(mask.sum()))  # consistent (J is singular)
    return msh.num_dofs, pat, out["J"], upload(mask.astype(np.uint8), np.uint8), upload(b, np.float64)


def _solve(name, n, pat, J, fm, b, x0=None, maxiter=-1, expect_rc=0):
    """One call through the C ABI; returns (x, iterations, final ||r||) after checking the status."""
    from snoopy_b200 import _lib
    from snoopy_b200.device import upload, zeros

    x = zeros(n) if x0 is None else upload(x0, np.float64)
    its = ctypes.c_int64()
    res = ctypes.c_double()
    fn = getattr(_lib.load(), name)
    rc = fn(n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(J), _lib.ptr(fm), _lib.ptr(b), _lib.ptr(x), 1e-9,
            0.0, maxiter, ctypes.byref(its), ctypes.byref(res), _lib.stream_ptr())
    assert rc == expect_rc, (name, rc, _lib.load().snp_last_error())
    return x[:n].cpu().numpy(), its.value, res.value


def _same(*args, **kw):
    """The allocating and the allocation-free entry point agree on iterations, x and ||r||."""
    x_ref, its_ref, res_ref = _solve("snp_pcg", *args, **kw)
    for _ in range(2):
        x, its, res = _solve("snp_pcg_noalloc", *args, **kw)
        assert its == its_ref
        assert rel_max(x, x_ref) < 1e-12
        assert abs(res - res_ref) <= 1e-12 * max(res_ref, 1e-300) + 1e-300
    return x_ref, its_ref


def test_noalloc_pcg_matches_allocating_pcg():
    n, pat, J, fm, b = _system()
    assert n <= 262144
    x_ref, its_ref, res_ref = _solve("snp_pcg", n, pat, J, fm, b)
    for _ in range(2):
        x, its, res = _solve("snp_pcg_noalloc", n, pat, J, fm, b)
        assert its == its_ref
        assert rel_max(x, x_ref) < 1e-12
        assert abs(res - res_ref) <= 1e-12 * max(res_ref, 1e-300) + 1e-300


def test_noalloc_pcg_other_paths_match_allocating_pcg():
    """No free mask (every row free), a nonzero initial guess, the iteration cap, and a zero
    diagonal on a free row: same iterations, iterate and status as snp_pcg."""
    from snoopy_b200.device import upload

    n, pat, J, fm, b = _system()
    rng = np.random.default_rng(5)
    # every row free: a regularised copy keeps the system definite (J + 1e-3 max|J_ii| I)
    Jreg = J.clone()
    diag = pat.diag_pos.long()
    Jreg[diag] += 1e-3 * float(J[diag].abs().max())
    _same(n, pat, Jreg, None, b)
    # warm start from a random guess on the free DoFs
    _same(n, pat, J, fm, b, x0=rng.normal(0, 1e-3, n))
    # the cap: one iteration, SNP_NOT_CONVERGED, the last iterate returned
    _, its = _same(n, pat, J, fm, b, maxiter=1, expect_rc=3)
    assert its == 1
    # a zeroed diagonal entry on a free row: SNP_ZERO_PIVOT before any iteration
    free_rows = np.flatnonzero(fm.cpu().numpy())
    Jz = J.clone()
    Jz[diag[int(free_rows[len(free_rows) // 2])]] = 0.0
    for name in ("snp_pcg", "snp_pcg_noalloc", "snp_pcg_noalloc"):
        _solve(name, n, pat, Jz, fm, b, expect_rc=5)
    # and a good call right after the failed ones
    _same(n, pat, J, fm, upload(b.cpu().numpy(), np.float64))


def test_noalloc_pcg_rejects_oversized_systems():
    from snoopy_b200 import _lib

    n, pat, J, fm, b = _system()
    rc = _lib.load().snp_pcg_noalloc(262145, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(J), _lib.ptr(fm),
                                     _lib.ptr(b), _lib.ptr(b), 1e-9, 0.0, -1, None, None, _lib.stream_ptr())
    assert rc == 1
    assert b"static work space" in _lib.load().snp_last_error()
