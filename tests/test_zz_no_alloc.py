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


def _solve(name, n, pat, J, fm, b):
    from snoopy_b200 import _lib
    from snoopy_b200.device import zeros

    x = zeros(n)
    its = ctypes.c_int64()
    res = ctypes.c_double()
    _lib.call(name, n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(J), _lib.ptr(fm), _lib.ptr(b),
              _lib.ptr(x), 1e-9, 0.0, -1, ctypes.byref(its), ctypes.byref(res), _lib.stream_ptr())
    return x[:n].cpu().numpy(), its.value, res.value


def test_noalloc_pcg_matches_allocating_pcg():
    n, pat, J, fm, b = _system()
    assert n <= 262144
    x_ref, its_ref, res_ref = _solve("snp_pcg", n, pat, J, fm, b)
    for _ in range(2):
        x, its, res = _solve("snp_pcg_noalloc", n, pat, J, fm, b)
        assert its == its_ref
        assert rel_max(x, x_ref) < 1e-12
        assert abs(res - res_ref) <= 1e-12 * max(res_ref, 1e-300) + 1e-300


def test_noalloc_pcg_rejects_oversized_systems():
    from snoopy_b200 import _lib

    n, pat, J, fm, b = _system()
    rc = _lib.load().snp_pcg_noalloc(262145, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(J), _lib.ptr(fm),
                                     _lib.ptr(b), _lib.ptr(b), 1e-9, 0.0, -1, None, None, _lib.stream_ptr())
    assert rc == 1
    assert b"static work space" in _lib.load().snp_last_error()
