"""The C-ABI library: it loads without a GPU and exports every function include/*.h declares."""

import ctypes
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?\w+\s*\*?\s*(snp_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert "snp_curlcurl_assemble" in names and "snp_pcg" in names and "snp_solver_solve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from snoopy_b200 import _lib

    L = _lib.load()
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing
    assert L.snp_version() == 1


def test_binding_covers_header():
    from snoopy_b200 import _lib

    assert _declared() <= set(_lib.EXPORTED)


def test_error_path_without_gpu():
    """A NULL handle is rejected on the host with a message, before any device work."""
    from snoopy_b200 import _lib

    L = _lib.load()
    rc = L.snp_pattern_info(None, None, None, None, None)
    assert rc == 1
    assert b"NULL" in L.snp_last_error()


def test_library_is_sm100a_build():
    from snoopy_b200 import _lib

    path = _lib.LIB_PATH
    assert os.path.exists(path)
    blob = open(path, "rb").read()
    assert b"sm_100a" in blob


def test_galerkin_spd_solve_on_host():
    """snp_spd_solve (the host solve of the Galerkin step) against numpy: badly scaled SPD
    systems, a dependent basis column left out, and a zero diagonal rejected."""
    import ctypes

    import numpy as np

    from snoopy_b200 import _lib

    L = _lib.load()
    P = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(3)
    for m in (1, 7, 64, 128):
        B = rng.normal(size=(m, m))
        D = np.diag(np.exp(rng.normal(size=m) * 3))
        A = D @ (B @ B.T + 1e-2 * np.eye(m)) @ D
        g = rng.normal(size=m)
        c = np.zeros(m)
        assert L.snp_spd_solve(m, A.ctypes.data_as(P), g.ctypes.data_as(P), c.ctypes.data_as(P)) == 0
        want = -np.linalg.solve(A, g)
        assert np.abs(c - want).max() <= 1e-8 * np.abs(want).max(), m
    # a repeated column: the dependent direction is dropped and the system is still solved
    m = 6
    B = rng.normal(size=(m, m))
    A = B @ B.T
    A[:, 5] = A[:, 4]
    A[5, :] = A[4, :]
    g = rng.normal(size=m)
    g[5] = g[4]
    c = np.zeros(m)
    assert L.snp_spd_solve(m, A.ctypes.data_as(P), g.ctypes.data_as(P), c.ctypes.data_as(P)) == 0
    assert c[5] == 0.0 and np.abs(A @ c + g).max() <= 1e-10 * np.abs(g).max()
    A = np.eye(3)
    A[1, 1] = 0.0
    g = np.ones(3)
    assert L.snp_spd_solve(3, A.ctypes.data_as(P), g.ctypes.data_as(P), c.ctypes.data_as(P)) == 1
    assert b"diagonal" in L.snp_last_error()


def test_two_phase_assembly_block_counts():
    """The element-value blocks of the two-phase curl-curl assembly (no GPU needed): 21 per
    matrix (upper triangle of the 6 x 6 element matrix), 6 per vector; unknown bits refused."""
    import ctypes

    from snoopy_b200 import _lib

    L = _lib.load()
    out = ctypes.c_int32()
    for parts, want in ((_lib.TERMS_K, 21), (_lib.TERMS_K | _lib.TERMS_DK, 42), (_lib.TERMS_J | _lib.TERMS_F, 27),
                        (_lib.TERMS_K | _lib.TERMS_DK | _lib.TERMS_RHS, 48), (_lib.TERMS_F, 6), (0, 0)):
        assert L.snp_curlcurl_terms_stride(parts, ctypes.byref(out)) == 0
        assert out.value == want, (parts, out.value)
    assert L.snp_curlcurl_terms_stride(64, ctypes.byref(out)) != 0
    assert b"unknown bits" in L.snp_last_error()
