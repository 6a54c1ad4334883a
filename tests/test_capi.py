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
