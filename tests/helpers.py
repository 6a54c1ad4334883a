"""Comparison helpers shared by the tests."""

import numpy as np
from scipy.sparse import csr_array


class TableReluctance:
    """A PCHIP reluctance given by its stored PP tables (duck-typed like ``Reluctance``)."""

    def __init__(self, c, x):
        self.c, self.x = np.asarray(c), np.asarray(x)

    def get_type_spec(self):
        return 1

    def get_spline_information(self):
        return self.c, self.x


class TablePermeability:
    """A B-spline permeability given by its stored tables (duck-typed like ``Permeability``)."""

    def __init__(self, t, c, k, hmin, muhmin):
        self.t, self.c, self.k, self.H_min, self.muhmin = np.asarray(t), np.asarray(c), int(k), float(hmin), float(muhmin)

    def get_type_spec(self):
        return 1

    def get_spline_information(self):
        return self.t, self.c, self.k, self.H_min, self.muhmin


def golden_materials(g):
    return (TableReluctance(g["rel_c"], g["rel_x"]),
            TablePermeability(g["perm_t"], g["perm_c"], g["perm_k"], g["perm_hmin"], g["perm_muhmin"]))


def csr_from(g, prefix, n):
    return csr_array((g[prefix + "_data"], g[prefix + "_indices"], g[prefix + "_indptr"]), shape=(n, n))


def abs_contrib(ti, tj, v, n):
    """Sum of absolute triplet contributions per CSR entry: the scale of its rounding error."""
    return csr_array((np.abs(v), (ti, tj)), shape=(n, n))


def assert_same_pattern(A, B):
    """CSR structure identical: same row pointers and the same (sorted) column indices."""
    A = csr_array(A)
    B = csr_array(B)
    A.sort_indices()
    B.sort_indices()
    assert A.shape == B.shape
    assert np.array_equal(A.indptr, B.indptr), "row pointers differ"
    assert np.array_equal(A.indices, B.indices), "column indices differ"


def assert_csr_close(A, B, rtol=1e-12, scale=None, atol_rel=0.0):
    """Same pattern and |A - B| <= rtol * (|B| + scale) entrywise.

    ``scale`` (CSR with B's pattern) is the sum of absolute element contributions of each
    entry; for entries whose contributions cancel it bounds the rounding error that any
    summation order makes, so the tolerance stays relative to the data.
    """
    assert_same_pattern(A, B)
    a = csr_array(A)
    b = csr_array(B)
    a.sort_indices()
    b.sort_indices()
    ref = np.abs(b.data)
    if scale is not None:
        s = csr_array(scale)
        s.sort_indices()
        assert np.array_equal(s.indices, b.indices)
        ref = np.maximum(ref, s.data)
    bound = rtol * ref + atol_rel * (np.abs(b.data).max() if b.nnz else 0.0)
    err = np.abs(a.data - b.data)
    bad = err > bound
    assert not bad.any(), (f"{bad.sum()} of {b.nnz} entries off: max err {err.max():.3e}, "
                           f"worst rel {(err / np.maximum(ref, 1e-300)).max():.3e}")


def rel_max(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
