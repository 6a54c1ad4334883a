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


def scale_csr(ti, tj, s, n):
    """CSR of the per-entry sums of term magnitudes (``scales`` output of the oracle)."""
    return csr_array((s, (ti, tj)), shape=(n, n))


def _at(M, rows, cols):
    if len(rows) == 0:
        return np.zeros(0)
    return np.asarray(M[rows, cols]).reshape(-1)


def assert_csr_close(A, B, rtol=1e-12, scale=None, atol_rel=0.0, zero_pattern_diff=False):
    """CSR parity: same structure and |A - B| <= rtol * max(|B|, scale) entrywise.

    ``scale`` (CSR, any superset of the pattern) holds, per entry, the sum of the magnitudes
    of the terms that make it up; rounding error of any evaluation order is bounded by a
    small multiple of it, so the bound stays relative to the data even where terms cancel.
    ``zero_pattern_diff``: for matrices with exact zeros dropped (scipy's ``K += this_K``),
    an entry stored on one side only is accepted when it is zero up to that scale (one
    side's arithmetic gave an exact 0, the other a rounding residue); their number is
    returned.
    """
    a = csr_array(A)
    b = csr_array(B)
    a.sort_indices()
    b.sort_indices()
    n_diff = 0
    if not zero_pattern_diff:
        assert_same_pattern(a, b)
    else:
        pa = csr_array((np.ones(a.nnz), a.indices, a.indptr), shape=a.shape)
        pb = csr_array((np.ones(b.nnz), b.indices, b.indptr), shape=b.shape)
        n_diff = int((pa - pb).count_nonzero())
    d = csr_array(a - b)
    d.eliminate_zeros()
    if d.nnz == 0:
        return n_diff
    rows, cols = d.nonzero()
    err = np.abs(_at(d, rows, cols))
    ref = np.abs(_at(b, rows, cols))
    if scale is not None:
        ref = np.maximum(ref, np.abs(_at(csr_array(scale), rows, cols)))
    bound = rtol * ref + atol_rel * (np.abs(b.data).max() if b.nnz else 0.0)
    bad = err > bound
    assert not bad.any(), (f"{bad.sum()} of {b.nnz} entries off: max err {err.max():.3e}, "
                           f"worst rel {(err / np.maximum(ref, 1e-300)).max():.3e}")
    return n_diff


def rel_max(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


NU0 = 0.25 / np.pi * 1e7


def oracle_total_rhs(oracle_mod, msh, Phi, tag=None):
    """rhs of the total-potential formulation from the coil's electric potential: the oracle's
    Laplace solve (``laplace_subdomain_solver.py:117-158``) and a numpy statement of
    ``compute_rhs_electric_potential`` (``curl_curl_assembler.py:1154-1284``)."""
    from snoopy_b200 import finite_element as FE
    from snoopy_b200 import mesh as M

    tag = M.TAG_COIL_1 if tag is None else tag
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    t1, t2 = msh.coil_terminals[tag]
    el = msh.domain_elements(tag)
    phi = oracle_mod.laplace_subdomain_solve(msh.nodes, msh.cells[el], np.concatenate([t1, t2]),
                                             msh.domain_nodes_mask(tag), Phi, t1, t2, w, q, dphi)
    X = msh.nodes[msh.cells[el]]
    Jm = np.einsum("eid,il->edl", X, dphi[0])
    Ji = np.linalg.inv(Jm)
    det = np.linalg.det(Jm)
    G = np.einsum("eld,el->ed", Ji, np.einsum("il,ei->el", dphi[0], phi[msh.cells[el]]))
    s = FE.orientation_signs(msh.orientations[el])
    wq = np.einsum("eld,qjl->eqjd", Ji, FE.edge_basis_functions(q)) * s[:, None, :, None]
    rhs = np.zeros(msh.num_dofs)
    np.add.at(rhs, msh.elem_edges[el].reshape(-1), np.einsum("eqjd,ed,q,e->ej", wq, G, w, det).reshape(-1))
    return rhs


def oracle_relative_residual(oracle_mod, ins, x):
    """||F_free(x)|| / ||F_free(0)|| of a batched-family instance (``snoopy_b200.batch.Instance``)
    by the oracle on the reference's C kernels: its Biot-Savart source (reduced variants) or its
    electric-potential rhs (total-potential variants), its materials, its Dirichlet mask."""
    import snoopy_b200 as S
    from snoopy_b200 import mesh as M

    msh = ins.mesh
    tb = ins.solver.curl_curl_factory.tables(2)
    mats_list = ins.solver.curl_curl_factory.material_list
    if ins.v["kind"] == "reduced":
        iron = msh.domain_elements(M.TAG_IRON)
        air = msh.domain_elements(M.TAG_AIR)
        P = np.einsum("qi,eid->eqd", tb.phi.reshape(tb.nq, 4), msh.nodes[msh.cells[iron]]).reshape(-1, 3)
        Bs = sum(oracle_mod.compute_B_line_segs_cpp(c.get_segments(), P, c.current, c.rad, backend="ref")
                 for c in ins.solver.coil_list)
        mats = [dict(cells=msh.cells[iron], glob_ids=msh.elem_edges[iron], orientations=msh.orientations[iron],
                     reluctance=mats_list[0]),
                dict(cells=msh.cells[air], glob_ids=msh.elem_edges[air], orientations=msh.orientations[air],
                     reluctance=S.ConstantReluctance(NU0))]
        sf, extra = [Bs, np.zeros((0, 3))], 0.0
    else:
        mats = []
        for tag in (M.TAG_COIL_1, M.TAG_IRON, M.TAG_AIR):
            e = msh.domain_elements(tag)
            mats.append(dict(cells=msh.cells[e], glob_ids=msh.elem_edges[e], orientations=msh.orientations[e],
                             reluctance=mats_list[1] if tag == M.TAG_IRON else S.ConstantReluctance(NU0)))
        sf, extra = (), oracle_total_rhs(oracle_mod, msh, ins.phi)
    O = oracle_mod.OracleCurlCurlAssembler(msh.nodes, mats, msh.num_dofs, tb.w, tb.q, tb.d_phi, tb.curls,
                                           backend="ref")
    mask = ins.solver.make_boundary_mask()
    _, _, r0 = O.compute_stiffness_and_jacobi_matrix_c(np.zeros(msh.num_dofs), sf)
    K, _, r = O.compute_stiffness_and_jacobi_matrix_c(x, sf)
    F0 = -(r0 + extra)
    F = K @ x - (r + extra)
    return float(np.linalg.norm(F[mask]) / np.linalg.norm(F0[mask]))
