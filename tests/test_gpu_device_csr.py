"""The opt-in device outputs of the drop-in assembly (``device=True``): torch sparse CSR
tensors on the GPU with the same structure and values as the host scipy matrices."""

import numpy as np
import pytest
import torch
from scipy.sparse import csr_array

import snoopy_b200 as S
from snoopy_b200 import fem_c
from snoopy_b200 import finite_element as FE
from snoopy_b200 import materials as MAT
from snoopy_b200 import mesh as M

pytestmark = pytest.mark.gpu

NU0 = 0.25 / np.pi * 1e7


def _host(T):
    """scipy csr_array of a torch sparse CSR tensor (explicit zeros kept)."""
    return csr_array((T.values().cpu().numpy(), T.col_indices().cpu().numpy(), T.crow_indices().cpu().numpy()),
                     shape=tuple(T.shape))


def _same(Td, A, drop_zeros=False):
    """Same structure; values of two separate assemblies agree to rounding (the CSR path sums an
    entry's element contributions with atomics, in no fixed order)."""
    assert Td.is_cuda and Td.layout == torch.sparse_csr and Td.dtype == torch.float64
    H = _host(Td)
    if drop_zeros:
        H.eliminate_zeros()
    A = csr_array(A)
    assert np.array_equal(H.indptr, A.indptr) and np.array_equal(H.indices, A.indices)
    assert np.abs(H.data - A.data).max() <= 1e-13 * np.abs(A.data).max()


def _close(a, b):
    return np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


def test_fem_c_device_outputs():
    msh = M.window_frame_mesh(4000, jitter=0.15, seed=2)
    w, q = FE.quadrature_rule(2)
    dphi = FE.evaluate_basis_derivative(q)
    phi = FE.evaluate_basis(q)
    curls, _ = FE.curl_edge_basis_functions(q)
    el = msh.domain_elements(M.TAG_IRON)
    rng = np.random.default_rng(0)
    x = rng.normal(0, 2e-3, msh.num_dofs)
    Bs = rng.normal(0, 0.5, (len(el) * len(w), 3))
    rel = MAT.atan_reluctance()
    args = (msh.nodes, msh.cells[el], msh.elem_edges[el], curls, dphi, msh.orientations[el], x, Bs, rel, q, w,
            msh.num_dofs, 6)
    K, dK, rhs = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(*args)
    Kd, dKd, rhsd = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl(*args, device=True)
    _same(Kd, K)
    _same(dKd, dK)
    assert rhsd.is_cuda and _close(rhsd.cpu().numpy(), rhs)
    v = rng.normal(size=msh.num_dofs)
    got = torch.sparse.mm(Kd, torch.as_tensor(v, device="cuda")[:, None])[:, 0].cpu().numpy()
    assert np.abs(got - K @ v).max() <= 1e-12 * np.abs(K @ v).max()
    dil = MAT.Dilution(0.0, 0.30, 0.35, 0.75, 0.02, 0.40, 0.45, 0.80, z_pos=-0.25, z_len=0.5)
    dargs = args[:4] + (phi,) + args[4:9] + (dil,) + args[9:]
    K2, _, r2 = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(*dargs)
    K2d, _, r2d = fem_c.compute_stiffness_and_jacobi_matrix_curl_curl_diluted(*dargs, device=True)
    _same(K2d, K2)
    assert _close(r2d.cpu().numpy(), r2)
    xn = rng.normal(0, 50.0, msh.num_nodes)
    G, dG = fem_c.compute_stiffness_and_jacobi_matrix(msh.nodes, msh.cells, dphi, xn, MAT.atan_permeability(), q, w)
    Gd, dGd = fem_c.compute_stiffness_and_jacobi_matrix(msh.nodes, msh.cells, dphi, xn, MAT.atan_permeability(), q, w,
                                                        device=True)
    _same(Gd, G)
    _same(dGd, dG)


def test_assembler_device_outputs():
    msh = M.window_frame_mesh(6000, jitter=0.15, seed=4)
    rel = MAT.atan_reluctance()
    A = S.CurlCurlAssembler(msh, [M.TAG_IRON, M.TAG_AIR], [rel, S.ConstantReluctance(NU0)])
    rng = np.random.default_rng(1)
    x = rng.normal(0, 2e-3, msh.num_dofs)
    Bs = rng.normal(0, 0.5, (len(msh.domain_elements(M.TAG_IRON)) * 4, 3))
    sf = [Bs, np.zeros((0, 3))]
    K, J, rhs = A.compute_stiffness_and_jacobi_matrix_c(x, quad_order=2, source_fields=sf)
    Kd, Jd, rhsd = A.compute_stiffness_and_jacobi_matrix_c(x, quad_order=2, source_fields=sf, device=True)
    # the host matrices drop exact zeros (scipy's K +=); the device ones keep the structure
    _same(Kd, K, drop_zeros=True)
    _same(Jd, J, drop_zeros=True)
    assert _close(rhsd.cpu().numpy(), rhs)
    GA = S.GradGradAssembler(msh, [M.TAG_IRON, M.TAG_AIR])
    xn = rng.normal(0, 50.0, msh.num_nodes)
    mus = [MAT.atan_permeability(), S.ConstantPermeability(4e-7 * np.pi)]
    Gk, Gj = GA.compute_stiffness_and_jacobi_matrix_c(xn, mus, quad_order=2)
    Gkd, Gjd = GA.compute_stiffness_and_jacobi_matrix_c(xn, mus, quad_order=2, device=True)
    _same(Gkd, Gk, drop_zeros=True)
    _same(Gjd, Gj, drop_zeros=True)
