"""Drop-in for the reference's native module ``fem_c_mod`` (``fem_c/interface_c.pyx``).

Same function names, arguments and return types; the arithmetic runs in the sm_100a
kernels of ``libsnoopy_b200.so``.  Inputs are host arrays like the reference's (they are
uploaded), and results come back as numpy arrays and scipy ``csr_array`` matrices with the
reference's semantics: per call, duplicates summed and explicit zeros kept
(``csr_array((vals, (i, j)))``, ``interface_c.pyx:154-155, 367-368``).

Only first-order tetrahedra are supported (4 nodes, 6 edge DoFs), as in every call the
reference's solvers make with ``element_order=1``.
"""

import ctypes
import os

import numpy as np

from . import _lib
from .device import Pattern, check_affine, permeability_tables, reluctance_tables, torch, upload, zeros


def _n_quad(w):
    return int(np.asarray(w).reshape(-1).shape[0])


def _check_range(name, a, hi):
    """Indices that the kernels gather with must lie in [0, hi); checked on the host."""
    a = np.asarray(a)
    if a.size and (a.min() < 0 or a.max() >= hi):
        raise ValueError(f"{name} holds indices outside [0, {hi})")


def _check_mesh(nodes, cells, glob_ids=None, num_dofs=None, orientations=None, n_orient=None):
    _check_range("cells", cells, np.asarray(nodes).reshape(-1, 3).shape[0])
    if glob_ids is not None:
        _check_range("glob_ids", glob_ids, int(num_dofs))
    if orientations is not None:
        _check_range("orientations", orientations, int(n_orient))
        if np.asarray(orientations).size * 6 != np.asarray(glob_ids).size:
            raise ValueError("one orientation and six glob_ids per element are required")


def compute_stiffness_and_jacobi_matrix(nodes, cells, d_phi, x, permeability, q, w, device=False):
    """Grad-grad stiffness matrix and Jacobian of the scalar potential (``interface_c.pyx:11-160``).

    :return: ``(K, dK)`` scipy CSR (num_nodes x num_nodes); with ``device=True`` torch sparse
        CSR tensors on the GPU (same structure and values, nothing copied to the host).
    """
    _lib.require_cuda()
    nodes = np.asarray(nodes, dtype=np.float64)
    num_nodes = nodes.shape[0]
    el_nodes = np.asarray(d_phi).shape[1]
    if el_nodes != 4:
        raise ValueError("only 4-node tetrahedra are supported")
    nq = _n_quad(w)
    check_affine(np.zeros((1, nq, 6, 3)), d_phi, nq)
    _check_mesh(nodes, cells)
    cells_d = upload(cells, np.int32)
    num_el = cells_d.numel() // el_nodes
    pat = Pattern(cells_d, num_el, 4, num_nodes)
    typ, k, n, t, c, hmin, muh = permeability_tables(permeability)
    K = zeros(pat.nnz)
    dK = zeros(pat.nnz)
    # every device buffer stays referenced until after the launch (freed blocks are reused)
    nodes_d, dphi_d, w_d, x_d = (upload(nodes, np.float64), upload(d_phi, np.float64), upload(w, np.float64),
                                 upload(x, np.float64))
    _lib.call("snp_gradgrad_assemble", pat.handle, 0, num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d), _lib.ptr(dphi_d),
              _lib.ptr(w_d), nq, _lib.ptr(x_d), typ, k, n, _lib.ptr(t), _lib.ptr(c), hmin, muh, _lib.ptr(K),
              _lib.ptr(dK), None, _lib.stream_ptr())
    if device:
        return pat.to_torch(K), pat.to_torch(dK)
    return pat.to_scipy(K), pat.to_scipy(dK)


def _curlcurl_K_dK_rhs(pat, num_el, num_dofs, nodes_d, cells_d, gids_d, or_d, curls_d, n_orient, phi_d, dphi_d, w_d,
                       nq, x_d, bs_d, n_int, rc, rx, dil):
    """K, dK and the reduced rhs of all elements of ``pat`` (device float64).  Element values and
    one sum per CSR entry (deterministic) where the pattern allows it and ``SNP_ASSEMBLY`` is not
    ``atomic``; otherwise the element kernel adding into the CSR (diluted when ``dil`` is set)."""
    if pat.rows_supported and os.environ.get("SNP_ASSEMBLY", "rows") != "atomic":
        t = torch()
        parts = _lib.TERMS_K | _lib.TERMS_DK | _lib.TERMS_RHS
        stride = ctypes.c_int32()
        _lib.call("snp_curlcurl_terms_stride", parts, ctypes.byref(stride))
        terms = t.empty(max(num_el * stride.value, 1), dtype=t.float64, device="cuda")
        K = t.empty(max(pat.nnz, 1), dtype=t.float64, device="cuda")
        dK = t.empty(max(pat.nnz, 1), dtype=t.float64, device="cuda")
        rhs = t.empty(max(num_dofs, 1), dtype=t.float64, device="cuda")
        _lib.call("snp_curlcurl_terms", pat.handle, 0, num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d), _lib.ptr(gids_d),
                  _lib.ptr(or_d), _lib.ptr(curls_d), n_orient, _lib.ptr(phi_d) if dil is not None else None,
                  _lib.ptr(dphi_d), _lib.ptr(w_d), nq, _lib.ptr(x_d), _lib.ptr(bs_d), n_int, _lib.ptr(rc), _lib.ptr(rx),
                  dil, parts, _lib.ptr(terms), _lib.stream_ptr())
        _lib.call("snp_curlcurl_rows", pat.handle, _lib.ptr(terms), parts, _lib.ptr(K), _lib.ptr(dK), None, None,
                  _lib.ptr(rhs), None, _lib.stream_ptr())
        return K[: pat.nnz], dK[: pat.nnz], rhs
    K = zeros(pat.nnz)
    dK = zeros(pat.nnz)
    rhs = zeros(num_dofs)
    if dil is None:
        _lib.call("snp_curlcurl_assemble", pat.handle, 0, num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d),
                  _lib.ptr(gids_d), _lib.ptr(or_d), _lib.ptr(curls_d), n_orient, _lib.ptr(dphi_d), _lib.ptr(w_d), nq,
                  _lib.ptr(x_d), _lib.ptr(bs_d), n_int, _lib.ptr(rc), _lib.ptr(rx), _lib.ptr(K), _lib.ptr(dK), None,
                  _lib.ptr(rhs), None, _lib.stream_ptr())
    else:
        _lib.call("snp_curlcurl_assemble_diluted", pat.handle, 0, num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d),
                  _lib.ptr(gids_d), _lib.ptr(or_d), _lib.ptr(curls_d), n_orient, _lib.ptr(phi_d), _lib.ptr(dphi_d),
                  _lib.ptr(w_d), nq, _lib.ptr(x_d), _lib.ptr(bs_d), n_int, _lib.ptr(rc), _lib.ptr(rx), dil,
                  _lib.ptr(K), _lib.ptr(dK), None, _lib.ptr(rhs), None, _lib.stream_ptr())
    return K, dK, rhs


def compute_stiffness_and_jacobi_matrix_curl_curl(nodes, cells, glob_ids, curls, d_phi, orientations, x, B_s,
                                                  reluctance, q, w, num_dofs, num_el_dofs, device=False):
    """Curl-curl stiffness matrix, Jacobian correction and reduced rhs (``interface_c.pyx:162-374``).

    ``B_s`` empty selects the plain kernel, otherwise the reduced one.
    :return: ``(K, dK, rhs)``: scipy CSR (num_dofs x num_dofs) and float64[num_dofs]; with
        ``device=True`` torch sparse CSR tensors and a CUDA tensor, left on the GPU.
    """
    _lib.require_cuda()
    if num_el_dofs != 6:
        raise ValueError("only first-order edge elements (6 DoFs per element) are supported")
    if np.asarray(d_phi).shape[1] != 4:
        raise ValueError("only 4-node tetrahedra are supported")
    nq = _n_quad(w)
    check_affine(curls, d_phi, nq)
    n_orient = int(np.asarray(curls).size // (nq * 18))
    _check_mesh(nodes, cells, glob_ids, num_dofs, orientations, n_orient)
    cells_d = upload(cells, np.int32)
    num_el = cells_d.numel() // 4
    gids_d = upload(glob_ids, np.int32)
    pat = Pattern(gids_d, num_el, 6, int(num_dofs))
    n_int, rc, rx = reluctance_tables(reluctance)
    B_s = np.asarray(B_s)
    bs_d = upload(B_s, np.float64) if B_s.size > 0 else None
    n_orient = int(np.asarray(curls).size // (nq * 18))
    nodes_d, or_d, curls_d = upload(nodes, np.float64), upload(orientations, np.int32), upload(curls, np.float64)
    dphi_d, w_d, x_d = upload(d_phi, np.float64), upload(w, np.float64), upload(x, np.float64)
    K, dK, rhs = _curlcurl_K_dK_rhs(pat, num_el, int(num_dofs), nodes_d, cells_d, gids_d, or_d, curls_d, n_orient,
                                    None, dphi_d, w_d, nq, x_d, bs_d, n_int, rc, rx, None)
    if device:
        return pat.to_torch(K), pat.to_torch(dK), rhs[: int(num_dofs)]
    return pat.to_scipy(K), pat.to_scipy(dK), rhs[: int(num_dofs)].cpu().numpy()


def compute_stiffness_and_jacobi_matrix_curl_curl_diluted(nodes, cells, glob_ids, curls, phi, d_phi, orientations, x,
                                                          B_s, reluctance, dilution, q, w, num_dofs, num_el_dofs,
                                                          device=False):
    """Curl-curl Newton system of diluted steel (``interface_c.pyx:698-926``).

    With ``B_s`` the reluctance at each quadrature point is s nu(s |B|) with the dilution
    factor s(z) of ``dilution`` (``materials.Dilution``); ``B_s`` empty selects the plain
    kernel, as the reference does for air.
    :return: ``(K, dK, rhs)``: scipy CSR (num_dofs x num_dofs) and float64[num_dofs]; with
        ``device=True`` torch sparse CSR tensors and a CUDA tensor, left on the GPU.
    """
    _lib.require_cuda()
    if num_el_dofs != 6:
        raise ValueError("only first-order edge elements (6 DoFs per element) are supported")
    if np.asarray(d_phi).shape[1] != 4:
        raise ValueError("only 4-node tetrahedra are supported")
    nq = _n_quad(w)
    if np.asarray(phi).size != 4 * nq:
        raise ValueError("phi must hold the 4 nodal basis functions at every quadrature point")
    check_affine(curls, d_phi, nq)
    n_orient = int(np.asarray(curls).size // (nq * 18))
    _check_mesh(nodes, cells, glob_ids, num_dofs, orientations, n_orient)
    cells_d = upload(cells, np.int32)
    num_el = cells_d.numel() // 4
    gids_d = upload(glob_ids, np.int32)
    pat = Pattern(gids_d, num_el, 6, int(num_dofs))
    n_int, rc, rx = reluctance_tables(reluctance)
    B_s = np.asarray(B_s)
    bs_d = upload(B_s, np.float64) if B_s.size > 0 else None
    dil = (ctypes.c_double * 4)(dilution.c_num, dilution.m_num, dilution.c_den, dilution.m_den)
    nodes_d, or_d, curls_d = upload(nodes, np.float64), upload(orientations, np.int32), upload(curls, np.float64)
    phi_d, dphi_d, w_d, x_d = (upload(phi, np.float64), upload(d_phi, np.float64), upload(w, np.float64),
                               upload(x, np.float64))
    K, dK, rhs = _curlcurl_K_dK_rhs(pat, num_el, int(num_dofs), nodes_d, cells_d, gids_d, or_d, curls_d, n_orient,
                                    phi_d, dphi_d, w_d, nq, x_d, bs_d, n_int, rc, rx, dil)
    if device:
        return pat.to_torch(K), pat.to_torch(dK), rhs[: int(num_dofs)]
    return pat.to_scipy(K), pat.to_scipy(dK), rhs[: int(num_dofs)].cpu().numpy()


def compute_rhs_Hcurl_red_c(nodes, cells, glob_ids, curls, d_phi, orientations, B_s, reluctance, x, q, w, num_dofs,
                            num_el_dofs):
    """rhs of the reduced vector potential formulation (``interface_c.pyx:377-552``)."""
    _lib.require_cuda()
    if num_el_dofs != 6:
        raise ValueError("only first-order edge elements (6 DoFs per element) are supported")
    nq = _n_quad(w)
    check_affine(curls, d_phi, nq)
    _check_mesh(nodes, cells, glob_ids, num_dofs, orientations, int(np.asarray(curls).size // (nq * 18)))
    cells_d = upload(cells, np.int32)
    num_el = cells_d.numel() // 4
    n_int, rc, rx = reluctance_tables(reluctance)
    n_orient = int(np.asarray(curls).size // (nq * 18))
    rhs = zeros(int(num_dofs))
    nodes_d, gids_d, or_d = upload(nodes, np.float64), upload(glob_ids, np.int32), upload(orientations, np.int32)
    curls_d, dphi_d, w_d = upload(curls, np.float64), upload(d_phi, np.float64), upload(w, np.float64)
    x_d, bs_d = upload(x, np.float64), upload(B_s, np.float64)
    _lib.call("snp_curlcurl_rhs_red", num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d), _lib.ptr(gids_d), _lib.ptr(or_d),
              _lib.ptr(curls_d), n_orient, _lib.ptr(dphi_d), _lib.ptr(w_d), nq, _lib.ptr(x_d), _lib.ptr(bs_d), n_int,
              _lib.ptr(rc), _lib.ptr(rx), _lib.ptr(rhs), _lib.stream_ptr())
    return rhs[: int(num_dofs)].cpu().numpy()


def compute_B_Hcurl(nodes, cells, glob_ids, curls, phi, d_phi, orientations, x, q, w, num_dofs, num_el_dofs):
    """Quadrature points and B there (``interface_c.pyx:555-696``): two float64[E*Q, 3] arrays."""
    _lib.require_cuda()
    if num_el_dofs != 6:
        raise ValueError("only first-order edge elements (6 DoFs per element) are supported")
    nq = _n_quad(w)
    n_orient = int(np.asarray(curls).size // (nq * 18))
    _check_mesh(nodes, cells, glob_ids, num_dofs, orientations, n_orient)
    cells_d = upload(cells, np.int32)
    num_el = cells_d.numel() // 4
    pts = zeros(3 * num_el * nq)
    B = zeros(3 * num_el * nq)
    nodes_d, gids_d, or_d = upload(nodes, np.float64), upload(glob_ids, np.int32), upload(orientations, np.int32)
    curls_d, phi_d, dphi_d, x_d = (upload(curls, np.float64), upload(phi, np.float64), upload(d_phi, np.float64),
                                   upload(x, np.float64))
    _lib.call("snp_b_hcurl", num_el, _lib.ptr(nodes_d), _lib.ptr(cells_d), _lib.ptr(gids_d), _lib.ptr(or_d),
              _lib.ptr(curls_d), n_orient, _lib.ptr(phi_d), _lib.ptr(dphi_d), nq, _lib.ptr(x_d), _lib.ptr(pts),
              _lib.ptr(B), _lib.stream_ptr())
    n = 3 * num_el * nq
    return pts[:n].cpu().numpy().reshape(-1, 3), B[:n].cpu().numpy().reshape(-1, 3)


def compute_B_line_segs_cpp(src, tar, current, radius):
    """Biot-Savart of line segments (``interface_c.pyx:928-991``): float64[M, 3].

    Wrong shapes print the reference's message and return -1, as it does.
    """
    src = np.asarray(src, dtype=np.float64)
    tar = np.asarray(tar, dtype=np.float64)
    if src.ndim != 2 or src.shape[1] != 6:
        print("Error! The source array must be of dimension N x 6!")
        return -1
    if tar.ndim != 2 or tar.shape[1] != 3:
        print("Error! The target array must be of dimension M x 3!")
        return -1
    _lib.require_cuda()
    B = zeros(3 * tar.shape[0])
    src_d, tar_d = upload(src, np.float64), upload(tar, np.float64)
    _lib.call("snp_biot_savart", _lib.ptr(src_d), src.shape[0], _lib.ptr(tar_d), tar.shape[0], float(current),
              float(radius), _lib.ptr(B), _lib.stream_ptr())
    return B[: 3 * tar.shape[0]].cpu().numpy().reshape(-1, 3).copy()


def biot_savart_device(src_t, tar_t, current, radius, out=None):
    """Biot-Savart on device tensors (src [S*6], tar [T*3]) -> B [T*3] device tensor."""
    n_tar = tar_t.numel() // 3
    B = out if out is not None else zeros(3 * n_tar)
    _lib.call("snp_biot_savart", _lib.ptr(src_t), src_t.numel() // 6, _lib.ptr(tar_t), n_tar, float(current),
              float(radius), _lib.ptr(B), _lib.stream_ptr())
    return B
