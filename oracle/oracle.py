"""CPU oracle for snoo.py's nonlinear magnetostatic path.

TEST INFRASTRUCTURE ONLY: ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference leg may import this module, as the checker or as the timed
CPU reference.  The product (``snoo.py_b200``) never imports it.

Two arithmetic backends with one interface:

* ``"oracle"``: ``oracle/_build/liboracle.so``, this project's C restatement (``restated.c``);
* ``"ref"``:    ``oracle/_ref/libctools_ref.so``, the reference's own ``fem_c/ctools.c``
  compiled from its sources (``build_oracle.py``).

The glue around them restates the reference's Python/Cython layers:

* ``compute_stiffness_and_jacobi_matrix_curl_curl``  ``fem_c/interface_c.pyx:162-374``
  (triplets -> ``csr_array((v, (i, j)))``: duplicates summed, explicit zeros kept)
* ``compute_stiffness_and_jacobi_matrix``            ``fem_c/interface_c.pyx:11-160``
* ``compute_rhs_Hcurl_red_c``                        ``fem_c/interface_c.pyx:377-552``
* ``compute_B_Hcurl``                                ``fem_c/interface_c.pyx:555-696``
* ``compute_B_line_segs_cpp``                        ``fem_c/interface_c.pyx:928-991``
* ``OracleCurlCurlAssembler.compute_stiffness_and_jacobi_matrix_c``
                                                     ``snoopy/curl_curl_assembler.py:815-932``
  (per-material loop, ``K += this_K`` drops exact zeros, returns ``(K, dK + K, rhs)``)
* ``OracleGradGradAssembler``                        ``snoopy/matrix_assembly.py:1059-1135``
* ``newton_reference``                               ``snoopy/red_mvp_solver.py:121-224``
* ``newton_residual``: the same loop driven to a relative Newton residual
  ||F_free(x)|| / ||F_free(x0)|| with F(x) = K(x) x - rhs(x) and a tight inner CG.
* ``laplace_subdomain_solve``                        ``snoopy/laplace_subdomain_solver.py:117-158``
* ``locate_points``, ``element_B``, ``nodal_fields``, ``interpolate_nodal``: field-map output
  (``snoopy/evaluators.py:155-410``, ``snoopy/curl_curl_assembler.py:2089-2196``)
* ``probe_B``: the total field at probe points (``RedMVPSolver``'s output, curl A + B_s)
"""

import ctypes
import os
import time

import numpy as np
from scipy.sparse import csr_array, diags
from scipy.sparse.linalg import cg, spsolve

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libctools_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64 = ctypes.c_int64


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(-1))


# ------------------------------------------------------------------ library loading

class _Mesh(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int), ("num_elements", ctypes.c_int),
                ("num_nodes_per_element", ctypes.c_int), ("nodes", _dp), ("cells", _ip)]


class _Triplets(ctypes.Structure):
    _fields_ = [("counter", ctypes.c_int), ("row", _ip), ("col", _ip), ("vals", _dp),
                ("num_triplets", ctypes.c_int)]


class _Quad(ctypes.Structure):
    _fields_ = [("num_points", ctypes.c_int), ("points", _dp), ("weights", _dp)]


class _Perm(ctypes.Structure):
    _fields_ = [("type_spec", ctypes.c_int), ("degree", ctypes.c_int), ("num_control_points", ctypes.c_int),
                ("knots", _dp), ("control_points", _dp), ("H_min", ctypes.c_double),
                ("mu_H_min", ctypes.c_double)]


class _Rel(ctypes.Structure):
    _fields_ = [("type_spec", ctypes.c_int), ("num_intervals", ctypes.c_int),
                ("coefficients", _dp), ("knots", _dp)]


class _Dil(ctypes.Structure):
    _fields_ = [("c_num", ctypes.c_double), ("m_num", ctypes.c_double), ("c_den", ctypes.c_double),
                ("m_den", ctypes.c_double)]


_LIBS = {}


def _ensure_built():
    if not os.path.exists(LIB_ORACLE):
        import importlib.util

        spec = importlib.util.spec_from_file_location("_oracle_build", os.path.join(HERE, "build_oracle.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()


def ref_available():
    return os.path.exists(LIB_REF)


def lib(backend="oracle"):
    if backend in _LIBS:
        return _LIBS[backend]
    if backend == "oracle":
        _ensure_built()
        L = ctypes.CDLL(LIB_ORACLE)
        L.or_pchip.restype = ctypes.c_double
        L.or_pchip.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp]
        L.or_mu.restype = ctypes.c_double
        L.or_mu.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_double,
                            ctypes.c_double, ctypes.c_double, _dp]
        L.or_curlcurl.restype = _i64
        L.or_curlcurl.argtypes = [_i64, ctypes.c_int, _dp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp,
                                  ctypes.c_int, _dp, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.or_rhs_red.restype = ctypes.c_int
        L.or_rhs_red.argtypes = [_i64, ctypes.c_int, _dp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp,
                                 ctypes.c_int, _dp, _dp, _dp]
        L.or_B_hcurl.restype = ctypes.c_int
        L.or_B_hcurl.argtypes = [_i64, ctypes.c_int, _dp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp]
        L.or_gradgrad.restype = _i64
        L.or_gradgrad.argtypes = [_i64, ctypes.c_int, _dp, _ip, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double, _ip, _ip, _dp, _dp, _dp,
                                  _dp]
        L.or_biot_savart.restype = None
        L.or_biot_savart.argtypes = [_dp, _i64, _dp, _i64, ctypes.c_double, ctypes.c_double, _dp]
    elif backend == "ref":
        if not os.path.exists(LIB_REF):
            raise FileNotFoundError(f"{LIB_REF} not built (needs the reference sources; run oracle/build_oracle.py)")
        L = ctypes.CDLL(LIB_REF)
        P = ctypes.POINTER
        L.compute_K_dK_Hcurl.restype = None
        L.compute_K_dK_Hcurl.argtypes = [P(_Triplets), P(_Triplets), _ip, P(_Rel), P(_Mesh), P(_Quad), _dp, _dp, _ip, _dp]
        L.compute_K_dK_Hcurl_red.restype = None
        L.compute_K_dK_Hcurl_red.argtypes = [P(_Triplets), P(_Triplets), _dp, _ip, P(_Rel), P(_Mesh), P(_Quad),
                                             _dp, _dp, _ip, _dp, _dp]
        L.compute_K_dK_Hcurl_red_dil.restype = None
        L.compute_K_dK_Hcurl_red_dil.argtypes = [P(_Triplets), P(_Triplets), _dp, P(_Dil), _ip, P(_Rel), P(_Mesh),
                                                 P(_Quad), _dp, _dp, _dp, _ip, _dp, _dp]
        L.compute_rhs_Hcurl_red.restype = None
        L.compute_rhs_Hcurl_red.argtypes = [_dp, _ip, P(_Rel), P(_Mesh), P(_Quad), _dp, _dp, _ip, _dp, _dp, ctypes.c_int]
        L.compute_B_Hcurl.restype = None
        L.compute_B_Hcurl.argtypes = [_dp, _dp, ctypes.c_int, _ip, P(_Mesh), P(_Quad), _dp, _dp, _dp, _ip, _dp]
        L.compute_K_dK.restype = None
        L.compute_K_dK.argtypes = [P(_Triplets), P(_Triplets), P(_Mesh), P(_Quad), _dp, _dp, P(_Perm)]
        L.compute_B_line_segs.restype = None
        L.compute_B_line_segs.argtypes = [_dp, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.eval_pchip_interpolator.restype = ctypes.c_double
        L.eval_pchip_interpolator.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double]
        L.eval_pchip_interpolator_derivative.restype = ctypes.c_double
        L.eval_pchip_interpolator_derivative.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double]
        L.compute_mu.restype = ctypes.c_double
        L.compute_mu.argtypes = [P(_Perm), ctypes.c_double]
        L.compute_mu_derivative.restype = ctypes.c_double
        L.compute_mu_derivative.argtypes = [P(_Perm), ctypes.c_double]
    else:
        raise ValueError(backend)
    _LIBS[backend] = L
    return L


# ------------------------------------------------------------------ material marshalling

def reluctance_arrays(reluctance):
    """(n_int, c flat, x) as ``interface_c.pyx:226-234`` builds them for the C struct."""
    if reluctance.get_type_spec() == 1:
        spl_c, spl_x = reluctance.get_spline_information()
        c = _f64(np.asarray(spl_c).flatten())
        x = _f64(spl_x)
        return len(x) - 1, c, x
    if reluctance.get_type_spec() == 0:
        return -1, _f64([reluctance.value]), np.zeros(1)
    raise ValueError("Type specifyer of reluctance not found!")


def permeability_arrays(permeability):
    """(type, k, n, t, c, H_min, mu_H_min) as ``interface_c.pyx:56-68`` builds them."""
    spl_t, spl_c, spl_k, spl_H_min, spl_mu_H_min, n = np.zeros(1), np.zeros(1), 1, 0.0, 4 * np.pi * 1e-7, 0
    if permeability.get_type_spec() == 0:
        spl_mu_H_min = float(np.asarray(permeability.evaluate_mu(0.0)).reshape(-1)[0])
    elif permeability.get_type_spec() == 1:
        spl_t, spl_c, spl_k, spl_H_min, spl_mu_H_min = permeability.get_spline_information()
        n = len(spl_t) - spl_k - 1
    else:
        raise ValueError("Type specifyer of permeability not found!")
    return int(permeability.get_type_spec()), int(spl_k), int(n), _f64(spl_t), _f64(spl_c), float(spl_H_min), float(spl_mu_H_min)


def pchip_eval(reluctance, B, backend="oracle"):
    """nu and dnu/dB at the points B through the chosen backend."""
    n_int, c, x = reluctance_arrays(reluctance)
    L = lib(backend)
    B = _f64(B)
    nu = np.empty_like(B)
    dnu = np.empty_like(B)
    if backend == "oracle":
        tmp = ctypes.c_double()
        for i, b in enumerate(B):
            nu[i] = L.or_pchip(n_int, _d(c), _d(x), float(b), ctypes.byref(tmp))
            dnu[i] = tmp.value
    else:
        for i, b in enumerate(B):
            nu[i] = L.eval_pchip_interpolator(n_int, _d(c), _d(x), float(b))
            dnu[i] = L.eval_pchip_interpolator_derivative(n_int, _d(c), _d(x), float(b))
    return nu, dnu


def mu_eval(permeability, H, backend="oracle"):
    """mu and dmu/dH at |H| values through the chosen backend."""
    typ, k, n, t, c, hmin, muhmin = permeability_arrays(permeability)
    L = lib(backend)
    H = _f64(H)
    mu = np.empty_like(H)
    dmu = np.empty_like(H)
    if backend == "oracle":
        tmp = ctypes.c_double()
        for i, h in enumerate(H):
            mu[i] = L.or_mu(typ, k, n, _d(t), _d(c), hmin, muhmin, float(h), ctypes.byref(tmp))
            dmu[i] = tmp.value
    else:
        perm = _Perm(typ, k, n, _d(t), _d(c), hmin, muhmin)
        for i, h in enumerate(H):
            mu[i] = L.compute_mu(ctypes.byref(perm), float(h))
            dmu[i] = L.compute_mu_derivative(ctypes.byref(perm), float(h))
    return mu, dmu


# ------------------------------------------------------------------ fem_c_mod restatement

def curl_curl_triplets(nodes, cells, glob_ids, curls, d_phi, orientations, x, B_s, reluctance, q, w,
                       num_dofs, num_el_dofs, backend="oracle", scales=None, phi=None, dilution=None):
    """Triplets (i, j, vK, vdK) and rhs of one material, as the C kernels emit them.

    ``scales``: an optional dict that receives "K" and "dK", the per-triplet sums of term
    magnitudes (restatement only), the scale of any evaluation order's rounding error.
    ``phi``/``dilution``: diluted steel (``compute_K_dK_Hcurl_red_dil``, ctools.c:1565-1759),
    used only with a source field, as ``interface_c.pyx:874-901`` does; ``dilution`` is any
    object with ``c_num, m_num, c_den, m_den``."""
    if num_el_dofs != 6:
        raise ValueError("only first-order edge elements (6 DoFs) are supported")
    nodes_c, cells_c, gid_c = _f64(nodes), _i32(cells), _i32(glob_ids)
    curls_c, dphi_c, or_c = _f64(curls), _f64(d_phi), _i32(orientations)
    x_c, q_c, w_c = _f64(x), _f64(q), _f64(w)
    Bs_c = _f64(B_s)
    E = len(cells_c) // 4
    Q = len(w_c)
    nt = E * num_el_dofs * num_el_dofs
    ti = np.empty(nt, dtype=np.int32)
    tj = np.empty(nt, dtype=np.int32)
    vK = np.empty(nt)
    vdK = np.empty(nt)
    rhs = np.zeros(num_dofs)
    n_int, rc, rx = reluctance_arrays(reluctance)
    L = lib(backend)
    dil = None
    if dilution is not None and len(Bs_c) > 0:
        dil = np.array([dilution.c_num, dilution.m_num, dilution.c_den, dilution.m_den], dtype=np.float64)
        phi_c = _f64(phi)
        assert len(phi_c) == 4 * Q, "phi must hold 4 nodal basis values per quadrature point"
    if backend == "oracle":
        bs_ptr = _d(Bs_c) if len(Bs_c) > 0 else None
        sK = np.empty(nt) if scales is not None else None
        sdK = np.empty(nt) if scales is not None else None
        got = L.or_curlcurl(E, Q, _d(nodes_c), _i(cells_c), _i(gid_c), _i(or_c), _d(curls_c), _d(dphi_c),
                            _d(w_c), _d(x_c), bs_ptr, n_int, _d(rc), _d(rx), _i(ti), _i(tj), _d(vK), _d(vdK), _d(rhs),
                            _d(sK) if sK is not None else None, _d(sdK) if sdK is not None else None,
                            _d(phi_c) if dil is not None else None, _d(dil) if dil is not None else None)
        assert got == nt, got
        if scales is not None:
            scales["K"], scales["dK"] = sK, sdK
    else:
        tK = _Triplets(0, _i(ti), _i(tj), _d(vK), nt)
        ti2 = np.empty(nt, dtype=np.int32)
        tj2 = np.empty(nt, dtype=np.int32)
        tdK = _Triplets(0, _i(ti2), _i(tj2), _d(vdK), nt)
        rel = _Rel(reluctance.get_type_spec(), n_int, _d(rc), _d(rx))
        msh = _Mesh(len(nodes_c) // 3, E, 4, _d(nodes_c), _i(cells_c))
        quad = _Quad(Q, _d(q_c), _d(w_c))
        if dil is not None:
            dc = _Dil(*[float(v) for v in dil])
            L.compute_K_dK_Hcurl_red_dil(ctypes.byref(tK), ctypes.byref(tdK), _d(rhs), ctypes.byref(dc), _i(gid_c),
                                         ctypes.byref(rel), ctypes.byref(msh), ctypes.byref(quad), _d(curls_c),
                                         _d(phi_c), _d(dphi_c), _i(or_c), _d(x_c), _d(Bs_c))
        elif len(Bs_c) == 0:
            L.compute_K_dK_Hcurl(ctypes.byref(tK), ctypes.byref(tdK), _i(gid_c), ctypes.byref(rel), ctypes.byref(msh),
                                 ctypes.byref(quad), _d(curls_c), _d(dphi_c), _i(or_c), _d(x_c))
        else:
            L.compute_K_dK_Hcurl_red(ctypes.byref(tK), ctypes.byref(tdK), _d(rhs), _i(gid_c), ctypes.byref(rel),
                                     ctypes.byref(msh), ctypes.byref(quad), _d(curls_c), _d(dphi_c), _i(or_c),
                                     _d(x_c), _d(Bs_c))
        assert tK.counter == nt and tdK.counter == nt
    return ti, tj, vK, vdK, rhs


def compute_stiffness_and_jacobi_matrix_curl_curl(nodes, cells, glob_ids, curls, d_phi, orientations, x, B_s,
                                                  reluctance, q, w, num_dofs, num_el_dofs, backend="oracle"):
    """(K, dK, rhs) of one material (``interface_c.pyx:162-374``)."""
    ti, tj, vK, vdK, rhs = curl_curl_triplets(nodes, cells, glob_ids, curls, d_phi, orientations, x, B_s,
                                              reluctance, q, w, num_dofs, num_el_dofs, backend)
    K = csr_array((vK, (ti, tj)), shape=(num_dofs, num_dofs))
    dK = csr_array((vdK, (ti, tj)), shape=(num_dofs, num_dofs))
    return K, dK, rhs


def compute_stiffness_and_jacobi_matrix_curl_curl_diluted(nodes, cells, glob_ids, curls, phi, d_phi, orientations,
                                                          x, B_s, reluctance, dilution, q, w, num_dofs, num_el_dofs,
                                                          backend="oracle"):
    """(K, dK, rhs) of one diluted-steel material (``interface_c.pyx:698-926``): the diluted
    reduced kernel with a source field, the plain kernel without one."""
    ti, tj, vK, vdK, rhs = curl_curl_triplets(nodes, cells, glob_ids, curls, d_phi, orientations, x, B_s,
                                              reluctance, q, w, num_dofs, num_el_dofs, backend, phi=phi,
                                              dilution=dilution)
    K = csr_array((vK, (ti, tj)), shape=(num_dofs, num_dofs))
    dK = csr_array((vdK, (ti, tj)), shape=(num_dofs, num_dofs))
    return K, dK, rhs


def compute_rhs_Hcurl_red_c(nodes, cells, glob_ids, curls, d_phi, orientations, B_s, reluctance, x, q, w,
                            num_dofs, num_el_dofs, backend="oracle"):
    """Reduced-formulation rhs only (``interface_c.pyx:377-552``)."""
    nodes_c, cells_c, gid_c = _f64(nodes), _i32(cells), _i32(glob_ids)
    curls_c, dphi_c, or_c = _f64(curls), _f64(d_phi), _i32(orientations)
    x_c, q_c, w_c, Bs_c = _f64(x), _f64(q), _f64(w), _f64(B_s)
    E, Q = len(cells_c) // 4, len(w_c)
    rhs = np.zeros(num_dofs)
    n_int, rc, rx = reluctance_arrays(reluctance)
    L = lib(backend)
    if backend == "oracle":
        L.or_rhs_red(E, Q, _d(nodes_c), _i(cells_c), _i(gid_c), _i(or_c), _d(curls_c), _d(dphi_c), _d(w_c),
                     _d(x_c), _d(Bs_c), n_int, _d(rc), _d(rx), _d(rhs))
    else:
        rel = _Rel(reluctance.get_type_spec(), n_int, _d(rc), _d(rx))
        msh = _Mesh(len(nodes_c) // 3, E, 4, _d(nodes_c), _i(cells_c))
        quad = _Quad(Q, _d(q_c), _d(w_c))
        L.compute_rhs_Hcurl_red(_d(rhs), _i(gid_c), ctypes.byref(rel), ctypes.byref(msh), ctypes.byref(quad),
                                _d(curls_c), _d(dphi_c), _i(or_c), _d(Bs_c), _d(x_c), num_el_dofs)
    return rhs


def compute_B_Hcurl(nodes, cells, glob_ids, curls, phi, d_phi, orientations, x, q, w, num_dofs, num_el_dofs,
                    backend="oracle"):
    """Quadrature points and B there (``interface_c.pyx:555-696``)."""
    nodes_c, cells_c, gid_c = _f64(nodes), _i32(cells), _i32(glob_ids)
    curls_c, phi_c, dphi_c, or_c = _f64(curls), _f64(phi), _f64(d_phi), _i32(orientations)
    x_c, q_c, w_c = _f64(x), _f64(q), _f64(w)
    E, Q = len(cells_c) // 4, len(w_c)
    pts = np.empty(3 * E * Q)
    B = np.empty(3 * E * Q)
    L = lib(backend)
    if backend == "oracle":
        L.or_B_hcurl(E, Q, _d(nodes_c), _i(cells_c), _i(gid_c), _i(or_c), _d(curls_c), _d(phi_c), _d(dphi_c),
                     _d(x_c), _d(pts), _d(B))
    else:
        msh = _Mesh(len(nodes_c) // 3, E, 4, _d(nodes_c), _i(cells_c))
        quad = _Quad(Q, _d(q_c), _d(w_c))
        L.compute_B_Hcurl(_d(pts), _d(B), num_el_dofs, _i(gid_c), ctypes.byref(msh), ctypes.byref(quad),
                          _d(curls_c), _d(phi_c), _d(dphi_c), _i(or_c), _d(x_c))
    return pts.reshape(-1, 3), B.reshape(-1, 3)


def grad_grad_triplets(nodes, cells, d_phi, x, permeability, q, w, backend="oracle", scales=None):
    nodes_c, cells_c, dphi_c, x_c, q_c, w_c = _f64(nodes), _i32(cells), _f64(d_phi), _f64(x), _f64(q), _f64(w)
    E, Q = len(cells_c) // 4, len(w_c)
    nt = E * 16
    ti = np.empty(nt, dtype=np.int32)
    tj = np.empty(nt, dtype=np.int32)
    vK = np.empty(nt)
    vdK = np.empty(nt)
    typ, k, n, t, c, hmin, muhmin = permeability_arrays(permeability)
    L = lib(backend)
    if backend == "oracle":
        sK = np.empty(nt) if scales is not None else None
        sdK = np.empty(nt) if scales is not None else None
        got = L.or_gradgrad(E, Q, _d(nodes_c), _i(cells_c), _d(dphi_c), _d(w_c), _d(x_c), typ, k, n, _d(t), _d(c),
                            hmin, muhmin, _i(ti), _i(tj), _d(vK), _d(vdK), _d(sK) if sK is not None else None,
                            _d(sdK) if sdK is not None else None)
        assert got == nt
        if scales is not None:
            scales["K"], scales["dK"] = sK, sdK
    else:
        tK = _Triplets(0, _i(ti), _i(tj), _d(vK), nt)
        ti2 = np.empty(nt, dtype=np.int32)
        tj2 = np.empty(nt, dtype=np.int32)
        tdK = _Triplets(0, _i(ti2), _i(tj2), _d(vdK), nt)
        perm = _Perm(typ, k, n, _d(t), _d(c), hmin, muhmin)
        msh = _Mesh(len(nodes_c) // 3, E, 4, _d(nodes_c), _i(cells_c))
        quad = _Quad(Q, _d(q_c), _d(w_c))
        L.compute_K_dK(ctypes.byref(tK), ctypes.byref(tdK), ctypes.byref(msh), ctypes.byref(quad), _d(dphi_c),
                       _d(x_c), ctypes.byref(perm))
    return ti, tj, vK, vdK


def compute_stiffness_and_jacobi_matrix(nodes, cells, d_phi, x, permeability, q, w, backend="oracle"):
    """(K, dK) of the P1 grad-grad operator (``interface_c.pyx:11-160``)."""
    n = np.asarray(nodes).reshape(-1, 3).shape[0]
    ti, tj, vK, vdK = grad_grad_triplets(nodes, cells, d_phi, x, permeability, q, w, backend)
    K = csr_array((vK, (ti, tj)), shape=(n, n))
    dK = csr_array((vdK, (ti, tj)), shape=(n, n))
    return K, dK


def compute_B_line_segs_cpp(src, tar, current, radius, backend="oracle"):
    """Biot-Savart of line segments (``interface_c.pyx:928-991``)."""
    src = np.asarray(src, dtype=np.float64)
    tar = np.asarray(tar, dtype=np.float64)
    if src.ndim != 2 or src.shape[1] != 6:
        raise ValueError("The source array must be of dimension N x 6!")
    if tar.ndim != 2 or tar.shape[1] != 3:
        raise ValueError("The target array must be of dimension M x 3!")
    s, t = _f64(src), _f64(tar)
    B = np.empty(3 * tar.shape[0])
    L = lib(backend)
    if backend == "oracle":
        L.or_biot_savart(_d(s), src.shape[0], _d(t), tar.shape[0], float(current), float(radius), _d(B))
    else:
        L.compute_B_line_segs(_d(B), _d(s), _d(t), float(current), float(radius), src.shape[0], tar.shape[0])
    return B.reshape(-1, 3)


# ------------------------------------------------------------------ assembler glue

class OracleCurlCurlAssembler:
    """Per-material assembly loop of ``CurlCurlAssembler.compute_stiffness_and_jacobi_matrix_c``
    (``curl_curl_assembler.py:815-932``) over explicit arrays.

    ``materials``: list of dicts with 0-based ``cells`` [E_m, 4], ``glob_ids`` [E_m, 6],
    ``orientations`` [E_m] and ``reluctance``, optionally ``dilution`` (diluted steel, the
    loop of ``curl_curl_assembler_diluted.py:204-300``; needs ``phi``).
    """

    def __init__(self, nodes, materials, num_dofs, w, q, d_phi, curls, backend="oracle", phi=None):
        self.nodes = nodes
        self.materials = materials
        self.num_dofs = num_dofs
        self.w, self.q, self.d_phi, self.curls, self.phi = w, q, d_phi, curls, phi
        self.backend = backend
        self.timings = {"kernel": 0.0, "csr": 0.0}

    def compute_stiffness_and_jacobi_matrix_c(self, x, source_fields=()):
        n = self.num_dofs
        K = csr_array((n, n))
        dK = csr_array((n, n))
        rhs = np.zeros(n)
        use_sf = len(source_fields) == len(self.materials)
        for m, mat in enumerate(self.materials):
            B_s = source_fields[m] if use_sf and len(source_fields[m]) > 0 else np.zeros((0, 3))
            t0 = time.perf_counter()
            ti, tj, vK, vdK, this_rhs = curl_curl_triplets(self.nodes, mat["cells"], mat["glob_ids"], self.curls,
                                                           self.d_phi, mat["orientations"], x, B_s,
                                                           mat["reluctance"], self.q, self.w, n, 6, self.backend,
                                                           phi=self.phi, dilution=mat.get("dilution"))
            t1 = time.perf_counter()
            this_K = csr_array((vK, (ti, tj)), shape=(n, n))
            this_dK = csr_array((vdK, (ti, tj)), shape=(n, n))
            K += this_K
            dK += this_dK
            rhs += this_rhs
            self.timings["kernel"] += t1 - t0
            self.timings["csr"] += time.perf_counter() - t1
        t1 = time.perf_counter()
        J = dK + K
        self.timings["csr"] += time.perf_counter() - t1
        return K, J, rhs

    def scales(self, x, source_fields=()):
        """Per-entry sums of term magnitudes of K and of J = K + dK (comparison scales)."""
        n = self.num_dofs
        sK = csr_array((n, n))
        sJ = csr_array((n, n))
        use_sf = len(source_fields) == len(self.materials)
        for m, mat in enumerate(self.materials):
            B_s = source_fields[m] if use_sf and len(source_fields[m]) > 0 else np.zeros((0, 3))
            sc = {}
            ti, tj, _, _, _ = curl_curl_triplets(self.nodes, mat["cells"], mat["glob_ids"], self.curls, self.d_phi,
                                                 mat["orientations"], x, B_s, mat["reluctance"], self.q, self.w, n, 6,
                                                 "oracle", scales=sc, phi=self.phi, dilution=mat.get("dilution"))
            sK = sK + csr_array((sc["K"], (ti, tj)), shape=(n, n))
            sJ = sJ + csr_array((sc["K"] + sc["dK"], (ti, tj)), shape=(n, n))
        return sK, sJ


class OracleGradGradAssembler:
    """``GradGradAssembler.compute_stiffness_and_jacobi_matrix_c`` (``matrix_assembly.py:1059-1135``)."""

    def __init__(self, nodes, cells_list, w, q, d_phi, backend="oracle"):
        self.nodes = nodes
        self.cells_list = cells_list
        self.w, self.q, self.d_phi = w, q, d_phi
        self.backend = backend

    def compute_stiffness_and_jacobi_matrix_c(self, x, mu_list):
        n = self.nodes.shape[0]
        K = csr_array((n, n))
        dK = csr_array((n, n))
        for m, perm in enumerate(mu_list):
            my_K, my_dK = compute_stiffness_and_jacobi_matrix(self.nodes, self.cells_list[m], self.d_phi, x, perm,
                                                              self.q, self.w, self.backend)
            K += my_K
            dK += my_dK
            dK += K
        return K, dK

    def scales(self, x, mu_list):
        """Comparison scales of K and of the returned J (with the reference's per-material
        ``dK += K``, J sums the running K after every material)."""
        n = self.nodes.shape[0]
        sK = csr_array((n, n))
        sJ = csr_array((n, n))
        for m, perm in enumerate(mu_list):
            sc = {}
            ti, tj, _, _ = grad_grad_triplets(self.nodes, self.cells_list[m], self.d_phi, x, perm, self.q, self.w,
                                              "oracle", scales=sc)
            sK = sK + csr_array((sc["K"], (ti, tj)), shape=(n, n))
            sJ = sJ + csr_array((sc["dK"], (ti, tj)), shape=(n, n)) + sK
        return sK, sJ


# ------------------------------------------------------------------ Newton loops

def newton_reference(assembler, mask, source_fields=(), tolerance=1e-4, x_0=None, maxiter=-1,
                     max_newton_iterations=25, verbose=False):
    """``RedMVPSolver.solve`` (``red_mvp_solver.py:121-224``) over an oracle assembler.

    Increment test max|h| < tol max|x|; scipy CG with atol=tol (rtol 1e-5) and a Jacobi
    preconditioner on the Dirichlet-reduced Jacobian; exit codes ignored.
    """
    n = assembler.num_dofs
    x_n = np.zeros(n) if x_0 is None or len(x_0) == 0 else np.array(x_0, dtype=np.float64)
    x_np1 = x_n.copy()
    stats = {"newton": 0, "cg": []}
    for i in range(max_newton_iterations):
        K, J, rhs = assembler.compute_stiffness_and_jacobi_matrix_c(x_n, source_fields)
        b = J @ x_n - K @ x_n + rhs
        if max(abs(b)) < 1e-14:
            x_np1 = 0.0 * x_n
            break
        J_c = J[mask, :][:, mask]
        M = diags(1.0 / J_c.diagonal(), shape=J_c.shape)
        its = [0]

        def cb(_):
            its[0] += 1

        kw = {} if maxiter < 0 else {"maxiter": maxiter}
        xx, _ = cg(J_c, b[mask], atol=tolerance, x0=x_n[mask], M=M, callback=cb, **kw)
        stats["cg"].append(its[0])
        x_np1 = 0.0 * x_n
        x_np1[mask] = xx
        h = x_np1 - x_n
        stats["newton"] = i + 1
        if verbose:
            print(f"  step {i}: max relative increment {max(abs(h)) / max(abs(x_np1)):.3e}, cg its {its[0]}")
        if max(abs(h)) < tolerance * max(abs(x_np1)):
            break
        x_n = x_np1.copy()
    return x_np1, stats


def ew_forcing(it, fn, fprev, eta_prev, F0, tol, eta_max=0.1, fp32=False):
    """Inner CG tolerance of the device Newton (Eisenstat-Walker choice 2 with safeguards):
    eta_0 = eta_max; eta_k = 0.9 (|F_k| / |F_k-1|)^2, kept >= 0.9 eta_k-1^2 when that exceeds 0.1,
    capped at eta_max; never below 0.5 tol |F_0| / |F_k| (no solving past the target)."""
    eta_max = min(eta_max if eta_max > 0 else 0.1, 0.5)
    eta = eta_max
    if it > 0:
        eta = 0.9 * (fn / fprev) ** 2
        sg = 0.9 * eta_prev * eta_prev
        if sg > 0.1 and sg > eta:
            eta = sg
        eta = min(eta, eta_max)
    eta = max(eta, 0.5 * tol * F0 / fn)
    if fp32:
        eta = max(eta, 1e-6)
    return min(eta, 0.5)


def block_jacobi_inverse(J, meta, mask):
    """Block-Jacobi preconditioner of the free Jacobian J[mask][:, mask] as a scipy matrix:
    the inverse of each diagonal block of the partition ``meta`` (uint16 per DoF: offset in
    the block | block size << 8, constrained DoFs alone; the product's ``newton.dof_blocks``).
    Restates the product's block build (per-DoF block rows of J, each block inverted) in
    float64, with its fallback to 1/diag for a block that is not positive definite."""
    from scipy.sparse import coo_matrix

    J = J.tocsr()
    n = J.shape[0]
    rows, cols, vals = [], [], []
    i = 0
    while i < n:
        s = int(meta[i]) >> 8
        if mask[i]:
            idx = np.arange(i, i + s)
            B = J[idx][:, idx].toarray()
            B = np.triu(B) + np.triu(B, 1).T  # the upper triangle, as the device reads it
            try:
                np.linalg.cholesky(B)
                X = np.linalg.inv(B)
            except np.linalg.LinAlgError:
                X = np.diag(1.0 / np.diag(B))
            ii, jj = np.meshgrid(idx, idx, indexing="ij")
            rows.append(ii.ravel())
            cols.append(jj.ravel())
            vals.append(X.ravel())
        i += s
    M = coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)).tocsr()
    return M[mask][:, mask]


def newton_residual(assembler, mask, source_fields=(), rtol=1e-8, x_0=None, cg_rtol=1e-12, cg_maxiter=None,
                    max_newton_iterations=50, verbose=False, forcing="fixed", line_search=False, blocks=None):
    """Newton on F(x) = K(x) x - rhs(x) until ||F_free|| <= rtol ||F_free(x_0)||.

    Each step solves J_free h = -F_free with Jacobi-preconditioned scipy CG to the
    relative tolerance ``cg_rtol``, but never below the absolute level 0.1 * rtol * ||F_free(x_0)||:
    the curl-curl Jacobian is singular (gradients), and rounding in F leaves a small
    inconsistent component that a CG asked for more drives along that null space.
    With ``line_search`` the step is damped by Armijo backtracking on ||F_free||: from alpha = 1,
    each rejected alpha is replaced by the minimiser of the quadratic model of ||F||^2 along h,
    kept within [0.1, 0.5] alpha, until ||F(x + alpha h)|| <= (1 - 1e-4 alpha) ||F(x)|| (at most
    30 reductions).  ``forcing="ew"`` uses the device solver's inner tolerances (``ew_forcing``).
    ``blocks`` (a block partition, see ``block_jacobi_inverse``) replaces the point-Jacobi
    preconditioner by block Jacobi, as the device solver's residual mode does by default.
    Returns x and stats (residual history, CG counts, step lengths).
    """
    n = assembler.num_dofs
    x = np.zeros(n) if x_0 is None or len(x_0) == 0 else np.array(x_0, dtype=np.float64)
    x[~mask] = 0.0
    stats = {"newton": 0, "cg": [], "res": [], "eta": [], "alpha": [], "assemblies": 0}
    F0 = None
    fprev = eta_prev = 0.0
    cached = None
    for i in range(max_newton_iterations + 1):
        if cached is None:
            K, J, rhs = assembler.compute_stiffness_and_jacobi_matrix_c(x, source_fields)
            stats["assemblies"] += 1
            F = K @ x - rhs
            fn = np.linalg.norm(F[mask])
        else:
            K, J, rhs, F, fn = cached
            cached = None
        if F0 is None:
            F0 = fn
        stats["res"].append(fn)
        if verbose:
            print(f"  newton {i}: |F| = {fn:.3e} rel {fn / F0 if F0 > 0 else 0:.3e}")
        if F0 == 0 or fn <= rtol * F0 or i == max_newton_iterations:
            break
        J_c = J[mask, :][:, mask]
        if blocks is None:
            M = diags(1.0 / J_c.diagonal(), shape=J_c.shape)
        else:
            M = block_jacobi_inverse(J, blocks, mask)
        its = [0]

        def cb(_):
            its[0] += 1

        if forcing == "ew":
            eta = ew_forcing(i, fn, fprev, eta_prev, F0, rtol, cg_rtol)
            fprev, eta_prev = fn, eta
            stats["eta"].append(eta)
            h, _ = cg(J_c, -F[mask], rtol=eta, atol=0.0, M=M, callback=cb, maxiter=cg_maxiter)
        else:
            h, _ = cg(J_c, -F[mask], rtol=cg_rtol, atol=0.1 * rtol * F0, M=M, callback=cb, maxiter=cg_maxiter)
        stats["cg"].append(its[0])
        if line_search == "energy":
            # F is the gradient of the magnetic energy W (convex for a monotone B-H law), so
            # phi'(a) = F(x + a h) . h increases along h: keep the full step unless
            # phi'(1) > 0.5 |phi'(0)|, else bracket phi'(a) ~ 0 by a safeguarded secant and
            # accept |phi'(a)| <= 0.5 |phi'(0)| (undershoots raise the lower end)
            g0 = float(F[mask] @ h)
            a_lo, g_lo, a_hi, g_hi = 0.0, g0, 1.0, 0.0
            alpha = 1.0
            c = 0.5 * abs(g0)
            for ls in range(12):
                xt = x.copy()
                xt[mask] += alpha * h
                Kt, Jt, rt = assembler.compute_stiffness_and_jacobi_matrix_c(xt, source_fields)
                stats["assemblies"] += 1
                Ft = Kt @ xt - rt
                g = float(Ft[mask] @ h)
                if g != g or ls == 11:
                    break
                if (g <= c) if ls == 0 else (abs(g) <= c):
                    break
                if g < -c:
                    a_lo, g_lo = alpha, g
                else:
                    a_hi, g_hi = alpha, g
                a_new = a_lo - g_lo * (a_hi - a_lo) / (g_hi - g_lo)
                width = a_hi - a_lo
                alpha = min(max(a_new, a_lo + 0.01 * width), a_hi - 0.01 * width)
            ft = np.linalg.norm(Ft[mask])
            x = xt
            cached = (Kt, Jt, rt, Ft, ft)
            stats["alpha"].append(alpha)
        elif line_search:
            alpha = 1.0
            for ls in range(31):
                xt = x.copy()
                xt[mask] += alpha * h
                Kt, Jt, rt = assembler.compute_stiffness_and_jacobi_matrix_c(xt, source_fields)
                stats["assemblies"] += 1
                Ft = Kt @ xt - rt
                ft = np.linalg.norm(Ft[mask])
                if (ft == ft and ft <= (1.0 - 1e-4 * alpha) * fn) or ls >= 30:
                    break
                # minimiser of the quadratic through phi(0) = fn^2, phi'(0) = -2 fn^2, phi(alpha) = ft^2,
                # kept within [0.1, 0.5] alpha (the device solver's rule)
                a_new = 0.5 * alpha
                if ft == ft:
                    den = ft * ft - fn * fn + 2.0 * fn * fn * alpha
                    if den > 0:
                        a_new = fn * fn * alpha * alpha / den
                alpha = min(max(a_new, 0.1 * alpha), 0.5 * alpha)
            x = xt
            cached = (Kt, Jt, rt, Ft, ft)
            stats["alpha"].append(alpha)
        else:
            x[mask] += h
        stats["newton"] = i + 1
    stats["rel_res"] = stats["res"][-1] / F0 if F0 else 0.0
    return x, stats


def laplace_subdomain_solve(nodes, cells, term_tags, subdomain_mask, Phi, tags_term_1, tags_term_2, w, q, d_phi,
                            backend="oracle"):
    """``LaplaceSubdomainSolver.solve`` (``laplace_subdomain_solver.py:117-158``)."""
    from scipy.sparse import csr_array as _csr

    num_all = nodes.shape[0]
    x_l = np.zeros(num_all)
    x_l[tags_term_1] = -0.5 * Phi
    x_l[tags_term_2] = 0.5 * Phi

    class _Const:
        def __init__(self, mu):
            self.mu = mu

        def get_type_spec(self):
            return 0

        def evaluate_mu(self, H, relative=False):
            return self.mu + 0.0 * np.asarray(H)

    K, _ = compute_stiffness_and_jacobi_matrix(nodes, cells, d_phi, 0.0 * x_l, _Const(1.0), q, w, backend)
    K = _csr(K)
    rhs = -K @ x_l
    keep = np.ones(num_all, dtype=bool)
    keep[term_tags] = False
    K_c = K[np.flatnonzero(keep), :][:, np.flatnonzero(keep)]
    rhs_c = np.delete(rhs, term_tags)
    mask_c = np.delete(subdomain_mask, term_tags)
    num_dof_red = len(rhs_c)
    K_c = K_c[mask_c, :][:, mask_c]
    rhs_c = rhs_c[mask_c]
    x_c = spsolve(K_c, rhs_c)
    x = np.zeros(num_dof_red)
    x[mask_c] = x_c
    out = x_l.copy()
    out[np.flatnonzero(keep)] = x
    return out


# ------------------------------------------------------------------ field maps

def locate_points(nodes, cells, points, tol=1e-12):
    """Element index (-1 outside) and barycentric coordinates of each point.

    The bucket search of the device mesh index, in numpy: elements bucketed by centroid on a
    uniform grid whose cell is at least the largest element extent, the 27 buckets around the
    point searched, the candidate with the largest smallest barycentric coordinate kept (the
    first one on ties; coordinates by LU solve).  The reference locates with gmsh's
    ``get_element_by_coordinates`` (``snoopy/evaluators.py:155-295``).
    """
    nodes = np.asarray(nodes, dtype=np.float64).reshape(-1, 3)
    cells = np.asarray(cells, dtype=np.int64).reshape(-1, 4)
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    p = nodes[cells]  # [E,4,3]
    ext = (p.max(axis=1) - p.min(axis=1)).max()
    cen = p.mean(axis=1)
    bmin = nodes.min(axis=0)
    bmax = nodes.max(axis=0)
    nb = np.maximum(1, np.floor((bmax - bmin) / ext).astype(np.int64))
    h = (bmax - bmin) / nb
    cb = np.minimum(((cen - bmin) / h).astype(np.int64), nb - 1)
    key = cb[:, 0] + nb[0] * (cb[:, 1] + nb[1] * cb[:, 2])
    order = np.argsort(key, kind="stable")
    skey = key[order]
    elem = np.full(pts.shape[0], -1, dtype=np.int64)
    bary = np.zeros((pts.shape[0], 4))
    fin = np.isfinite(pts).all(axis=1)
    r = np.where(fin[:, None], (pts - bmin) / h, -10.0)
    ip = np.floor(np.clip(r, -2.0, nb + 1.0)).astype(np.int64)
    offs = np.array([(i, j, k) for i in (-1, 0, 1) for j in (-1, 0, 1) for k in (-1, 0, 1)])
    for n, x in enumerate(pts):
        if not fin[n]:
            continue
        b = ip[n] + offs
        ok = np.all((b >= 0) & (b < nb), axis=1)
        b = b[ok]
        keys = b[:, 0] + nb[0] * (b[:, 1] + nb[1] * b[:, 2])
        lo = np.searchsorted(skey, keys, side="left")
        hi = np.searchsorted(skey, keys, side="right")
        cand = np.concatenate([order[a:c] for a, c in zip(lo, hi)]) if len(keys) else np.zeros(0, np.int64)
        if cand.size == 0:
            continue
        pc = p[cand]
        T = np.stack([pc[:, 1] - pc[:, 0], pc[:, 2] - pc[:, 0], pc[:, 3] - pc[:, 0]], axis=2)
        lam123 = np.linalg.solve(T, (x - pc[:, 0])[:, :, None])[:, :, 0]
        lam = np.concatenate([1.0 - lam123.sum(axis=1, keepdims=True), lam123], axis=1)
        score = lam.min(axis=1)
        best = int(np.argmax(score))
        if score[best] >= -tol:
            elem[n] = cand[best]
            bary[n] = lam[best]
    return elem, bary


def element_B(nodes, cells, glob_ids, orientations, curls, n_orient, d_phi, x):
    """B = sum_k J curl_hat_k x_k / det in every listed element, at the first point of the
    tables (first order: constant), the loop body of ``compute_nodal_fields``
    (``snoopy/curl_curl_assembler.py:2160-2183``)."""
    nodes = np.asarray(nodes, dtype=np.float64).reshape(-1, 3)
    cells = np.asarray(cells, dtype=np.int64).reshape(-1, 4)
    gids = np.asarray(glob_ids, dtype=np.int64).reshape(-1, 6)
    ori = np.asarray(orientations, dtype=np.int64).reshape(-1)
    dphi = np.asarray(d_phi, dtype=np.float64).reshape(-1, 4, 3)[0]
    ct = np.asarray(curls, dtype=np.float64).reshape(int(n_orient), -1, 6, 3)[:, 0]  # [n_orient, 6, 3], first point
    X = nodes[cells]                                   # [E, 4, 3]
    J = np.einsum("eik,il->ekl", X, dphi)              # J[k][l] = sum_i X_i[k] dphi_i[l]
    det = np.linalg.det(J)
    xv = np.asarray(x, dtype=np.float64)[gids]         # [E, 6]
    B = np.zeros((len(cells), 3))
    for k in range(6):
        B += np.einsum("ekl,el->ek", J, ct[ori, k]) * (xv[:, k] / det)[:, None]
    return B


def nodal_fields(num_nodes, cells, B_elem):
    """Element values averaged at the nodes (``compute_nodal_fields``,
    ``snoopy/curl_curl_assembler.py:2185-2196``): per node the sum over its listed elements
    divided by their number; nodes with none keep 0."""
    cells = np.asarray(cells, dtype=np.int64).reshape(-1, 4)
    out = np.zeros((num_nodes, B_elem.shape[1]))
    mult = np.zeros(num_nodes, dtype=np.int64)
    for i in range(4):
        np.add.at(out, cells[:, i], B_elem)
        np.add.at(mult, cells[:, i], 1)
    m = mult != 0
    out[m] /= mult[m][:, None]
    return out


def interpolate_nodal(cells, elem, bary, nodal_sets, point_set):
    """sum_i phi_i v[cells[e][i]] at located points (``evaluate_interpolation``,
    ``snoopy/evaluators.py:390-406``), v = nodal_sets[point_set[p]]; 0 for unlocated points."""
    cells = np.asarray(cells, dtype=np.int64).reshape(-1, 4)
    nc = nodal_sets[0].reshape(len(nodal_sets[0]), -1).shape[1]
    out = np.zeros((len(elem), nc))
    for p, (e, s) in enumerate(zip(elem, point_set)):
        if e < 0 or s < 0:
            continue
        v = nodal_sets[s].reshape(-1, nc)
        out[p] = bary[p] @ v[cells[e]]
    return out


def probe_B(nodes, cells, glob_ids, orientations, curls, phi, d_phi, q, w, num_dofs, x, points, coils=(),
            backend="ref"):
    """Total field B = curl A + B_s at points, all arithmetic on the CPU: points located by
    ``locate_points``, curl A from ``compute_B_Hcurl`` (``interface_c.pyx:555-696``, through the
    chosen backend) on the located elements (first order: constant per element, so its first
    quadrature point serves), the source field of ``coils`` (objects with ``get_segments()``,
    ``current`` and ``rad``) from ``compute_B_line_segs_cpp`` (``interface_c.pyx:928-991``), as
    ``RedMVPSolver``'s field output adds it.  Returns (B [P, 3], element index [P])."""
    el, _ = locate_points(nodes, cells, points)
    if (el < 0).any():
        raise ValueError(f"{int((el < 0).sum())} points lie outside the mesh")
    cells = np.asarray(cells).reshape(-1, 4)
    gids = np.asarray(glob_ids).reshape(-1, 6)
    ori = np.asarray(orientations).reshape(-1)
    _, B = compute_B_Hcurl(nodes, cells[el], gids[el], curls, phi, d_phi, ori[el], x, q, w, num_dofs, 6, backend)
    B = B.reshape(len(el), -1, 3)[:, 0].copy()
    for c in coils:
        B += compute_B_line_segs_cpp(c.get_segments(), points, c.current, c.rad, backend=backend)
    return B, el
