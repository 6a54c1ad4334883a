"""``CurlCurlAssembler`` with the reference's interface (``snoopy/curl_curl_assembler.py``).

The reference gathers per-material cells and edge ids from gmsh (``:19-137``), and every
Newton step re-queries element orientations from gmsh, re-creates reference tables, calls
the C kernel per material, converts triplets to CSR and adds the matrices (``:815-932``).
Here the mesh arrays, tables and one CSR pattern over all materials are uploaded once and
cached.  Each call stores every element's matrix values (one launch per material) and then
sums every CSR entry from its element contributions in element order (one launch): the values
are bitwise repeatable and each is written once.  ``SNP_ASSEMBLY=atomic`` (or ``method="atomic"``)
selects the one-launch-per-material kernels that add element values into the CSR with atomics.

``mesh`` is a ``snoopy_b200.mesh.TetMesh`` (gmsh is not a dependency); ``volume_tags`` are
its volume tags, in the order of ``material_list``.
"""

import ctypes
import os

import numpy as np

from . import _lib
from . import finite_element as fe
from .device import Pattern, check_affine, reluctance_tables, torch, upload, zeros


class _QuadTables:
    def __init__(self, quad_order):
        self.quad_order = quad_order
        self.w, self.q = fe.quadrature_rule(quad_order)
        self.nq = len(self.w)
        self.d_phi = fe.evaluate_basis_derivative(self.q)
        self.phi = fe.evaluate_basis(self.q)
        self.curls, self.n_orient = fe.curl_edge_basis_functions(self.q)
        check_affine(self.curls, self.d_phi, self.nq)
        self.w_d = upload(self.w, np.float64)
        self.d_phi_d = upload(self.d_phi, np.float64)
        self.phi_d = upload(self.phi, np.float64)
        self.curls_d = upload(self.curls, np.float64)


class CurlCurlAssembler:
    """Assembler of the Newton system of the curl-curl operator (``curl_curl_assembler.py:17``)."""

    def __init__(self, mesh, volume_tags, material_list, element_order=1):
        if element_order > 4:
            print("Warning! Elements order {} not implemented. Using 1".format(element_order))
            element_order = 1
        if element_order != 1:
            raise NotImplementedError("only first-order edge elements (element_order=1) are implemented")
        self.mesh = mesh
        self.element_order = 1
        self.num_dofs = int(mesh.num_dofs)
        self.material_list = material_list
        self.nodes = mesh.nodes
        self.cell_types = []
        self.cells = []
        self.global_ids = []
        self.cell_tags = []
        self.orientations = []
        self._elems = []
        tags = list(volume_tags) if len(volume_tags) > 0 else [-1]
        self.num_materials = len(material_list) if len(volume_tags) > 0 else 1
        for tag in tags:
            el = mesh.domain_elements(tag)
            self._elems.append(el)
            self.cell_types.append(np.array([4]))
            self.cells.append([(mesh.cells[el].astype(np.int64) + 1).reshape(-1)])
            self.cell_tags.append(el + 1)
            self.global_ids.append((mesh.elem_edges[el] + 1).astype(np.int32))
            self.orientations.append(mesh.orientations[el])
        self.volume_tags = volume_tags
        self._dev = None
        self._tables = {}

    # ---------------------------------------------------------------- device state
    def _device_state(self):
        if self._dev is None:
            _lib.require_cuda()
            d = {"nodes": upload(self.nodes, np.float64), "mats": [], "offsets": []}
            off = 0
            all_gids = []
            for n in range(self.num_materials):
                el = self._elems[n]
                d["mats"].append({"cells": upload(self.mesh.cells[el], np.int32),
                                  "gids": upload(self.mesh.elem_edges[el], np.int32),
                                  "orient": upload(self.mesh.orientations[el], np.int32),
                                  "count": len(el), "offset": off})
                off += len(el)
                all_gids.append(self.mesh.elem_edges[el])
            gids = upload(np.concatenate(all_gids) if all_gids else np.zeros((0, 6)), np.int32)
            d["pattern"] = Pattern(gids, off, 6, self.num_dofs)
            d["rel"] = [reluctance_tables(m) for m in self.material_list[: self.num_materials]]
            self._dev = d
        return self._dev

    def tables(self, quad_order):
        if quad_order not in self._tables:
            self._tables[quad_order] = _QuadTables(quad_order)
        return self._tables[quad_order]

    @property
    def pattern(self):
        return self._device_state()["pattern"]

    def upload_source_fields(self, source_fields):
        """Per-material device tensors (or None) from the reference's ``source_fields`` list."""
        use = len(source_fields) == self.num_materials
        out = []
        for n in range(self.num_materials):
            if use and len(source_fields[n]) > 0:
                sf = source_fields[n]
                out.append(sf if hasattr(sf, "data_ptr") else upload(sf, np.float64))
            else:
                out.append(None)
        return out

    def assemble_device(self, x, quad_order=2, source_fields=(), K=True, J=True, rhs=True, F=False, dK=False,
                        stream=None, method=None):
        """Assemble on the device into the cached pattern.

        :param x: float64 DoF vector (numpy or CUDA tensor).
        :param method: ``"rows"`` (element values, then one sum per CSR entry: deterministic),
            ``"atomic"`` (element kernels adding into the CSR), or None: ``$SNP_ASSEMBLY``, else
            rows where the pattern allows it.
        :return: dict of CUDA tensors ``K``, ``J`` (= K + dK), ``dK`` [nnz], ``rhs``, ``F`` [n]
            (those requested), plus ``pattern``.
        """
        d = self._device_state()
        tb = self.tables(quad_order)
        pat = d["pattern"]
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        bs = self.upload_source_fields(source_fields)
        out = {"pattern": pat}
        method = method or os.environ.get("SNP_ASSEMBLY", "rows")
        s = _lib.stream_ptr(stream)
        if method != "atomic" and pat.rows_supported:
            t = torch()
            for key, want, size in (("K", K, pat.nnz), ("J", J, pat.nnz), ("dK", dK, pat.nnz),
                                    ("rhs", rhs, self.num_dofs), ("F", F, self.num_dofs)):
                out[key] = t.empty(max(size, 1), dtype=t.float64, device="cuda") if want else None
            parts = ((_lib.TERMS_K if (K or J) else 0) | (_lib.TERMS_DK if (dK or J) else 0)
                     | (_lib.TERMS_F if F else 0) | (_lib.TERMS_RHS if rhs else 0))
            stride = ctypes.c_int32()
            _lib.call("snp_curlcurl_terms_stride", parts, ctypes.byref(stride))
            need = pat.n_elems * stride.value
            if d.get("terms") is None or d["terms"].numel() < need:
                d["terms"] = t.empty(max(need, 1), dtype=t.float64, device="cuda")
            for n, m in enumerate(d["mats"]):
                n_int, rc, rx = d["rel"][n]
                coef = self._dilution_coef(n)
                _lib.call("snp_curlcurl_terms", pat.handle, m["offset"], m["count"], _lib.ptr(d["nodes"]),
                          _lib.ptr(m["cells"]), _lib.ptr(m["gids"]), _lib.ptr(m["orient"]), _lib.ptr(tb.curls_d),
                          tb.n_orient, _lib.ptr(tb.phi_d) if coef is not None else None, _lib.ptr(tb.d_phi_d),
                          _lib.ptr(tb.w_d), tb.nq, _lib.ptr(x_d), _lib.ptr(bs[n]), n_int, _lib.ptr(rc), _lib.ptr(rx),
                          coef, parts, _lib.ptr(d["terms"]), s)
            _lib.call("snp_curlcurl_rows", pat.handle, _lib.ptr(d["terms"]), parts, _lib.ptr(out["K"]),
                      _lib.ptr(out["dK"]), _lib.ptr(out["J"]), None, _lib.ptr(out["rhs"]), _lib.ptr(out["F"]), s)
            for key, want, size in (("K", K, pat.nnz), ("J", J, pat.nnz), ("dK", dK, pat.nnz),
                                    ("rhs", rhs, self.num_dofs), ("F", F, self.num_dofs)):
                if want:
                    out[key] = out[key][:size]
            return out
        for key, want, size in (("K", K, pat.nnz), ("J", J, pat.nnz), ("dK", dK, pat.nnz), ("rhs", rhs, self.num_dofs),
                                ("F", F, self.num_dofs)):
            out[key] = zeros(size) if want else None
        for n, m in enumerate(d["mats"]):
            n_int, rc, rx = d["rel"][n]
            coef = self._dilution_coef(n)
            common = (pat.handle, m["offset"], m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]),
                      _lib.ptr(m["gids"]), _lib.ptr(m["orient"]), _lib.ptr(tb.curls_d), tb.n_orient)
            outs = (_lib.ptr(out["K"]), _lib.ptr(out["dK"]), _lib.ptr(out["J"]), _lib.ptr(out["rhs"]),
                    _lib.ptr(out["F"]), s)
            if coef is None:
                _lib.call("snp_curlcurl_assemble", *common, _lib.ptr(tb.d_phi_d), _lib.ptr(tb.w_d), tb.nq,
                          _lib.ptr(x_d), _lib.ptr(bs[n]), n_int, _lib.ptr(rc), _lib.ptr(rx), *outs)
            else:
                _lib.call("snp_curlcurl_assemble_diluted", *common, _lib.ptr(tb.phi_d), _lib.ptr(tb.d_phi_d),
                          _lib.ptr(tb.w_d), tb.nq, _lib.ptr(x_d), _lib.ptr(bs[n]), n_int, _lib.ptr(rc), _lib.ptr(rx),
                          coef, *outs)
        return out

    def _dilution_coef(self, n):
        """Dilution coefficients {c_num, m_num, c_den, m_den} of material ``n`` as a ctypes array,
        or None for plain steel and air (the diluted assembler overrides this)."""
        return None

    # ---------------------------------------------------------------- reference API
    def compute_stiffness_and_jacobi_matrix_c(self, x, quad_order=2, source_fields=[], device=False):
        """``(K, dK + K, rhs)`` like ``curl_curl_assembler.py:815-932``: scipy CSR without exact zeros.
        With ``device=True``: torch sparse CSR tensors on the GPU with the full structural pattern
        (exact zeros kept) and a CUDA rhs, nothing copied to the host."""
        out = self.assemble_device(x, quad_order, source_fields, K=True, J=True, rhs=True)
        pat = out["pattern"]
        if device:
            return pat.to_torch(out["K"]), pat.to_torch(out["J"]), out["rhs"][: self.num_dofs]
        K = pat.to_scipy(out["K"], drop_zeros=True)
        J = pat.to_scipy(out["J"], drop_zeros=True)
        return K, J, out["rhs"][: self.num_dofs].cpu().numpy()

    def get_quadrature_points(self, quad_order=3, domain_ids=[]):
        """Physical quadrature points, one [E_m * Q, 3] array per material (``:1521-1593``)."""
        d = self._device_state()
        tb = self.tables(quad_order)
        n_list = domain_ids if len(domain_ids) > 0 else range(self.num_materials)
        out = []
        for n in n_list:
            m = d["mats"][n]
            pts = zeros(3 * m["count"] * tb.nq)
            _lib.call("snp_quad_points", m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]), _lib.ptr(tb.phi_d),
                      tb.nq, _lib.ptr(pts), _lib.stream_ptr())
            out.append(pts[: 3 * m["count"] * tb.nq].cpu().numpy().reshape(-1, 3))
        return out

    def get_quadrature_points_device(self, quad_order, n):
        d = self._device_state()
        tb = self.tables(quad_order)
        m = d["mats"][n]
        pts = zeros(3 * m["count"] * tb.nq)
        _lib.call("snp_quad_points", m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]), _lib.ptr(tb.phi_d),
                  tb.nq, _lib.ptr(pts), _lib.stream_ptr())
        return pts[: 3 * m["count"] * tb.nq]

    def compute_B(self, x, quad_order=8):
        """Quadrature points and B = curl A there over all materials (``:1722-1802``)."""
        d = self._device_state()
        tb = self.tables(quad_order)
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        P, B = [], []
        for m in d["mats"]:
            n = 3 * m["count"] * tb.nq
            pts = zeros(n)
            b = zeros(n)
            _lib.call("snp_b_hcurl", m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]), _lib.ptr(m["gids"]),
                      _lib.ptr(m["orient"]), _lib.ptr(tb.curls_d), tb.n_orient, _lib.ptr(tb.phi_d), _lib.ptr(tb.d_phi_d),
                      tb.nq, _lib.ptr(x_d), _lib.ptr(pts), _lib.ptr(b), _lib.stream_ptr())
            P.append(pts[:n].cpu().numpy().reshape(-1, 3))
            B.append(b[:n].cpu().numpy().reshape(-1, 3))
        return np.concatenate(P, axis=0), np.concatenate(B, axis=0)

    def compute_rhs_electric_potential(self, x_p, quad_order=8, select_mat="all"):
        """rhs from a nodal electric potential over the selected materials (``:1154-1284``)."""
        d = self._device_state()
        materials = range(self.num_materials) if isinstance(select_mat, str) else select_mat
        w, q = fe.quadrature_rule(quad_order)
        nq = len(w)
        basis = fe.edge_basis_functions(q)  # [Q, 6, 3], orientation 0
        signs = fe.orientation_signs(np.arange(fe.N_ORIENT))
        basis_t = upload(signs[:, None, :, None] * basis[None], np.float64)
        dphi_t = upload(fe.evaluate_basis_derivative(q), np.float64)
        w_t = upload(w, np.float64)
        xp = x_p if hasattr(x_p, "data_ptr") else upload(x_p, np.float64)
        rhs = zeros(self.num_dofs)
        for n in materials:
            m = d["mats"][n]
            _lib.call("snp_rhs_grad_potential", m["count"], _lib.ptr(d["nodes"]), _lib.ptr(m["cells"]),
                      _lib.ptr(m["gids"]), _lib.ptr(m["orient"]), _lib.ptr(basis_t), fe.N_ORIENT, _lib.ptr(dphi_t),
                      _lib.ptr(w_t), nq, _lib.ptr(xp), _lib.ptr(rhs), _lib.stream_ptr())
        return rhs[: self.num_dofs].cpu().numpy()

    def element_B_device(self, x):
        """Device [E, 3]: B = curl A in every element of the mesh (first order: constant)."""
        d = self._device_state()
        tb = self.tables(1)
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        if "all" not in d:
            d["all"] = (upload(self.mesh.cells, np.int32), upload(self.mesh.elem_edges, np.int32),
                        upload(self.mesh.orientations, np.int32))
        if "arange" not in d:
            d["arange"] = upload(np.arange(self.mesh.num_elements), np.int32)
        cells_d, gids_d, or_d = d["all"]
        E = self.mesh.num_elements
        B = zeros(3 * E)[: 3 * E]
        _lib.call("snp_b_at_elements", E, _lib.ptr(d["arange"]), _lib.ptr(d["nodes"]), _lib.ptr(cells_d),
                  _lib.ptr(gids_d), _lib.ptr(or_d), _lib.ptr(tb.curls_d), tb.n_orient, _lib.ptr(tb.d_phi_d), tb.nq,
                  _lib.ptr(x_d), _lib.ptr(B), _lib.stream_ptr())
        return B.view(E, 3)

    def compute_nodal_fields(self, x, mat_ids):
        """B at the mesh nodes by averaging the element fields of the materials ``mat_ids``
        (volume tags) around each node (``curl_curl_assembler.py:2089-2196``); nodes outside
        them get 0.  Returns float64 [N, 3] (numpy)."""
        mask = np.zeros(self.mesh.num_elements, dtype=np.uint8)
        for mid in mat_ids:
            n = list(self.volume_tags).index(mid)
            mask[self._elems[n]] = 1
        B = self.element_B_device(x)
        out = self.mesh.index().nodal_average(B, 3, upload(mask, np.uint8))
        return out.cpu().numpy()

    def compute_B_at_points(self, x, points, elements=None):
        """B = curl A at arbitrary points (element constant for first order); points outside give 0."""
        d = self._device_state()
        tb = self.tables(1)
        if elements is None:
            elements, _ = self.mesh.locate(points)
        elements = np.asarray(elements, dtype=np.int64)
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        B = zeros(3 * len(elements))
        if "all" not in d:
            d["all"] = (upload(self.mesh.cells, np.int32), upload(self.mesh.elem_edges, np.int32),
                        upload(self.mesh.orientations, np.int32))
        cells_d, gids_d, or_d = d["all"]
        el_d = upload(elements, np.int32)
        _lib.call("snp_b_at_elements", len(elements), _lib.ptr(el_d), _lib.ptr(d["nodes"]), _lib.ptr(cells_d),
                  _lib.ptr(gids_d), _lib.ptr(or_d), _lib.ptr(tb.curls_d), tb.n_orient, _lib.ptr(tb.d_phi_d), tb.nq,
                  _lib.ptr(x_d), _lib.ptr(B), _lib.stream_ptr())
        return B[: 3 * len(elements)].cpu().numpy().reshape(-1, 3)
