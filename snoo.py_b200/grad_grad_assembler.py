"""``GradGradAssembler`` with the reference's interface (``snoopy/matrix_assembly.py:92-1135``,
duplicated as ``snoopy/grad_grad_assembler.py``), plus the sparse row/column helpers of
``matrix_assembly.py:16-90``.

Nodal P1 assembly of div(mu grad phi) and its Newton Jacobian through the sm_100a kernel
``snp_gradgrad_assemble``; one CSR pattern over all domains is built once and cached.
"""

import numpy as np

from . import _lib
from . import finite_element as fe
from .device import Pattern, permeability_tables, upload, zeros


def recover_full_solution(u, u_g, b):
    """Insert the reduced solution into the lifting vector (``matrix_assembly.py:16-46``)."""
    num_nodes = len(u_g)
    indx_rem = np.delete(np.arange(num_nodes, dtype=np.int64), b)
    u_ret = np.array(u_g, dtype=np.float64).copy()
    u_ret[indx_rem] = u
    return u_ret


def delete_rows_sparse(M, rows):
    """``matrix_assembly.py:48-68``."""
    mask = np.ones(M.shape[0], dtype=bool)
    mask[rows] = False
    return M[np.flatnonzero(mask), :]


def delete_cols_sparse(M, cols):
    """``matrix_assembly.py:70-90``."""
    mask = np.ones(M.shape[1], dtype=bool)
    mask[cols] = False
    return M[:, np.flatnonzero(mask)]


class GradGradAssembler:
    """P1 scalar-potential assembler (``matrix_assembly.py:92``)."""

    def __init__(self, mesh, domain_tags):
        self.mesh = mesh
        self.nodes = mesh.nodes
        self.num_materials = len(domain_tags)
        self.cell_types = []
        self.cells = []
        self._elems = []
        for tag in domain_tags:
            el = mesh.domain_elements(tag)
            self._elems.append(el)
            self.cell_types.append(np.array([4]))
            self.cells.append([(mesh.cells[el].astype(np.int64) + 1).reshape(-1)])
        self.domain_tags = list(domain_tags)
        self._dev = None
        self._tables = {}

    def get_quadrature_rule(self, ct, quad_order):
        w, q = fe.quadrature_rule(quad_order)
        return q, w

    def _device_state(self):
        if self._dev is None:
            _lib.require_cuda()
            cells = [self.mesh.cells[el] for el in self._elems]
            allc = np.concatenate(cells) if cells else np.zeros((0, 4), dtype=np.int32)
            cd = upload(allc, np.int32)
            offs = np.cumsum([0] + [len(el) for el in self._elems])
            self._dev = {"nodes": upload(self.nodes, np.float64), "cells": cd, "offsets": offs,
                         "pattern": Pattern(cd, len(allc), 4, self.nodes.shape[0])}
        return self._dev

    def _tabs(self, quad_order):
        if quad_order not in self._tables:
            w, q = fe.quadrature_rule(quad_order)
            self._tables[quad_order] = (len(w), upload(w, np.float64), upload(fe.evaluate_basis_derivative(q), np.float64))
        return self._tables[quad_order]

    @property
    def pattern(self):
        return self._device_state()["pattern"]

    def assemble_device(self, x, mu_list, quad_order=8, K=True, dK=False, J=True):
        """Assemble into the cached pattern; returns CUDA tensors (those requested) and ``pattern``."""
        d = self._device_state()
        nq, w_d, dphi_d = self._tabs(quad_order)
        pat = d["pattern"]
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        out = {"pattern": pat, "K": zeros(pat.nnz) if K else None, "dK": zeros(pat.nnz) if dK else None,
               "J": zeros(pat.nnz) if J else None}
        for n, perm in enumerate(mu_list):
            typ, k, nc, t, c, hmin, muh = permeability_tables(perm)
            off, cnt = int(d["offsets"][n]), int(d["offsets"][n + 1] - d["offsets"][n])
            _lib.call("snp_gradgrad_assemble", pat.handle, off, cnt, _lib.ptr(d["nodes"]),
                      _lib.ptr(d["cells"][4 * off:]) if cnt else _lib.ptr(d["cells"]), _lib.ptr(dphi_d), _lib.ptr(w_d),
                      nq, _lib.ptr(x_d), typ, k, nc, _lib.ptr(t), _lib.ptr(c), hmin, muh, _lib.ptr(out["K"]),
                      _lib.ptr(out["dK"]), _lib.ptr(out["J"]), _lib.stream_ptr())
        return out

    def compute_stiffness_and_jacobi_matrix_c(self, x, mu_list, quad_order=8, device=False):
        """``(K, J)`` (``matrix_assembly.py:1059-1135``), scipy CSR without exact zeros; with
        ``device=True`` torch sparse CSR tensors on the GPU (full structural pattern).

        The reference adds the running K to dK after every material (``dK += K`` inside the
        material loop), so J = dK + sum_n (K of materials 0..n).  This is kept as is: with one
        domain, the Laplace subdomain case, it is K + dK.
        """
        d = self._device_state()
        nq, w_d, dphi_d = self._tabs(quad_order)
        pat = d["pattern"]
        x_d = x if hasattr(x, "data_ptr") else upload(x, np.float64)
        K = zeros(pat.nnz)
        dK = zeros(pat.nnz)
        Ksum = zeros(pat.nnz)
        for n, perm in enumerate(mu_list):
            typ, k, nc, t, c, hmin, muh = permeability_tables(perm)
            off, cnt = int(d["offsets"][n]), int(d["offsets"][n + 1] - d["offsets"][n])
            _lib.call("snp_gradgrad_assemble", pat.handle, off, cnt, _lib.ptr(d["nodes"]),
                      _lib.ptr(d["cells"][4 * off:]) if cnt else _lib.ptr(d["cells"]), _lib.ptr(dphi_d), _lib.ptr(w_d),
                      nq, _lib.ptr(x_d), typ, k, nc, _lib.ptr(t), _lib.ptr(c), hmin, muh, _lib.ptr(K), _lib.ptr(dK),
                      None, _lib.stream_ptr())
            Ksum += K
        J = dK + Ksum
        if device:
            return pat.to_torch(K), pat.to_torch(J)
        return pat.to_scipy(K, drop_zeros=True), pat.to_scipy(J, drop_zeros=True)
