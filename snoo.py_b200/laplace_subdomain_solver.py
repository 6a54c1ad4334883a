"""``LaplaceSubdomainSolver`` (``snoopy/laplace_subdomain_solver.py``): the electric scalar
potential in a coil subdomain, driven by a potential difference between two terminals.

The reference assembles K with mu = 1 (``GradGradAssembler``), lifts the terminal values
+-Phi/2, deletes the terminal rows/columns, restricts to the subdomain and calls scipy's
direct ``spsolve`` (``:117-158``).  Here K is assembled by the grad-grad kernel and the
restricted SPD system is solved by the device Jacobi-PCG to a relative residual of 1e-14.
"""

import ctypes

import numpy as np

from . import _lib
from .device import upload, zeros
from .grad_grad_assembler import GradGradAssembler
from .materials import ConstantPermeability


class LaplaceSubdomainSolver:
    """:param mesh: ``TetMesh``; :param subdomain_tag: the coil volume tag;
    :param terminal_groups: two arrays of terminal node indices (the terminal surfaces)."""

    def __init__(self, mesh, subdomain_tag, terminal_groups, quad_order=4):
        self.mesh = mesh
        self.matrix_factory = GradGradAssembler(mesh, [subdomain_tag])
        self.terminal_1 = terminal_groups[0]
        self.terminal_2 = terminal_groups[1]
        self.setup_boundary_conditions()
        self.subdomain_mask = self.get_subdomain_mask(subdomain_tag)
        nodes_all = self.matrix_factory.nodes
        self.num_dofs_all = nodes_all.shape[0]
        self.num_dofs = int(self.subdomain_mask.sum())
        self.quad_order = quad_order
        self.rtol = 1e-14
        self.last_iterations = 0

    def setup_boundary_conditions(self):
        """Terminal node ids (``laplace_subdomain_solver.py:71-115`` finds them by coordinates)."""
        self.tags_term_1 = np.asarray(self.terminal_1, dtype=np.int32)
        self.tags_term_2 = np.asarray(self.terminal_2, dtype=np.int32)
        self.term_tags = np.append(self.tags_term_1, self.tags_term_2, axis=0)

    def get_subdomain_mask(self, subdomain_tag):
        return self.mesh.domain_nodes_mask(subdomain_tag)

    def make_lifting_vector(self, Phi):
        x_l = np.zeros((self.num_dofs_all,))
        x_l[self.tags_term_1] = -0.5 * Phi
        x_l[self.tags_term_2] = 0.5 * Phi
        return x_l

    def solve(self, Phi, return_device=False):
        """Potential for the terminal difference Phi, float64[num_nodes]."""
        x_l = self.make_lifting_vector(Phi)
        xl_d = upload(x_l, np.float64)
        out = self.matrix_factory.assemble_device(0.0 * xl_d, [ConstantPermeability(1.0)], self.quad_order, K=True,
                                                  J=False)
        pat = out["pattern"]
        n = self.num_dofs_all
        rhs = zeros(n)
        _lib.call("snp_spmv", n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["K"]), None,
                  _lib.ptr(xl_d), _lib.ptr(rhs), _lib.stream_ptr())
        rhs = -rhs
        free = self.subdomain_mask.copy()
        free[self.term_tags] = False
        free_d = upload(free.astype(np.uint8), np.uint8)
        x = zeros(n)
        its = ctypes.c_int64()
        res = ctypes.c_double()
        _lib.call("snp_pcg", n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["K"]), _lib.ptr(free_d),
                  _lib.ptr(rhs), _lib.ptr(x), self.rtol, 0.0, 100 * n, ctypes.byref(its), ctypes.byref(res),
                  _lib.stream_ptr())
        self.last_iterations = int(its.value)
        fm = free_d.bool()
        sol = xl_d.clone()
        sol[fm] = x[:n][fm]
        return sol if return_device else sol.cpu().numpy()
