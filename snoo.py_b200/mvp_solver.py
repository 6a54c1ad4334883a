"""``MVPSolver``: total magnetic vector potential with coil currents from Laplace subdomain
solves (``snoopy/mvp_solver.py``).  ``solve_nonlin`` keeps the reference's Newton loop
(``mvp_solver.py:222-334``) with every step on the device; the coil source rhs comes from
``CurlCurlAssembler.compute_rhs_electric_potential`` on the device.
"""

import numpy as np

from .curl_curl_assembler import CurlCurlAssembler
from .device import to_host, upload, zeros
from .laplace_subdomain_solver import LaplaceSubdomainSolver
from .materials import ConstantReluctance
from .newton import MODE_REFERENCE, MODE_RESIDUAL, DeviceNewton


class MVPSolver:
    """:param gmsh_model: ``TetMesh``; :param coil_terminals: per coil, two terminal node-index arrays."""

    def __init__(self, gmsh_model, coil_tags, iron_tags, air_tags, coil_terminals, reluctances,
                 max_newton_iterations=25, element_order=1, quad_order=-1):
        self.coil_sd_solvers = [LaplaceSubdomainSolver(gmsh_model.mesh, ct, coil_terminals[i])
                                for i, ct in enumerate(coil_tags)]
        domain_tags = list(coil_tags) + list(iron_tags) + list(air_tags)
        nu0 = ConstantReluctance(0.25 / np.pi * 1e7)
        material_properties = [nu0] * len(coil_tags) + list(reluctances) + [nu0] * len(air_tags)
        self.max_newton_iterations = max_newton_iterations
        self.element_order = element_order
        if element_order > 3:
            print("Error! Element order {} not implemented! Choosing 1.")
            element_order = 1
        self.quad_order = element_order + 2 if quad_order < 0 else quad_order
        self.dirichlet_dofs = gmsh_model.get_edge_boundary_dofs(["Dirichlet Boundary"], element_order)
        self.curl_curl_factory = CurlCurlAssembler(gmsh_model.mesh, domain_tags, material_properties, element_order)
        self.num_dofs_mvp = self.curl_curl_factory.num_dofs
        self.verbose = True
        self._newton = None
        self._rhs_key = None

    def get_global_ids(self):
        return self.curl_curl_factory.global_ids

    def make_boundary_mask(self):
        mask = np.ones((self.num_dofs_mvp,), dtype=bool)
        mask[np.asarray(self.dirichlet_dofs, dtype=np.int64) - 1] = False
        return mask

    def compute_source_rhs(self, phi_list):
        """rhs_mvp: sum over coils of the rhs from each coil's Laplace potential (``mvp_solver.py:256-271``)."""
        rhs = np.zeros((self.num_dofs_mvp,))
        self.sol_sp = []
        for i, sol in enumerate(self.coil_sd_solvers):
            self.sol_sp.append(sol.solve(phi_list[i]))
            rhs += self.curl_curl_factory.compute_rhs_electric_potential(self.sol_sp[-1], quad_order=self.quad_order,
                                                                         select_mat=[i])
        return rhs

    def _engine(self, phi_list, apply_gauge=False):
        key = (tuple(float(p) for p in phi_list), bool(apply_gauge))
        if self._newton is None or self._rhs_key != key:
            rhs_mvp = self.compute_source_rhs(phi_list)
            mask = self.make_boundary_mask()
            if apply_gauge:
                # tree-cotree gauge: the spanning tree's edges are fixed too (mvp_solver.py:257-260)
                tree_dofs, _ = self.curl_curl_factory.mesh.get_cotree_dofs()
                mask[tree_dofs] = False
            self._newton = DeviceNewton(self.curl_curl_factory, mask, (), self.quad_order, rhs_extra=rhs_mvp,
                                        stream=getattr(self, "stream", None))
            self._rhs_key = key
        return self._newton

    def solve_lin(self, phi_list, tolerance=1e-4, xcg_0=np.zeros((0,)), maxiter=-1, apply_gauge=False):
        """Linear solve K(0) x = rhs with the reluctances at |B| = 0 (``mvp_solver.py:128-220``):
        Jacobi-PCG on the free DoFs with scipy cg's rules as the reference calls it (relative
        tolerance 1e-5; ``tolerance`` is the absolute tolerance when a start ``xcg_0`` or
        ``maxiter`` is given; ``maxiter`` -1: 10 x free DoFs).  The reference's diagnostic plots
        are not drawn; the CG exit code (0 converged, else the iteration count) is kept in
        ``last_exit_code``.  Returns float64[num_dofs] (numpy), 0 on the constrained DoFs."""
        import ctypes

        from . import _lib

        n = self.num_dofs_mvp
        rhs_d = upload(self.compute_source_rhs(phi_list), np.float64)
        out = self.curl_curl_factory.assemble_device(np.zeros(n), self.quad_order, K=True, J=False, rhs=False)
        pat = out["pattern"]
        mask = self.make_boundary_mask()
        if apply_gauge:
            tree_dofs, _ = self.curl_curl_factory.mesh.get_cotree_dofs()
            mask[tree_dofs] = False
        x = zeros(n)
        has_x0 = len(xcg_0) == n
        if has_x0:
            x[:n] = upload(np.where(mask, np.asarray(xcg_0, dtype=np.float64), 0.0), np.float64)
        atol = float(tolerance) if (has_x0 or maxiter >= 0) else 0.0
        free_d = upload(mask.astype(np.uint8), np.uint8)
        its, res = ctypes.c_int64(), ctypes.c_double()
        rc = _lib.load().snp_pcg(n, _lib.ptr(pat.row_ptr), _lib.ptr(pat.col_idx), _lib.ptr(out["K"]),
                                 _lib.ptr(free_d), _lib.ptr(rhs_d), _lib.ptr(x), 1e-5, atol, int(maxiter),
                                 ctypes.byref(its), ctypes.byref(res), _lib.stream_ptr())
        if rc not in (0, 3):  # 3: maxiter reached, which scipy reports through its exit code
            _lib.check(rc)
        self.last_exit_code = 0 if rc == 0 else int(its.value)
        return to_host(x[:n])

    def solve_nonlin(self, phi_list, tolerance=1e-4, x_0=np.zeros((0,)), maxiter=-1, apply_gauge=False,
                     plot_current_density=False):
        """Newton with the reference's increment test; returns float64[num_dofs] (numpy)."""
        eng = self._engine(phi_list, apply_gauge)
        x0 = None if len(x_0) == 0 else np.asarray(x_0, dtype=np.float64)
        if self.verbose:
            print("***********************")
            print("start Newton iterations")
        x, stats = eng.solve(x0, mode=MODE_REFERENCE, tol=tolerance, cg_maxiter=maxiter,
                             max_newton=self.max_newton_iterations, cg_rtol=1e-5, verbose=self.verbose)
        self.last_stats = stats
        return to_host(x)

    def solve_to_residual(self, phi_list, rtol=1e-8, x_0=None, precision="fp64", max_newton=None, cg_maxiter=50000):
        """Newton until ||F_free(x)|| <= rtol ||F_free(x_0)|| (see ``RedMVPSolver.solve_to_residual``)."""
        eng = self._engine(phi_list)
        x, stats = eng.solve(x_0, mode=MODE_RESIDUAL, tol=rtol, max_newton=max_newton or self.max_newton_iterations,
                             precision={"fp64": 0, "mixed": 1}[precision], cg_maxiter=cg_maxiter)
        self.last_stats = stats
        return to_host(x), stats
