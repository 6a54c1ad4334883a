"""``RedMVPSolver``: the reduced magnetic vector potential solver (``snoopy/red_mvp_solver.py``).

Coils give the source field B_s at the iron quadrature points through Biot-Savart; the
unknown is the reduced potential on first-order edge elements; iron is nonlinear through
its PCHIP reluctance; air is nu0.  ``solve`` keeps the reference's Newton loop and stopping
rules (``red_mvp_solver.py:121-224``) but runs every step on the device.
``solve_to_residual`` drives the same Newton iteration to a relative residual
||F_free(x)|| <= rtol ||F_free(x0)||, F(x) = K(x) x - rhs(x), optionally with float32
Krylov solves.
"""

import numpy as np

from . import _lib
from .curl_curl_assembler import CurlCurlAssembler
from .device import to_host, torch, upload, zeros
from .fem_c import biot_savart_device
from .materials import ConstantReluctance
from .newton import MODE_REFERENCE, MODE_RESIDUAL, DeviceNewton


class RedMVPSolver:
    """Reduced vector potential solver (``red_mvp_solver.py:14-93``).

    :param gmsh_model: a ``TetMesh`` (stands in for the gmsh model: it provides ``.mesh`` and the
        "Dirichlet Boundary" edge set).
    """

    def __init__(self, gmsh_model, coil_list, iron_tags, air_tags, reluctances, max_newton_iterations=25,
                 element_order=1, quad_order=6):
        self.iron_tags = list(iron_tags)
        self.air_tags = list(air_tags)
        self.coil_list = coil_list
        self.domain_tags = self.iron_tags + self.air_tags
        material_properties = list(reluctances) + [ConstantReluctance(0.25 / np.pi * 1e7)] * len(self.air_tags)
        self.max_newton_iterations = max_newton_iterations
        self.element_order = element_order
        if element_order > 3:
            print("Error! Element order {} not implemented! Choosing 1.")
            element_order = 1
        self.quad_order = quad_order
        self.dirichlet_dofs = gmsh_model.get_edge_boundary_dofs(["Dirichlet Boundary"], element_order)
        self.curl_curl_factory = CurlCurlAssembler(gmsh_model.mesh, self.domain_tags, material_properties,
                                                   element_order)
        self.num_dofs_mvp = self.curl_curl_factory.num_dofs
        self.verbose = True
        self._newton = None
        self._source_fields = None

    def get_global_ids(self):
        return self.curl_curl_factory.global_ids

    def make_boundary_mask(self):
        """Boolean mask of the non-Dirichlet DoFs (``red_mvp_solver.py:105-119``)."""
        mask = np.ones((self.num_dofs_mvp,), dtype=bool)
        mask[np.asarray(self.dirichlet_dofs, dtype=np.int64) - 1] = False
        return mask

    def compute_source_fields(self, refresh=False):
        """B_s at the iron quadrature points, summed over coils (``red_mvp_solver.py:149-166``),
        as device tensors; empty entries for the air domains.  Computed once and kept, or again
        with ``refresh`` (then also handed to the Newton engines built so far)."""
        if self._source_fields is None or refresh:
            fields = []
            groups = self._coil_groups()
            for i in range(len(self.iron_tags)):
                pts = self.curl_curl_factory.get_quadrature_points_device(self.quad_order, i)
                B = None
                for segs, current, rad in groups:
                    Bg = biot_savart_device(segs, pts, current, rad)[: pts.numel()]
                    B = Bg if B is None else B + Bg
                if B is None:
                    B = zeros(pts.numel())[: pts.numel()]
                fields.append(B)
            for _ in self.air_tags:
                fields.append(np.zeros((0, 3)))
            self._source_fields = fields
            for eng in (self._newton, getattr(self, "_newton_gauged", None)):
                if eng is not None:
                    for i in range(len(self.iron_tags)):
                        eng.set_source(i, fields[i])
        return self._source_fields

    def _coil_groups(self):
        """The coils' filament segments on the device, coils of equal current and core radius
        concatenated (one Biot-Savart launch per group); re-uploaded only when a coil's
        segments, current or radius change."""
        key = [(c.current, c.rad, c.get_segments()) for c in self.coil_list]
        cached = getattr(self, "_coil_cache", None)
        if cached is not None and len(cached[0]) == len(key) and all(
                a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2]) for a, b in zip(cached[0], key)):
            return cached[1]
        groups = {}
        for current, rad, segs in key:
            groups.setdefault((float(current), float(rad)), []).append(np.asarray(segs, dtype=np.float64))
        dev = [(upload(np.concatenate(v), np.float64), cur, rad) for (cur, rad), v in groups.items()]
        self._coil_cache = (key, dev)
        return dev

    def gauge_mask(self):
        """Free-DoF mask of the tree-cotree gauged formulation: the Dirichlet edges and the
        spanning tree's edges are fixed (``red_mvp_solver.py:169-171``)."""
        mask = self.make_boundary_mask()
        tree_dofs, _ = self.curl_curl_factory.mesh.get_cotree_dofs()
        mask[tree_dofs] = False
        return mask

    def newton_engine(self, apply_gauge=False):
        if apply_gauge:
            if getattr(self, "_newton_gauged", None) is None:
                self._newton_gauged = DeviceNewton(self.curl_curl_factory, self.gauge_mask(),
                                                   self.compute_source_fields(), self.quad_order,
                                                   stream=getattr(self, "stream", None))
            return self._newton_gauged
        if self._newton is None:
            self._newton = DeviceNewton(self.curl_curl_factory, self.make_boundary_mask(), self.compute_source_fields(),
                                        self.quad_order, stream=getattr(self, "stream", None))
        return self._newton

    def _engine_for_solve(self, apply_gauge=False):
        """The Newton engine with the coils' source field evaluated now: every solve evaluates it,
        as the reference's does (``red_mvp_solver.py:149-166``), so coil changes between solves
        are seen."""
        built = (getattr(self, "_newton_gauged", None) if apply_gauge else self._newton) is not None
        eng = self.newton_engine(apply_gauge)
        if built:
            self.compute_source_fields(refresh=True)
        return eng

    def solve(self, tolerance=1e-4, x_0=np.zeros((0,)), maxiter=-1, apply_gauge=False):
        """Newton with the reference's increment test (``red_mvp_solver.py:121-224``).  The coils'
        source field is evaluated on every call, as the reference does (``:149-166``).

        :return: the solution vector, float64[num_dofs] (numpy).
        """
        eng = self._engine_for_solve(apply_gauge)
        x0 = None if len(x_0) == 0 else np.asarray(x_0, dtype=np.float64)
        if self.verbose:
            print("***********************")
            print("start Newton iterations")
        x, stats = eng.solve(x0, mode=MODE_REFERENCE, tol=tolerance, cg_maxiter=maxiter,
                             max_newton=self.max_newton_iterations, cg_rtol=1e-5, verbose=self.verbose)
        self.last_stats = stats
        return to_host(x)

    def solve_to_residual(self, rtol=1e-8, x_0=None, precision="fp64", max_newton=None, cg_maxiter=50000,
                          return_device=False, verbose=False):
        """Newton until ||F_free(x)|| <= rtol ||F_free(x_0)||.

        :param precision: "fp64", or "mixed" for float32 Jacobian values and CG inside the
            float64 Newton residual and update.
        :param cg_maxiter: cap on CG iterations per Newton step (-1: 10 x free DoFs, as scipy).
        :return: (x, stats); x is numpy unless ``return_device``.  The source field is evaluated
        on every call, as in ``solve``.
        """
        eng = self._engine_for_solve()
        prec = {"fp64": 0, "mixed": 1}[precision]
        x, stats = eng.solve(x_0, mode=MODE_RESIDUAL, tol=rtol, cg_maxiter=cg_maxiter,
                             max_newton=max_newton or self.max_newton_iterations, precision=prec, verbose=verbose)
        self.last_stats = stats
        return (x if return_device else to_host(x)), stats

    def evaluate_B(self, x, points, elements=None):
        """Total field B = B_s + curl A_r at points (reduced formulation)."""
        Br = self.curl_curl_factory.compute_B_at_points(x, points, elements)
        pts = upload(points, np.float64)
        Bs = zeros(pts.numel())[: pts.numel()]
        for coil in self.coil_list:
            segs = upload(coil.get_segments(), np.float64)
            Bs += biot_savart_device(segs, pts, coil.current, coil.rad)[: pts.numel()]
        return Br + Bs.cpu().numpy().reshape(-1, 3)
