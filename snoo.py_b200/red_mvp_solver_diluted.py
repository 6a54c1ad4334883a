"""``RedMVPSolverDiluted``: the reduced vector potential solver for magnets of diluted steel
(``snoopy/red_mvp_solver_diluted.py``).

As ``RedMVPSolver``, with one ``materials.Dilution`` per iron domain (air is never diluted,
``red_mvp_solver_diluted.py:73-75``); the device Newton solver evaluates the diluted
reluctance in every assembly of the loop.
"""

import numpy as np

from .curl_curl_assembler_diluted import CurlCurlAssemblerDiluted
from .materials import ConstantReluctance
from .red_mvp_solver import RedMVPSolver


class RedMVPSolverDiluted(RedMVPSolver):
    """Reduced vector potential solver with diluted iron (``red_mvp_solver_diluted.py:14-103``).

    :param dilutions: one ``Dilution`` (or None) per entry of ``iron_tags``.
    """

    def __init__(self, gmsh_model, coil_list, iron_tags, air_tags, reluctances, dilutions, max_newton_iterations=25,
                 element_order=1, quad_order=6):
        if len(dilutions) != len(iron_tags):
            raise ValueError("one dilution (or None) per iron domain is required")
        super().__init__(gmsh_model, coil_list, iron_tags, air_tags, reluctances, max_newton_iterations,
                         element_order, quad_order)
        self.dilutions = list(dilutions) + [None] * len(self.air_tags)
        material_properties = list(reluctances) + [ConstantReluctance(0.25 / np.pi * 1e7)] * len(self.air_tags)
        self.curl_curl_factory = CurlCurlAssemblerDiluted(gmsh_model.mesh, self.domain_tags, material_properties,
                                                          self.dilutions, self.element_order)

    def solve(self, tolerance=1e-4, x_0=np.zeros((0,)), maxiter=-1):
        """Newton with the reference's increment test (``red_mvp_solver_diluted.py:129-229``)."""
        return super().solve(tolerance=tolerance, x_0=x_0, maxiter=maxiter)
