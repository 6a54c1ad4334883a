"""snoopy_b200: sm_100a implementation of snoo.py's nonlinear magnetostatic path.

Drop-in pieces, with the reference's names and call signatures:

* ``fem_c``                      the native module ``fem_c_mod`` (``fem_c/interface_c.pyx``)
* ``CurlCurlAssembler``          ``snoopy/curl_curl_assembler.py``
* ``GradGradAssembler``          ``snoopy/matrix_assembly.py`` / ``snoopy/grad_grad_assembler.py``
* ``RedMVPSolver``               ``snoopy/red_mvp_solver.py``
* ``MVPSolver``                  ``snoopy/mvp_solver.py``
* ``LaplaceSubdomainSolver``     ``snoopy/laplace_subdomain_solver.py``
* ``CurlCurlAssemblerDiluted``  ``snoopy/curl_curl_assembler_diluted.py``
* ``RedMVPSolverDiluted``        ``snoopy/red_mvp_solver_diluted.py``
* ``Reluctance``, ``ConstantReluctance``, ``Permeability``, ``ConstantPermeability``,
  ``Dilution``                   ``snoopy/materials.py``
* ``RacetrackCoil``              ``snoopy/racetrack_coil.py``
* ``ship.get_vector_field_mag_1`` ``snoopy/SHiP_functions.py`` (template 1, meshed without gmsh)
* ``evaluators``                 ``snoopy/evaluators.py``

gmsh is replaced by ``mesh.TetMesh`` and its generators, and by ``finite_element``'s tables.
All arithmetic runs in ``libsnoopy_b200.so`` (CUDA, sm_100a); there is no CPU fallback.
"""

from . import finite_element, materials, mesh
from .materials import ConstantPermeability, ConstantReluctance, Dilution, Permeability, Reluctance
from .mesh import TetMesh, kuhn_microbench_mesh, window_frame_mesh
from .racetrack_coil import RacetrackCoil

__version__ = "0.1.0"


def __getattr__(name):
    # modules that touch the native library are imported on first use
    if name in ("CurlCurlAssembler",):
        from .curl_curl_assembler import CurlCurlAssembler

        return CurlCurlAssembler
    if name in ("GradGradAssembler",):
        from .grad_grad_assembler import GradGradAssembler

        return GradGradAssembler
    if name == "RedMVPSolver":
        from .red_mvp_solver import RedMVPSolver

        return RedMVPSolver
    if name == "CurlCurlAssemblerDiluted":
        from .curl_curl_assembler_diluted import CurlCurlAssemblerDiluted

        return CurlCurlAssemblerDiluted
    if name == "RedMVPSolverDiluted":
        from .red_mvp_solver_diluted import RedMVPSolverDiluted

        return RedMVPSolverDiluted
    if name == "MVPSolver":
        from .mvp_solver import MVPSolver

        return MVPSolver
    if name == "LaplaceSubdomainSolver":
        from .laplace_subdomain_solver import LaplaceSubdomainSolver

        return LaplaceSubdomainSolver
    if name == "DeviceNewton":
        from .newton import DeviceNewton

        return DeviceNewton
    raise AttributeError(name)
