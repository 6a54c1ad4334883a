"""Import name of the package in ``snoo.py_b200/``.

A directory name containing a dot cannot be imported directly, so this module loads
``snoo.py_b200/__init__.py`` as the package ``snoopy_b200`` (its submodules resolve from
that directory): ``import snoopy_b200`` or ``from snoopy_b200 import RedMVPSolver``.
"""

import importlib.util
import os
import sys

_PKG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "snoo.py_b200")
_spec = importlib.util.spec_from_file_location(__name__, os.path.join(_PKG_DIR, "__init__.py"),
                                               submodule_search_locations=[_PKG_DIR])
_module = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _module
_spec.loader.exec_module(_module)
