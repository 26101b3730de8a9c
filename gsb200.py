"""Import shim for the package in ``geometricsolvers.jl_b200/``, whose directory name is not a
Python identifier: ``import gsb200`` loads that package under the name ``gsb200``."""

import importlib.util
import os
import sys

_dir = os.path.join(os.path.dirname(os.path.abspath(__file__)), "geometricsolvers.jl_b200")
_spec = importlib.util.spec_from_file_location(
    __name__, os.path.join(_dir, "__init__.py"), submodule_search_locations=[_dir]
)
_mod = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
