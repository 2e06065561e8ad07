"""Import shim: the package lives in the directory ``pyscf-forge_b200/``
(a name Python cannot import directly).  ``import pyscf_forge_b200`` loads
that directory as the package ``pyscf_forge_b200``."""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pyscf-forge_b200")
_spec = importlib.util.spec_from_file_location(__name__, os.path.join(_DIR, "__init__.py"),
                                               submodule_search_locations=[_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
