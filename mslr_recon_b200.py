"""Import alias for the ``mslr-recon_b200/`` package directory.

The package directory name contains a hyphen, which the import statement
cannot spell; ``import mslr_recon_b200`` loads it from that directory and
registers it under this name (submodules resolve normally).
"""
import importlib.util
import os
import sys

_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mslr-recon_b200")
_spec = importlib.util.spec_from_file_location(
    __name__, os.path.join(_DIR, "__init__.py"), submodule_search_locations=[_DIR])
_mod = importlib.util.module_from_spec(_spec)
sys.modules[__name__] = _mod
_spec.loader.exec_module(_mod)
