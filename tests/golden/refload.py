"""Import the waam_twin reference on top of the serial Taichi stand-in.

TEST INFRASTRUCTURE ONLY: used by ``make_golden.py`` in a container that has
the reference checkout; nothing on the GPU box or in the product imports it.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_ROOT = os.environ.get("WAAM_REFERENCE_ROOT", "")


def load():
    """Return the imported reference package ``waam_twin`` (shim-backed).

    ``WAAM_REFERENCE_ROOT`` names the reference checkout (the folder that
    holds ``kernels.py`` and ``twin.py``)."""
    if not REFERENCE_ROOT or not os.path.isfile(os.path.join(REFERENCE_ROOT, "kernels.py")):
        raise RuntimeError("set WAAM_REFERENCE_ROOT to the waam_twin reference checkout "
                           "(the folder with kernels.py); got %r" % REFERENCE_ROOT)
    shim = os.path.join(HERE, "taichi_shim")
    if shim not in sys.path:
        sys.path.insert(0, shim)
    import taichi  # noqa: F401  (the shim)

    if "waam_twin" not in sys.modules:
        pkg = types.ModuleType("waam_twin")
        pkg.__path__ = [REFERENCE_ROOT]
        pkg.__file__ = os.path.join(REFERENCE_ROOT, "__init__.py")
        sys.modules["waam_twin"] = pkg
        twin_mod = importlib.import_module("waam_twin.twin")
        pkg.WAAMTwin = twin_mod.WAAMTwin
    return sys.modules["waam_twin"]
