"""B200-native (sm_100a) coupled melt-pool step of the waam_twin WAAM digital twin.

Drop-in for the reference's operator API (``physics``), its step driver
(``coupled_step``) and ``WAAMTwin.step`` / ``run_path``.  All field work runs in
hand-written CUDA kernels of ``_lib/libwaam_b200.so`` through a C ABI
(``include/waam_b200.h``); there is no CPU path.
"""
from . import _native  # noqa: F401
from .coupled_step import coupled_step, coupled_step_fused, coupled_step_operators  # noqa: F401
from .grid import WAAMGrid  # noqa: F401
from .materials import MaterialProps, er70s6_constants, from_constants, load_material  # noqa: F401
from .twin import WAAMTwin  # noqa: F401

__version__ = "0.1.0"
__all__ = ["WAAMTwin", "WAAMGrid", "MaterialProps", "coupled_step", "load_material",
           "er70s6_constants", "from_constants"]
