"""Operator API of the coupled step, module for module as the reference's
``physics/`` package (lbm, thermal, phase_change, free_surface, forces, arc,
deposition, weld_forces), backed by the sm_100a kernels."""
from . import arc, deposition, deposition_balance, electrical_stickout, forces, free_surface  # noqa: F401
from . import lbm, phase_change, thermal, weld_forces  # noqa: F401
