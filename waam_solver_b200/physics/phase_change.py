"""Enthalpy-porosity phase recovery (reference physics/phase_change.py)."""
from .. import kernels

update_phase = kernels.update_phase

__all__ = ["update_phase"]
