"""Thermal operators (reference physics/thermal.py)."""
from .. import kernels

advect_diffuse_temperature = kernels.advect_diffuse_temperature
apply_boundary_losses = kernels.apply_thermal_boundary_losses
update_T_max = kernels.update_T_max
update_cooling_rate = kernels.update_cooling_rate
prescribe_gaussian_pulse = kernels.prescribe_gaussian_pulse
sync_T_from_H = kernels.sync_T_from_H
init_stefan_liquid_column = kernels.init_stefan_liquid_column
clamp_substrate_enthalpy = kernels.clamp_substrate_enthalpy
clamp_enthalpy_floor_scalar = kernels.clamp_enthalpy_floor_scalar
clamp_enthalpy_ceiling_scalar = kernels.clamp_enthalpy_ceiling_scalar

__all__ = [
    "advect_diffuse_temperature", "apply_boundary_losses", "update_T_max", "update_cooling_rate",
    "prescribe_gaussian_pulse", "sync_T_from_H", "init_stefan_liquid_column",
    "clamp_substrate_enthalpy", "clamp_enthalpy_floor_scalar", "clamp_enthalpy_ceiling_scalar",
]
