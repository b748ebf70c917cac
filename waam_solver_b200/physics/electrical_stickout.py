"""Droplet entry temperature with optional stick-out preheat and the
open-loop CTWD update (reference physics/electrical_stickout.py:15-59)."""
from __future__ import annotations

import math

from .deposition_balance import wire_mass_flux_kg_s


def stickout_resistance_ohm(twin) -> float:
    r = 0.5 * twin.wire_diameter_m
    return twin.rho_e_ohm_m * max(twin.stickout_m, 1e-6) / max(math.pi * r * r, 1e-12)


def droplet_entry_temperature_K(twin) -> float:
    base = twin.mat.T_liquidus + twin.deposition_superheat_K
    if not twin.enable_ctwd:
        return base
    mdot = wire_mass_flux_kg_s(twin)
    if mdot <= 0:
        return base
    I = twin.welding_current_A
    dT = twin.eta_stick * I * I * stickout_resistance_ohm(twin) / (mdot * twin.mat.cp)
    return min(twin.T_vapor_cap_K - 50.0, base + dT)


def measure_bead_height_m(twin, g) -> float:
    """Max height of deposited SOLID above nz_solid (one device reduction)."""
    from .bead_geometry import measure_bead_height_m as _m
    return _m(twin, g)


def update_ctwd(twin, g) -> None:
    """electrical_stickout.py:53-59: CTWD from the measured bead height."""
    if not twin.enable_ctwd:
        return
    h_meas = measure_bead_height_m(twin, g)
    twin._bead_height_m = h_meas
    twin.ctwd_m = max(twin.ctwd_nominal_m, twin.ctwd_nominal_m + (h_meas - twin.layer_height_m))
