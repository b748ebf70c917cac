"""Weld body forces: arc pressure model, droplet impact (reference
physics/weld_forces.py:22-193).  Recoil and shielding-gas shear are not
built (they are off in every supported configuration) and raise if enabled.
"""
from __future__ import annotations

import math

from .. import kernels
from .._native import WaamError
from .deposition_balance import droplet_mass_kg, infer_transfer_mode

MU0 = 4.0e-7 * math.pi
_IMPACT_MODE_SCALE = {"globular": 0.78, "spray": 1.18, "pulsed": 1.05}


def lin_eagar_peak_pa(current_A: float, sigma_p_m: float) -> float:
    """Lin & Eagar peak arc pressure mu0*I^2/(4*pi^2*sigma^2) [Pa]."""
    s = max(float(sigma_p_m), 1.0e-6)
    i = max(float(current_A), 0.0)
    return MU0 * i * i / (4.0 * math.pi * math.pi * s * s)


def arc_pressure_sigma_m(twin) -> float:
    s = getattr(twin, "pressure_sigma_m", None)
    return float(s) if s is not None and s > 0.0 else float(twin.arc_sigma_m)


def arc_pressure_sigma_cells(twin) -> float:
    return arc_pressure_sigma_m(twin) / twin.grid.dx


def arc_pressure_peak_pa(twin) -> float:
    model = str(getattr(twin, "arc_pressure_model", "constant")).strip().lower()
    if model in ("lin_eagar", "lineagar", "lin-eagar"):
        return lin_eagar_peak_pa(twin.welding_current_A, arc_pressure_sigma_m(twin))
    return float(twin.arc_pressure)


def droplet_impact_velocity_m_s(twin, m_drop_kg=None) -> float:
    """Impact speed: max(feed speed, free fall over one drop length + pinch assist),
    scaled by transfer mode and a bounded mass correction, capped at 5 m/s."""
    drop_len = 3e-3
    if twin.droplet_freq > 0 and twin.wire_feed_m_s > 0:
        drop_len = twin.wire_feed_m_s / twin.droplet_freq
    if m_drop_kg is None:
        m_drop_kg = droplet_mass_kg(twin)
    v_feed = max(twin.wire_feed_m_s, 0.0)
    v_fall = math.sqrt(max(0.0, 2.0 * 9.81 * drop_len))
    pinch = 0.35 * math.sqrt(max(twin.welding_current_A, 0.0) / 200.0) * \
        math.sqrt(1.2e-3 / max(twin.wire_diameter_m, 1e-6))
    scale = _IMPACT_MODE_SCALE.get(infer_transfer_mode(twin), 1.0)
    mass_term = 1.0
    if m_drop_kg > 0:
        mass_term = min(1.25, max(0.8, math.sqrt(droplet_mass_kg(twin) / m_drop_kg)))
    return min(5.0, scale * max(v_feed, v_fall + pinch) * mass_term)


def droplet_velocity_lu(twin, m_drop_kg=None):
    g = twin.grid
    v = droplet_impact_velocity_m_s(twin, m_drop_kg)
    lead = math.radians(float(getattr(twin, "impact_lead_angle_deg", 0.0)))
    dx_, dy_, _ = getattr(twin, "_torch_dir_xyz", (1.0, 0.0, 0.0))
    h = math.hypot(dx_, dy_)
    if h < 1e-9:
        dx_, dy_, h = 1.0, 0.0, 1.0
    dx_, dy_ = dx_ / h, dy_ / h
    v_xy = min(0.65 * v, max(twin.travel_speed_m_s, abs(v) * math.tan(lead)))
    v_z = -math.sqrt(max(v * v - v_xy * v_xy, 0.20 * v * v))
    k = g.dt / g.dx
    return v_xy * dx_ * k, v_xy * dy_ * k, v_z * k


def droplet_impact_pressure_pa(twin, m_drop_kg=None, drop_r_m=None) -> float:
    """Kinetic pressure 0.5*m*v^2 / (pi r^2)."""
    m = droplet_mass_kg(twin) if m_drop_kg is None else m_drop_kg
    if m <= 0:
        return 0.0
    v = droplet_impact_velocity_m_s(twin, m)
    r = drop_r_m if drop_r_m is not None else max(1.5 * twin.grid.dx, 0.5 * twin.wire_diameter_m)
    return 0.5 * m * v * v / max(math.pi * r * r, 1e-12)


def apply_droplet_impact(twin, g, arc_i, arc_j, arc_k, drop_r, drop_mass_kg=None):
    if not twin.enable_deposition_momentum:
        return
    vx, vy, vz = droplet_velocity_lu(twin, drop_mass_kg)
    kernels.feed_wire_momentum_impact(g.f_src, g.rho, g.ux, g.uy, g.uz, g.flags, g.f_l, arc_i,
                                      arc_j, arc_k, drop_r, vx, vy, vz, g.FLAG_GAS, g.nx, g.ny,
                                      g.nz)
    if twin.enable_droplet_impact_pressure:
        kernels.apply_droplet_impact_pressure(
            g.Fz, g.flags, g.phi, g.f_l, arc_i, arc_j, arc_k, drop_r,
            droplet_impact_pressure_pa(twin, drop_mass_kg, drop_r * g.dx), g.dt, g.dx,
            twin.mat.rho, g.FLAG_SOLID, g.FLAG_GAS)


def gas_shear_tau_pa(twin):
    """physics/weld_forces.py:126-131: dynamic shear of the argon jet, capped."""
    rho_gas = 1.6
    v = twin.gas_jet_velocity_m_s
    tau = 0.5 * rho_gas * v * v * twin.gas_shear_coeff
    return min(tau, 5000.0)


def recoil_accommodation(twin):
    return float(getattr(twin, "recoil_accommodation", 0.54))


def apply_recoil(twin, g, arc_i, arc_j, arc_k):
    """physics/weld_forces.py:134-158."""
    if not twin.enable_recoil:
        return
    if twin.use_recoil_clausius_clapeyron:
        kernels.apply_vapor_recoil_clausius_clapeyron(
            g.Fz, g.T, g.phi, g.flags, arc_i, arc_j, arc_k, twin.sigma_cells,
            twin.P_vapor_ref_Pa, twin.T_boiling_K, twin.L_vapor_J_kg, twin.R_spec_vapor_J_kgK,
            recoil_accommodation(twin), g.dt, g.dx, twin.mat.rho, g.FLAG_SOLID, g.FLAG_GAS)
    else:
        kernels.apply_vapor_recoil(g.Fz, g.T, g.phi, g.flags, arc_i, arc_j, arc_k,
                                   twin.sigma_cells, twin.recoil_pressure_pa, twin.mat.T_liquidus,
                                   g.dt, g.dx, twin.mat.rho, g.FLAG_SOLID, g.FLAG_GAS)


def apply_gas_shear(twin, g, arc_i, arc_j, arc_k):
    """physics/weld_forces.py:180-193."""
    if not twin.enable_gas_shear:
        return
    kernels.apply_gas_shear_stress(g.Fx, g.Fy, g.phi, g.flags, arc_i, arc_j, arc_k,
                                   twin.sigma_cells, gas_shear_tau_pa(twin), g.dt, g.dx,
                                   twin.mat.rho, g.FLAG_SOLID, g.FLAG_GAS)


def solve_lorentz(twin, g, arc_i, arc_j, arc_k, apply_force=True, arc_k_dev=None):
    if twin.enable_lorentz:
        from . import lorentz
        lorentz.solve_lorentz(twin, g, arc_i, arc_j, arc_k, apply_force=apply_force,
                              arc_k_dev=arc_k_dev)
