"""Deterministic wire mass and droplet sizing (host arithmetic).

Restates the process relations of the reference's
physics/deposition_balance.py:12-86: wire mass flux rho*pi*d^2/4*v_feed, a
transfer-mode-dependent droplet period with a sinusoidal size jitter, droplet
mass = flux * interval, and an equivalent-sphere radius in cells clamped to
[1, 10].
"""
from __future__ import annotations

import math

_MODE_PERIOD_SCALE = {"globular": 1.55, "spray": 0.72}


def wire_mass_flux_kg_s(twin) -> float:
    r = 0.5 * twin.wire_diameter_m
    return twin.mat.rho * (math.pi * r * r) * twin.wire_feed_m_s


def infer_transfer_mode(twin) -> str:
    mode = str(getattr(twin, "droplet_transfer_mode", "auto")).strip().lower()
    if mode in ("globular", "spray", "pulsed"):
        return mode
    if getattr(twin, "pulse_frequency_hz", 0.0) > 0.0:
        return "pulsed"
    return "globular" if float(getattr(twin, "welding_current_A", 0.0)) < 180.0 else "spray"


def base_droplet_period_s(twin) -> float:
    f = float(getattr(twin, "droplet_freq", 0.0))
    return 1.0 / max(f, 1e-9) if f > 0.0 else 1.0 / 50.0


def droplet_period_s(twin) -> float:
    base = base_droplet_period_s(twin)
    mode = infer_transfer_mode(twin)
    if mode == "pulsed":
        pulse = max(float(getattr(twin, "pulse_frequency_hz", 0.0)), 1e-9)
        scale = min(4.0, max(0.25, (1.0 / pulse) / base))
    else:
        scale = _MODE_PERIOD_SCALE.get(mode, 1.0)
    nth = float(getattr(twin, "_n_droplets_fired", 0) + 1)
    amp = min(max(float(getattr(twin, "droplet_size_jitter", 0.0)), 0.0), 0.35)
    jitter = 1.0 + amp * math.sin(0.73 * nth + 0.31)
    return max(0.20 * base, base * scale * jitter)


def droplet_mass_for_interval_kg(twin, dt_drop_s: float) -> float:
    return max(0.0, wire_mass_flux_kg_s(twin) * max(dt_drop_s, 0.0))


def droplet_mass_kg(twin) -> float:
    if twin.droplet_freq <= 0:
        return 0.0
    return droplet_mass_for_interval_kg(twin, droplet_period_s(twin))


def droplet_radius_cells_from_mass_kg(twin, m_drop: float) -> float:
    if m_drop <= 0:
        return 3.0
    cells = (m_drop / twin.mat.rho) / (twin.grid.dx ** 3)
    r = (3.0 * cells / (4.0 * math.pi)) ** (1.0 / 3.0)
    return min(10.0, max(1.0, r))


def droplet_radius_cells(twin) -> float:
    return droplet_radius_cells_from_mass_kg(twin, droplet_mass_kg(twin))


def expected_deposited_mass_kg(twin) -> float:
    return wire_mass_flux_kg_s(twin) * twin._step_n * twin.grid.dt
