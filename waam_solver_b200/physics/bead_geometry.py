"""Bead geometry telemetry (reference physics/bead_geometry.py:13-47).

The toe column and the bead height come from the device: a telemetry record
(kernels.telemetry_pool) or a one-value reduction (kernels.bead_height_k),
never a full-volume copy.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .. import kernels


def toe_angle_from_column(phi_col, flags_col, k0, contact_angle_deg, dx, FLAG_GAS=2):
    """bead_geometry.py:21-40 over the column phi[nx//3, ny//2, k0:k0+len]
    (float32 arithmetic on the phi values, as the numpy original)."""
    phi_col = np.asarray(phi_col, dtype=np.float32)
    best_angle = float(contact_angle_deg)
    best_phi = np.float32(0.0)
    for q in range(len(phi_col)):
        k = k0 + q
        if int(flags_col[q]) == FLAG_GAS and phi_col[q] > best_phi:
            best_phi = phi_col[q]
        if phi_col[q] > 0.45 and k > k0:
            dz = dx
            dphi = phi_col[q] - phi_col[q - 1]
            if abs(dphi) > 1e-4:
                slope = abs(dphi) * dx / max(dz, 1e-9)
                angle = math.degrees(math.atan(1.0 / max(slope, 1e-6)))
                best_angle = min(89.0, max(10.0, angle))
    return best_angle


def estimate_toe_angle_deg(twin, g) -> float:
    i, j = g.nx // 3, g.ny // 2
    k0 = max(0, twin.nz_solid - 1)
    k1 = min(g.nz - 1, twin.nz_solid + 8)
    if k1 <= k0:
        return float(twin.contact_angle_deg)
    phi = g.phi[i, j, k0:k1].cpu().numpy()
    flags = g.flags[i, j, k0:k1].cpu().numpy()
    return toe_angle_from_column(phi, flags, k0, twin.contact_angle_deg, g.dx, g.FLAG_GAS)


def bead_height_m_from_k(k_max, nz_solid, dx) -> float:
    """electrical_stickout.py:39-50: (max deposited solid k - nz_solid + 1) * dx."""
    return 0.0 if k_max < 0 else float((k_max - nz_solid + 1) * dx)


def measure_bead_height_m(twin, g) -> float:
    buf = getattr(g, "_bead_k_buf", None)
    if buf is None:
        buf = g._bead_k_buf = torch.zeros((), dtype=torch.int32, device=g.device)
    kernels.bead_height_k(g.flags, twin.nz_solid, buf)
    return bead_height_m_from_k(int(buf.item()), twin.nz_solid, g.dx)


def bead_reinforcement_height_mm(twin, g) -> float:
    return measure_bead_height_m(twin, g) * 1000.0
