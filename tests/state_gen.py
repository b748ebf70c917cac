"""Seeded synthetic melt-pool states for parity tests (numpy, float32).

A state mimics a WAAM bead-on-plate snapshot: a solid plate below
``nz_solid``, a wavy metal/gas interface (tanh profile of a smooth random
height map) a few cells above it, a Gaussian hot spot that melts part of the
metal, random melt velocities, and D3Q19 populations near equilibrium.
Flags follow the reference's flag rules (kernels.py:2394-2419).
"""
from __future__ import annotations

import numpy as np

EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12)

FLAG_FLUID, FLAG_SOLID, FLAG_GAS, FLAG_IFACE = 0, 1, 2, 4

# ER70S-6-like constants used by every benchmark configuration.
MATERIAL = dict(
    k=30.0, rho=7800.0, cp=680.0, T_solidus=1723.0, T_liquidus=1783.0,
    L_fusion=2.7e5, gamma_0=1.8, dgamma_dT=-4.3e-4, mu=0.0065, beta_T=1.2e-4,
)


def _smooth_noise(rng, nx, ny, passes=3):
    a = rng.standard_normal((nx, ny))
    for _ in range(passes):
        a = 0.25 * (np.roll(a, 1, 0) + np.roll(a, -1, 0) + np.roll(a, 1, 1) + np.roll(a, -1, 1))
    a -= a.min()
    a /= max(a.max(), 1e-12)
    return a


def feq(rho, ux, uy, uz):
    u2 = ux * ux + uy * uy + uz * uz
    out = np.empty((19,) + rho.shape, dtype=np.float64)
    for q in range(19):
        eu = EX[q] * ux + EY[q] * uy + EZ[q] * uz
        out[q] = W[q] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * u2)
    return out


def phase_from_H(H, cp_rho, L_rho, Ts, Tl):
    H_sol = cp_rho * Ts
    H_liq = H_sol + L_rho
    fl = np.clip((H - H_sol) / L_rho, 0.0, 1.0)
    T = np.where(H <= H_sol, H / cp_rho,
                 np.where(H >= H_liq, Tl + (H - H_liq) / cp_rho, Ts + fl * (Tl - Ts)))
    fl = np.where(H <= H_sol, 0.0, np.where(H >= H_liq, 1.0, fl))
    return T, fl


def flags_from(phi, fl, nz_solid):
    nx, ny, nz = phi.shape
    k = np.arange(nz)[None, None, :]
    flags = np.full(phi.shape, FLAG_IFACE, dtype=np.int32)
    flags[phi < 0.05] = FLAG_GAS
    flags[(phi > 0.55) & (fl > 0.1)] = FLAG_FLUID
    flags[(phi > 0.85) & (fl < 0.05)] = FLAG_SOLID
    flags[np.broadcast_to(k < nz_solid, phi.shape)] = FLAG_SOLID
    return flags


def seeded_state(nx, ny, nz, seed=0, nz_solid=None, T_peak=3000.0, hot=None):
    """Return a dict of float32 / int32 numpy fields named like the reference grid."""
    rng = np.random.default_rng(seed)
    m = MATERIAL
    cp_rho = m["rho"] * m["cp"]
    L_rho = m["rho"] * m["L_fusion"]
    if nz_solid is None:
        nz_solid = max(2, nz // 3)
    i = np.arange(nx)[:, None, None].astype(np.float64)
    j = np.arange(ny)[None, :, None].astype(np.float64)
    k = np.arange(nz)[None, None, :].astype(np.float64)

    hm = nz_solid - 0.5 + 4.0 * _smooth_noise(rng, nx, ny)
    phi = 0.5 * (1.0 - np.tanh((k - hm[:, :, None]) / 0.8))
    phi = phi + rng.uniform(-0.01, 0.01, phi.shape)
    phi = np.clip(phi, 0.0, 1.0)
    phi[:, :, :nz_solid] = 1.0

    cx, cy, cz = (hot or (0.45 * nx, 0.5 * ny, nz_solid + 1.0))
    s = max(2.0, 0.22 * min(nx, ny))
    r2 = (i - cx) ** 2 + (j - cy) ** 2 + (k - cz) ** 2
    T = 300.0 + (T_peak - 300.0) * np.exp(-r2 / (2 * s * s)) + rng.normal(0.0, 5.0, phi.shape)
    H_sol = cp_rho * m["T_solidus"]
    H_liq = H_sol + L_rho
    fl_t = np.clip((T - m["T_solidus"]) / (m["T_liquidus"] - m["T_solidus"]), 0, 1)
    H = np.where(T < m["T_solidus"], cp_rho * T,
                 np.where(T > m["T_liquidus"], H_liq + cp_rho * (T - m["T_liquidus"]), H_sol + fl_t * L_rho))
    H = H.astype(np.float32).astype(np.float64)
    T, fl = phase_from_H(H, cp_rho, L_rho, m["T_solidus"], m["T_liquidus"])

    flags = flags_from(phi, fl, nz_solid)
    ux = rng.uniform(-0.03, 0.03, phi.shape)
    uy = rng.uniform(-0.03, 0.03, phi.shape)
    uz = rng.uniform(-0.03, 0.03, phi.shape)
    rho = 1.0 + rng.normal(0.0, 1e-3, phi.shape)
    fa = feq(rho, ux, uy, uz) + rng.normal(0.0, 1e-5, (19,) + phi.shape)
    fb = feq(rho, ux, uy, uz) + rng.normal(0.0, 1e-5, (19,) + phi.shape)
    F = rng.uniform(-2e-3, 2e-3, (3,) + phi.shape)

    st = dict(
        f_a=fa, f_b=fb, rho=rho, ux=ux, uy=uy, uz=uz, T=T, H=H, f_l=fl, phi=phi,
        T_max=T + rng.uniform(0.0, 50.0, phi.shape), T_prev=T + rng.normal(0.0, 2.0, phi.shape),
        dT_dt=rng.normal(0.0, 1e3, phi.shape),
        time_above_800_s=rng.uniform(0, 1e-3, phi.shape),
        time_above_1100_s=rng.uniform(0, 1e-3, phi.shape),
        time_above_solidus_s=rng.uniform(0, 1e-3, phi.shape),
        Fx=F[0], Fy=F[1], Fz=F[2],
        Fx_snap=np.zeros(phi.shape), Fy_snap=np.zeros(phi.shape), Fz_snap=np.zeros(phi.shape),
    )
    out = {k2: np.ascontiguousarray(v, dtype=np.float32) for k2, v in st.items()}
    out["flags"] = flags
    out["nz_solid"] = nz_solid
    return out
