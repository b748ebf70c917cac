"""The reference's validation scripts run through this package's CUDA path.

Each test builds the case of one script in ``validation/`` of the reference
with this package's operator API (``waam_solver_b200.kernels``) or its
``WAAMTwin``, computes the script's metric with the script's own formula,
asserts the script's own threshold, and compares the value with the one the
reference's unmodified script returned when it ran on the serial Taichi
stand-in (``tests/golden/kat_reference.json``, written by
``tests/golden/make_golden.py kats``).  The material the scripts load
(materials/placeholders/ER70S-6.yaml) comes from
``tests/golden/kat_materials.json``.

Closeness to the reference value: the CUDA kernels agree with the reference
kernels to ~1e-6 relative per step, so each metric is asserted within a
small tolerance of the reference's value (written per test).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np
import pytest
import torch

from cases import GOLDEN

pytestmark = pytest.mark.gpu


def _kat(name, value):
    """The reference script's value for ``name``; prints this run's value."""
    print("validation %s: %.9g" % (name, value))
    with open(os.path.join(GOLDEN, "kat_reference.json")) as fh:
        return json.load(fh)[name]


def _placeholder_material():
    from waam_solver_b200.materials import from_constants
    with open(os.path.join(GOLDEN, "kat_materials.json")) as fh:
        rec = json.load(fh)["ER70S-6-placeholder"]
    m = from_constants(rec["name"], rec["constants"], status=rec["status"],
                       contact_angle_deg=rec["contact_angle_deg"])
    assert not any(rec["tables"].values())
    return m


def _twin(**kw):
    from waam_solver_b200 import WAAMTwin
    kw.setdefault("material", _placeholder_material())
    return WAAMTwin(device="cuda:0", **kw)


def _np(t):
    return t.detach().cpu().numpy()


def _channel(n_steps):
    """validation/test_lbm_poiseuille.py:20-62 and test_lbm_cavity.py:19-59:
    a force-driven channel (walls at j and k ends), SRT at tau 1, no Darcy
    term, collide -> stream -> swap in the reference's buffer order."""
    from waam_solver_b200 import kernels
    nx, ny, nz = 64, 32, 6
    tau, fx = 1.0, 1e-4
    nu = (tau - 0.5) / 3.0
    tw = _twin(nx=nx, ny=ny, nz=nz, dx=3e-4, C_darcy=0.0, max_tracers=10)
    g = tw.grid
    kernels.init_poiseuille_channel(g.f_a, g.rho, g.ux, g.uy, g.uz, g.f_l, g.phi, g.flags, 1.0,
                                    g.ny, g.nz, fx, nu, g.FLAG_FLUID, g.FLAG_SOLID)
    kernels.init_aux_fields(g.T_max, g.T_prev, g.dT_dt, g.time_above_800_s,
                            g.time_above_1100_s, g.time_above_solidus_s, g.Fx_snap, g.Fy_snap,
                            g.Fz_snap, g.Fx, g.Fy, g.Fz, tw.T_amb, g.porosity_active,
                            g.tracer_head, g.max_tracers)
    kernels.stream(g.f_a, g.f_b, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
    for _ in range(n_steps):
        kernels.set_uniform_Fx(g.Fx, g.Fy, g.Fz, fx, g.flags, g.FLAG_FLUID)
        kernels.collide_srt(g.f_src, g.f_dst, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l,
                            g.flags, tau, 1.0 / tau, 1.0, 0.0, g.FLAG_SOLID, g.FLAG_GAS, g.nx,
                            g.ny, g.nz)
        kernels.stream(g.f_dst, g.f_src, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        g.swap_buffers()
    torch.cuda.synchronize()
    return tw, fx, nu


def test_poiseuille_profile():
    """validation/test_lbm_poiseuille.py:16-87: profile L2 (%) of the mid-plane
    velocity against the parabola, threshold 8 %."""
    tw, fx, nu = _channel(100)
    g = tw.grid
    nx, ny, nz = g.nx, g.ny, g.nz
    h = ny - 2
    y = np.arange(1, ny - 1, dtype=np.float64) - 1.0
    u_anal = (fx / (2.0 * nu)) * y * (h - 1.0 - y)
    ux, flags = _np(g.ux), _np(g.flags)
    u = np.array([float(ux[nx // 2, j, nz // 2]) for j in range(1, ny - 1)
                  if flags[nx // 2, j, nz // 2] == g.FLAG_FLUID])
    l2 = float(np.sqrt(np.mean((u / (u.max() + 1e-12) - u_anal / (u_anal.max() + 1e-12)) ** 2))
               * 100.0)
    assert l2 < 8.0
    ref = _kat("test_lbm_poiseuille", l2)
    assert abs(l2 - ref) <= 1e-4 * ref, (l2, ref)


def test_lid_cavity_flow():
    """validation/test_lbm_cavity.py:18-71: mean |ux| over the fluid cells after
    150 forced steps, at least 1e-6."""
    tw, _, _ = _channel(150)
    g = tw.grid
    ux, flags = _np(g.ux), _np(g.flags)
    fluid = flags == g.FLAG_FLUID
    u_mean = float(np.abs(ux[fluid]).mean())
    assert u_mean >= 1e-6
    ref = _kat("test_lbm_cavity", u_mean)
    assert abs(u_mean - ref) <= 1e-5 * ref, (u_mean, ref)


def test_thermal_diffusion_gaussian_pulse():
    """validation/test_thermal_diffusion.py:23-78: a Gaussian pulse in an
    all-fluid 48^3 box diffused for 400 steps (advect_diffuse_temperature +
    T = H / rho cp), L2 error (%) of the interior against the analytical
    solution, threshold 1 %."""
    from waam_solver_b200 import kernels
    n, dx, T_bg, sigma0, A = 48, 3e-4, 300.0, 1.2e-3, 500.0
    tw = _twin(nx=n, ny=n, nz=n, dx=dx, use_srt=True, C_darcy=0.0, max_tracers=100)
    tw.reset(T_ambient=T_bg, test_fluid_domain=True)
    g = tw.grid
    c = (n // 2) * dx
    kernels.prescribe_gaussian_pulse(g.T, g.H, g.f_l, g.flags, T_bg, A, sigma0, c, c, c, dx,
                                     tw.cp_rho, g.FLAG_GAS)
    for _ in range(400):
        kernels.advect_diffuse_temperature(g.H, g.T, g.ux, g.uy, g.uz, g.flags, tw.alpha_lu, 1.0,
                                           g.FLAG_SOLID, g.FLAG_GAS, tw.cp_rho, g.nx, g.ny, g.nz)
        kernels.sync_T_from_H(g.H, g.T, tw.cp_rho)
    T = _np(g.T)
    t = 400 * g.dt
    x = (np.arange(n) - n // 2) * dx
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    R = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    s2 = sigma0 ** 2 + 2.0 * tw.mat.alpha * t
    T_anal = T_bg + A * (sigma0 ** 2 / s2) ** 1.5 * np.exp(-R ** 2 / (2.0 * s2))
    inner = np.s_[4:-4, 4:-4, 4:-4]
    l2 = float(np.sqrt(np.sum((T[inner] - T_anal[inner]) ** 2) /
                       np.sum((T_anal[inner] - T_bg) ** 2)) * 100.0)
    assert l2 < 1.0
    ref = _kat("test_thermal_diffusion", l2)
    assert abs(l2 - ref) <= 1e-3 * ref, (l2, ref)


def _stefan_lambda(ste):
    """validation/test_stefan_solidification.py:18-36 (bisection)."""
    def res(lam):
        return math.sqrt(math.pi) * lam * math.exp(lam * lam) * math.erf(lam) - ste
    lo, hi = 1e-6, 5.0
    while res(hi) < 0:
        hi *= 2.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if res(mid) > 0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def _interface_height(fl, T, flags, nz_solid, dx, Ts, Tl, FLUID):
    """validation/test_stefan_solidification.py:39-79."""
    mi, mj = fl.shape[0] // 2, fl.shape[1] // 2
    cf, cT, cg = fl[mi, mj, :], T[mi, mj, :], flags[mi, mj, :]
    Tm = 0.5 * (Ts + Tl)
    for k in range(nz_solid, fl.shape[2] - 1):
        if cg[k] != FLUID:
            continue
        lo, hi = float(cT[k]), float(cT[k + 1])
        if lo < Tm <= hi:
            return (k - nz_solid + (Tm - lo) / max(hi - lo, 1e-9)) * dx
        if lo >= Tm > hi:
            return (k - nz_solid + 1.0 - (lo - Tm) / max(lo - hi, 1e-9)) * dx
    for k in range(nz_solid, fl.shape[2] - 1):
        if cg[k] != FLUID:
            continue
        lo, hi = float(cf[k]), float(cf[k + 1])
        if lo < 0.5 <= hi:
            return (k - nz_solid + (0.5 - lo) / max(hi - lo, 1e-12)) * dx
    if cf[nz_solid] >= 0.5:
        return 0.0
    return (fl.shape[2] - nz_solid) * dx


def test_stefan_solidification_front():
    """validation/test_stefan_solidification.py:82-163: a liquid column above a
    300 K substrate; the front of the mid isotherm against the Stefan
    sqrt(t) law, slope error (%) with threshold 8 %, front monotonic."""
    from waam_solver_b200 import kernels
    tw = _twin(nx=4, ny=4, nz=80, dx=1.0e-4, C_darcy=0.0, max_tracers=10)
    g = tw.grid
    m = tw.mat
    nz_solid, T_amb = 8, 300.0
    T_init = m.T_liquidus + 50.0
    kernels.init_stefan_liquid_column(g.T, g.H, g.f_l, g.phi, g.flags, nz_solid, T_amb, T_init,
                                      tw.cp_rho, tw.L_rho, m.T_solidus, m.T_liquidus,
                                      g.FLAG_FLUID, g.FLAG_SOLID)
    lam = _stefan_lambda(m.cp * (T_init - T_amb) / m.L_fusion)
    slope_anal = 2.0 * lam * math.sqrt(m.alpha)
    sq, hist = [], []
    for step in range(1, 801):
        kernels.clamp_substrate_enthalpy(g.H, g.T, g.f_l, g.flags, nz_solid, T_amb, tw.cp_rho,
                                         g.FLAG_SOLID)
        kernels.advect_diffuse_temperature(g.H, g.T, g.ux, g.uy, g.uz, g.flags, tw.alpha_lu, 1.0,
                                           g.FLAG_SOLID, g.FLAG_GAS, tw.cp_rho, g.nx, g.ny, g.nz)
        kernels.update_phase(g.H, g.T, g.f_l, tw.cp_rho, tw.L_rho, m.T_solidus, m.T_liquidus)
        if step in (200, 300, 400, 500, 600, 700):
            sq.append(math.sqrt(step * g.dt))
            hist.append(_interface_height(_np(g.f_l), _np(g.T), _np(g.flags), nz_solid, g.dx,
                                          m.T_solidus, m.T_liquidus, g.FLAG_FLUID))
    assert all(a <= b for a, b in zip(hist, hist[1:]))
    slope = float(np.polyfit(sq, hist, 1)[0])
    err = abs(slope - slope_anal) / slope_anal * 100.0
    assert err < 8.0
    ref = _kat("test_stefan_solidification", err)
    assert abs(err - ref) <= 1e-3 * ref, (err, ref)


def test_vof_mass_conservation():
    """validation/test_vof_mass.py:14-41: phi sum drift (%) under uniform
    advection (ux = 0.02 in the fluid) over 80 steps, threshold 0.5 %."""
    from waam_solver_b200 import kernels
    tw = _twin(nx=32, ny=32, nz=16, dx=3e-4, C_darcy=0.0, max_tracers=10, enable_vof=True)
    tw.reset(test_fluid_domain=True)
    g = tw.grid
    phi0 = float(_np(g.phi).sum())
    g.ux.copy_(torch.where(g.flags == g.FLAG_FLUID, torch.full_like(g.ux, 0.02), g.ux))
    for _ in range(80):
        kernels.advect_phi(g.phi_tmp, g.phi, g.ux, g.uy, g.uz, g.flags, g.FLAG_SOLID, g.FLAG_GAS,
                           g.nx, g.ny, g.nz)
        g.phi.copy_(g.phi_tmp)
        kernels.reinitialize_phi(g.phi, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.FLAG_FLUID)
    phi1 = float(_np(g.phi).sum())
    drift = abs(phi1 - phi0) / max(phi0, 1e-9) * 100.0
    assert drift < 0.5
    assert abs(drift - _kat("test_vof_mass", drift)) <= 1e-6


def test_goldak_energy_and_asymmetry():
    """validation/test_goldak_energy.py:16-69: one Goldak injection deposits
    eta Q dt within 1 %, ff + fr normalised to 2, more heat behind the torch."""
    from waam_solver_b200.physics.arc import Goldak3D, normalize_goldak_fractions
    ff, fr = normalize_goldak_fractions(0.6, 0.4)
    assert abs(ff + fr - 2.0) < 1e-9
    ff2, fr2 = normalize_goldak_fractions(0.6, 1.4)
    assert abs(ff2 - 0.6) < 1e-12 and abs(fr2 - 1.4) < 1e-12
    tw = _twin(nx=32, ny=24, nz=20, dx=3e-4, heat_source="goldak", arc_efficiency=0.8,
               arc_power_W=3600.0, enable_vof=False, max_tracers=10)
    tw.reset(test_fluid_domain=True)
    tw.arc_source = Goldak3D(ff=0.6, fr=1.4, a_front=4.0, a_rear=8.0, b=4.0, c=3.0)
    g = tw.grid
    H0 = float(_np(g.H).sum()) * g.dx ** 3
    ai, aj = (g.nx - 1) * 0.5, (g.ny - 1) * 0.5
    tw.arc_source.inject(tw, g, ai, aj, float(tw.nz_solid + 2))
    H = _np(g.H)
    dH = float(H.sum()) * g.dx ** 3 - H0
    expected = tw.eta * tw.Q_w * g.dt
    err = abs(dH - expected) / expected
    assert err <= 0.01
    # the float32 sums of two 15k-cell fields (as the script takes them): the
    # value is reproduced to their rounding
    assert abs(err - _kat("test_goldak_energy", err)) <= 2e-4, err
    i0 = int(round(ai))
    assert float(H[:i0].sum()) > float(H[i0 + 1:].sum())


def test_rosenthal_far_field_tail():
    """validation/test_rosenthal_farfield.py:18-68: the twin's full coupled step
    (reference defaults: SRT, Gaussian arc, 50 Hz droplet schedule without
    wire) for 1200 steps at 5 mm/s; the substrate temperature 2, 3 and 4 mm
    behind the torch against the Rosenthal thick-plate tail
    (validation/rosenthal.py:7-61), mean error (%) -- the script's gate is
    55 %, which the reference itself misses here; the test pins the value."""
    travel, Q, eta, T0 = 0.005, 2800.0, 0.72, 300.0
    tw = _twin(nx=80, ny=40, nz=32, dx=2.5e-4, arc_power_W=Q, arc_efficiency=eta,
               travel_speed_m_s=travel, enable_heat_loss=False, C_darcy=1.6e5,
               max_tracers=100)
    tw.reset(T_ambient=T0)
    g = tw.grid
    cy = (g.ny // 2) * g.dx
    x0 = 0.012
    for s in range(1200):
        tw.step(x0 + s * travel * g.dt, cy, is_welding=True)
    torch.cuda.synchronize()
    x_t = x0 + 1199 * travel * g.dt
    T, flags = _np(g.T), _np(g.flags)
    m = tw.mat
    k_sub = max(1, tw.nz_solid - 1)
    errs = []
    for back in (2.0, 3.0, 4.0):
        i = int((x_t - back * 1e-3) / g.dx)
        j = g.ny // 2
        if i < 0 or flags[i, j, k_sub] == g.FLAG_GAS:
            continue
        Ts = float(T[i, j, k_sub])
        R = back * 1e-3
        Ta = T0 + eta * Q / (2.0 * math.pi * m.k * R)   # on the trailing centreline R + xi = 0
        if Ta > T0 + 5.0 and Ts > T0 + 1.0:
            errs.append(abs(Ts - Ta) / (Ta - T0) * 100.0)
    assert errs
    err = float(np.mean(errs))
    # The unmodified script misses its own 55 % gate on this case (96.63 % on
    # the stand-in): the tail runs hotter than the thick-plate solution.  The
    # drop-in reproduces the reference's value, not the gate.
    ref = _kat("test_rosenthal_farfield", err)
    assert ref > 55.0
    assert abs(err - ref) <= 1e-3 * ref, (err, ref)
