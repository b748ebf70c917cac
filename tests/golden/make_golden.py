"""Generate the golden fixtures in this folder from the waam_twin reference.

TEST INFRASTRUCTURE ONLY.  Run in a container that has the reference
checkout, named by ``WAAM_REFERENCE_ROOT``::

    WAAM_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py [what ...]

``what``: ``kernels``, ``kernel=<name>``, ``steps``, ``table_steps``,
``telemetry``, ``run_path``, ``kat_materials``, ``kats`` or ``kat=<script>`` (one validation script, merged
into the existing ``kat_reference.json``).

Every fixture is produced by the reference's own, unmodified Taichi kernels
(kernels.py, cumulant_kernel.py) or its own ``WAAMTwin.step`` /
``coupled_step`` (twin.py:533-567, solvers/coupled_step.py:73-464), executed
serially by the numpy stand-in in ``taichi_shim/`` with the deterministic
semantics documented there.  Inputs are seeded synthetic states from
``tests/state_gen.py``.  Outputs are small ``.npz`` files:

* ``k_<case>.npz``: one kernel call -- ``in_<field>``/``out_<field>`` arrays,
  ``args`` (JSON of the scalar arguments) and ``fields`` (JSON list).
* ``step_<case>.npz``: a short ``WAAMTwin.step`` run -- the full state before
  each step and after the last one (``s<n>_<field>``), the torch positions and
  the twin's derived scalars.
* ``kat_reference.json``: known-answer values of the reference's validation
  scripts executed on the stand-in (Poiseuille, VOF mass, Goldak energy,
  Stefan, thermal diffusion, lid cavity, Rosenthal far field).
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import refload  # noqa: E402
from state_gen import MATERIAL, seeded_state  # noqa: E402

wt = refload.load()
from waam_twin import kernels as K  # noqa: E402
from waam_twin.cumulant_kernel import collide_mrt  # noqa: E402
from waam_twin.materials import MaterialProps  # noqa: E402
from waam_twin.physics import arc as arc_mod  # noqa: E402

FIELDS3 = ["rho", "ux", "uy", "uz", "T", "H", "f_l", "phi", "T_max", "T_prev", "dT_dt",
           "time_above_800_s", "time_above_1100_s", "time_above_solidus_s",
           "Fx", "Fy", "Fz", "Fx_snap", "Fy_snap", "Fz_snap", "flags"]


def material(theta_deg=30.0):
    m = MATERIAL
    return MaterialProps(
        name="ER70S-6-constants", k=m["k"], rho=m["rho"], cp=m["cp"],
        alpha=m["k"] / (m["rho"] * m["cp"]), T_solidus=m["T_solidus"],
        T_liquidus=m["T_liquidus"], L_fusion=m["L_fusion"], gamma_0=m["gamma_0"],
        dgamma_dT=m["dgamma_dT"], T_ref_gamma=m["T_liquidus"], mu=m["mu"],
        beta_T=m["beta_T"], contact_angle_deg=theta_deg, status="synthetic",
    )


def table_material():
    """The reference's validated ER70S-6 file: cp, k, mu and dgamma/dT tables."""
    from waam_twin.materials import load_material
    return load_material(os.path.join(refload.REFERENCE_ROOT, "materials", "validated",
                                      "ER70S-6.v1.yaml"))


def table_args(tw):
    """The twin's GPU tables (float32 knots as uploaded) and reference values."""
    t = tw.gpu_tables
    out = {}
    for name in ("cp", "k", "mu", "dgamma"):
        out[name + "_T"] = [float(v) for v in getattr(t, name + "_T").to_numpy()]
        out[name + "_V"] = [float(v) for v in getattr(t, name + "_V").to_numpy()]
        out["n_" + name] = int(getattr(t, "n_" + name)[None])
    out.update(cp_fallback=t.cp_fallback, k_fallback=t.k_fallback, mu_fallback=t.mu_fallback,
               dgamma_fallback=t.dgamma_fallback, rho=tw.mat.rho,
               force_scale=tw.force_scale / tw.grid.dx, cp_rho_ref=tw.cp_rho,
               alpha_lu_ref=tw.alpha_lu, dgamma_lu_ref=tw.dgamma_dT_lu, tau_ref=tw.grid.tau,
               marangoni_scale=tw.marangoni_scale, H_sol_t=tw.H_sol, H_liq_t=tw.H_liq,
               T_solidus_t=tw.mat.T_solidus, T_liquidus_t=tw.mat.T_liquidus,
               L_rho_t=tw.L_rho, T_cap=tw.T_vapor_cap_K, C_darcy=tw.C_darcy)
    return out


def refresh(tw, g):
    t = tw.gpu_tables
    K.refresh_thermal_properties(
        g.T, g.cp_rho_field, g.alpha_lu_field, g.dgamma_lu_field, g.tau_field,
        t.cp_T, t.cp_V, t.k_T, t.k_V, t.mu_T, t.mu_V, t.dgamma_T, t.dgamma_V,
        t.n_cp, t.n_k, t.n_mu, t.n_dgamma, tw.mat.rho, g.dt, g.dx,
        t.cp_fallback, t.k_fallback, t.mu_fallback, t.dgamma_fallback,
        tw.force_scale / g.dx, tw.cp_rho, tw.alpha_lu, tw.dgamma_dT_lu, g.tau,
        tw.marangoni_scale, 1, g.flags, g.FLAG_SOLID, g.FLAG_GAS)


def make_twin(nx, ny, nz, dx=2e-4, **kw):
    if kw.pop("tables", False):
        kw.setdefault("use_srt", False)
        kw.setdefault("enable_vof", True)
        kw.setdefault("max_tracers", 64)
        kw.setdefault("droplet_freq_hz", 0.0)
        return wt.WAAMTwin(material=table_material(), nx=nx, ny=ny, nz=nz, dx=dx, **kw)
    kw.setdefault("use_srt", False)
    kw.setdefault("enable_vof", True)
    kw.setdefault("max_tracers", 64)
    kw.setdefault("droplet_freq_hz", 0.0)
    return wt.WAAMTwin(material=material(kw.pop("theta", 30.0)), nx=nx, ny=ny, nz=nz, dx=dx, **kw)


def load_state(g, st):
    for name in FIELDS3:
        getattr(g, name).from_numpy(st[name])
    g.f_a.from_numpy(st["f_a"])
    g.f_b.from_numpy(st["f_b"])
    if hasattr(g, "phi_tmp"):
        g.phi_tmp.from_numpy(np.zeros_like(st["phi"]))


def dump_state(g, prefix, out):
    for name in FIELDS3:
        out[prefix + name] = getattr(g, name).to_numpy()
    out[prefix + "f_a"] = g.f_a.to_numpy()
    out[prefix + "f_b"] = g.f_b.to_numpy()


def save(name, payload):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **payload)
    print("wrote", name, os.path.getsize(path), "bytes")


# ---------------------------------------------------------------------------
# kernel cases
# ---------------------------------------------------------------------------
NX, NY, NZ = 13, 11, 12


ONLY = set()   # kernel case names given as ``kernel=<name>`` on the command line


def kernel_case(name, call, fields, seed=0, twin_kw=None, state_kw=None, extra_in=None):
    if ONLY and name not in ONLY:
        return
    tw = make_twin(NX, NY, NZ, **(twin_kw or {}))
    g = tw.grid
    st = seeded_state(NX, NY, NZ, seed=seed, **(state_kw or {}))
    tw.nz_solid = st["nz_solid"]
    load_state(g, st)
    if extra_in:
        extra_in(tw, g)
    payload = {}
    for f in fields:
        payload["in_" + f] = getattr(g, f).to_numpy()
    args = call(tw, g)
    for f in fields:
        payload["out_" + f] = getattr(g, f).to_numpy()
    payload["args"] = np.array(json.dumps(args))
    payload["fields"] = np.array(json.dumps(fields))
    save("k_%s.npz" % name, payload)


def scal(tw):
    g = tw.grid
    m = tw.mat
    return dict(cp_rho=float(np.float32(tw.cp_rho)), L_rho=float(np.float32(tw.L_rho)),
                T_solidus=m.T_solidus, T_liquidus=m.T_liquidus, T_cap=tw.T_vapor_cap_K,
                alpha_lu=tw.alpha_lu, dt=g.dt, dx=g.dx, nz_solid=tw.nz_solid,
                nx=g.nx, ny=g.ny, nz=g.nz)


def c_inject_gauss(tw, g):
    a = dict(arc_i=5.3, arc_j=4.6, arc_k=float(tw.nz_solid + 1), Q_w=3000.0, sigma=3.2,
             dt=g.dt, dx3=g.dx ** 3, eta=0.75, pen=tw.arc_penetration_m / g.dx, enable=1)
    K.inject_arc_heat(g.H, g.flags, g.phi, g.f_l, g.arc_norm_buf, a["arc_i"], a["arc_j"], a["arc_k"],
                      a["Q_w"], a["sigma"], a["dt"], a["dx3"], a["eta"], a["pen"], a["enable"],
                      g.FLAG_SOLID, g.FLAG_GAS)
    a["norm"] = float(g.arc_norm_buf[None])
    return a


def c_inject_goldak(tw, g):
    a = dict(arc_i=6.1, arc_j=5.2, arc_k=float(tw.nz_solid + 1), Q_w=4000.0, dt=g.dt,
             dx3=g.dx ** 3, eta=0.78, sign=-1.0, ff=0.6, fr=1.4, a_front=3.0, a_rear=6.5,
             b=2.5, c=2.0, pen=tw.arc_penetration_m / g.dx, enable=1)
    K.inject_goldak_heat(g.H, g.flags, g.phi, g.f_l, g.arc_norm_buf, a["arc_i"], a["arc_j"], a["arc_k"],
                         a["Q_w"], a["dt"], a["dx3"], a["eta"], a["sign"], a["ff"], a["fr"],
                         a["a_front"], a["a_rear"], a["b"], a["c"], a["pen"], a["enable"],
                         g.FLAG_SOLID, g.FLAG_GAS)
    a["norm"] = float(g.arc_norm_buf[None])
    return a


def c_ceiling(tw, g):
    a = scal(tw)
    a["T_cap"] = 2500.0
    K.clamp_enthalpy_ceiling_scalar(g.H, g.flags, tw.cp_rho, a["T_solidus"], a["T_liquidus"],
                                    a["T_cap"], tw.L_rho, g.FLAG_GAS)
    return a


def c_thermal(tw, g):
    a = scal(tw)
    K.advect_diffuse_temperature(g.H, g.T, g.ux, g.uy, g.uz, g.flags, tw.alpha_lu, 1.0,
                                 g.FLAG_SOLID, g.FLAG_GAS, tw.cp_rho, g.nx, g.ny, g.nz)
    return a


def c_phase(tw, g):
    a = scal(tw)
    K.update_phase(g.H, g.T, g.f_l, tw.cp_rho, tw.L_rho, a["T_solidus"], a["T_liquidus"])
    return a


def c_tmax_cool(tw, g):
    a = scal(tw)
    K.update_T_max(g.T, g.T_max, g.flags, g.FLAG_GAS)
    K.update_cooling_rate(g.T, g.T_prev, g.dT_dt, g.flags, g.dt, g.FLAG_GAS)
    return a


def c_vof_chain(wetting):
    def run(tw, g):
        a = scal(tw)
        a["theta"] = tw.theta_rad
        a["wetting"] = int(wetting)
        K.advect_phi(g.phi_tmp, g.phi, g.ux, g.uy, g.uz, g.flags, g.FLAG_SOLID, g.FLAG_GAS,
                     g.nx, g.ny, g.nz)
        g.phi.copy_from(g.phi_tmp)
        K.reinitialize_phi(g.phi, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.FLAG_FLUID)
        if wetting:
            K.apply_contact_angle_phi_bc(g.phi, g.flags, tw.theta_rad, g.FLAG_SOLID, g.FLAG_GAS,
                                         g.nx, g.ny, g.nz)
        K.update_flags_from_phi(g.phi, g.f_l, g.flags, tw.nz_solid, g.FLAG_FLUID, g.FLAG_SOLID,
                                g.FLAG_GAS, g.FLAG_IFACE)
        K.sync_phi_liquid_fraction(g.phi, g.f_l, g.flags, g.FLAG_GAS, g.FLAG_SOLID)
        return a
    return run


def c_contact(tw, g):
    a = scal(tw)
    a["theta"] = tw.theta_rad
    K.apply_contact_angle_phi_bc(g.phi, g.flags, tw.theta_rad, g.FLAG_SOLID, g.FLAG_GAS,
                                 g.nx, g.ny, g.nz)
    return a


def c_forces(wetting, welding=True, hydro=True):
    def run(tw, g):
        a = scal(tw)
        a.update(gamma_lu=tw.gamma_lu, dgamma_lu=tw.dgamma_dT_lu, theta=tw.theta_rad,
                 wetting=int(wetting), arc_i=6.4, arc_j=5.1, arc_k=float(tw.nz_solid + 1),
                 p_sigma=3.0, pressure=500.0, rho_phys=tw.mat.rho, g_lu=tw.g_lu,
                 beta=tw.beta_T, F_cap=0.05, welding=int(welding), hydro=int(hydro))
        K.clear_forces(g.Fx, g.Fy, g.Fz)
        K.compute_csf_tension(g.phi, g.flags, g.Fx, g.Fy, g.Fz, tw.gamma_lu, g.FLAG_SOLID,
                              g.FLAG_GAS, g.nx, g.ny, g.nz, int(wetting), float(tw.theta_rad))
        K.compute_marangoni_force(g.T, g.phi, g.f_l, g.Fx, g.Fy, g.Fz, g.flags, tw.dgamma_dT_lu,
                                  g.dx, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        if welding:
            K.apply_arc_pressure(g.Fz, g.flags, g.phi, a["arc_i"], a["arc_j"], a["arc_k"],
                                 a["p_sigma"], a["pressure"], g.dt, g.dx, tw.mat.rho,
                                 g.FLAG_SOLID, g.FLAG_GAS)
        if hydro:
            K.add_hydrostatic_gravity(g.Fz, g.f_l, g.flags, 1.0, tw.g_lu, g.FLAG_SOLID, g.FLAG_GAS)
        K.add_buoyancy(g.T, g.Fz, g.f_l, g.flags, tw.g_lu, tw.beta_T, tw.mat.T_liquidus, 1.0,
                       g.FLAG_SOLID, g.FLAG_GAS)
        K.clamp_body_force_magnitude(g.Fx, g.Fy, g.Fz, g.flags, 0.05, g.FLAG_SOLID, g.FLAG_GAS)
        return a
    return run


def c_csf_only(wetting):
    def run(tw, g):
        a = scal(tw)
        a.update(gamma_lu=tw.gamma_lu * 50.0, theta=tw.theta_rad, wetting=int(wetting))
        K.compute_csf_tension(g.phi, g.flags, g.Fx, g.Fy, g.Fz, a["gamma_lu"], g.FLAG_SOLID,
                              g.FLAG_GAS, g.nx, g.ny, g.nz, int(wetting), float(tw.theta_rad))
        return a
    return run


def c_collide(kind):
    def run(tw, g):
        a = scal(tw)
        a.update(omega=tw.omega, omega_b=tw.omega_bulk, C_darcy=tw.C_darcy, tau=g.tau, u_cap=0.08)
        if kind == "mrt":
            collide_mrt(g.f_a, g.f_b, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l, g.flags,
                        g.ex, g.ey, g.ez, g.w, g.opp, tw.omega, tw.omega_bulk, tw.C_darcy,
                        g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        else:
            K.collide_srt(g.f_a, g.f_b, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l, g.flags,
                          g.tau, tw.omega, 1.0, tw.C_darcy, g.FLAG_SOLID, g.FLAG_GAS,
                          g.nx, g.ny, g.nz)
        K.clamp_velocity_mach(g.ux, g.uy, g.uz, g.flags, 0.08, g.FLAG_SOLID, g.FLAG_GAS)
        return a
    return run


def c_stream(tw, g):
    a = scal(tw)
    K.stream(g.f_b, g.f_a, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
    return a


def c_tail(tw, g):
    a = scal(tw)
    a.update(arc_i=9.5, arc_j=5.0, arc_k=float(tw.nz_solid + 1), dir=[1.0, 0.0, 0.0],
             lookback=2.0, T_freeze=tw.mat.T_liquidus + 35.0)
    K.update_time_above_T(g.T, g.flags, g.time_above_800_s, g.time_above_1100_s,
                          g.time_above_solidus_s, g.dt, 800.0 + 273.15, 1100.0 + 273.15,
                          tw.mat.T_solidus, g.FLAG_GAS)
    K.snapshot_forces(g.Fx, g.Fy, g.Fz, g.Fx_snap, g.Fy_snap, g.Fz_snap)
    K.remelt_hot_solid_scalar(g.T, g.H, g.f_l, g.phi, g.flags, tw.cp_rho, tw.mat.T_solidus,
                              tw.mat.T_liquidus, tw.L_rho, g.FLAG_SOLID, g.FLAG_FLUID)
    K.solidify_trailing_pool_scalar(g.T, g.H, g.f_l, g.phi, g.flags, g.ux, g.uy, g.uz, tw.cp_rho,
                                    a["arc_i"], a["arc_j"], a["arc_k"], 1.0, 0.0, 0.0,
                                    a["lookback"], a["T_freeze"], tw.mat.T_solidus,
                                    g.FLAG_SOLID, g.FLAG_FLUID, g.FLAG_GAS)
    K.solidify_cooled_metal(g.T, g.f_l, g.phi, g.flags, g.ux, g.uy, g.uz, tw.mat.T_solidus, 1,
                            g.FLAG_SOLID, g.FLAG_FLUID, g.FLAG_GAS)
    return a


def c_heat_loss(tw, g):
    a = scal(tw)
    a.update(T_amb=300.0, h_conv=25.0, eps_rad=0.3, conv=1, rad=1, sigma_sb=5.670374419e-8)
    K.apply_thermal_boundary_losses(g.H, g.T, g.flags, 300.0, 25.0, 0.3, 1, 1, tw.cp_rho, g.dt,
                                    g.dx, a["sigma_sb"], g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
    K.clamp_enthalpy_floor_scalar(g.H, tw.cp_rho, g.flags, 300.0, g.FLAG_GAS)
    return a


def c_surface_height(tw, g):
    out = {}
    for (i0, j0) in [(3, 4), (7, 2), (12, 10), (0, 0)]:
        K.surface_height_at(g.phi, g.flags, g.surface_k_buf, i0, j0, tw.nz_solid, g.FLAG_GAS, g.nz)
        out["%d_%d" % (i0, j0)] = float(g.surface_k_buf[None])
    a = scal(tw)
    a["heights"] = out
    return a


def c_deposit(tw, g):
    a = scal(tw)
    a.update(arc_i=6.2, arc_j=5.4, arc_k=float(tw.nz_solid + 1), foot_r=3.5, drop_r=2.2,
             T_drop=tw.mat.T_liquidus + 500.0, cell_vol=g.dx ** 3)
    a["target_vol"] = 30.0 * g.dx ** 3
    placed = []
    r_try = a["foot_r"]
    placed_real = 0.0
    for _ in range(3):
        g.deposit_vol_buf[None] = placed_real
        g.deposit_real_buf[None] = placed_real
        K.feed_wire_surface(g.f_a, g.flags, g.f_l, g.phi, g.H, g.T, g.rho, a["arc_i"], a["arc_j"],
                            a["arc_k"], r_try, a["drop_r"], a["target_vol"], a["T_drop"], tw.cp_rho,
                            tw.L_rho, 1.0, g.deposit_vol_buf, g.deposit_real_buf, g.dx ** 3,
                            g.FLAG_GAS, g.FLAG_FLUID, g.FLAG_SOLID, g.nx, g.ny, g.nz)
        placed_real = float(g.deposit_real_buf[None])
        placed.append([r_try, placed_real, float(g.deposit_vol_buf[None])])
        r_try = min(r_try + 1.5, 16.0)
    a["placed"] = placed
    a.update(vel=[0.004, -0.002, -0.03])
    K.feed_wire_momentum_impact(g.f_a, g.rho, g.ux, g.uy, g.uz, g.flags, g.f_l, a["arc_i"],
                                a["arc_j"], a["arc_k"], a["drop_r"], 0.004, -0.002, -0.03,
                                g.FLAG_GAS, g.nx, g.ny, g.nz)
    a.update(impact_pa=2.0e4)
    K.apply_droplet_impact_pressure(g.Fz, g.flags, g.phi, g.f_l, a["arc_i"], a["arc_j"], a["arc_k"],
                                    a["drop_r"], a["impact_pa"], g.dt, g.dx, tw.mat.rho,
                                    g.FLAG_SOLID, g.FLAG_GAS)
    return a


def c_feed_wire(tw, g):
    """feed_wire (kernels.py:177-242) twice: the second call starts from the
    budget the first one left, so the cut falls inside its box."""
    a = scal(tw)
    a.update(arc_i=6.3, arc_j=5.2, arc_k=float(tw.nz_solid), drop_rs=[0.6, 1.7],
             arc_ks=[float(g.nz - 2), float(tw.nz_solid)], cell_vol=g.dx ** 3,
             T_drop=tw.mat.T_liquidus + 500.0, rho0=1.0)
    a["target_vol"] = 40.0 * g.dx ** 3
    acc = []
    for arc_k, drop_r in zip(a["arc_ks"], a["drop_rs"]):
        K.feed_wire(g.f_a, g.flags, g.f_l, g.phi, g.H, g.T, g.rho, a["arc_i"], a["arc_j"], arc_k,
                    drop_r, a["target_vol"], a["T_drop"], tw.cp_rho, tw.L_rho, a["rho0"],
                    g.deposit_vol_buf, a["cell_vol"], g.FLAG_GAS, g.FLAG_FLUID, g.nx, g.ny, g.nz)
        acc.append(float(g.deposit_vol_buf[None]))
    a["vol_acc_after"] = acc
    return a


def c_feed_wire_momentum(tw, g):
    a = scal(tw)
    a.update(arc_i=5.6, arc_j=4.4, arc_k=float(tw.nz_solid - 2), drop_r=3.3, vz_lu=0.021)
    K.feed_wire_momentum(g.ux, g.uy, g.uz, g.flags, g.f_l, a["arc_i"], a["arc_j"], a["arc_k"],
                         a["drop_r"], a["vz_lu"], g.FLAG_GAS, g.nx, g.ny, g.nz)
    return a


LORENTZ_FIELDS = ["sigma_elec", "elec_source", "phi_elec", "phi_elec_tmp", "Jx", "Jy", "Jz",
                  "Bx", "By", "Bz", "elec_rad_bins", "Fx", "Fy", "Fz"]


def weld_forces_setup(tw, g):
    """Some interface cells above the boiling point (the Clausius-Clapeyron
    recoil acts only there) and non-zero starting forces."""
    T = g.T.to_numpy()
    rng = np.random.default_rng(41)
    hot = rng.uniform(0.0, 1.0, T.shape) < 0.35
    T = np.where(hot, rng.uniform(3000.0, 3600.0, T.shape), T).astype(np.float32)
    g.T.from_numpy(T)
    for name in ("Fx", "Fy", "Fz"):
        fld = getattr(g, name)
        fld.from_numpy(rng.normal(0.0, 1e-3, fld.shape).astype(np.float32))


def c_weld_forces(tw, g):
    """kernels.py:995-1141: shielding-gas shear, vapour recoil (T-ratio form) and
    vapour recoil (Clausius-Clapeyron form), added to F one after the other."""
    a = scal(tw)
    a.update(arc_i=6.3, arc_j=5.4, arc_k=float(tw.nz_solid + 1), sigma=2.5, tau_pa=115.2,
             recoil_pa=5000.0, T_ref=tw.mat.T_liquidus, P_ref=101325.0, T_boil=3100.0,
             L_vap=6.0e6, R_spec=450.0, C_acc=0.54, rho_ref=tw.mat.rho)
    K.apply_gas_shear_stress(g.Fx, g.Fy, g.phi, g.flags, a["arc_i"], a["arc_j"], a["arc_k"],
                             a["sigma"], a["tau_pa"], g.dt, g.dx, a["rho_ref"], g.FLAG_SOLID,
                             g.FLAG_GAS)
    K.apply_vapor_recoil(g.Fz, g.T, g.phi, g.flags, a["arc_i"], a["arc_j"], a["arc_k"],
                         a["sigma"], a["recoil_pa"], a["T_ref"], g.dt, g.dx, a["rho_ref"],
                         g.FLAG_SOLID, g.FLAG_GAS)
    K.apply_vapor_recoil_clausius_clapeyron(g.Fz, g.T, g.phi, g.flags, a["arc_i"], a["arc_j"],
                                            a["arc_k"], a["sigma"], a["P_ref"], a["T_boil"],
                                            a["L_vap"], a["R_spec"], a["C_acc"], g.dt, g.dx,
                                            a["rho_ref"], g.FLAG_SOLID, g.FLAG_GAS)
    return a


def lorentz_setup(tw, g):
    g.ensure_lorentz_fields()
    rng = np.random.default_rng(31)
    g.phi_elec.from_numpy(rng.uniform(0.0, 0.05, (g.nx, g.ny, g.nz)).astype(np.float32))
    g.phi_elec_tmp.from_numpy(np.zeros((g.nx, g.ny, g.nz), np.float32))


def c_lorentz(tw, g):
    """physics/weld_forces.py:196-281 with a fixed budget of 30 Jacobi sweeps."""
    from waam_twin.physics.weld_forces import MU0
    a = scal(tw)
    a.update(arc_i=6.3, arc_j=5.4, arc_k=float(tw.nz_solid + 1), sigma_cells=2.5, current=200.0,
             s_liq=1.0e6, s_sol=1.0e5, omega=0.85, iters=30, n_bins=int(g.n_elec_bins),
             mu0=MU0, rho_ref=tw.mat.rho)
    a["bin_dr"] = max(float(max(g.nx, g.ny)) / (2.0 * g.n_elec_bins), 0.5)
    K.elec_build_sigma(g.sigma_elec, g.f_l, g.flags, a["s_liq"], a["s_sol"], g.FLAG_GAS)
    K.elec_clear_source(g.elec_source)
    K.elec_inject_arc_source(g.elec_source, a["arc_i"], a["arc_j"], a["arc_k"], a["sigma_cells"],
                             a["current"], g.dx, g.nz)
    K.elec_normalize_source(g.elec_source, a["current"], g.dx)
    res = []
    for it in range(a["iters"]):
        K.elec_jacobi_step(g.phi_elec, g.phi_elec_tmp, g.sigma_elec, g.elec_source, g.flags,
                           g.dx, a["omega"], g.FLAG_GAS, g.FLAG_SOLID, tw.nz_solid, g.nx, g.ny,
                           g.nz)
        K.elec_l1_diff(g.phi_elec_tmp, g.phi_elec, g.elec_res_buf, g.elec_norm_buf)
        g.phi_elec.copy_from(g.phi_elec_tmp)
        if it % 10 == 9:
            res.append([float(g.elec_res_buf[None]), float(g.elec_norm_buf[None])])
    a["l1"] = res
    K.elec_compute_J(g.Jx, g.Jy, g.Jz, g.phi_elec, g.sigma_elec, g.flags, g.dx, g.FLAG_GAS,
                     g.nx, g.ny, g.nz)
    K.elec_bin_axial_current(g.Jz, g.elec_rad_bins, a["arc_i"], a["arc_j"], g.dx, a["bin_dr"],
                             a["n_bins"], g.nz)
    K.elec_prefix_bins(g.elec_rad_bins, a["n_bins"], g.nz)
    K.elec_B_axisymmetric(g.Bx, g.By, g.Bz, g.elec_rad_bins, a["arc_i"], a["arc_j"], g.dx,
                          a["bin_dr"], MU0, a["n_bins"], g.nz)
    K.apply_lorentz_JxB(g.Fx, g.Fy, g.Fz, g.Jx, g.Jy, g.Jz, g.Bx, g.By, g.Bz, g.f_l, g.flags,
                        g.dt, g.dx, tw.mat.rho, g.FLAG_GAS)
    return a


def tracer_setup(tw, g):
    rng = np.random.default_rng(41)
    m = g.max_tracers
    ext = np.array([g.nx, g.ny, g.nz], np.float64) * g.dx
    pos = rng.uniform(-0.05, 1.05, (m, 3)) * ext          # some outside the grid
    hot = np.array([0.45 * g.nx, 0.5 * g.ny, tw.nz_solid + 1.0]) * g.dx
    pos[: m // 2] = hot + rng.uniform(-3.0, 3.0, (m // 2, 3)) * g.dx   # near the melt
    act = rng.choice([0, 1, 1, 1, 2], size=m).astype(np.int32)
    g.porosity_pos.from_numpy(pos.astype(np.float32))
    g.porosity_active.from_numpy(act)


def c_tracers(tw, g):
    a = scal(tw)
    a["max_tracers"] = int(g.max_tracers)
    K.advect_tracers(g.porosity_pos, g.porosity_active, g.ux, g.uy, g.uz, g.f_l, g.flags, g.dx,
                     g.dt, g.max_tracers, g.FLAG_SOLID, g.FLAG_GAS)
    return a


PROP_FIELDS = ["cp_rho_field", "alpha_lu_field", "dgamma_lu_field", "tau_field"]


def c_refresh(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    refresh(tw, g)
    return a


def props_setup(tw, g):
    refresh(tw, g)        # realistic per-cell properties as the kernel inputs


def c_thermal_var(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    K.advect_diffuse_temperature_variable(g.H, g.T, g.ux, g.uy, g.uz, g.flags, g.alpha_lu_field,
                                          g.cp_rho_field, 1.0, g.FLAG_SOLID, g.FLAG_GAS,
                                          g.nx, g.ny, g.nz)
    return a


def c_phase_var(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    K.clamp_enthalpy_floor(g.H, g.cp_rho_field, g.flags, 300.0, g.FLAG_GAS)
    K.update_phase_variable_cp(g.H, g.T, g.f_l, g.cp_rho_field, tw.L_rho, tw.mat.T_solidus,
                               tw.mat.T_liquidus, tw.H_sol, tw.H_liq)
    K.clamp_enthalpy_ceiling_variable_cp(g.H, g.flags, g.cp_rho_field, tw.H_liq,
                                         tw.mat.T_liquidus, 2500.0, g.FLAG_GAS)
    K.update_phase_variable_cp(g.H, g.T, g.f_l, g.cp_rho_field, tw.L_rho, tw.mat.T_solidus,
                               tw.mat.T_liquidus, tw.H_sol, tw.H_liq)
    a["T_floor"] = 300.0
    a["T_cap_case"] = 2500.0
    return a


def c_forces_var(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    K.clear_forces(g.Fx, g.Fy, g.Fz)
    K.compute_marangoni_force_variable(g.T, g.phi, g.f_l, g.Fx, g.Fy, g.Fz, g.flags,
                                       g.dgamma_lu_field, g.FLAG_SOLID, g.FLAG_GAS,
                                       g.nx, g.ny, g.nz)
    return a


def c_srt_var(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    K.collide_srt_variable_tau(g.f_a, g.f_b, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l,
                               g.flags, g.tau_field, tw.C_darcy, g.FLAG_SOLID, g.FLAG_GAS,
                               g.nx, g.ny, g.nz)
    return a


def c_tail_var(tw, g):
    a = scal(tw)
    a.update(table_args(tw))
    a.update(arc_i=9.5, arc_j=5.0, arc_k=float(tw.nz_solid + 1), lookback=2.0,
             T_freeze=tw.mat.T_liquidus + 35.0)
    K.remelt_hot_solid(g.T, g.H, g.f_l, g.phi, g.flags, g.cp_rho_field, tw.mat.T_solidus,
                       tw.mat.T_liquidus, tw.L_rho, g.FLAG_SOLID, g.FLAG_FLUID)
    K.solidify_trailing_pool(g.T, g.H, g.f_l, g.phi, g.flags, g.ux, g.uy, g.uz, g.cp_rho_field,
                             a["arc_i"], a["arc_j"], a["arc_k"], 1.0, 0.0, 0.0, a["lookback"],
                             a["T_freeze"], tw.mat.T_solidus, g.FLAG_SOLID, g.FLAG_FLUID,
                             g.FLAG_GAS)
    return a


SHIFT_FIELDS = ["T", "H", "f_l", "phi", "flags", "T_max", "T_prev", "dT_dt", "time_above_800_s",
                "time_above_1100_s", "time_above_solidus_s", "rho", "ux", "uy", "uz", "Fx", "Fy",
                "Fz"] + PROP_FIELDS + ["f_a", "f_b"]


def shift_setup(tw, g):
    """Every shifted field distinct and non-zero (kernels.py:2620-2723 moves 22
    scalar fields and both population buffers)."""
    refresh(tw, g)
    rng = np.random.default_rng(77)
    for name in ("T_max", "T_prev", "dT_dt", "time_above_800_s", "time_above_1100_s",
                 "time_above_solidus_s", "Fx", "Fy", "Fz"):
        fld = getattr(g, name)
        fld.from_numpy(rng.uniform(-1.0, 2.0, fld.shape).astype(np.float32))
    fb = g.f_b.to_numpy()
    g.f_b.from_numpy((fb * rng.uniform(0.9, 1.1, fb.shape)).astype(np.float32))


def c_shift(tw, g):
    a = scal(tw)
    a.update(n_shift=3, T_amb=300.0, rho0=1.0)
    K.shift_simulation_window_x(
        3, g.f_a, g.f_b, g.T, g.H, g.f_l, g.phi, g.flags, g.T_max, g.T_prev, g.dT_dt,
        g.time_above_800_s, g.time_above_1100_s, g.time_above_solidus_s, g.rho, g.ux, g.uy, g.uz,
        g.Fx, g.Fy, g.Fz, g.cp_rho_field, g.alpha_lu_field, g.dgamma_lu_field, g.tau_field,
        300.0, tw.cp_rho, 1.0, tw.nz_solid, g.FLAG_SOLID, g.FLAG_GAS, g.FLAG_FLUID,
        g.nx, g.ny, g.nz)
    return a


def c_derived(tw, g):
    a = scal(tw)
    g.ensure_export_buffers()
    K.compute_curvature_field(g.phi, g.flags, g.kappa_field, g.FLAG_GAS, g.nx, g.ny, g.nz)
    K.compute_vorticity_magnitude(g.ux, g.uy, g.uz, g.flags, g.vorticity_mag, g.dx, g.dt,
                                  g.FLAG_GAS, g.nx, g.ny, g.nz)
    return a


def derived_setup(tw, g):
    g.ensure_export_buffers()
    g.kappa_field.from_numpy(np.full((g.nx, g.ny, g.nz), 7.0, np.float32))
    g.vorticity_mag.from_numpy(np.full((g.nx, g.ny, g.nz), 7.0, np.float32))


def c_reset(tw, g):
    a = scal(tw)
    tw.reset()
    a["nz_solid"] = tw.nz_solid
    return a


def kernel_cases():
    base = ["H", "T", "f_l", "phi", "flags"]
    kernel_case("inject_gauss", c_inject_gauss, ["H"])
    kernel_case("inject_goldak", c_inject_goldak, ["H"], seed=1)
    kernel_case("ceiling", c_ceiling, ["H"])
    kernel_case("thermal", c_thermal, ["H"])
    kernel_case("thermal_s2", c_thermal, ["H"], seed=2)
    kernel_case("phase", c_phase, ["H", "T", "f_l"])
    kernel_case("tmax_cool", c_tmax_cool, ["T_max", "T_prev", "dT_dt"])
    kernel_case("vof", c_vof_chain(False), ["phi", "flags", "f_l", "phi_tmp"])
    kernel_case("vof_wet", c_vof_chain(True), ["phi", "flags", "f_l", "phi_tmp"], seed=3)
    kernel_case("contact", c_contact, ["phi"], seed=4)
    kernel_case("contact_s5", c_contact, ["phi"], seed=5, twin_kw=dict(theta=60.0))
    kernel_case("forces", c_forces(False), ["Fx", "Fy", "Fz"])
    kernel_case("forces_wet", c_forces(True), ["Fx", "Fy", "Fz"], seed=6)
    kernel_case("csf", c_csf_only(False), ["Fx", "Fy", "Fz"], seed=7)
    kernel_case("csf_wet", c_csf_only(True), ["Fx", "Fy", "Fz"], seed=8)
    kernel_case("collide_mrt", c_collide("mrt"), ["f_b", "rho", "ux", "uy", "uz"])
    kernel_case("collide_srt", c_collide("srt"), ["f_b", "rho", "ux", "uy", "uz"], seed=9)
    kernel_case("stream", c_stream, ["f_a"])
    kernel_case("tail", c_tail, base + ["time_above_800_s", "time_above_1100_s",
                                        "time_above_solidus_s", "Fx_snap", "Fy_snap", "Fz_snap",
                                        "ux", "uy", "uz"], seed=10)
    kernel_case("heat_loss", c_heat_loss, ["H"], seed=11)
    kernel_case("surface_height", c_surface_height, ["phi"], seed=12)
    kernel_case("deposit", c_deposit, base + ["rho", "f_a", "ux", "uy", "uz", "Fz"], seed=13)
    kernel_case("feed_wire", c_feed_wire, base + ["rho", "f_a"], seed=27)
    kernel_case("feed_wire_momentum", c_feed_wire_momentum, ["ux", "uy", "uz"], seed=28)
    kernel_case("lorentz", c_lorentz, LORENTZ_FIELDS, seed=14, extra_in=lorentz_setup)
    kernel_case("weld_forces", c_weld_forces, ["T", "Fx", "Fy", "Fz"], seed=26,
                extra_in=weld_forces_setup)
    kernel_case("tracers", c_tracers, ["porosity_pos", "porosity_active"], seed=15,
                extra_in=tracer_setup)
    tb = dict(tables=True)
    kernel_case("refresh", c_refresh, PROP_FIELDS, seed=16, twin_kw=tb)
    kernel_case("thermal_var", c_thermal_var, ["H"] + PROP_FIELDS, seed=17, twin_kw=tb,
                extra_in=props_setup)
    kernel_case("phase_var", c_phase_var, ["H", "T", "f_l"] + PROP_FIELDS, seed=18,
                twin_kw=tb, extra_in=props_setup)
    kernel_case("forces_var", c_forces_var, ["Fx", "Fy", "Fz"] + PROP_FIELDS, seed=19,
                twin_kw=tb, extra_in=props_setup)
    kernel_case("srt_var", c_srt_var, ["f_b", "rho", "ux", "uy", "uz"] + PROP_FIELDS, seed=20,
                twin_kw=tb, extra_in=props_setup)
    kernel_case("tail_var", c_tail_var, base + ["ux", "uy", "uz"] + PROP_FIELDS, seed=21,
                twin_kw=tb, extra_in=props_setup)
    kernel_case("shift", c_shift, SHIFT_FIELDS, seed=24, twin_kw=tb, extra_in=shift_setup)
    kernel_case("derived", c_derived, ["kappa_field", "vorticity_mag"], seed=25,
                extra_in=derived_setup)
    kernel_case("reset", c_reset, base + ["rho", "ux", "uy", "uz", "f_a", "f_b", "T_max",
                                          "T_prev", "dT_dt", "time_above_800_s", "Fx", "Fx_snap"])


# ---------------------------------------------------------------------------
# full-step cases
# ---------------------------------------------------------------------------
def twin_scalars(tw):
    g = tw.grid
    return dict(
        nx=g.nx, ny=g.ny, nz=g.nz, dx=g.dx, dt=g.dt, tau=g.tau, alpha_lu=tw.alpha_lu,
        omega=tw.omega, omega_bulk=tw.omega_bulk, cp_rho=tw.cp_rho, L_rho=tw.L_rho,
        sigma_cells=tw.sigma_cells, g_lu=tw.g_lu, gamma_lu=tw.gamma_lu,
        dgamma_dT_lu=tw.dgamma_dT_lu, theta_rad=tw.theta_rad, nz_solid=tw.nz_solid,
        Q_w=tw.Q_w, eta=tw.eta, C_darcy=tw.C_darcy,
    )


def material_record(tw):
    """Constants and tables of the twin's material after the surfactant model."""
    m = tw.mat
    consts = {k: float(getattr(m, k)) for k in (
        "k", "rho", "cp", "alpha", "T_solidus", "T_liquidus", "L_fusion", "gamma_0",
        "dgamma_dT", "T_ref_gamma", "mu", "beta_T")}
    tables = {k: [list(map(float, r)) for r in getattr(m.tables, k)]
              for k in ("cp", "k", "mu", "dgamma_dT")}
    return dict(constants=consts, tables=tables, contact_angle_deg=m.contact_angle_deg)


def step_case(name, nx, ny, nz, n_steps, positions, twin_kw, setup=None, seeded=None,
              after_load=None):
    tw = make_twin(nx, ny, nz, **dict(twin_kw))
    if setup:
        setup(tw)
    tw.reset()
    g = tw.grid
    if seeded is not None:
        st = seeded_state(nx, ny, nz, seed=seeded, nz_solid=tw.nz_solid)
        load_state(g, st)
    if after_load:
        after_load(tw, g)
    props = bool(twin_kw.get("tables"))
    payload = {}
    log = []
    for s in range(n_steps):
        dump_state(g, "s%d_" % s, payload)
        if props:
            for f in PROP_FIELDS:
                payload["s%d_%s" % (s, f)] = getattr(g, f).to_numpy()
        payload["s%d_read_is_a" % s] = np.array(g.f_src is g.f_a)
        x, y = positions[s]
        tw.step(x, y, True)
        log.append(dict(arc=list(tw._last_arc_ijk), droplets=tw._n_droplets_fired,
                        deposited=tw._deposited_volume_m3, dir=list(tw._torch_dir_xyz),
                        last_drop=tw._last_droplet_time))
    dump_state(g, "s%d_" % n_steps, payload)
    if props:
        for f in PROP_FIELDS:
            payload["s%d_%s" % (n_steps, f)] = getattr(g, f).to_numpy()
    payload["s%d_read_is_a" % n_steps] = np.array(g.f_src is g.f_a)
    payload["positions"] = np.array(positions, dtype=np.float64)
    sc = twin_scalars(tw)
    if props:
        sc.update(material=material_record(tw), H_sol=tw.H_sol, H_liq=tw.H_liq)
    payload["scalars"] = np.array(json.dumps(sc))
    payload["twin_kw"] = np.array(json.dumps(twin_kw))
    payload["log"] = np.array(json.dumps(log))
    save("step_%s.npz" % name, payload)


def step_cases():
    # Config-1-like: Gaussian2D arc, MRT, VOF, no wire feed, plate 4 cells.
    nx, ny, nz = 16, 12, 12
    dx = 2.5e-4
    cy = (ny // 2) * dx
    pos = [(0.0012 + s * 0.008 * dx * 0.1, cy) for s in range(4)]
    kw1 = dict(dx=dx, heat_source="gaussian2d", arc_power_W=3000.0, arc_efficiency=0.75,
               arc_sigma_mm=0.75, travel_speed_m_s=0.008)
    step_case("c1_plate", nx, ny, nz, 3, pos, kw1,
              setup=lambda tw: setattr(tw, "plate_thickness_mm", 1.0))
    # Same config from a seeded molten state (exercises collide/stream/forces).
    step_case("c1_seeded", nx, ny, nz, 3, pos, kw1,
              setup=lambda tw: setattr(tw, "plate_thickness_mm", 1.0), seeded=21)

    # Config-2-like: Goldak, 100 Hz droplets (first fires at step 0), wetting 30 deg,
    # CSF, hydrostatic gravity, buoyancy, Marangoni, MRT.
    dx2 = 2e-4
    cy2 = (ny // 2) * dx2
    pos2 = [(0.0014 + s * 0.008 * dx2 * 0.1, cy2) for s in range(4)]
    kw2 = dict(dx=dx2, heat_source="goldak", arc_power_W=4000.0, arc_efficiency=0.78,
               arc_sigma_mm=0.6, droplet_freq_hz=100.0, enable_wetting=True,
               enable_csf_tension=True, enable_hydrostatic_gravity=True,
               travel_speed_m_s=0.008)

    def setup2(tw):
        tw.plate_thickness_mm = 0.8
        tw.wire_feed_m_s = 0.1
        tw.droplet_transfer_mode = "pulsed"
        tw.pulse_frequency_hz = 100.0
        tw.droplet_size_jitter = 0.0
        tw.arc_source = arc_mod.Goldak3D(ff=0.6, fr=1.4, a_front=3.0 / (dx2 * 1e3) / 4,
                                         a_rear=9.0 / (dx2 * 1e3) / 4, b=3.0 / (dx2 * 1e3) / 4,
                                         c=3.0 / (dx2 * 1e3) / 4)

    def run2(name, seeded):
        tw_setup = setup2

        def s(tw):
            tw_setup(tw)
        tw = make_twin(nx, ny, nz, **kw2)
        s(tw)
        tw.reset()
        tw._last_droplet_time = -1.0  # first step fires a droplet
        g = tw.grid
        if seeded is not None:
            st = seeded_state(nx, ny, nz, seed=seeded, nz_solid=tw.nz_solid)
            load_state(g, st)
        payload = {}
        log = []
        for step in range(3):
            dump_state(g, "s%d_" % step, payload)
            payload["s%d_read_is_a" % step] = np.array(g.f_src is g.f_a)
            payload["s%d_last_drop" % step] = np.array(tw._last_droplet_time)
            payload["s%d_n_drops" % step] = np.array(tw._n_droplets_fired)
            x, y = pos2[step]
            tw.step(x, y, True)
            log.append(dict(arc=list(tw._last_arc_ijk), droplets=tw._n_droplets_fired,
                            deposited=tw._deposited_volume_m3, dir=list(tw._torch_dir_xyz),
                            last_drop=tw._last_droplet_time))
        dump_state(g, "s3_", payload)
        payload["s3_read_is_a"] = np.array(g.f_src is g.f_a)
        payload["positions"] = np.array(pos2, dtype=np.float64)
        sc = twin_scalars(tw)
        sc.update(goldak=dict(ff=tw.arc_source.ff, fr=tw.arc_source.fr,
                              a_front=tw.arc_source.a_front, a_rear=tw.arc_source.a_rear,
                              b=tw.arc_source.b, c=tw.arc_source.c))
        payload["scalars"] = np.array(json.dumps(sc))
        payload["twin_kw"] = np.array(json.dumps(kw2))
        payload["log"] = np.array(json.dumps(log))
        save("step_%s.npz" % name, payload)

    run2("c2_drop", None)
    run2("c2_seeded", 22)
    table_step_cases()


def table_step_cases():
    """The material-table path (solvers/coupled_step.py:168-458 with
    use_material_tables): the validated ER70S-6 file, c1-like Gaussian arc,
    heat losses on.  t1_plate starts from reset, where the property fields
    are still zero at the first enthalpy ceiling; t1_seeded starts from a
    molten state with refreshed fields, with substrate growth and the
    trailing freeze on, and runs the variable-tau SRT collision."""
    nx, ny, nz = 16, 12, 12
    dx = 2.5e-4
    cy = (ny // 2) * dx
    pos = [(0.0012 + s * 0.008 * dx * 0.1, cy) for s in range(4)]
    kw = dict(dx=dx, heat_source="gaussian2d", arc_power_W=3000.0, arc_efficiency=0.75,
              arc_sigma_mm=0.75, travel_speed_m_s=0.008, enable_heat_loss=True, tables=True)
    step_case("t1_plate", nx, ny, nz, 3, pos, kw,
              setup=lambda tw: setattr(tw, "plate_thickness_mm", 1.0))
    kw2 = dict(kw, enable_substrate_growth=True, enable_bead_freeze=True)
    step_case("t1_seeded", nx, ny, nz, 3, pos, kw2,
              setup=lambda tw: setattr(tw, "plate_thickness_mm", 1.0), seeded=23,
              after_load=refresh)


# ---------------------------------------------------------------------------
# telemetry: the reference's get_telemetry on seeded states
# ---------------------------------------------------------------------------
TELEM_FIELDS = ["T", "H", "f_l", "phi", "dT_dt", "ux", "uy", "uz", "flags"]


def telemetry_cases():
    """twin.py:706-821 on three states: a seeded pool with tracers, deposited
    solid above the plate and wetting on (toe angle); the same state with the
    pool frozen out (no liquid); the reset state."""
    nx, ny, nz = 20, 14, 14
    out = {}
    for name, seed in (("pool", 31), ("frozen", 32), ("reset", None)):
        tw = make_twin(nx, ny, nz, enable_wetting=True, droplet_freq_hz=100.0)
        tw.plate_thickness_mm = 0.8
        tw.wire_feed_m_s = 0.1
        tw.reset()
        tw.enable_force_diagnostics = False
        g = tw.grid
        if seed is not None:
            st = seeded_state(nx, ny, nz, seed=seed, nz_solid=tw.nz_solid)
            rng = np.random.default_rng(seed)
            st["dT_dt"] = rng.normal(0.0, 2e4, st["T"].shape).astype(np.float32)
            if name == "frozen":
                st["f_l"] = np.minimum(st["f_l"], np.float32(0.4))
            # a few deposited solid cells above the plate
            st["flags"][3:6, 5:8, tw.nz_solid:tw.nz_solid + 3] = 1
            load_state(g, st)
            act = np.zeros(g.max_tracers, np.int32)
            act[:30] = 1
            act[30:41] = 2
            g.porosity_active.from_numpy(act)
            tw._deposited_volume_m3 = 3.1e-9
            tw._n_droplets_fired = 4
            tw._step_n = 123
        tele = tw.get_telemetry()
        tele.pop("force_diagnostics", None)
        for f in TELEM_FIELDS:
            out["%s_%s" % (name, f)] = getattr(g, f).to_numpy()
        out["%s_porosity_active" % name] = g.porosity_active.to_numpy()
        out["%s_telemetry" % name] = np.array(json.dumps(tele))
        out["%s_state" % name] = np.array(json.dumps(dict(
            nz_solid=tw.nz_solid, step=tw._step_n, deposited=tw._deposited_volume_m3,
            n_drops=tw._n_droplets_fired, material=material_record(tw),
            twin_kw=dict(nx=nx, ny=ny, nz=nz, enable_wetting=True, droplet_freq_hz=100.0,
                         use_srt=False, enable_vof=True, wire_feed_m_s=0.1,
                         plate_thickness_mm=0.8))))
    save("telemetry.npz", out)


# ---------------------------------------------------------------------------
# known-answer values of the reference validation scripts
# ---------------------------------------------------------------------------
def kat_materials():
    """The material the validation scripts load (materials/placeholders/
    ER70S-6.yaml through the reference's load_material), as a record."""
    from waam_twin.materials import load_material
    m = load_material("materials/placeholders/ER70S-6.yaml")
    rec = {k: float(getattr(m, k)) for k in (
        "k", "rho", "cp", "alpha", "T_solidus", "T_liquidus", "L_fusion", "gamma_0",
        "dgamma_dT", "T_ref_gamma", "mu", "beta_T")}
    rec = dict(constants=rec, name=m.name, status=m.status,
               contact_angle_deg=float(m.contact_angle_deg),
               tables={k: [list(map(float, r)) for r in getattr(m.tables, k)]
                       for k in ("cp", "k", "mu", "dgamma_dT")})
    with open(os.path.join(HERE, "kat_materials.json"), "w") as fh:
        json.dump({"ER70S-6-placeholder": rec}, fh, indent=1, sort_keys=True)
    print("kat materials", rec)


class _PathRecorder:
    """Stands in for a twin in the reference's ``WAAMTwin.run_path``: the
    attributes that method reads, and a ``step`` that records its call."""

    def __init__(self, nx, ny, dx, travel, interpass_attr=0, window_offset=0.0):
        import types
        self.grid = types.SimpleNamespace(nx=nx, ny=ny, dx=dx, dt=dx * 0.05 / 0.5)
        self.travel_speed_m_s = travel
        self._interpass_cooling_steps = interpass_attr
        self._window_offset_x_m = window_offset
        self._torch_dir_xyz = (1.0, 0.0, 0.0)
        self.calls = []

    def step(self, x, y, is_welding=True, torch_z_m=None):
        self.calls.append([float(x), float(y), bool(is_welding), torch_z_m])


RUN_PATH_CASES = {
    # name: (job given as, n_steps, interpass argument, interpass attribute, window offset)
    "yaml_interpass": ("yaml", 180, 7, 0, 0.0),
    "yaml_attr_interpass": ("yaml", 150, 0, 5, 0.0),
    "dict_default_steps": ("dict", None, 0, 0, 0.0),
    "dict_window": ("dict", 120, 3, 0, 1.5e-3),
    "empty_path": ("empty", 40, 0, 0, 0.0),
}


def run_path_cases():
    """The reference's run_path (twin.py:632-704) on the recorder: every step
    call (x, y, welding, z) and the seeded torch direction, for a job YAML, a
    job dict, and a job without a path (tests/golden/job_path.yaml)."""
    import yaml
    job_file = os.path.join(HERE, "job_path.yaml")
    with open(job_file) as fh:
        job = yaml.safe_load(fh)
    out = {}
    for name, (kind, n, ip_arg, ip_attr, off) in RUN_PATH_CASES.items():
        rec = _PathRecorder(48, 32, 2.5e-4, 2.5, ip_attr, off)
        arg = {"yaml": job_file, "dict": job, "empty": {"job_name": "no_path"}}[kind]
        wt.WAAMTwin.run_path(rec, arg, n_steps=n, interpass_steps=ip_arg)
        out[name] = dict(calls=rec.calls, torch_dir=list(rec._torch_dir_xyz),
                         nx=48, ny=32, dx=2.5e-4, travel=2.5, n_steps=n,
                         interpass_steps=ip_arg, interpass_attr=ip_attr, window_offset=off,
                         job=kind)
        print("run_path", name, len(rec.calls), "steps")
    with open(os.path.join(HERE, "run_path_reference.json"), "w") as fh:
        json.dump(out, fh)


KAT_SCRIPTS = ["test_vof_mass", "test_goldak_energy", "test_lbm_poiseuille",
               "test_stefan_solidification", "test_thermal_diffusion", "test_lbm_cavity",
               "test_rosenthal_farfield"]


def kats(names=None):
    """Run validation scripts of the reference (their own ``run()`` with its
    default arguments) and merge their returned values into
    kat_reference.json.  A script's pass/fail threshold is set to infinity so
    that it returns its value even where the reference itself misses its own
    threshold; the value does not depend on it, and the tests apply the
    thresholds."""
    import importlib
    import inspect
    import time
    path = os.path.join(HERE, "kat_reference.json")
    out = {}
    for name in names or KAT_SCRIPTS:
        t0 = time.time()
        mod = importlib.import_module("waam_twin.validation." + name)
        params = inspect.signature(mod.run).parameters
        kw = {p: float("inf") for p in ("threshold", "threshold_pct") if p in params}
        out[name] = float(mod.run(**kw))
        print("kat", name, out[name], "%.0f s" % (time.time() - t0), flush=True)
        # merge into the file as it is now (another run may have added values)
        cur = {}
        if os.path.exists(path):
            with open(path) as fh:
                cur = json.load(fh)
        cur[name] = out[name]
        with open(path, "w") as fh:
            json.dump(cur, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    what = sys.argv[1:] or ["kernels", "steps", "kats"]
    ONLY.update(w.split("=", 1)[1] for w in what if w.startswith("kernel="))
    KAT_ONLY = [w.split("=", 1)[1] for w in what if w.startswith("kat=")]
    if "kernels" in what or ONLY:
        kernel_cases()
    if "steps" in what:
        step_cases()
    if "table_steps" in what:
        table_step_cases()
    if "telemetry" in what:
        telemetry_cases()
    if "run_path" in what:
        run_path_cases()
    if "kat_materials" in what:
        kat_materials()
    if "kats" in what or KAT_ONLY:
        kats(KAT_ONLY or None)
