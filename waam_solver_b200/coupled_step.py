"""One coupled physics timestep (reference solvers/coupled_step.py:73-464).

Two drivers produce the same state:

* ``coupled_step_operators`` calls the operator API one kernel at a time in
  the reference's order -- the drop-in path for callers that interleave
  their own operators;
* ``coupled_step_fused`` runs the B200 pipeline of ``waam_step_pre`` /
  ``waam_step_main`` (about eight kernels per step, no host synchronisation
  except on droplet steps, where the deposition budget is read back exactly
  as the reference does).

``coupled_step`` dispatches on ``twin.step_mode`` ("fused" by default).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native, kernels
from ._native import WaamError
from .physics import deposition, forces, free_surface, lbm, phase_change, thermal, weld_forces
from .grid import raw_field
from .physics.electrical_stickout import droplet_entry_temperature_K, update_ctwd

T_800 = 800.0 + 273.15
T_1100 = 1100.0 + 273.15


def _clamp_ceiling(twin, g):
    """solvers/coupled_step.py:17-31."""
    if not twin.enable_enthalpy_cap:
        return
    if twin.use_material_tables:
        thermal.clamp_enthalpy_ceiling_variable_cp(g.H, g.flags, g.cp_rho_field, twin.H_liq,
                                                   twin.mat.T_liquidus, twin.T_vapor_cap_K,
                                                   g.FLAG_GAS)
    else:
        thermal.clamp_enthalpy_ceiling_scalar(g.H, g.flags, twin.cp_rho, twin.mat.T_solidus,
                                              twin.mat.T_liquidus, twin.T_vapor_cap_K, twin.L_rho,
                                              g.FLAG_GAS)


def _update_phase(twin, g):
    if twin.use_material_tables:
        thermal.update_phase_variable_cp(g.H, g.T, g.f_l, g.cp_rho_field, twin.L_rho,
                                         twin.mat.T_solidus, twin.mat.T_liquidus, twin.H_sol,
                                         twin.H_liq)
    else:
        phase_change.update_phase(g.H, g.T, g.f_l, twin.cp_rho, twin.L_rho, twin.mat.T_solidus,
                                  twin.mat.T_liquidus)


def _refresh_properties(twin, g):
    """solvers/coupled_step.py:168-181 (the knots travel by value, no device read)."""
    t = twin.gpu_tables
    thermal.refresh_properties(
        g.T, g.cp_rho_field, g.alpha_lu_field, g.dgamma_lu_field, g.tau_field, t.cp_T, t.cp_V,
        t.k_T, t.k_V, t.mu_T, t.mu_V, t.dgamma_T, t.dgamma_V, t.n_cp, t.n_k, t.n_mu, t.n_dgamma,
        g.mat.rho, g.dt, g.dx, t.cp_fallback, t.k_fallback, t.mu_fallback, t.dgamma_fallback,
        twin.force_scale / g.dx, twin.cp_rho, twin.alpha_lu, twin.dgamma_dT_lu, g.tau,
        twin.marangoni_scale, 1, g.flags, g.FLAG_SOLID, g.FLAG_GAS)


def _resolve_arc_k(twin, g, arc_i, arc_j, torch_z_m=None):
    """solvers/coupled_step.py:34-59 (host read of the surface height)."""
    i0 = max(0, min(int(arc_i), g.nx - 1))
    j0 = max(0, min(int(arc_j), g.ny - 1))
    free_surface.surface_height_at(g.phi, g.flags, g.surface_k_buf, i0, j0, twin.nz_solid,
                                   g.FLAG_GAS, g.nz)
    k = float(g.surface_k_buf.item())
    if k < 1.0:
        k = float(max(1, twin.nz_solid - 1))
    return _robot_z(twin, g, k, torch_z_m)


def _robot_z(twin, g, k_surface, torch_z_m):
    if getattr(twin, "use_torch_z", False) and torch_z_m is not None:
        z_bead = max(twin.substrate_z_m, torch_z_m - twin.ctwd_m)
        k_robot = twin.nz_solid + (z_bead - twin.substrate_z_m) / g.dx - 1.0
        k_robot = max(float(twin.nz_solid) + 0.5, min(k_robot, float(g.nz) - 2.0))
        return max(k_surface, k_robot)
    return k_surface


def _footprint_radii(r_try):
    """The retry radii of solvers/coupled_step.py:130-151 (10 attempts)."""
    radii = []
    for _ in range(10):
        radii.append(r_try)
        r_try = min(r_try + 1.5, 16.0)
    return radii


def _droplet(twin, g, arc_i, arc_j, arc_k, torch_x_m, torch_y_m, device_retries=False):
    """Droplet schedule and deposition (solvers/coupled_step.py:110-166).

    ``device_retries`` runs the footprint retry loop in one launch
    (``kernels.deposit_droplet``) instead of one ``feed_wire_surface`` call and
    one read-back per attempt; the results are identical.  Returns True when a
    droplet fired this step."""
    if twin.droplet_freq <= 0:
        return False
    sim_time = twin._step_n * g.dt
    period = deposition.droplet_period_s(twin)
    if sim_time - twin._last_droplet_time < period:
        return False
    drop_dt = sim_time - twin._last_droplet_time
    twin._last_droplet_time = sim_time
    drop_mass = deposition.droplet_mass_for_interval_kg(twin, drop_dt)
    drop_r = deposition.droplet_radius_cells_from_mass_kg(twin, drop_mass)
    drop_vol = drop_mass / twin.mat.rho
    T_drop = droplet_entry_temperature_K(twin)
    _spawn_tracers(twin, g, torch_x_m, torch_y_m, arc_k)
    r_try = deposition.deposition_footprint_cells(twin, drop_r)
    placed_real = 0.0
    if device_retries:
        g.deposit_vol_buf.zero_()
        g.deposit_real_buf.zero_()
        kernels.deposit_droplet(
            g.f_src, g.flags, g.f_l, g.phi, g.H, g.T, g.rho, arc_i, arc_j, arc_k,
            _footprint_radii(r_try), drop_vol * 0.98, drop_r, drop_vol, T_drop, twin.cp_rho,
            twin.L_rho, 1.0, g.deposit_vol_buf, g.deposit_real_buf, g.dx ** 3, g.FLAG_GAS,
            g.FLAG_FLUID, g.FLAG_SOLID, g.nx, g.ny, g.nz)
        placed_real = float(g.deposit_real_buf.item())
    for _ in range(0 if device_retries else 10):
        g.deposit_vol_buf.fill_(placed_real)
        g.deposit_real_buf.fill_(placed_real)
        deposition.feed_wire_surface(
            g.f_src, g.flags, g.f_l, g.phi, g.H, g.T, g.rho, arc_i, arc_j, arc_k, r_try, drop_r,
            drop_vol, T_drop, twin.cp_rho, twin.L_rho, 1.0, g.deposit_vol_buf,
            g.deposit_real_buf, g.dx ** 3, g.FLAG_GAS, g.FLAG_FLUID, g.FLAG_SOLID, g.nx, g.ny,
            g.nz)
        placed_real = float(g.deposit_real_buf.item())
        if placed_real >= drop_vol * 0.98:
            break
        r_try = min(r_try + 1.5, 16.0)
    if placed_real < drop_vol * 0.98:
        twin._deposition_overflow += 1
    twin._deposited_volume_m3 += placed_real
    twin._n_droplets_fired += 1
    weld_forces.apply_droplet_impact(twin, g, arc_i, arc_j, arc_k, drop_r, drop_mass)
    return True


def coupled_step_operators(twin, torch_x_m, torch_y_m, is_welding, torch_z_m=None):
    """The reference step, operator by operator (constants or table path)."""
    g = twin.grid
    arc_i = torch_x_m / g.dx
    arc_j = torch_y_m / g.dx
    arc_k = _resolve_arc_k(twin, g, arc_i, arc_j, torch_z_m)
    twin._last_arc_ijk = (float(arc_i), float(arc_j), float(arc_k))
    forces.clear_forces(g.Fx, g.Fy, g.Fz)
    if twin.enable_ctwd:
        update_ctwd(twin, g)
    pressure = weld_forces.arc_pressure_peak_pa(twin)
    p_sigma = weld_forces.arc_pressure_sigma_cells(twin)
    if is_welding:
        twin.arc_source.inject(twin, g, arc_i, arc_j, arc_k)
        _clamp_ceiling(twin, g)
        _droplet(twin, g, arc_i, arc_j, arc_k, torch_x_m, torch_y_m)
    tables = twin.use_material_tables
    if tables:
        _refresh_properties(twin, g)
        thermal.advect_diffuse_variable(g.H, g.T, g.ux, g.uy, g.uz, g.flags, g.alpha_lu_field,
                                        g.cp_rho_field, 1.0, g.FLAG_SOLID, g.FLAG_GAS, g.nx,
                                        g.ny, g.nz)
    else:
        thermal.advect_diffuse_temperature(g.H, g.T, g.ux, g.uy, g.uz, g.flags, twin.alpha_lu,
                                           1.0, g.FLAG_SOLID, g.FLAG_GAS, twin.cp_rho, g.nx,
                                           g.ny, g.nz)
    if twin.enable_heat_loss:
        thermal.apply_boundary_losses(g.H, g.T, g.flags, twin.T_amb, twin.h_conv, twin.eps_rad,
                                      int(twin.enable_convection), int(twin.enable_radiation),
                                      twin.cp_rho, g.dt, g.dx, twin.sigma_sb, g.FLAG_SOLID,
                                      g.FLAG_GAS, g.nx, g.ny, g.nz)
        if tables:
            thermal.clamp_enthalpy_floor(g.H, g.cp_rho_field, g.flags, twin.T_amb, g.FLAG_GAS)
        else:
            thermal.clamp_enthalpy_floor_scalar(g.H, twin.cp_rho, g.flags, twin.T_amb,
                                                g.FLAG_GAS)
    _update_phase(twin, g)
    _clamp_ceiling(twin, g)
    _update_phase(twin, g)
    thermal.update_T_max(g.T, g.T_max, g.flags, g.FLAG_GAS)
    thermal.update_cooling_rate(g.T, g.T_prev, g.dT_dt, g.flags, g.dt, g.FLAG_GAS)
    if twin.enable_vof:
        g.ensure_vof_buffers()
        free_surface.advect_phi(g.phi_tmp, g.phi, g.ux, g.uy, g.uz, g.flags, g.FLAG_SOLID,
                                g.FLAG_GAS, g.nx, g.ny, g.nz)
        g.phi.copy_(g.phi_tmp)
        free_surface.reinitialize_phi(g.phi, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.FLAG_FLUID)
        if twin.enable_wetting:
            free_surface.apply_contact_angle_phi_bc(g.phi, g.flags, twin.theta_rad, g.FLAG_SOLID,
                                                    g.FLAG_GAS, g.nx, g.ny, g.nz)
        free_surface.update_flags_from_phi(g.phi, g.f_l, g.flags, twin.nz_solid, g.FLAG_FLUID,
                                           g.FLAG_SOLID, g.FLAG_GAS, g.FLAG_IFACE)
        free_surface.sync_phi_liquid_fraction(g.phi, g.f_l, g.flags, g.FLAG_GAS, g.FLAG_SOLID)
    if twin.enable_csf_tension:
        forces.compute_csf_tension(g.phi, g.flags, g.Fx, g.Fy, g.Fz, twin.gamma_lu, g.FLAG_SOLID,
                                   g.FLAG_GAS, g.nx, g.ny, g.nz,
                                   enable_wetting=twin.enable_wetting, theta_rad=twin.theta_rad)
    if tables:
        forces.compute_marangoni_force_variable(g.T, g.phi, g.f_l, g.Fx, g.Fy, g.Fz, g.flags,
                                                g.dgamma_lu_field, g.FLAG_SOLID, g.FLAG_GAS,
                                                g.nx, g.ny, g.nz)
    else:
        forces.compute_marangoni_force(g.T, g.phi, g.f_l, g.Fx, g.Fy, g.Fz, g.flags,
                                       twin.dgamma_dT_lu, g.dx, g.FLAG_SOLID, g.FLAG_GAS, g.nx,
                                       g.ny, g.nz)
    if is_welding:
        weld_forces.apply_gas_shear(twin, g, arc_i, arc_j, arc_k)
        forces.apply_arc_pressure(g.Fz, g.flags, g.phi, arc_i, arc_j, arc_k, p_sigma, pressure,
                                  g.dt, g.dx, twin.mat.rho, g.FLAG_SOLID, g.FLAG_GAS)
        weld_forces.apply_recoil(twin, g, arc_i, arc_j, arc_k)
    if twin.enable_hydrostatic_gravity:
        forces.add_hydrostatic_gravity(g.Fz, g.f_l, g.flags, 1.0, twin.g_lu, g.FLAG_SOLID,
                                       g.FLAG_GAS)
    forces.add_buoyancy(g.T, g.Fz, g.f_l, g.flags, twin.g_lu, twin.beta_T, twin.mat.T_liquidus,
                        1.0, g.FLAG_SOLID, g.FLAG_GAS)
    if is_welding and twin.enable_lorentz:
        weld_forces.solve_lorentz(twin, g, arc_i, arc_j, arc_k)
    u_cap = float(getattr(twin, "u_mach_limit_lu", 0.08))
    F_cap = float(getattr(twin, "force_limit_lu", 0.05))
    if F_cap > 0.0:
        kernels.clamp_body_force_magnitude(g.Fx, g.Fy, g.Fz, g.flags, F_cap, g.FLAG_SOLID,
                                           g.FLAG_GAS)
    if tables and twin.use_variable_tau:
        lbm.collide_srt_variable_tau(g.f_src, g.f_dst, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz,
                                     g.f_l, g.flags, g.tau_field, twin.C_darcy, g.FLAG_SOLID,
                                     g.FLAG_GAS, g.nx, g.ny, g.nz)
    elif twin.use_srt:
        lbm.collide_srt(g.f_src, g.f_dst, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l,
                        g.flags, g.tau, twin.omega, 1.0, twin.C_darcy, g.FLAG_SOLID, g.FLAG_GAS,
                        g.nx, g.ny, g.nz)
    else:
        lbm.collide_mrt(g.f_src, g.f_dst, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l,
                        g.flags, g.ex, g.ey, g.ez, g.w, g.opp, twin.omega, twin.omega_bulk,
                        twin.C_darcy, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
    if u_cap > 0.0:
        kernels.clamp_velocity_mach(g.ux, g.uy, g.uz, g.flags, u_cap, g.FLAG_SOLID, g.FLAG_GAS)
    lbm.stream(g.f_dst, g.f_src, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
    kernels.advect_tracers(g.porosity_pos, g.porosity_active, g.ux, g.uy, g.uz, g.f_l, g.flags,
                           g.dx, g.dt, g.max_tracers, g.FLAG_SOLID, g.FLAG_GAS)
    kernels.update_time_above_T(g.T, g.flags, g.time_above_800_s, g.time_above_1100_s,
                                g.time_above_solidus_s, g.dt, T_800, T_1100, twin.mat.T_solidus,
                                g.FLAG_GAS)
    kernels.snapshot_forces(g.Fx, g.Fy, g.Fz, g.Fx_snap, g.Fy_snap, g.Fz_snap)
    if twin.enable_substrate_growth or twin.enable_bead_freeze:
        if tables:
            free_surface.remelt_hot_solid(g.T, g.H, g.f_l, g.phi, g.flags, g.cp_rho_field,
                                          twin.mat.T_solidus, twin.mat.T_liquidus, twin.L_rho,
                                          g.FLAG_SOLID, g.FLAG_FLUID)
        else:
            free_surface.remelt_hot_solid_scalar(g.T, g.H, g.f_l, g.phi, g.flags, twin.cp_rho,
                                                 twin.mat.T_solidus, twin.mat.T_liquidus,
                                                 twin.L_rho, g.FLAG_SOLID, g.FLAG_FLUID)
        if is_welding and twin.enable_bead_freeze:
            dx_, dy_, dz_ = getattr(twin, "_torch_dir_xyz", (1.0, 0.0, 0.0))
            lookback = max(2.0, twin.trailing_solidify_lookback_mm / (g.dx * 1000.0))
            T_freeze = twin.mat.T_liquidus + twin.trailing_solidify_temp_margin_K
            if tables:
                kernels.solidify_trailing_pool(g.T, g.H, g.f_l, g.phi, g.flags, g.ux, g.uy, g.uz,
                                               g.cp_rho_field, arc_i, arc_j, arc_k, dx_, dy_, dz_,
                                               lookback, T_freeze, twin.mat.T_solidus,
                                               g.FLAG_SOLID, g.FLAG_FLUID, g.FLAG_GAS)
            else:
                kernels.solidify_trailing_pool_scalar(g.T, g.H, g.f_l, g.phi, g.flags, g.ux,
                                                      g.uy, g.uz, twin.cp_rho, arc_i, arc_j,
                                                      arc_k, dx_, dy_, dz_, lookback, T_freeze,
                                                      twin.mat.T_solidus, g.FLAG_SOLID,
                                                      g.FLAG_FLUID, g.FLAG_GAS)
        free_surface.solidify_cooled_metal(g.T, g.f_l, g.phi, g.flags, g.ux, g.uy, g.uz,
                                           twin.mat.T_solidus, True, g.FLAG_SOLID, g.FLAG_FLUID,
                                           g.FLAG_GAS)
    g.swap_buffers()
    twin._step_n += 1
    g._forces_dirty = True


def _fields(g):
    f = _native.WaamFields()
    g.ensure_vof_buffers()
    r = lambda name: raw_field(g, name)  # noqa: E731  (no flush of pending work)
    for name, t in (("f_src", r("f_src")), ("f_dst", r("f_dst")), ("rho", r("rho")), ("ux", r("ux")),
                    ("uy", r("uy")), ("uz", r("uz")), ("T", g.T), ("T_next", g.T_next), ("H", g.H),
                    ("H_next", g.H_next), ("f_l", g.f_l), ("phi", g.phi),
                    ("phi_tmp", g.phi_tmp), ("flags", g.flags), ("T_max", g.T_max),
                    ("T_prev", g.T_prev), ("dT_dt", g.dT_dt), ("t800", g.time_above_800_s),
                    ("t1100", g.time_above_1100_s), ("tsol", g.time_above_solidus_s),
                    ("Fx", r("Fx")), ("Fy", r("Fy")), ("Fz", r("Fz")),
                    ("step_scalars", g.step_scalars)):
        setattr(f, name, t.data_ptr())
    f.nx, f.ny, f.nz = g.nx, g.ny, g.nz
    if getattr(g, "_tracers_live", False):   # advected once the first droplet spawned some
        f.tracer_pos = r("porosity_pos").data_ptr()
        f.tracer_active = r("porosity_active").data_ptr()
        f.max_tracers = g.max_tracers
    f.cp_rho_f, f.alpha_f = g.cp_rho_field.data_ptr(), g.alpha_lu_field.data_ptr()
    f.dgamma_f, f.tau_f = g.dgamma_lu_field.data_ptr(), g.tau_field.data_ptr()
    copies = getattr(g, "flags_copies", None)
    if copies is not None:
        # rotation of three: this step writes w, the step before wrote r, the
        # one before that rr
        w = getattr(g, "_flags_copy_i", 0)
        f.flags_copy_w = copies[w].data_ptr()
        f.flags_copy_r = copies[(w + 2) % 3].data_ptr()
        f.flags_copy_rr = copies[(w + 1) % 3].data_ptr()
    f.status = g.step_status.data_ptr()
    caches = getattr(g, "pop_caches", None)
    if caches is not None:
        # each compact copy goes with its population buffer
        a_first = g._read_buf is raw_field(g, "f_a")
        f.pop_cache_src = caches[0 if a_first else 1].data_ptr()
        f.pop_cache_dst = caches[1 if a_first else 0].data_ptr()
        f.pop_cache_stamp = g.pop_cache_stamp.data_ptr()
    if g.nz > 32:
        # quiet tiles need a k tile above the plate's: with one 32-cell k tile
        # every tile holds metal, and the list would only add a kernel
        f.tile_bits = g.tile_bits.data_ptr()
        f.tile_list = g.tile_list.data_ptr()
        f.tile_part = g.tile_part.data_ptr()
    return f


def _spawn_tracers(twin, g, torch_x_m, torch_y_m, arc_k):
    """solvers/coupled_step.py:120-125: 50 porosity tracers per droplet."""
    kernels.inject_tracers(g.porosity_pos, g.porosity_active, g.tracer_head, g.max_tracers,
                           torch_x_m, torch_y_m, float(arc_k + 1) * g.dx,
                           float(twin.sigma_cells * g.dx), 50, seed=twin._step_n)
    if not getattr(g, "_tracers_live", False):
        g._tracers_live = True
        g.__dict__.pop("_fields_cache", None)    # the fused step now advects them
        twin.__dict__["_graphs"] = {}


def step_params(twin):
    """WaamStepParams with every per-twin constant (per-step fields filled later)."""
    g = twin.grid
    m = twin.mat
    p = _native.WaamStepParams()
    p.nz_solid = twin.nz_solid
    terms = twin.arc_source.fused_terms(twin)
    for k, v in terms.items():
        setattr(p, k, v)
    p.Q_w, p.eta, p.dt, p.dx, p.dx3 = twin.Q_w, twin.eta, g.dt, g.dx, g.dx ** 3
    p.pen = twin.arc_penetration_m / g.dx
    p.surface_weighting = 1 if twin.arc_surface_weighting else 0
    p.cp_rho, p.L_rho, p.Ts, p.Tl = twin.cp_rho, twin.L_rho, m.T_solidus, m.T_liquidus
    p.T_cap, p.alpha_lu = twin.T_vapor_cap_K, twin.alpha_lu
    p.cap_enabled = 1 if twin.enable_enthalpy_cap else 0
    p.heat_loss = 1 if twin.enable_heat_loss else 0
    p.T_amb, p.h_conv, p.eps_rad, p.sigma_sb = twin.T_amb, twin.h_conv, twin.eps_rad, twin.sigma_sb
    p.conv, p.rad = int(twin.enable_convection), int(twin.enable_radiation)
    p.vof, p.wetting, p.theta = int(twin.enable_vof), int(twin.enable_wetting), twin.theta_rad
    p.csf, p.hydro = int(twin.enable_csf_tension), int(twin.enable_hydrostatic_gravity)
    p.gamma_lu, p.dgamma_lu = twin.gamma_lu, twin.dgamma_dT_lu
    p.p_sigma = weld_forces.arc_pressure_sigma_cells(twin)
    p.pressure = weld_forces.arc_pressure_peak_pa(twin)
    p.rho_phys, p.g_lu, p.beta, p.T_ref = m.rho, twin.g_lu, twin.beta_T, m.T_liquidus
    p.F_cap = float(getattr(twin, "force_limit_lu", 0.05))
    p.collision = 1 if twin.use_srt else 0
    p.omega = twin.omega
    p.omega_b = twin.omega_bulk
    p.C_darcy = twin.C_darcy
    p.u_cap = float(getattr(twin, "u_mach_limit_lu", 0.08))
    p.T800, p.T1100 = T_800, T_1100
    p.substrate_growth, p.bead_freeze = int(twin.enable_substrate_growth), int(twin.enable_bead_freeze)
    p.lookback = max(2.0, twin.trailing_solidify_lookback_mm / (g.dx * 1000.0))
    p.T_freeze = m.T_liquidus + twin.trailing_solidify_temp_margin_K
    p.f_storage = g.population_storage
    p.use_tables = 1 if twin.use_material_tables else 0
    p.variable_tau = 1 if twin.use_variable_tau else 0
    p.rho_mat = m.rho
    p.force_scale_lu = twin.force_scale / g.dx
    p.marangoni_scale = twin.marangoni_scale
    p.H_sol_t, p.H_liq_t = twin.H_sol, twin.H_liq
    p.tau_ref = g.tau
    p.tables = twin.gpu_tables.struct
    # shielding-gas shear and vapour recoil (physics/weld_forces.py:126-193)
    p.gas_shear = 1 if twin.enable_gas_shear else 0
    p.gs_tau_pa = weld_forces.gas_shear_tau_pa(twin)
    p.recoil = (2 if twin.use_recoil_clausius_clapeyron else 1) if twin.enable_recoil else 0
    p.recoil_pa, p.recoil_T_ref = twin.recoil_pressure_pa, m.T_liquidus
    p.P_ref, p.T_boil = twin.P_vapor_ref_Pa, twin.T_boiling_K
    p.L_vap, p.R_spec = twin.L_vapor_J_kg, twin.R_spec_vapor_J_kgK
    p.C_acc = weld_forces.recoil_accommodation(twin)
    p.weld_sigma = twin.sigma_cells
    p.rho_lo, p.rho_hi = getattr(twin, "health_rho_band", (0.5, 2.0))
    return p


def _check_fused_supported(twin):
    supported = not getattr(twin, "use_torch_z", False)
    if not supported and twin.grid.population_storage:
        raise WaamError("16-bit population storage runs on the fused step only; this "
                        "configuration needs the operator path")
    return supported


class _PositionRing:
    """Pinned host slots for the per-step torch position (a 2-float H2D copy).

    A slot is rewritten only after the copy that last read it has completed,
    so the host can run ahead of the GPU without racing its own copies."""

    SLOTS = 1024

    def __init__(self):
        self.host = torch.zeros((self.SLOTS, 2), dtype=torch.float32, pin_memory=True)
        self.host_np = self.host.numpy()
        self.views = [self.host[i] for i in range(self.SLOTS)]
        self.events = [None] * self.SLOTS
        self.i = 0

    def upload(self, dst, arc_i, arc_j):
        slot = self.i % self.SLOTS
        self.i += 1
        ev = self.events[slot]
        if ev is not None:
            ev.synchronize()
        self.host_np[slot, 0] = arc_i
        self.host_np[slot, 1] = arc_j
        dst.copy_(self.views[slot], non_blocking=True)
        if ev is None:
            ev = self.events[slot] = torch.cuda.Event()
        ev.record()


def upload_position(twin, arc_i, arc_j):
    g = twin.grid
    src = getattr(twin, "_device_position", None)
    if src is not None:
        # caller-provided device tensor with the position (cells); no host copy
        g._pos_dst.copy_(src)
        return
    ring = getattr(g, "_pos_ring", None)
    if ring is None:
        ring = g._pos_ring = _PositionRing()
    ring.upload(g._pos_dst, arc_i, arc_j)


def _fields_cached(g, lorentz=False):
    """WaamFields for the current buffer parity (device pointers never move);
    ``lorentz``: with the current density and self field the collision adds."""
    key = (g._read_buf is raw_field(g, "f_a"), g._cur, lorentz, getattr(g, "_flags_copy_i", 0))
    cache = g.__dict__.setdefault("_fields_cache", {})
    f = cache.get(key)
    if f is None:
        f = cache[key] = _fields(g)
        if lorentz:
            for q, t in enumerate((g.Jx, g.Jy, g.Jz)):
                f.lorentz_J[q] = t.data_ptr()
            for q, t in enumerate((g.Bx, g.By, g.Bz)):
                f.lorentz_B[q] = t.data_ptr()
        g._pos_dst = g.step_scalars[4:6]
    return f


def flush_stream(g):
    """Run the work a pipelined step left pending (WaamStepParams.defer_stream /
    defer_collide), so that populations, density, velocity, forces and tracers
    hold the step's result.  A no-op otherwise."""
    collide = g.__dict__.get("_collide_pending", False)
    if not (collide or g.__dict__.get("_stream_pending", False)):
        return
    g._stream_pending = False
    g._collide_pending = False
    g._lag_pending = False      # a held stream is pending only with a collision (_pending_params)
    kernels.PENDING_GRIDS.discard(g)
    st = torch.cuda.current_stream().cuda_stream
    if collide:
        p = g._pending_params
        _native.call("waam_step_finish", ctypes.byref(_fields_cached(g)), ctypes.byref(p),
                     g.workspace.data_ptr(), g.workspace.numel(), st)
        return
    p = _native.WaamStepParams()
    p.f_storage = g.population_storage
    _native.call("waam_step_stream", ctypes.byref(_fields_cached(g)), ctypes.byref(p), st)


def _droplet_due(twin, g, is_welding):
    if not is_welding or twin.droplet_freq <= 0:
        return False
    sim_time = twin._step_n * g.dt
    return sim_time - twin._last_droplet_time >= deposition.droplet_period_s(twin)


def _run_graph(twin, g, f, p, ws, key):
    """Replay (capturing on first reuse) the CUDA graph of one non-droplet step."""
    graphs = twin.__dict__.setdefault("_graphs", {})
    entry = graphs.get(key)
    if entry is None:
        graphs[key] = entry = {"seen": 0, "graph": None}
    if entry["graph"] is None:
        entry["seen"] += 1
        if entry["seen"] < 3:      # eager the first two times: modules load outside capture
            return False
        graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(graph, stream=side):
            st = torch.cuda.current_stream().cuda_stream
            _native.call("waam_step_pre", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(),
                         ws.numel(), st)
            _native.call("waam_step_main", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(),
                         ws.numel(), st)
        torch.cuda.current_stream().wait_stream(side)
        entry["graph"] = graph
    entry["graph"].replay()
    return True


def coupled_step_fused(twin, torch_x_m, torch_y_m, is_welding, torch_z_m=None):
    """The B200 pipeline (waam_step_pre -> [droplet] -> waam_step_main).

    Steps without a droplet replay a captured CUDA graph of the two stages
    (``twin.use_cuda_graphs``); droplet steps and instrumented steps run the
    stages eagerly because they read back or record events in between.  With
    the welding current's Lorentz force, waam_step_main runs as its two
    halves around the potential solve (solvers/coupled_step.py:352-353), whose
    convergence checks read back; the collision then adds J x B before the
    force clamp."""
    if not _check_fused_supported(twin):
        flush_stream(twin.grid)
        return coupled_step_operators(twin, torch_x_m, torch_y_m, is_welding, torch_z_m)
    g = twin.grid
    if twin.enable_ctwd:
        # solvers/coupled_step.py:99-100: bead height from the flags at step start
        update_ctwd(twin, g)
    arc_i = torch_x_m / g.dx
    arc_j = torch_y_m / g.dx
    p = twin._fused_params
    if p is None:
        p = twin._fused_params = step_params(twin)
        twin.__dict__["_graphs"] = {}
    p.arc_i, p.arc_j = arc_i, arc_j
    p.welding = 1 if is_welding else 0
    p.forces_from_buffer = 0
    p.clear_forces = 1 if getattr(g, "_forces_dirty", True) else 0
    dx_, dy_, dz_ = getattr(twin, "_torch_dir_xyz", (1.0, 0.0, 0.0))
    p.dir_x, p.dir_y, p.dir_z = dx_, dy_, dz_
    if getattr(g, "flags_copies", None) is None:
        # the flags of each step, copied by its column pass, for its pending
        # stream -- kept for two steps, for the lagged stream
        g.flags_copies = tuple(torch.zeros_like(g.flags) for _ in range(3))
        g._flags_copy_i = 0
        g.__dict__.pop("_fields_cache", None)
    if (getattr(g, "pop_caches", None) is None and getattr(twin, "population_cache", True) and
            g.nz > 32):
        # the compact copies of the collision's output (WaamFields.pop_cache_*):
        # two slots per 32-cell column chunk, 96 or 48 bytes each, filled with
        # 0xff bytes (a cell index no cell has).  Not on grids of one 32-cell k
        # tile: their collision is launch-bound (measured on 64x32x32: 0.0234
        # against 0.0230 ms per step without the copy)
        slot = 96 if g.population_storage == 0 else 48
        nbytes = g.nx * g.ny * ((g.nz + 31) // 32) * 2 * slot
        g.pop_caches = tuple(torch.full((nbytes,), 255, dtype=torch.uint8, device=g.device)
                             for _ in range(2))
        g.pop_cache_stamp = torch.zeros(1, dtype=torch.int32, device=g.device)
        g.__dict__.pop("_fields_cache", None)
    f = _fields_cached(g)
    ws = g.workspace
    upload_position(twin, arc_i, arc_j)
    twin._last_arc_ijk = _LazyArc(g, arc_i, arc_j)
    events = getattr(twin, "_stage_events", None)
    due = _droplet_due(twin, g, is_welding)
    lorentz = bool(is_welding and twin.enable_lorentz)
    # Pipelined stream: this step's stream is left to run beside the next
    # step's first stages.  Droplet steps (the deposition writes populations),
    # instrumented steps and the remelt / solidify tail run it in order.
    # Pipelined collision: a step that may leave its stream pending also
    # leaves its collision and tracers pending, to run beside the next step's
    # arc stage -- except droplet steps (force buffer) and Lorentz steps.
    if due or events is not None:
        flush_stream(g)
    collide_prev = bool(g.__dict__.get("_collide_pending", False))
    p.collide_prev = 1 if collide_prev else 0
    p.collide_prev_welding = g.__dict__.get("_pending_welding", 0) if collide_prev else 0
    # the pending collision reads the population copy as its own step decided
    p.collide_prev_cache_read = g.__dict__.get("_pending_cache_read", 0) if collide_prev else 0
    p.stream_prev = 1 if (collide_prev or g.__dict__.get("_stream_pending", False)) else 0
    p.defer_stream = 1 if (getattr(twin, "pipeline_stream", True) and events is None and
                           not (twin.enable_bead_freeze or twin.enable_substrate_growth)) else 0
    p.defer_collide = 1 if (p.defer_stream and not due and not lorentz and
                            getattr(twin, "pipeline_collide", True)) else 0
    # Lagged stream: a step that leaves its collision pending also holds back
    # the previous step's stream, which the next step runs beside that
    # collision, on the cells that collision does not write
    p.stream_lag = 1 if g.__dict__.get("_lag_pending", False) else 0
    p.hold_stream = 1 if (p.stream_prev and p.defer_collide and
                          getattr(twin, "pipeline_lag_stream", True)) else 0
    # quiet tiles: skipped only while the tile history is the fused step's own
    # (no droplet deposition in the middle of this step, no force clear, no
    # remelt / solidify tail rewriting flags, nothing changed the state since)
    p.tile_skip = 1 if (getattr(twin, "skip_quiet_tiles", True) and g._tiles_valid and
                        g.__dict__.get("_tile_epoch") == kernels.STATE_EPOCH[0] and not due and
                        not p.clear_forces and
                        not (twin.enable_bead_freeze or twin.enable_substrate_growth)) else 0
    # population cache: read only while nothing but the fused step has written
    # the populations since the previous collision (the conditions of the
    # tile history that concern them: no state change since the previous
    # fused step completed, no droplet deposition before this collision)
    p.cache_read = 1 if (getattr(g, "pop_caches", None) is not None and
                         getattr(twin, "population_cache", True) and g._tiles_valid and
                         g.__dict__.get("_tile_epoch") == kernels.STATE_EPOCH[0] and
                         not due) else 0
    # until this step completes: a step that raises part-way leaves the next
    # one a tile-history restart (which also zeroes the work-list count)
    g._tiles_valid = False
    done = False
    if not due and not lorentz and events is None and getattr(twin, "use_cuda_graphs", True):
        key = (g._read_buf is raw_field(g, "f_a"), g._cur, p.welding, p.clear_forces, p.stream_prev,
               p.defer_stream, p.collide_prev, p.collide_prev_welding,
               p.collide_prev_cache_read, p.defer_collide,
               g._flags_copy_i, p.tile_skip, p.stream_lag, p.hold_stream, p.cache_read,
               (dx_, dy_, dz_) if twin.enable_bead_freeze else None)
        done = _run_graph(twin, g, f, p, ws, key)
    if not done:
        stream = torch.cuda.current_stream().cuda_stream
        _native.call("waam_step_pre", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(),
                     ws.numel(), stream)
        if due:
            arc_k = float(g.step_scalars[0].item())
            twin._synced_this_step = True
            forces.clear_forces(g.Fx, g.Fy, g.Fz)
            _droplet(twin, g, arc_i, arc_j, arc_k, torch_x_m, torch_y_m, device_retries=True)
            f = _fields_cached(g)     # the first droplet switches tracer advection on
            p.forces_from_buffer = 1
            p.clear_forces = 0
        if lorentz:
            # stage events (if any) go to both halves; _lorentz_events, if set,
            # bracket the potential solve between them
            handles, n_ev = None, 0
            if events is not None:
                handles = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
                n_ev = len(events)
            _native.call("waam_step_main_stage", ctypes.byref(f), ctypes.byref(p), 0,
                         ws.data_ptr(), ws.numel(), handles, n_ev, stream)
            lz_events = getattr(twin, "_lorentz_events", None)
            if lz_events is not None:
                lz_events[0].record()
            weld_forces.solve_lorentz(twin, g, arc_i, arc_j, None, apply_force=False,
                                      arc_k_dev=g.step_scalars[0:1])
            if lz_events is not None:
                lz_events[1].record()
            _native.call("waam_step_main_stage", ctypes.byref(_fields_cached(g, lorentz=True)),
                         ctypes.byref(p), 1, ws.data_ptr(), ws.numel(), handles, n_ev, stream)
        elif events is None:
            _native.call("waam_step_main", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(),
                         ws.numel(), stream)
        else:
            # stage timing for measurement: 7 cudaEvent handles recorded in-stream
            handles = (ctypes.c_void_p * len(events))(*[e.cuda_event for e in events])
            _native.call("waam_step_main_events", ctypes.byref(f), ctypes.byref(p),
                         ws.data_ptr(), ws.numel(), handles, len(events), stream)
    # the droplet impact load (and J x B on SOLID cells, which only runs
    # without VOF) stays in F outside the active cells until the next step
    g._forces_dirty = bool(p.forces_from_buffer) or (lorentz and not twin.enable_vof)
    g._stream_pending = bool(p.defer_stream)
    g._collide_pending = bool(p.defer_collide)
    g._lag_pending = bool(p.hold_stream)
    if p.defer_stream:
        kernels.PENDING_GRIDS.add(g)
    if p.defer_collide:
        q = _native.WaamStepParams.from_buffer_copy(p)
        q.collide_prev, q.collide_prev_welding = 1, p.welding
        q.collide_prev_cache_read = p.cache_read
        q.stream_lag, q.hold_stream = p.hold_stream, 0
        g._pending_params = q
        g._pending_welding = p.welding
        g._pending_cache_read = p.cache_read
    g._flags_copy_i = (g._flags_copy_i + 1) % 3    # this step's copy is read by the next two
    g._tiles_valid = True                    # this step's column pass wrote the chunk bits
    g._tile_epoch = kernels.STATE_EPOCH[0]
    g.flip_thermal()
    g.swap_buffers()
    twin._step_n += 1


class _LazyArc(tuple):
    """(arc_i, arc_j, arc_k) whose arc_k is read from the device on first use."""

    def __new__(cls, g, arc_i, arc_j):
        obj = super().__new__(cls, (arc_i, arc_j, None))
        obj._g = g
        return obj

    def __getitem__(self, idx):
        if idx == 2 or idx == -1:
            return float(self._g.step_scalars[0].item())
        return tuple.__getitem__(self, idx)

    def __iter__(self):
        yield self[0]
        yield self[1]
        yield self[2]


def coupled_step(twin, torch_x_m, torch_y_m, is_welding, torch_z_m=None):
    if getattr(twin, "step_mode", "fused") == "operators":
        flush_stream(twin.grid)
        coupled_step_operators(twin, torch_x_m, torch_y_m, is_welding, torch_z_m)
    else:
        kernels.IN_FUSED_STEP[0] = True
        try:
            coupled_step_fused(twin, torch_x_m, torch_y_m, is_welding, torch_z_m)
        finally:
            kernels.IN_FUSED_STEP[0] = False
    rec = getattr(twin, "probe_recorder", None)
    if rec is not None:
        rec.record_step(twin)
