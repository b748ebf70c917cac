"""Operator API of the coupled step, reference names and signatures.

Each function here has the name and positional arguments of the waam_twin
Taichi kernel it replaces (kernels.py / cumulant_kernel.py of the reference)
and runs the matching sm_100a entry point of ``libwaam_b200.so`` on the
current torch CUDA stream.  Fields are torch CUDA tensors laid out like the
reference grid.  The ``FLAG_*`` arguments are accepted for signature
compatibility and must carry the reference values (FLUID=0, SOLID=1, GAS=2,
IFACE=4).  There is no CPU path: a missing library or a non-CUDA tensor
raises.
"""
from __future__ import annotations

import ctypes
import weakref
import math

import torch

from . import _native
from ._native import WaamError

FLAG_VALUES = {"FLAG_FLUID": 0, "FLAG_SOLID": 1, "FLAG_GAS": 2, "FLAG_IFACE": 4}
_W = [1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12


def _flags_ok(**kw):
    for k, v in kw.items():
        if int(v) != FLAG_VALUES[k]:
            raise WaamError("%s=%s differs from the built-in value %d" % (k, v, FLAG_VALUES[k]))


def _f(t, n=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise WaamError("expected a CUDA tensor, got %r" % type(t))
    if t.dtype != torch.float32 or not t.is_contiguous():
        raise WaamError("expected a contiguous float32 CUDA tensor, got %s" % t.dtype)
    if n is not None and t.numel() != n:
        raise WaamError("field has %d elements, expected %d" % (t.numel(), n))
    return t.data_ptr()


POP_STORAGE = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2}


def _pop(t, n=None):
    """(pointer, storage code) of a population tensor: float32 f_q, or float16 /
    bfloat16 offsets f_q - w_q (see WaamStepParams.f_storage)."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise WaamError("expected a CUDA tensor, got %r" % type(t))
    if t.dtype not in POP_STORAGE or not t.is_contiguous():
        raise WaamError("populations must be a contiguous float32, float16 or bfloat16 CUDA "
                        "tensor, got %s" % t.dtype)
    if n is not None and t.numel() != n:
        raise WaamError("populations have %d elements, expected %d" % (t.numel(), n))
    return t.data_ptr(), POP_STORAGE[t.dtype]


def _i(t, n=None):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise WaamError("expected a CUDA tensor, got %r" % type(t))
    if t.dtype != torch.int32 or not t.is_contiguous():
        raise WaamError("expected a contiguous int32 CUDA tensor (flags), got %s" % t.dtype)
    if n is not None and t.numel() != n:
        raise WaamError("flags has %d elements, expected %d" % (t.numel(), n))
    return t.data_ptr()


def _dims(t):
    if t.dim() == 4:
        return tuple(t.shape[1:])
    return tuple(t.shape)


def _stream():
    return torch.cuda.current_stream().cuda_stream


_WORKSPACES = {}


def workspace_for(t):
    """Device workspace for reducing entry points (cached per device and size)."""
    n = t.numel() if t.dim() == 3 else t[0].numel()
    key = (t.device, n)
    ws = _WORKSPACES.get(key)
    if ws is None:
        nbytes = int(_native.lib().waam_workspace_bytes(n))
        ws = torch.zeros(nbytes, dtype=torch.uint8, device=t.device)
        _WORKSPACES[key] = ws
    return ws.data_ptr(), ws.numel()


# Entry points that can change flags, phi, f_l, H, T or the material-property
# fields.  The fused step keeps a history of all-GAS tiles from step to step
# (quiet-tile skipping); a grid trusts it only while STATE_EPOCH is the value
# it saw at its last step.
_TILE_STATE_WRITERS = frozenset({
    "waam_advect_diffuse_temperature", "waam_advect_diffuse_temperature_variable",
    "waam_advect_phi", "waam_apply_contact_angle_phi_bc", "waam_apply_thermal_boundary_losses",
    "waam_clamp_enthalpy_ceiling_scalar", "waam_clamp_enthalpy_ceiling_variable_cp",
    "waam_clamp_enthalpy_floor", "waam_clamp_enthalpy_floor_scalar", "waam_deposit_droplet",
    "waam_feed_wire", "waam_feed_wire_surface", "waam_init_grid", "waam_inject_arc_heat",
    "waam_inject_goldak_heat", "waam_refresh_thermal_properties", "waam_reinitialize_phi",
    "waam_remelt_hot_solid", "waam_remelt_hot_solid_scalar", "waam_shift_window_x",
    "waam_solidify_cooled_metal", "waam_solidify_trailing_pool",
    "waam_solidify_trailing_pool_scalar", "waam_sync_phi_liquid_fraction",
    "waam_update_flags_from_phi", "waam_update_phase", "waam_update_phase_variable_cp"})
# Entry points that write populations (besides those above): they end the
# fused step's population cache as well.
_POPULATION_WRITERS = frozenset({
    "waam_collide_mrt", "waam_collide_srt", "waam_collide_srt_variable_tau", "waam_stream",
    "waam_feed_wire_momentum", "waam_feed_wire_momentum_impact_stored"})
STATE_EPOCH = [0]
# Grids whose last fused step left work pending (its stream, or its collision,
# tracers and stream): a state-writing operator call runs that work first,
# since the pending collision reads phi, T, f_l and flags.  IN_FUSED_STEP
# marks the fused step's own operator calls.
PENDING_GRIDS = weakref.WeakSet()
IN_FUSED_STEP = [False]


def state_changed():
    """Record a change of flags / phi / f_l / H / T made outside the fused step,
    after running the work a pipelined step left pending."""
    if not IN_FUSED_STEP[0]:
        for g in list(PENDING_GRIDS):
            g.flush_stream()
    STATE_EPOCH[0] += 1


def _call(name, *args):
    if name in _TILE_STATE_WRITERS or name in _POPULATION_WRITERS:
        state_changed()
    return _native.call(name, *args)


# ---------------------------------------------------------------- init ----
def init_grid(f, rho, ux, uy, uz, T, H, f_l, phi, flags, T_ambient, rho0, cp_rho, nz_solid,
              plate_i0, plate_i1, plate_j0, plate_j1, FLAG_FLUID, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_FLUID=FLAG_FLUID, FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(rho)
    n = nx * ny * nz
    _call("waam_init_grid", _f(f, 19 * n), _f(rho, n), _f(ux, n), _f(uy, n), _f(uz, n), _f(T, n),
          _f(H, n), _f(f_l, n), _f(phi, n), _i(flags, n), nx, ny, nz, float(T_ambient),
          float(rho0), float(cp_rho), int(nz_solid), int(plate_i0), int(plate_i1),
          int(plate_j0), int(plate_j1), _stream())


def init_aux_fields(T_max, T_prev, dT_dt, time_above_800, time_above_1100, time_above_solidus,
                    Fx_snap, Fy_snap, Fz_snap, Fx, Fy, Fz, T_ambient, porosity_active,
                    tracer_head, max_tracers):
    """kernels.py:123-158 (state reset; not on the step path)."""
    tracer_head.zero_()
    porosity_active.zero_()
    T_max.fill_(float(T_ambient))
    T_prev.fill_(float(T_ambient))
    for t in (dT_dt, time_above_800, time_above_1100, time_above_solidus, Fx_snap, Fy_snap,
              Fz_snap, Fx, Fy, Fz):
        t.zero_()


def clear_forces(Fx, Fy, Fz):
    n = Fx.numel()
    _call("waam_clear_forces", _f(Fx, n), _f(Fy, n), _f(Fz, n), n, _stream())


# ----------------------------------------------------------------- arc ----
def inject_arc_heat(H, flags, phi, f_l, norm_buf, arc_i, arc_j, arc_k, Q_w, sigma, dt, dx3, eta,
                    penetration_cells, enable_surface_weight, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(H)
    n = H.numel()
    ws, wsb = workspace_for(H)
    _call("waam_inject_arc_heat", _f(H, n), _i(flags, n), _f(f_l, n), _f(norm_buf, 1), nx, ny, nz,
          float(arc_i), float(arc_j), float(arc_k), float(Q_w), float(sigma), float(dt),
          float(dx3), float(eta), float(penetration_cells), int(enable_surface_weight), ws, wsb,
          _stream())


def inject_goldak_heat(H, flags, phi, f_l, norm_buf, arc_i, arc_j, arc_k, Q_w, dt, dx3, eta,
                       travel_sign, ff, fr, a_front, a_rear, b_axis, c_axis, penetration_cells,
                       enable_surface_weight, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(H)
    n = H.numel()
    ws, wsb = workspace_for(H)
    _call("waam_inject_goldak_heat", _f(H, n), _i(flags, n), _f(f_l, n), _f(norm_buf, 1), nx, ny,
          nz, float(arc_i), float(arc_j), float(arc_k), float(Q_w), float(dt), float(dx3),
          float(eta), float(travel_sign), float(ff), float(fr), float(a_front), float(a_rear),
          float(b_axis), float(c_axis), float(penetration_cells), int(enable_surface_weight), ws,
          wsb, _stream())


def surface_height_at(phi, flags, out, i0, j0, nz_fallback, FLAG_GAS, nz):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    nx, ny, nz_ = _dims(phi)
    if int(nz) != nz_:
        raise WaamError("surface_height_at: nz=%s does not match the field (%d)" % (nz, nz_))
    n = phi.numel()
    _call("waam_surface_height_at", _f(phi, n), _i(flags, n), _f(out, 1), nx, ny, nz_, int(i0),
          int(j0), int(nz_fallback), _stream())


# ---------------------------------------------------------- deposition ----
def feed_wire(f_src, flags, f_l, phi, H, T, rho, arc_i, arc_j, arc_k, droplet_radius, target_vol,
              T_drop, cp_rho, L_rho, rho0, vol_acc, cell_vol, FLAG_GAS, FLAG_FLUID, nx, ny, nz):
    """kernels.py:177-242: GAS cells in the droplet sphere or the column above
    the arc become liquid metal while ``vol_acc`` (0-d device float) is below
    ``target_vol``, in serial lexicographic order."""
    _flags_ok(FLAG_GAS=FLAG_GAS, FLAG_FLUID=FLAG_FLUID)
    n = int(nx) * int(ny) * int(nz)
    fp, storage = _pop(f_src, 19 * n)
    _call("waam_feed_wire", fp, storage, _i(flags, n), _f(f_l, n), _f(phi, n), _f(H, n), _f(T, n),
          _f(rho, n), int(nx), int(ny), int(nz), float(arc_i), float(arc_j), float(arc_k),
          float(droplet_radius), float(target_vol), float(T_drop), float(cp_rho), float(L_rho),
          float(rho0), _f(vol_acc, 1), float(cell_vol), _stream())


def feed_wire_momentum(ux, uy, uz, flags, f_l, arc_i, arc_j, arc_k, droplet_radius, vz_lu,
                       FLAG_GAS, nx, ny, nz):
    """kernels.py:644-676: uz = min(uz + vz_lu, 0.15) for the liquid, non-gas
    cells of the droplet's column (ux and uy are not touched)."""
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _f(ux, n)
    _f(uy, n)
    _call("waam_feed_wire_momentum", _f(uz, n), _i(flags, n), _f(f_l, n), int(nx), int(ny),
          int(nz), float(arc_i), float(arc_j), float(arc_k), float(droplet_radius), float(vz_lu),
          _stream())


def feed_wire_surface(f_src, flags, f_l, phi, H, T, rho, arc_i, arc_j, arc_k, footprint_r,
                      droplet_radius, target_vol, T_drop, cp_rho, L_rho, rho0, vol_acc, real_acc,
                      cell_vol, FLAG_GAS, FLAG_FLUID, FLAG_SOLID, nx, ny, nz):
    _flags_ok(FLAG_GAS=FLAG_GAS, FLAG_FLUID=FLAG_FLUID, FLAG_SOLID=FLAG_SOLID)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_feed_wire_surface", _f(f_src, 19 * n), _i(flags, n), _f(f_l, n), _f(phi, n),
          _f(H, n), _f(T, n), _f(rho, n), int(nx), int(ny), int(nz), float(arc_i), float(arc_j),
          float(arc_k), float(footprint_r), float(droplet_radius), float(target_vol),
          float(T_drop), float(cp_rho), float(L_rho), float(rho0), _f(vol_acc, 1),
          _f(real_acc, 1), float(cell_vol), _stream())


def deposit_droplet(f_src, flags, f_l, phi, H, T, rho, arc_i, arc_j, arc_k, footprint_radii,
                    accept_volume, droplet_radius, target_vol, T_drop, cp_rho, L_rho, rho0,
                    vol_acc, real_acc, cell_vol, FLAG_GAS, FLAG_FLUID, FLAG_SOLID, nx, ny, nz):
    """The footprint retry loop of solvers/coupled_step.py:126-151 in one launch.

    Attempt ``t`` is ``feed_wire_surface`` with ``footprint_radii[t]``; attempt
    ``t > 0`` runs only while ``real_acc`` is below ``accept_volume`` and starts
    with both budgets at ``real_acc``.  ``vol_acc``/``real_acc`` hold the
    starting budgets on entry and the final ones on return."""
    _flags_ok(FLAG_GAS=FLAG_GAS, FLAG_FLUID=FLAG_FLUID, FLAG_SOLID=FLAG_SOLID)
    n = int(nx) * int(ny) * int(nz)
    radii = (ctypes.c_float * len(footprint_radii))(*[float(r) for r in footprint_radii])
    fp, storage = _pop(f_src, 19 * n)
    _call("waam_deposit_droplet", fp, storage, _i(flags, n), _f(f_l, n), _f(phi, n),
          _f(H, n), _f(T, n), _f(rho, n), int(nx), int(ny), int(nz), float(arc_i), float(arc_j),
          float(arc_k), ctypes.cast(radii, ctypes.c_void_p), len(footprint_radii),
          float(accept_volume), float(droplet_radius), float(target_vol), float(T_drop),
          float(cp_rho), float(L_rho), float(rho0), _f(vol_acc, 1), _f(real_acc, 1),
          float(cell_vol), _stream())


def feed_wire_momentum_impact(f_src, rho, ux, uy, uz, flags, f_l, arc_i, arc_j, arc_k,
                              droplet_radius, vx_lu, vy_lu, vz_lu, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    fp, storage = _pop(f_src, 19 * n)
    _call("waam_feed_wire_momentum_impact_stored", fp, storage, _f(rho, n), _f(ux, n), _f(uy, n),
          _f(uz, n), _i(flags, n), _f(f_l, n), int(nx), int(ny), int(nz), float(arc_i),
          float(arc_j), float(arc_k), float(droplet_radius), float(vx_lu), float(vy_lu),
          float(vz_lu), _stream())


def apply_droplet_impact_pressure(Fz, flags, phi, f_l, arc_i, arc_j, arc_k, drop_radius,
                                  impact_pa, dt, dx, rho_ref, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(Fz)
    n = Fz.numel()
    _call("waam_apply_droplet_impact_pressure", _f(Fz, n), _i(flags, n), _f(phi, n), _f(f_l, n),
          nx, ny, nz, float(arc_i), float(arc_j), float(arc_k), float(drop_radius),
          float(impact_pa), float(dt), float(dx), float(rho_ref), _stream())


# ------------------------------------------------------------- thermal ----
def advect_diffuse_temperature(H, T, ux, uy, uz, flags, alpha_lu, dt, FLAG_SOLID, FLAG_GAS,
                               cp_rho, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    ws, wsb = workspace_for(H)
    _call("waam_advect_diffuse_temperature", _f(H, n), _f(T, n), _f(ux, n), _f(uy, n), _f(uz, n),
          _i(flags, n), int(nx), int(ny), int(nz), float(alpha_lu), float(dt), float(cp_rho), ws,
          wsb, _stream())


def update_phase(H, T, f_l, cp_rho, L_rho, T_solidus, T_liquidus):
    n = H.numel()
    _call("waam_update_phase", _f(H, n), _f(T, n), _f(f_l, n), n, float(cp_rho), float(L_rho),
          float(T_solidus), float(T_liquidus), _stream())


def clamp_enthalpy_ceiling_scalar(H, flags, cp_rho, T_solidus, T_liquidus, T_vapor_cap, L_rho,
                                  FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = H.numel()
    _call("waam_clamp_enthalpy_ceiling_scalar", _f(H, n), _i(flags, n), n, float(cp_rho),
          float(T_solidus), float(T_liquidus), float(T_vapor_cap), float(L_rho), _stream())


def clamp_enthalpy_floor_scalar(H, cp_rho, flags, T_floor, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = H.numel()
    _call("waam_clamp_enthalpy_floor_scalar", _f(H, n), float(cp_rho), _i(flags, n), n,
          float(T_floor), _stream())


def update_T_max(T, T_max, flags, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = T.numel()
    _call("waam_update_T_max", _f(T, n), _f(T_max, n), _i(flags, n), n, _stream())


def update_cooling_rate(T, T_prev, dT_dt, flags, dt_phys, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = T.numel()
    _call("waam_update_cooling_rate", _f(T, n), _f(T_prev, n), _f(dT_dt, n), _i(flags, n), n,
          float(dt_phys), _stream())


def apply_thermal_boundary_losses(H, T, flags, T_amb, h_conv, eps_rad, enable_conv, enable_rad,
                                  cp_rho, dt, dx, sigma_sb, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_apply_thermal_boundary_losses", _f(H, n), _f(T, n), _i(flags, n), int(nx),
          int(ny), int(nz), float(T_amb), float(h_conv), float(eps_rad), int(enable_conv),
          int(enable_rad), float(dt), float(dx), float(sigma_sb), _stream())


def apply_thermal_boundary_losses_variable(H, T, flags, cp_rho_field, T_amb, h_conv, eps_rad,
                                           enable_conv, enable_rad, dt, dx, sigma_sb, FLAG_SOLID,
                                           FLAG_GAS, nx, ny, nz):
    """kernels.py:1867-1918: the same loss as apply_thermal_boundary_losses (the
    q*dt/dx update does not use rho*cp); cp_rho_field is accepted and unused."""
    apply_thermal_boundary_losses(H, T, flags, T_amb, h_conv, eps_rad, enable_conv, enable_rad,
                                  0.0, dt, dx, sigma_sb, FLAG_SOLID, FLAG_GAS, nx, ny, nz)


# ------------------------------------------------------ material tables ----
def _host_knots(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu()
    return [float(v) for v in list(a)[:_native.TABLE_KNOTS]]


def material_tables_struct(cp_T, cp_V, k_T, k_V, mu_T, mu_V, dgamma_T, dgamma_V, n_cp, n_k, n_mu,
                           n_dgamma, cp_fallback, k_fallback, mu_fallback, dgamma_fallback):
    """WaamMaterialTables from knot arrays (lists, numpy arrays or tensors of up
    to 8 values) and counts (ints or 0-d tensors)."""
    tb = _native.WaamMaterialTables()
    for name, arr in (("cp_T", cp_T), ("cp_V", cp_V), ("k_T", k_T), ("k_V", k_V),
                      ("mu_T", mu_T), ("mu_V", mu_V), ("dgamma_T", dgamma_T),
                      ("dgamma_V", dgamma_V)):
        vals = _host_knots(arr)
        dst = getattr(tb, name)
        for q, v in enumerate(vals):
            dst[q] = v
    for name, v in (("n_cp", n_cp), ("n_k", n_k), ("n_mu", n_mu), ("n_dgamma", n_dgamma)):
        v = int(v.item() if isinstance(v, torch.Tensor) else v)
        if not 0 <= v <= _native.TABLE_KNOTS:
            raise WaamError("%s=%d outside [0, %d]" % (name, v, _native.TABLE_KNOTS))
        setattr(tb, name, v)
    tb.cp_fallback, tb.k_fallback = float(cp_fallback), float(k_fallback)
    tb.mu_fallback, tb.dgamma_fallback = float(mu_fallback), float(dgamma_fallback)
    return tb


def refresh_thermal_properties(T, cp_rho_field, alpha_lu_field, dgamma_lu_field, tau_field, cp_T,
                               cp_V, k_T, k_V, mu_T, mu_V, dgamma_T, dgamma_V, n_cp, n_k, n_mu,
                               n_dgamma, rho, dt, dx, cp_fallback, k_fallback, mu_fallback,
                               dgamma_fallback, force_scale, cp_rho_ref, alpha_lu_ref,
                               dgamma_lu_ref, tau_ref, marangoni_scale, use_tables, flags,
                               FLAG_SOLID, FLAG_GAS):
    """kernels.py:1710-1772.  The knots are read on the host (pass host arrays or
    a MaterialGPUTables' attributes to keep the call free of device reads)."""
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = T.numel()
    tb = material_tables_struct(cp_T, cp_V, k_T, k_V, mu_T, mu_V, dgamma_T, dgamma_V, n_cp, n_k,
                                n_mu, n_dgamma, cp_fallback, k_fallback, mu_fallback,
                                dgamma_fallback)
    _call("waam_refresh_thermal_properties", _f(T, n), _f(cp_rho_field, n), _f(alpha_lu_field, n),
          _f(dgamma_lu_field, n), _f(tau_field, n), _i(flags, n), n, ctypes.byref(tb),
          float(rho), float(dt), float(dx), float(force_scale), float(cp_rho_ref),
          float(alpha_lu_ref), float(dgamma_lu_ref), float(tau_ref), float(marangoni_scale),
          int(use_tables), _stream())


def advect_diffuse_temperature_variable(H, T, ux, uy, uz, flags, alpha_lu_field, cp_rho_field, dt,
                                        FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    ws, wsb = workspace_for(H)
    _call("waam_advect_diffuse_temperature_variable", _f(H, n), _f(T, n), _f(ux, n), _f(uy, n),
          _f(uz, n), _i(flags, n), _f(alpha_lu_field, n), _f(cp_rho_field, n), int(nx), int(ny),
          int(nz), float(dt), ws, wsb, _stream())


def update_phase_variable_cp(H, T, f_l, cp_rho_field, L_rho, T_solidus, T_liquidus, H_sol, H_liq):
    n = H.numel()
    _call("waam_update_phase_variable_cp", _f(H, n), _f(T, n), _f(f_l, n), _f(cp_rho_field, n), n,
          float(L_rho), float(T_solidus), float(T_liquidus), float(H_sol), float(H_liq), _stream())


def clamp_enthalpy_ceiling_variable_cp(H, flags, cp_rho_field, H_liq, T_liquidus, T_vapor_cap,
                                       FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = H.numel()
    _call("waam_clamp_enthalpy_ceiling_variable_cp", _f(H, n), _i(flags, n), _f(cp_rho_field, n),
          n, float(H_liq), float(T_liquidus), float(T_vapor_cap), _stream())


def clamp_enthalpy_floor(H, cp_rho_field, flags, T_floor, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = H.numel()
    _call("waam_clamp_enthalpy_floor", _f(H, n), _f(cp_rho_field, n), _i(flags, n), n,
          float(T_floor), _stream())


def compute_marangoni_force_variable(T, phi, f_l, Fx, Fy, Fz, flags, dgamma_lu_field, FLAG_SOLID,
                                     FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_compute_marangoni_force_variable", _f(T, n), _f(phi, n), _f(f_l, n), _f(Fx, n),
          _f(Fy, n), _f(Fz, n), _i(flags, n), _f(dgamma_lu_field, n), int(nx), int(ny), int(nz),
          _stream())


def remelt_hot_solid(T, H, f_l, phi, flags, cp_rho_field, T_solidus, T_liquidus, L_rho,
                     FLAG_SOLID, FLAG_FLUID):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_FLUID=FLAG_FLUID)
    n = T.numel()
    _call("waam_remelt_hot_solid", _f(T, n), _f(H, n), _f(f_l, n), _f(phi, n), _i(flags, n),
          _f(cp_rho_field, n), n, float(T_solidus), float(T_liquidus), float(L_rho), _stream())


def solidify_trailing_pool(T, H, f_l, phi, flags, ux, uy, uz, cp_rho_field, arc_i, arc_j, arc_k,
                           dir_x, dir_y, dir_z, lookback_cells, T_freeze, T_solidus, FLAG_SOLID,
                           FLAG_FLUID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_FLUID=FLAG_FLUID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(T)
    n = T.numel()
    _call("waam_solidify_trailing_pool", _f(T, n), _f(H, n), _f(f_l, n), _f(phi, n), _i(flags, n),
          _f(ux, n), _f(uy, n), _f(uz, n), _f(cp_rho_field, n), nx, ny, nz, float(arc_i),
          float(arc_j), float(arc_k), float(dir_x), float(dir_y), float(dir_z),
          float(lookback_cells), float(T_freeze), float(T_solidus), _stream())


def collide_srt_variable_tau(f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, tau_field,
                             C_darcy, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_collide_srt_variable_tau", _f(f_src, 19 * n), _f(f_dst, 19 * n), _f(rho, n),
          _f(ux, n), _f(uy, n), _f(uz, n), _f(Fx, n), _f(Fy, n), _f(Fz, n), _f(f_l, n),
          _i(flags, n), _f(tau_field, n), n, float(C_darcy), _stream())


def update_time_above_T(T, flags, time_above_800, time_above_1100, time_above_solidus, dt, T_800,
                        T_1100, T_solidus, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = T.numel()
    _call("waam_update_time_above_T", _f(T, n), _i(flags, n), _f(time_above_800, n),
          _f(time_above_1100, n), _f(time_above_solidus, n), n, float(dt), float(T_800),
          float(T_1100), float(T_solidus), _stream())


# ----------------------------------------------------------------- VOF ----
def advect_phi(phi_dst, phi_src, ux, uy, uz, flags, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_advect_phi", _f(phi_dst, n), _f(phi_src, n), _f(ux, n), _f(uy, n), _f(uz, n),
          _i(flags, n), int(nx), int(ny), int(nz), _stream())


def reinitialize_phi(phi, flags, FLAG_SOLID, FLAG_GAS, FLAG_FLUID):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS, FLAG_FLUID=FLAG_FLUID)
    n = phi.numel()
    _call("waam_reinitialize_phi", _f(phi, n), _i(flags, n), n, _stream())


def apply_contact_angle_phi_bc(phi, flags, theta_rad, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    ws, wsb = workspace_for(phi)
    _call("waam_apply_contact_angle_phi_bc", _f(phi, n), _i(flags, n), int(nx), int(ny), int(nz),
          float(theta_rad), ws, wsb, _stream())


def update_flags_from_phi(phi, f_l, flags, nz_solid, FLAG_FLUID, FLAG_SOLID, FLAG_GAS, FLAG_IFACE):
    _flags_ok(FLAG_FLUID=FLAG_FLUID, FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS,
              FLAG_IFACE=FLAG_IFACE)
    nx, ny, nz = _dims(phi)
    n = phi.numel()
    _call("waam_update_flags_from_phi", _f(phi, n), _f(f_l, n), _i(flags, n), nx, ny, nz,
          int(nz_solid), _stream())


def sync_phi_liquid_fraction(phi, f_l, flags, FLAG_GAS, FLAG_SOLID):
    _flags_ok(FLAG_GAS=FLAG_GAS, FLAG_SOLID=FLAG_SOLID)
    n = phi.numel()
    _call("waam_sync_phi_liquid_fraction", _f(phi, n), _f(f_l, n), _i(flags, n), n, _stream())


def remelt_hot_solid_scalar(T, H, f_l, phi, flags, cp_rho, T_solidus, T_liquidus, L_rho,
                            FLAG_SOLID, FLAG_FLUID):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_FLUID=FLAG_FLUID)
    n = T.numel()
    _call("waam_remelt_hot_solid_scalar", _f(T, n), _f(H, n), _f(f_l, n), _f(phi, n),
          _i(flags, n), n, float(cp_rho), float(T_solidus), float(T_liquidus), float(L_rho),
          _stream())


def solidify_trailing_pool_scalar(T, H, f_l, phi, flags, ux, uy, uz, cp_rho, arc_i, arc_j, arc_k,
                                  dir_x, dir_y, dir_z, lookback_cells, T_freeze, T_solidus,
                                  FLAG_SOLID, FLAG_FLUID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_FLUID=FLAG_FLUID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(T)
    n = T.numel()
    _call("waam_solidify_trailing_pool_scalar", _f(T, n), _f(H, n), _f(f_l, n), _f(phi, n),
          _i(flags, n), _f(ux, n), _f(uy, n), _f(uz, n), nx, ny, nz, float(cp_rho), float(arc_i),
          float(arc_j), float(arc_k), float(dir_x), float(dir_y), float(dir_z),
          float(lookback_cells), float(T_freeze), float(T_solidus), _stream())


def solidify_cooled_metal(T, f_l, phi, flags, ux, uy, uz, T_solidus, zero_velocity, FLAG_SOLID,
                          FLAG_FLUID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_FLUID=FLAG_FLUID, FLAG_GAS=FLAG_GAS)
    n = T.numel()
    _call("waam_solidify_cooled_metal", _f(T, n), _f(f_l, n), _f(phi, n), _i(flags, n), _f(ux, n),
          _f(uy, n), _f(uz, n), n, float(T_solidus), int(zero_velocity), _stream())


# -------------------------------------------------------------- forces ----
def compute_csf_tension(phi, flags, Fx, Fy, Fz, gamma_lu, FLAG_SOLID, FLAG_GAS, nx, ny, nz,
                        enable_wetting, theta_rad):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_compute_csf_tension", _f(phi, n), _i(flags, n), _f(Fx, n), _f(Fy, n), _f(Fz, n),
          int(nx), int(ny), int(nz), float(gamma_lu), int(enable_wetting), float(theta_rad),
          _stream())


compute_csf_wetting = compute_csf_tension


def compute_marangoni_force(T, phi, f_l, Fx, Fy, Fz, flags, dgamma_dT, dx, FLAG_SOLID, FLAG_GAS,
                            nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_compute_marangoni_force", _f(T, n), _f(phi, n), _f(f_l, n), _f(Fx, n), _f(Fy, n),
          _f(Fz, n), _i(flags, n), int(nx), int(ny), int(nz), float(dgamma_dT), _stream())


def apply_gas_shear_stress(Fx, Fy, phi, flags, arc_i, arc_j, arc_k, sigma, tau_peak_pa, dt, dx,
                           rho_ref, FLAG_SOLID, FLAG_GAS):
    """kernels.py:1094-1141 (arc_k is not used by the reference either)."""
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(Fx)
    n = Fx.numel()
    _call("waam_apply_gas_shear_stress", _f(Fx, n), _f(Fy, n), _f(phi, n), _i(flags, n), nx, ny,
          nz, float(arc_i), float(arc_j), float(sigma), float(tau_peak_pa), float(dt), float(dx),
          float(rho_ref), _stream())


def apply_vapor_recoil(Fz, T, phi, flags, arc_i, arc_j, arc_k, sigma, recoil_pa, T_ref, dt, dx,
                       rho_ref, FLAG_SOLID, FLAG_GAS):
    """kernels.py:995-1028."""
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(Fz)
    n = Fz.numel()
    _call("waam_apply_vapor_recoil", _f(Fz, n), _f(T, n), _f(phi, n), _i(flags, n), nx, ny, nz,
          float(arc_i), float(arc_j), float(sigma), float(recoil_pa), float(T_ref), float(dt),
          float(dx), float(rho_ref), _stream())


def apply_vapor_recoil_clausius_clapeyron(Fz, T, phi, flags, arc_i, arc_j, arc_k, sigma, P_ref_Pa,
                                          T_boil_K, L_vapor_J_kg, R_spec_J_kgK, C_acc, dt, dx,
                                          rho_ref, FLAG_SOLID, FLAG_GAS):
    """kernels.py:1046-1091."""
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(Fz)
    n = Fz.numel()
    _call("waam_apply_vapor_recoil_cc", _f(Fz, n), _f(T, n), _f(phi, n), _i(flags, n), nx, ny,
          nz, float(arc_i), float(arc_j), float(sigma), float(P_ref_Pa), float(T_boil_K),
          float(L_vapor_J_kg), float(R_spec_J_kgK), float(C_acc), float(dt), float(dx),
          float(rho_ref), _stream())


def apply_arc_pressure(Fz, flags, phi, arc_i, arc_j, arc_k, sigma, pressure_pa, dt, dx, rho_ref,
                       FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(Fz)
    n = Fz.numel()
    _call("waam_apply_arc_pressure", _f(Fz, n), _i(flags, n), _f(phi, n), nx, ny, nz,
          float(arc_i), float(arc_j), float(arc_k), float(sigma), float(pressure_pa), float(dt),
          float(dx), float(rho_ref), _stream())


def add_buoyancy(T, Fz, f_l, flags, g_lu, beta, T_ref, rho_ref, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = T.numel()
    _call("waam_add_buoyancy", _f(T, n), _f(Fz, n), _f(f_l, n), _i(flags, n), n, float(g_lu),
          float(beta), float(T_ref), float(rho_ref), _stream())


def add_hydrostatic_gravity(Fz, f_l, flags, rho_ref, g_lu, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = Fz.numel()
    _call("waam_add_hydrostatic_gravity", _f(Fz, n), _f(f_l, n), _i(flags, n), n, float(rho_ref),
          float(g_lu), _stream())


def clamp_body_force_magnitude(Fx, Fy, Fz, flags, F_max_lu, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = Fx.numel()
    _call("waam_clamp_body_force_magnitude", _f(Fx, n), _f(Fy, n), _f(Fz, n), _i(flags, n), n,
          float(F_max_lu), _stream())


def snapshot_forces(Fx, Fy, Fz, Fx_snap, Fy_snap, Fz_snap):
    if Fx_snap.data_ptr() == Fx.data_ptr():
        return  # the snapshot aliases the force field
    n = Fx.numel()
    _call("waam_snapshot_forces", _f(Fx, n), _f(Fy, n), _f(Fz, n), _f(Fx_snap, n),
          _f(Fy_snap, n), _f(Fz_snap, n), n, _stream())


# ------------------------------------------------------------------ LBM ----
def collide_srt(f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, tau, omega, dt_lu, C_darcy,
                FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_collide_srt", _f(f_src, 19 * n), _f(f_dst, 19 * n), _f(rho, n), _f(ux, n),
          _f(uy, n), _f(uz, n), _f(Fx, n), _f(Fy, n), _f(Fz, n), _f(f_l, n), _i(flags, n), n,
          float(omega), float(C_darcy), _stream())


def collide_mrt(f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, EX, EY, EZ, W, OPP,
                omega_s, omega_b, C_darcy, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_collide_mrt", _f(f_src, 19 * n), _f(f_dst, 19 * n), _f(rho, n), _f(ux, n),
          _f(uy, n), _f(uz, n), _f(Fx, n), _f(Fy, n), _f(Fz, n), _f(f_l, n), _i(flags, n), n,
          float(omega_s), float(omega_b), float(C_darcy), _stream())


def clamp_velocity_mach(ux, uy, uz, flags, u_max_lu, FLAG_SOLID, FLAG_GAS):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = ux.numel()
    _call("waam_clamp_velocity_mach", _f(ux, n), _f(uy, n), _f(uz, n), _i(flags, n), n,
          float(u_max_lu), _stream())


def stream(f_src, f_dst, flags, FLAG_SOLID, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_stream", _f(f_src, 19 * n), _f(f_dst, 19 * n), _i(flags, n), int(nx), int(ny),
          int(nz), _stream())


# ---------------------------------------------- verification set-ups ------
# The reference's validation scripts build their cases with these kernels
# (kernels.py:2085-2155, 3089-3179); they are set-up code, not step code.
def init_poiseuille_channel(f, rho, ux, uy, uz, f_l, phi, flags, rho0, ny, nz, fx_lu, nu_lu,
                            FLAG_FLUID, FLAG_SOLID):
    state_changed()
    nx = rho.shape[0]
    dev = rho.device
    j = torch.arange(ny, device=dev).view(1, ny, 1).expand(nx, ny, nz)
    k = torch.arange(nz, device=dev).view(1, 1, nz).expand(nx, ny, nz)
    wall = (j == 0) | (j == ny - 1) | (k == 0) | (k == nz - 1)
    flags.copy_(torch.where(wall, torch.full_like(flags, FLAG_SOLID), torch.full_like(flags, FLAG_FLUID)))
    rho.fill_(float(rho0))
    uy.zero_()
    uz.zero_()
    f_l.fill_(1.0)
    phi.fill_(1.0)
    h = torch.tensor(float(ny - 2), dtype=torch.float32, device=dev)
    y = (j - 1).to(torch.float32)
    c = torch.tensor(float(fx_lu), dtype=torch.float32) / (torch.tensor(2.0) * torch.tensor(float(nu_lu), dtype=torch.float32))
    prof = c.to(dev) * y * (h - 1.0 - y)
    ux.copy_(torch.where(wall, torch.zeros_like(prof), prof))
    u2 = ux * ux + uy * uy + uz * uz
    from .grid import EX as _EX, EY as _EY, EZ as _EZ
    for q in range(19):
        wq = torch.tensor(_W[q], dtype=torch.float32)
        eu = _EX[q] * ux + _EY[q] * uy + _EZ[q] * uz
        eq = wq.to(dev) * float(rho0) * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * u2)
        f[q].copy_(torch.where(wall, (wq * float(rho0)).to(dev).expand_as(eq), eq))


def set_uniform_Fx(Fx, Fy, Fz, fx_lu, flags, FLAG_FLUID):
    fluid = flags == FLAG_FLUID
    Fx.copy_(torch.where(fluid, torch.full_like(Fx, float(fx_lu)), torch.zeros_like(Fx)))
    Fy.zero_()
    Fz.zero_()


def prescribe_gaussian_pulse(T, H, f_l, flags, T_bg, A, sigma_m, cx, cy, cz, dx, cp_rho, FLAG_GAS):
    state_changed()
    nx, ny, nz = T.shape
    dev = T.device
    f32 = dict(dtype=torch.float32, device=dev)
    inv2s2 = torch.tensor(1.0, dtype=torch.float32) / (torch.tensor(2.0) * torch.tensor(float(sigma_m), dtype=torch.float32) ** 2)
    dxv = float(dx)
    px = torch.arange(nx, **f32).view(nx, 1, 1) * dxv - float(cx)
    py = torch.arange(ny, **f32).view(1, ny, 1) * dxv - float(cy)
    pz = torch.arange(nz, **f32).view(1, 1, nz) * dxv - float(cz)
    r2 = px * px + py * py + pz * pz
    Tc = float(T_bg) + float(A) * torch.exp(-r2 * inv2s2.to(dev))
    keep = flags == FLAG_GAS
    T.copy_(torch.where(keep, T, Tc))
    H.copy_(torch.where(keep, H, float(cp_rho) * Tc))
    f_l.copy_(torch.where(keep, f_l, torch.ones_like(f_l)))


def sync_T_from_H(H, T, cp_rho):
    state_changed()
    T.copy_(H / float(cp_rho))


def init_stefan_liquid_column(T, H, f_l, phi, flags, nz_solid, T_amb, T_init, cp_rho, L_rho,
                              T_solidus, T_liquidus, FLAG_FLUID, FLAG_SOLID):
    state_changed()
    nx, ny, nz = T.shape
    k = torch.arange(nz, device=T.device).view(1, 1, nz).expand(nx, ny, nz)
    sol = k < int(nz_solid)
    cp = torch.tensor(float(cp_rho), dtype=torch.float32)
    H_liq = cp * float(T_liquidus) + torch.tensor(float(L_rho), dtype=torch.float32)
    flags.copy_(torch.where(sol, torch.full_like(flags, FLAG_SOLID), torch.full_like(flags, FLAG_FLUID)))
    phi.fill_(1.0)
    f_l.copy_(torch.where(sol, torch.zeros_like(f_l), torch.ones_like(f_l)))
    T.copy_(torch.where(sol, torch.full_like(T, float(T_amb)), torch.full_like(T, float(T_init))))
    h_liq_val = (H_liq + cp * (torch.tensor(float(T_init), dtype=torch.float32) - float(T_liquidus))).item()
    h_sol_val = (cp * float(T_amb)).item()
    H.copy_(torch.where(sol, torch.full_like(H, h_sol_val), torch.full_like(H, h_liq_val)))


def clamp_substrate_enthalpy(H, T, f_l, flags, nz_solid, T_amb, cp_rho, FLAG_SOLID):
    state_changed()
    nx, ny, nz = T.shape
    k = torch.arange(nz, device=T.device).view(1, 1, nz).expand(nx, ny, nz)
    m = (k < int(nz_solid)) & (flags == FLAG_SOLID)
    h = (torch.tensor(float(cp_rho), dtype=torch.float32) * float(T_amb)).item()
    H.copy_(torch.where(m, torch.full_like(H, h), H))
    T.copy_(torch.where(m, torch.full_like(T, float(T_amb)), T))
    f_l.copy_(torch.where(m, torch.zeros_like(f_l), f_l))


def bind_velocity_set(grid):
    """Kept for API compatibility (kernels.py:54-56)."""
    return None


__all__ = [n for n in dir() if not n.startswith("_") and n not in ("math", "torch")]


# ------------------------------------------------------------- Lorentz ----
# kernels.py:1236-1513 (electric potential, current density, self field, J x B)

def elec_build_sigma(sigma, f_l, flags, sigma_liquid, sigma_solid, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = sigma.numel()
    _call("waam_elec_build_sigma", _f(sigma, n), _f(f_l, n), _i(flags, n), n,
          float(sigma_liquid), float(sigma_solid), _stream())


def elec_build_sigma_mask(sigma, fixed, f_l, flags, sigma_liquid, sigma_solid, nz_solid):
    """elec_build_sigma plus the uint8 mask of the cells the Jacobi sweep holds at 0."""
    nx, ny, nz = _dims(sigma)
    if fixed.dtype != torch.uint8 or tuple(fixed.shape) != (nx, ny, nz):
        raise WaamError("elec_build_sigma_mask: fixed must be uint8 (nx, ny, nz)")
    n = nx * ny * nz
    _call("waam_elec_build_sigma_mask", _f(sigma, n), fixed.data_ptr(), _f(f_l, n),
          _i(flags, n), nx, ny, nz, float(sigma_liquid), float(sigma_solid), int(nz_solid),
          _stream())


def elec_jacobi_chunk(phi_a, phi_b, sigma, source, fixed, dx, omega_j, n_sweeps, arc_k,
                      sigma_cells, diff_buf, norm_buf):
    """n_sweeps Jacobi sweeps phi_a -> phi_b -> ..., the last with the L1 check;
    the last iterate ends in phi_b when n_sweeps is odd, else in phi_a."""
    nx, ny, nz = _dims(phi_a)
    if fixed.dtype != torch.uint8 or tuple(fixed.shape) != (nx, ny, nz):
        raise WaamError("elec_jacobi_chunk: fixed must be uint8 (nx, ny, nz)")
    n = nx * ny * nz
    ws, wsb = workspace_for(phi_a)
    _call("waam_elec_jacobi_chunk", _f(phi_a, n), _f(phi_b, n), _f(sigma, n), _f(source, n),
          fixed.data_ptr(), nx, ny, nz, float(dx), float(omega_j), int(n_sweeps), float(arc_k),
          float(sigma_cells), _f(diff_buf, 1), _f(norm_buf, 1), ws, wsb, _stream())


def elec_prepare(sigma, fixed, phi_b, f_l, flags, sigma_liquid, sigma_solid, nz_solid, live,
                 zero, counts):
    """Conductivity map, fixed-cell mask and the live / newly fixed cell lists of
    one potential solve (zeroes phi_b at the newly fixed cells)."""
    nx, ny, nz = _dims(sigma)
    n = nx * ny * nz
    for t, name in ((live, "live"), (zero, "zero"), (counts, "counts")):
        if t.dtype != torch.int32 or not t.is_contiguous():
            raise WaamError("elec_prepare: %s must be contiguous int32" % name)
    if live.numel() < n or zero.numel() < n:
        raise WaamError("elec_prepare: live / zero lists need nx*ny*nz entries")
    _call("waam_elec_prepare", _f(sigma, n), fixed.data_ptr(), _f(phi_b, n), _f(f_l, n),
          _i(flags, n), nx, ny, nz, float(sigma_liquid), float(sigma_solid), int(nz_solid),
          live.data_ptr(), zero.data_ptr(), counts.data_ptr(), counts.numel(), _stream())


def elec_jacobi_live(phi_a, phi_b, sigma, source, live, zero, counts, dx, omega_j, n_sweeps,
                     first_chunk, arc_k_dev, sigma_cells, diff_buf, norm_buf):
    """n_sweeps sweeps over the live cells (see waam_elec_jacobi_live); arc_k_dev:
    a one-element float32 device tensor holding the arc height in cells."""
    nx, ny, nz = _dims(phi_a)
    n = nx * ny * nz
    ws, wsb = workspace_for(phi_a)
    _call("waam_elec_jacobi_live", _f(phi_a, n), _f(phi_b, n), _f(sigma, n), _f(source, n),
          live.data_ptr(), zero.data_ptr(), counts.data_ptr(), nx, ny, nz, float(dx),
          float(omega_j), int(n_sweeps), 1 if first_chunk else 0, _f(arc_k_dev, 1),
          float(sigma_cells), _f(diff_buf, 1), _f(norm_buf, 1), ws, wsb, _stream())


def elec_clear_source(source):
    source.zero_()


def elec_inject_arc_source(source, arc_i, arc_j, arc_k, sigma_cells, current_A, dx, nz):
    nx, ny, nz_ = _dims(source)
    if int(nz) != nz_:
        raise WaamError("elec_inject_arc_source: nz=%d does not match the field (%d)" % (nz, nz_))
    _call("waam_elec_inject_arc_source", _f(source), nx, ny, nz_, float(arc_i), float(arc_j),
          float(arc_k), float(sigma_cells), float(current_A), float(dx), _stream())


def elec_arc_source(source, arc_i, arc_j, arc_k, sigma_cells, current_A, dx):
    """elec_clear_source + elec_inject_arc_source + elec_normalize_source in one call."""
    nx, ny, nz = _dims(source)
    ws, wsb = workspace_for(source)
    _call("waam_elec_arc_source", _f(source), nx, ny, nz, float(arc_i), float(arc_j),
          float(arc_k), float(sigma_cells), float(current_A), float(dx), ws, wsb, _stream())


def elec_arc_source_dev(source, arc_i, arc_j, arc_k_dev, sigma_cells, current_A, dx):
    """elec_arc_source with the arc height in a one-element device tensor."""
    nx, ny, nz = _dims(source)
    ws, wsb = workspace_for(source)
    _call("waam_elec_arc_source_dev", _f(source), nx, ny, nz, float(arc_i), float(arc_j),
          _f(arc_k_dev, 1), float(sigma_cells), float(current_A), float(dx), ws, wsb, _stream())


def elec_fields(Jx, Jy, Jz, Bx, By, Bz, bins, phi, sigma, flags, arc_i, arc_j, dx, bin_dr_cells,
                mu0, n_bins):
    """elec_compute_J, elec_bin_axial_current, elec_prefix_bins, elec_B_axisymmetric."""
    nx, ny, nz = _dims(phi)
    n = nx * ny * nz
    if tuple(bins.shape) != (nz, int(n_bins)):
        raise WaamError("elec_fields: bins must be (nz, n_bins)")
    ws, wsb = workspace_for(phi)
    _call("waam_elec_fields", _f(Jx, n), _f(Jy, n), _f(Jz, n), _f(Bx, n), _f(By, n), _f(Bz, n),
          _f(bins, nz * int(n_bins)), _f(phi, n), _f(sigma, n), _i(flags, n), nx, ny, nz,
          float(arc_i), float(arc_j), float(dx), float(bin_dr_cells), float(mu0), int(n_bins),
          ws, wsb, _stream())


def elec_normalize_source(source, target_current_A, dx):
    ws, wsb = workspace_for(source)
    _call("waam_elec_normalize_source", _f(source), source.numel(), float(target_current_A),
          float(dx), ws, wsb, _stream())


def elec_init_ground(phi, flags, nz_solid, FLAG_SOLID):
    _flags_ok(FLAG_SOLID=FLAG_SOLID)
    _call("waam_elec_init_ground", _f(phi), phi.numel(), _stream())


def elec_jacobi_step(phi_in, phi_out, sigma, source, flags, dx, omega_j, FLAG_GAS, FLAG_SOLID,
                     nz_solid, nx, ny, nz):
    _flags_ok(FLAG_GAS=FLAG_GAS, FLAG_SOLID=FLAG_SOLID)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_elec_jacobi_step", _f(phi_in, n), _f(phi_out, n), _f(sigma, n), _f(source, n),
          _i(flags, n), int(nx), int(ny), int(nz), float(dx), float(omega_j), int(nz_solid),
          _stream())


def elec_jacobi_step_l1(phi_in, phi_out, sigma, source, flags, dx, omega_j, nz_solid, diff_buf,
                        norm_buf):
    """elec_jacobi_step then elec_l1_diff(phi_out, phi_in, diff_buf, norm_buf), one pass."""
    nx, ny, nz = _dims(phi_in)
    n = phi_in.numel()
    ws, wsb = workspace_for(phi_in)
    _call("waam_elec_jacobi_step_l1", _f(phi_in, n), _f(phi_out, n), _f(sigma, n),
          _f(source, n), _i(flags, n), nx, ny, nz, float(dx), float(omega_j), int(nz_solid),
          _f(diff_buf, 1), _f(norm_buf, 1), ws, wsb, _stream())


def elec_l1_diff(a, b, diff_buf, norm_buf):
    nx, ny, nz = _dims(a)
    ws, wsb = workspace_for(a)
    _call("waam_elec_l1_diff", _f(a), _f(b, a.numel()), _f(diff_buf, 1), _f(norm_buf, 1), nx,
          ny, nz, ws, wsb, _stream())


def elec_compute_J(Jx, Jy, Jz, phi, sigma, flags, dx, FLAG_GAS, nx, ny, nz):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_elec_compute_J", _f(Jx, n), _f(Jy, n), _f(Jz, n), _f(phi, n), _f(sigma, n),
          _i(flags, n), int(nx), int(ny), int(nz), float(dx), _stream())


def elec_bin_axial_current(Jz, bins, arc_i, arc_j, dx, bin_dr_cells, n_bins, nz):
    nx, ny, nz_ = _dims(Jz)
    if tuple(bins.shape) != (nz_, int(n_bins)):
        raise WaamError("elec_bin_axial_current: bins must be (nz, n_bins)")
    ws, wsb = workspace_for(Jz)
    _call("waam_elec_bin_axial_current", _f(Jz), _f(bins, nz_ * int(n_bins)), nx, ny, nz_,
          float(arc_i), float(arc_j), float(dx), float(bin_dr_cells), int(n_bins), ws, wsb,
          _stream())


def elec_prefix_bins(bins, n_bins, nz):
    _call("waam_elec_prefix_bins", _f(bins, int(n_bins) * int(nz)), int(n_bins), int(nz),
          _stream())


def elec_B_axisymmetric(Bx, By, Bz, bins, arc_i, arc_j, dx, bin_dr_cells, mu0, n_bins, nz):
    nx, ny, nz_ = _dims(Bx)
    n = Bx.numel()
    _call("waam_elec_B_axisymmetric", _f(Bx, n), _f(By, n), _f(Bz, n),
          _f(bins, nz_ * int(n_bins)), nx, ny, nz_, float(arc_i), float(arc_j), float(dx),
          float(bin_dr_cells), float(mu0), int(n_bins), _stream())


def apply_lorentz_JxB(Fx, Fy, Fz, Jx, Jy, Jz, Bx, By, Bz, f_l, flags, dt, dx, rho_ref, FLAG_GAS):
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = Fx.numel()
    _call("waam_apply_lorentz_JxB", _f(Fx, n), _f(Fy, n), _f(Fz, n), _f(Jx, n), _f(Jy, n),
          _f(Jz, n), _f(Bx, n), _f(By, n), _f(Bz, n), _f(f_l, n), _i(flags, n), n, float(dt),
          float(dx), float(rho_ref), _stream())


# ------------------------------------------------------------- tracers ----
# kernels.py:3182-3255 (porosity tracers; no feedback into the fields)
_tracer_calls = [0]


def inject_tracers(pos, active, head, max_tracers, arc_x, arc_y, arc_z, sigma_m, spawn_count,
                   seed=None):
    """Spawn ``spawn_count`` tracers into the ring buffer (kernels.py:3182-3205).

    ``seed`` selects the random offsets (a counter-based hash; the reference's
    ti.random() is not reproducible); by default successive calls use 0, 1, 2..."""
    if seed is None:
        seed = _tracer_calls[0]
        _tracer_calls[0] += 1
    m = int(max_tracers)
    if pos.shape != (m, 3) or active.numel() != m:
        raise WaamError("inject_tracers: pos must be (max_tracers, 3), active (max_tracers,)")
    _call("waam_inject_tracers", _f(pos), _i(active), _i(head, 1), m, float(arc_x),
          float(arc_y), float(arc_z), float(sigma_m), int(spawn_count),
          int(seed) & 0xFFFFFFFFFFFFFFFF, _stream())


def advect_tracers(pos, active, ux, uy, uz, f_l, flags, dx, dt, max_tracers, FLAG_SOLID,
                   FLAG_GAS):
    """kernels.py:3207-3255: nearest-cell velocity, pos += u * dx."""
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS)
    nx, ny, nz = _dims(ux)
    n = ux.numel()
    m = int(max_tracers)
    if pos.shape != (m, 3) or active.numel() != m:
        raise WaamError("advect_tracers: pos must be (max_tracers, 3), active (max_tracers,)")
    _call("waam_advect_tracers", _f(pos), _i(active), _f(ux, n), _f(uy, n), _f(uz, n),
          _f(f_l, n), _i(flags, n), nx, ny, nz, float(dx), m, _stream())


# ------------------------------------------------------------ telemetry ----
TELEMETRY_BYTES = ctypes.sizeof(_native.WaamTelemetry)


def telemetry_record(device):
    """Device buffer for one WaamTelemetry record."""
    return torch.zeros(TELEMETRY_BYTES, dtype=torch.uint8, device=device)


def telemetry_pool(T, f_l, phi, dT_dt, ux, uy, uz, H, flags, tracer_active, max_tracers,
                   nz_solid, record):
    """Every pool aggregate of get_telemetry into ``record`` (two launches, no sync)."""
    nx, ny, nz = _dims(T)
    n = T.numel()
    if record.numel() < TELEMETRY_BYTES or record.dtype != torch.uint8 or not record.is_cuda:
        raise WaamError("record must be a CUDA uint8 tensor of %d bytes" % TELEMETRY_BYTES)
    ws, wsb = workspace_for(T)
    act = _i(tracer_active) if tracer_active is not None and max_tracers > 0 else None
    _call("waam_telemetry_pool", _f(T, n), _f(f_l, n), _f(phi, n), _f(dT_dt, n), _f(ux, n),
          _f(uy, n), _f(uz, n), None if H is None else _f(H, n),
          None if flags is None else _i(flags, n), act, int(max_tracers), nx, ny, nz,
          int(nz_solid), record.data_ptr(), ws, wsb, _stream())


def read_telemetry(record):
    """The record as a WaamTelemetry struct (one device-to-host read)."""
    host = record[:TELEMETRY_BYTES].cpu().numpy().tobytes()
    return _native.WaamTelemetry.from_buffer_copy(host)


def telemetry_pool_reduce(T, f_l, phi, dT_dt, ux, uy, uz, n_buf, T_peak_buf, cool_buf, u2_buf,
                          i_sum_buf, i_min_buf, i_max_buf, T_global_buf):
    """kernels.py:3424-3468 with its 0-d output buffers (filled on the device)."""
    rec = telemetry_record(T.device)
    telemetry_pool(T, f_l, phi, dT_dt, ux, uy, uz, None, None, None, 0, 0, rec)
    d = rec[:40].view(torch.float64)
    q = rec[40:56].view(torch.int64)
    ints = rec[56:64].view(torch.int32)
    has = q[0] > 0
    n_buf.copy_(q[0].to(n_buf.dtype))
    T_global_buf.copy_(d[0].to(T_global_buf.dtype))
    T_peak_buf.copy_(d[1].to(T_peak_buf.dtype))
    cool_buf.copy_(d[2].to(cool_buf.dtype))
    u2_buf.copy_(d[3].to(u2_buf.dtype))
    i_sum_buf.copy_(q[1].to(i_sum_buf.dtype))
    i_min_buf.copy_(torch.where(has, ints[0].to(torch.float64),
                                torch.full_like(d[0], 1.0e9)).to(i_min_buf.dtype))
    i_max_buf.copy_(torch.where(has, ints[1].to(torch.float64),
                                torch.full_like(d[0], -1.0e9)).to(i_max_buf.dtype))


def extract_fl_yz_slice(f_l, out, i_slice, ny, nz):
    """kernels.py:3471-3481."""
    out.copy_(f_l[int(i_slice)].reshape(out.shape))


def probe_sample(T, f_l, cells, row):
    """T and f_l at cell indices ``cells`` (-1: outside) into ``row`` (device,
    2 floats per probe), export/probes.py:90-107."""
    if len(cells) > _native.MAX_PROBES:
        raise WaamError("at most %d probes" % _native.MAX_PROBES)
    ps = _native.WaamProbeSet()
    ps.n_probes = len(cells)
    for q, c in enumerate(cells):
        ps.cell[q] = int(c)
    _call("waam_probe_sample", _f(T), _f(f_l), ctypes.byref(ps), _f(row), _stream())


def bead_height_k(flags, nz_solid, out):
    """Max k of SOLID cells at or above nz_solid into the 0-d int32 ``out`` (-1: none)."""
    nx, ny, nz = _dims(flags)
    _call("waam_bead_height", _i(flags), nx, ny, nz, int(nz_solid), _i(out), _stream())


# -------------------------------------------------------- moving window ----
def _f32_bits(v):
    import numpy as np
    return int(np.array([v], dtype=np.float32).view(np.uint32)[0])


def _pop_reset_bits(t, q, rho0):
    """Raw bits of the reset population W[q] * rho0 in the storage of ``t``."""
    import numpy as np
    feq = np.float32(_W[q]) * np.float32(rho0)
    if t.dtype == torch.float32:
        return _f32_bits(feq)
    off = np.float32(feq - np.float32(_W[q]))
    h = torch.tensor([float(off)], dtype=torch.float32).to(t.dtype).view(torch.int16)
    return int(h.item()) & 0xFFFF


def shift_simulation_window_x(n_shift, f_a, f_b, T, H, f_l, phi, flags, T_max, T_prev, dT_dt,
                              time_above_800, time_above_1100, time_above_solidus, rho, ux, uy,
                              uz, Fx, Fy, Fz, cp_rho_field, alpha_lu_field, dgamma_lu_field,
                              tau_field, T_amb, cp_rho, rho0, nz_solid, FLAG_SOLID, FLAG_GAS,
                              FLAG_FLUID, nx, ny, nz):
    """kernels.py:2620-2723 in one launch (every plane moves in place)."""
    import numpy as np
    _flags_ok(FLAG_SOLID=FLAG_SOLID, FLAG_GAS=FLAG_GAS, FLAG_FLUID=FLAG_FLUID)
    n = int(nx) * int(ny) * int(nz)
    planes = []

    def add(t, mode, below=0, above=0, elem=4):
        planes.append(_native.WaamShiftPlane(t.data_ptr(), elem, mode, below, above))

    C_, K_, B_ = _native.SHIFT_CONST, _native.SHIFT_KEEP, _native.SHIFT_BY_K
    amb = _f32_bits(T_amb)
    for t, mode, below, above in (
            (T, C_, amb, 0), (H, C_, _f32_bits(np.float32(cp_rho) * np.float32(T_amb)), 0),
            (f_l, C_, 0, 0), (phi, B_, _f32_bits(1.0), 0), (T_max, C_, amb, 0),
            (T_prev, C_, amb, 0), (dT_dt, C_, 0, 0), (time_above_800, C_, 0, 0),
            (time_above_1100, C_, 0, 0), (time_above_solidus, C_, 0, 0),
            (rho, C_, _f32_bits(rho0), 0), (ux, C_, 0, 0), (uy, C_, 0, 0), (uz, C_, 0, 0),
            (Fx, C_, 0, 0), (Fy, C_, 0, 0), (Fz, C_, 0, 0), (cp_rho_field, K_, 0, 0),
            (alpha_lu_field, K_, 0, 0), (dgamma_lu_field, K_, 0, 0), (tau_field, K_, 0, 0)):
        _f(t, n)
        add(t, mode, below, above)
    _i(flags, n)
    add(flags, B_, int(FLAG_SOLID), int(FLAG_GAS))
    for buf in (f_a, f_b):
        _pop(buf, 19 * n)
        elem = buf.element_size()
        for q in range(19):
            add(buf[q], C_, _pop_reset_bits(buf, q, rho0), 0, elem)
    arr = (_native.WaamShiftPlane * len(planes))(*planes)
    _call("waam_shift_window_x", ctypes.cast(arr, ctypes.c_void_p), len(planes), int(n_shift),
          int(nx), int(ny), int(nz), int(nz_solid), _stream())


def shift_tracers_x(pos, max_tracers, shift_m):
    _call("waam_shift_tracers_x", _f(pos), int(max_tracers), float(shift_m), _stream())


# --------------------------------------------------------------- export ----
def compute_curvature_field(phi, flags, kappa_out, FLAG_GAS, nx, ny, nz):
    """kernels.py:3354-3376."""
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_compute_curvature_field", _f(phi, n), _i(flags, n), _f(kappa_out, n), int(nx),
          int(ny), int(nz), _stream())


def compute_vorticity_magnitude(ux, uy, uz, flags, vort_out, dx, dt, FLAG_GAS, nx, ny, nz):
    """kernels.py:3379-3418."""
    _flags_ok(FLAG_GAS=FLAG_GAS)
    n = int(nx) * int(ny) * int(nz)
    _call("waam_compute_vorticity_magnitude", _f(ux, n), _f(uy, n), _f(uz, n), _i(flags, n),
          _f(vort_out, n), int(nx), int(ny), int(nz), float(dx), float(dt), _stream())


def export_pack(channels, nx, ny, nz, out):
    """Pack channels (op, a, b, c, sources) into ``out`` (device, 4-byte
    elements, len(channels) * nx * ny * nz) in VTK cell order, one launch."""
    n = int(nx) * int(ny) * int(nz)
    if len(channels) > _native.MAX_EXPORT_CHANNELS:
        raise WaamError("at most %d export channels" % _native.MAX_EXPORT_CHANNELS)
    if out.numel() * out.element_size() < 4 * n * len(channels) or not out.is_cuda:
        raise WaamError("export staging buffer too small")
    arr = (_native.WaamExportChannel * max(1, len(channels)))()
    for q, (op, a, b, c, srcs) in enumerate(channels):
        arr[q].op, arr[q].a, arr[q].b, arr[q].c = op, a, b, c
        for s, t in enumerate(srcs):
            if t.numel() != n or not t.is_contiguous() or t.element_size() != 4 or not t.is_cuda:
                raise WaamError("export source must be a contiguous 4-byte CUDA field")
            arr[q].src[s] = t.data_ptr()
    _call("waam_export_pack", ctypes.cast(arr, ctypes.c_void_p), len(channels), int(nx), int(ny),
          int(nz), out.data_ptr(), _stream())
