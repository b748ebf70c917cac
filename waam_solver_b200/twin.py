"""WAAMTwin driver on the B200 backend (reference twin.py:37-869, the parts on
the step path: construction, derived lattice scalars, reset, step, run,
run_path, telemetry).

The constructor takes the reference's keyword arguments.  Features outside
the accelerated path (vapour recoil, gas shear, moving window) raise
instead of silently changing the physics.
"""
from __future__ import annotations

import logging
import math

import numpy as np
import torch

from . import kernels
from .coupled_step import coupled_step
from .gpu_tables import MaterialGPUTables
from .grid import WAAMGrid
from .materials import MaterialProps, load_material
from .physics.arc import create_heat_source
from .physics.bead_geometry import bead_height_m_from_k, toe_angle_from_column
from .physics.deposition_balance import (droplet_mass_kg, expected_deposited_mass_kg,
                                         infer_transfer_mode, wire_mass_flux_kg_s)
from .physics.electrical_stickout import droplet_entry_temperature_K
from .physics.weld_forces import arc_pressure_peak_pa, droplet_impact_velocity_m_s
from .torch_path import plan_path, run_path

RHO_LATTICE = 1.0
log = logging.getLogger("waam_solver_b200")


class WAAMTwin:
    def __init__(self, material="ER70S-6", nx=256, ny=128, nz=64, dx=2e-4, arc_power_W=2800.0,
                 arc_efficiency=0.8, high_sulphur=False, T_ambient=300.0, use_srt=True,
                 C_darcy=1.6e5, arc_pressure_pa=500.0, droplet_freq_hz=50.0, max_tracers=None,
                 enable_heat_loss=False, h_conv=25.0, eps_rad=0.3, enable_convection=True,
                 enable_radiation=False, heat_source="gaussian2d", enable_vof=False,
                 enable_recoil=False, enable_csf_tension=False, enable_deposition_momentum=True,
                 enable_lorentz=False, enable_gas_shear=False,
                 enable_droplet_impact_pressure=True, use_recoil_clausius_clapeyron=True,
                 enable_substrate_growth=False, enable_moving_window=False, enable_wetting=False,
                 enable_hydrostatic_gravity=False, enable_bead_freeze=False, enable_ctwd=False,
                 contact_angle_deg=None, deposition_superheat_K=500.0,
                 deposition_footprint_sigma_scale=1.0, stickout_mm=12.0, ctwd_mm=15.0,
                 layer_height_mm=1.2, recoil_pressure_pa=5000.0, welding_current_A=140.0,
                 sigma_liquid_Sm=1.0e6, sigma_solid_Sm=1.0e5, lorentz_jacobi_iters=40,
                 lorentz_jacobi_omega=0.85, gas_jet_velocity_m_s=12.0, gas_shear_coeff=1.0,
                 T_boiling_K=3100.0, P_vapor_ref_Pa=101325.0, L_vapor_J_kg=6.0e6,
                 R_spec_vapor_J_kgK=450.0, travel_speed_m_s=0.0, use_variable_tau=True,
                 enable_enthalpy_cap=True, T_vapor_cap_K=3200.0, arc_surface_weighting=True,
                 arc_penetration_mm=2.0, wire_diameter_mm=1.2, arc_sigma_mm=2.0, bulk_tau=None,
                 step_mode="fused", population_dtype="float32", device=None):
        if arc_power_W < 0:
            raise ValueError("arc_power_W must be >= 0, got %s" % arc_power_W)
        if not 0.0 < arc_efficiency <= 1.0:
            raise ValueError("arc_efficiency must be in (0, 1], got %s" % arc_efficiency)
        if wire_diameter_mm <= 0:
            raise ValueError("wire_diameter_mm must be > 0, got %s" % wire_diameter_mm)
        if arc_sigma_mm <= 0:
            raise ValueError("arc_sigma_mm must be > 0, got %s" % arc_sigma_mm)
        if contact_angle_deg is not None and not 0.0 < contact_angle_deg < 180.0:
            raise ValueError("contact_angle_deg must be in (0, 180), got %s" % contact_angle_deg)
        self.mat = material if isinstance(material, MaterialProps) else load_material(material, high_sulphur)
        self.Q_w = arc_power_W
        self.eta = arc_efficiency
        self.T_amb = T_ambient
        self.use_srt = use_srt
        self.C_darcy = C_darcy
        self.arc_pressure = arc_pressure_pa
        self.arc_pressure_model = "constant"
        self.pressure_sigma_m = None
        self.strict_mode = False
        self.u_mach_limit_lu = 0.08
        self.force_limit_lu = 0.05
        self.droplet_freq = droplet_freq_hz
        self.enable_heat_loss = enable_heat_loss
        self.h_conv = h_conv
        self.eps_rad = eps_rad
        self.enable_convection = enable_convection
        self.enable_radiation = enable_radiation
        self.sigma_sb = 5.670374419e-8
        self.heat_source_name = heat_source
        self.enable_vof = enable_vof
        self.enable_recoil = enable_recoil
        self.enable_csf_tension = enable_csf_tension
        self.enable_deposition_momentum = enable_deposition_momentum
        self.enable_lorentz = enable_lorentz
        self.enable_gas_shear = enable_gas_shear
        self.grid = WAAMGrid(nx, ny, nz, dx, self.mat, max_tracers=max_tracers or 50_000,
                             allocate_lorentz=enable_lorentz, allocate_vof=True, device=device,
                             population_dtype=population_dtype)
        if self.grid.population_storage and step_mode != "fused":
            raise NotImplementedError("16-bit population storage runs on the fused step only "
                                      "(step_mode='fused')")
        self.enable_droplet_impact_pressure = enable_droplet_impact_pressure
        self.use_recoil_clausius_clapeyron = use_recoil_clausius_clapeyron
        self.enable_substrate_growth = enable_substrate_growth
        self.enable_moving_window = enable_moving_window
        self.enable_wetting = enable_wetting
        self.enable_hydrostatic_gravity = enable_hydrostatic_gravity
        self.enable_bead_freeze = enable_bead_freeze
        self.enable_ctwd = enable_ctwd
        self.contact_angle_deg = (contact_angle_deg if contact_angle_deg is not None
                                  else self.mat.contact_angle_deg)
        self.theta_rad = math.radians(self.contact_angle_deg)
        self.deposition_superheat_K = deposition_superheat_K
        self.deposition_footprint_sigma_scale = deposition_footprint_sigma_scale
        self.stickout_m = stickout_mm * 1e-3
        self.ctwd_nominal_m = ctwd_mm * 1e-3
        self.ctwd_m = ctwd_mm * 1e-3
        self.layer_height_m = layer_height_mm * 1e-3
        self.rho_e_ohm_m = self.mat.rho_e_ohm_m
        self.eta_stick = self.mat.eta_stick
        self.recoil_pressure_pa = recoil_pressure_pa
        self.welding_current_A = welding_current_A
        self.sigma_liquid_Sm = sigma_liquid_Sm
        self.sigma_solid_Sm = sigma_solid_Sm
        self.lorentz_jacobi_iters = lorentz_jacobi_iters
        self.lorentz_jacobi_omega = lorentz_jacobi_omega
        self.gas_jet_velocity_m_s = gas_jet_velocity_m_s
        self.gas_shear_coeff = gas_shear_coeff
        self.T_boiling_K = T_boiling_K
        self.P_vapor_ref_Pa = P_vapor_ref_Pa
        self.L_vapor_J_kg = L_vapor_J_kg
        self.R_spec_vapor_J_kgK = R_spec_vapor_J_kgK
        self.travel_speed_m_s = travel_speed_m_s
        self.marangoni_scale = 1.0
        self.use_variable_tau = use_variable_tau
        self.enable_enthalpy_cap = enable_enthalpy_cap
        self.T_vapor_cap_K = T_vapor_cap_K
        self.arc_surface_weighting = arc_surface_weighting
        self.arc_penetration_m = arc_penetration_mm * 1e-3
        self.wire_diameter_m = wire_diameter_mm * 1e-3
        self.wire_feed_m_s = 0.0
        self.droplet_transfer_mode = "auto"
        self.pulse_frequency_hz = 0.0
        self.droplet_size_jitter = 0.12
        self.impact_lead_angle_deg = 0.0
        self.trailing_solidify_lookback_mm = 2.5
        self.trailing_solidify_temp_margin_K = 35.0
        self._deposited_volume_m3 = 0.0
        self._n_droplets_fired = 0
        self._deposition_overflow = 0
        self._lorentz_warm = False
        self._lorentz_unconverged = 0
        self._lorentz_unconverged_streak = 0
        self.lorentz_jacobi_tol = 1e-4
        self.plate_thickness_mm = None
        self.plate_size_mm = None
        self.plate_origin_mm = None
        self.nz_solid = max(1, nz // 5)
        self._step_n = 0
        self._last_droplet_time = 0.0
        self._window_offset_x_m = 0.0
        self._interpass_cooling_steps = 0
        self.probe_recorder = None
        self.use_torch_z = False
        self.substrate_z_m = 0.0
        self._sim_origin_offset_x_m = 0.0
        self._sim_origin_offset_y_m = 0.0
        self._last_torch_pos_m = None
        self._torch_dir_xyz = (1.0, 0.0, 0.0)
        self._warned_zero_wire_feed = False
        self._last_arc_ijk = None
        self.step_mode = step_mode
        # leave each step's LBM stream running beside the next step's first
        # stages (results identical; see coupled_step.coupled_step_fused)
        self.pipeline_stream = True
        # and its collision and tracers beside the next step's arc stage
        self.pipeline_collide = True
        # and hold each stream back one more step, to run beside the next
        # collision on the cells that collision does not write
        self.pipeline_lag_stream = True
        # non-droplet fused steps replay a captured CUDA graph of the step
        self.use_cuda_graphs = True
        self._fused_params = None

        # Derived lattice scalars (twin.py:244-274).
        g = self.grid
        mat = self.mat
        self.cp_rho = mat.rho * mat.cp
        self.L_rho = mat.rho * mat.L_fusion
        self.alpha_lu = mat.alpha * g.dt / (g.dx ** 2)
        self.omega = 1.0 / g.tau
        self.omega_bulk = 1.0 / bulk_tau if bulk_tau else self.omega
        self.arc_sigma_m = arc_sigma_mm * 1e-3
        self.sigma_cells = self.arc_sigma_m / g.dx
        self.g_lu = 9.81 * (g.dt ** 2) / g.dx
        self.beta_T = mat.beta_T
        scale_F = (g.dt ** 2) / (mat.rho * g.dx ** 2)
        self.force_scale = scale_F
        self.dgamma_dT_lu = mat.dgamma_dT * scale_F / g.dx
        self.gamma_lu = mat.gamma_0 * scale_F / g.dx
        # twin.py:269-273: the table path runs when the material has any table;
        # H_sol / H_liq use cp at the solidus
        self.gpu_tables = MaterialGPUTables(mat)
        self.use_material_tables = self.gpu_tables.enabled
        cp_sol = mat.cp_at(mat.T_solidus)
        self.H_sol = mat.rho * cp_sol * mat.T_solidus
        self.H_liq = self.H_sol + self.L_rho
        self.arc_source = create_heat_source(heat_source)

    # -- configuration ----------------------------------------------------
    def invalidate(self):
        """Drop cached step parameters after changing a twin attribute, and the
        fused step's quiet-tile history and population copy -- call it after
        writing grid fields (flags, phi, f_l, H, T, populations) directly,
        outside this package's operators."""
        self._fused_params = None
        self.grid.__dict__.pop("_fields_cache", None)
        self.grid._tiles_valid = False

    def resolve_nz_solid(self, test_fluid_domain=False):
        """Substrate layers from plate thickness (else nz//5), leaving gas headroom."""
        if test_fluid_domain:
            return 0
        g = self.grid
        headroom = max(6, g.nz // 4)
        max_solid = max(1, g.nz - headroom)
        thick = self.plate_thickness_mm
        if thick is not None and float(thick) > 0.0:
            n = int(round(float(thick) / (g.dx * 1000.0)))
            return max(1, min(n, max_solid))
        return max(1, min(g.nz // 5, max_solid))

    def resolve_plate_ij(self):
        g = self.grid
        if not self.plate_size_mm:
            return 0, g.nx, 0, g.ny
        dx_mm = g.dx * 1000.0
        ni = min(max(1, int(round(float(self.plate_size_mm[0]) / dx_mm))), g.nx)
        nj = min(max(1, int(round(float(self.plate_size_mm[1]) / dx_mm))), g.ny)
        if self.plate_origin_mm is not None:
            i0 = int(round(float(self.plate_origin_mm[0]) / dx_mm))
            j0 = int(round(float(self.plate_origin_mm[1]) / dx_mm))
        else:
            i0, j0 = (g.nx - ni) // 2, (g.ny - nj) // 2
        i0 = max(0, min(i0, g.nx - ni))
        j0 = max(0, min(j0, g.ny - nj))
        return i0, i0 + ni, j0, j0 + nj

    def apply_plate_geometry(self, *, plate_thickness_mm=None, plate_size_mm=None,
                             plate_origin_mm=None):
        if plate_thickness_mm is not None:
            self.plate_thickness_mm = float(plate_thickness_mm)
            self.nz_solid = self.resolve_nz_solid()
        if plate_size_mm is not None:
            self.plate_size_mm = (float(plate_size_mm[0]), float(plate_size_mm[1]))
        if plate_origin_mm is not None:
            self.plate_origin_mm = (float(plate_origin_mm[0]), float(plate_origin_mm[1]))
        self.invalidate()

    # -- state ------------------------------------------------------------
    def reset(self, T_ambient=None, test_fluid_domain=False):
        """twin.py:486-531: quiescent plate + gas, aux fields, one initial stream."""
        T0 = T_ambient or self.T_amb
        g = self.grid
        if test_fluid_domain:
            nz_solid = -1
            self.nz_solid = 0
            i0, i1, j0, j1 = 0, g.nx, 0, g.ny
        else:
            self.nz_solid = self.resolve_nz_solid(False)
            nz_solid = self.nz_solid
            i0, i1, j0, j1 = self.resolve_plate_ij()
        g._stream_pending = False          # the state is rebuilt below
        g._collide_pending = False
        g._lag_pending = False
        f_a, f_b = g.f_a, g.f_b
        if g.population_storage:
            # initialise and stream in float32, then store offsets; zeroed like
            # the float32 buffers, since the stream leaves SOLID cells alone
            f_a, f_b = torch.zeros(f_a.shape, device=g.device), torch.zeros(f_b.shape,
                                                                              device=g.device)
        kernels.init_grid(f_a, g.rho, g.ux, g.uy, g.uz, g.T, g.H, g.f_l, g.phi, g.flags, T0,
                          RHO_LATTICE, self.cp_rho, nz_solid, i0, i1, j0, j1, g.FLAG_FLUID,
                          g.FLAG_SOLID, g.FLAG_GAS)
        kernels.init_aux_fields(g.T_max, g.T_prev, g.dT_dt, g.time_above_800_s,
                                g.time_above_1100_s, g.time_above_solidus_s, g.Fx_snap, g.Fy_snap,
                                g.Fz_snap, g.Fx, g.Fy, g.Fz, T0, g.porosity_active,
                                g.tracer_head, g.max_tracers)
        kernels.stream(f_a, f_b, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        if g.population_storage:
            g.store_populations(g.f_a, f_a)
            g.store_populations(g.f_b, f_b)
            del f_a, f_b
        self._step_n = 0
        self._last_droplet_time = 0.0
        self._deposited_volume_m3 = 0.0
        self._n_droplets_fired = 0
        self._deposition_overflow = 0
        self._last_torch_pos_m = None
        self._torch_dir_xyz = (1.0, 0.0, 0.0)
        self._lorentz_warm = False
        self._lorentz_unconverged_streak = 0
        self._bead_height_m = 0.0
        self._warned_zero_wire_feed = False
        g.deposit_vol_buf.zero_()
        g.deposit_real_buf.zero_()
        g._tracers_live = False
        self.invalidate()

    def step(self, torch_x_m, torch_y_m, is_welding=True, torch_z_m=None):
        """twin.py:533-567."""
        z_now = 0.0 if torch_z_m is None else float(torch_z_m)
        if self._last_torch_pos_m is not None:
            px, py, pz = self._last_torch_pos_m
            d = (torch_x_m - px, torch_y_m - py, z_now - pz)
            norm = math.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
            if norm > 1e-12:
                self._torch_dir_xyz = (d[0] / norm, d[1] / norm, d[2] / norm)
        self._last_torch_pos_m = (torch_x_m, torch_y_m, z_now)
        if (is_welding and self.droplet_freq > 0 and self.wire_feed_m_s <= 0.0
                and not self._warned_zero_wire_feed):
            self._warned_zero_wire_feed = True
            log.warning("[WAAMTwin] welding step with wire_feed_m_s == 0: no metal will be "
                        "deposited; set twin.wire_feed_m_s")
        if self.enable_moving_window:
            self._maybe_shift_window(torch_x_m)
        sim_x = torch_x_m - self._window_offset_x_m - self._sim_origin_offset_x_m
        sim_y = torch_y_m - self._sim_origin_offset_y_m
        coupled_step(self, sim_x, sim_y, is_welding, torch_z_m)
        self._check_strict_mode()

    def _maybe_shift_window(self, torch_x_world):
        """twin.py:599-631: once the torch passes 62 % of the window, move every
        field max(8, nx // 10) cells back (one launch) and the tracers with it."""
        g = self.grid
        sim_x = torch_x_world - self._window_offset_x_m
        if sim_x < 0.62 * (g.nx - 8) * g.dx:
            return
        n_shift = max(8, g.nx // 10)
        from .coupled_step import flush_stream
        flush_stream(g)
        kernels.shift_simulation_window_x(
            n_shift, g.f_a, g.f_b, g.T, g.H, g.f_l, g.phi, g.flags, g.T_max, g.T_prev, g.dT_dt,
            g.time_above_800_s, g.time_above_1100_s, g.time_above_solidus_s, g.rho, g.ux, g.uy,
            g.uz, g.Fx, g.Fy, g.Fz, g.cp_rho_field, g.alpha_lu_field, g.dgamma_lu_field,
            g.tau_field, self.T_amb, self.cp_rho, RHO_LATTICE, self.nz_solid, g.FLAG_SOLID,
            g.FLAG_GAS, g.FLAG_FLUID, g.nx, g.ny, g.nz)
        self._window_offset_x_m += n_shift * g.dx
        kernels.shift_tracers_x(g.porosity_pos, g.max_tracers, n_shift * g.dx)
        # F may now be non-zero outside the active cells of the fused step
        g._forces_dirty = True
        log.info("[WAAMTwin] Moving window shift -%d cells  offset=%.2fmm", n_shift,
                 self._window_offset_x_m * 1e3)

    HEALTH_BITS = {"nonfinite_enthalpy": 1, "nonfinite_lbm": 2, "rho_out_of_band": 4}

    def health(self, clear=False):
        """The fused step's device health word since it was last cleared: a
        non-gas cell's enthalpy not finite, an active cell's density or
        velocity not finite, an active cell's density outside
        ``health_rho_band`` (default (0.5, 2.0)).  Reading it synchronises
        with the device (4 bytes)."""
        g = self.grid
        g.flush_stream()
        word = int(g.step_status.item())
        if clear:
            g.step_status.zero_()
        out = {k: bool(word & b) for k, b in self.HEALTH_BITS.items()}
        out["word"] = word
        return out

    def _check_health(self):
        """strict_mode on a step that already synchronised with the device: raise
        when the health word reports non-finite values (the reference's
        NaN/Inf check of its force diagnostics, twin.py:578-585, at the points
        where it can be read without an extra synchronisation)."""
        h = self.health()
        if h["nonfinite_enthalpy"] or h["nonfinite_lbm"]:
            raise RuntimeError("[strict_mode] NaN/Inf in the fused step (health word %d: %s) "
                               "after step %d" % (h["word"], ", ".join(
                                   k for k in self.HEALTH_BITS if h[k]), self._step_n))

    def _check_strict_mode(self):
        if not self.strict_mode:
            return
        if self.__dict__.pop("_synced_this_step", False):
            self._check_health()
        streak = int(getattr(self, "_lorentz_unconverged_streak", 0) or 0)
        if self.enable_lorentz and streak > 50:
            raise RuntimeError("[strict_mode] Lorentz Jacobi failed to converge for %d "
                               "consecutive steps -- raise lorentz_jacobi_iters or disable "
                               "strict_mode" % streak)
        if self._n_droplets_fired < 20:
            return
        ratio = self._deposited_volume_m3 * self.mat.rho / max(
            self._n_droplets_fired * droplet_mass_kg(self), 1e-12)
        if not 0.95 <= ratio <= 1.05:
            raise RuntimeError("[strict_mode] mass_balance_ratio=%.3f outside [0.95, 1.05] after "
                               "%d droplets" % (ratio, self._n_droplets_fired))

    def run(self, n_steps, torch_x_m=0.0, torch_y_m=0.0, is_welding=True):
        for _ in range(n_steps):
            self.step(torch_x_m, torch_y_m, is_welding)

    def path_positions(self, job, n_steps=None):
        """(driver, [(step, segment, x, y, z), ...]) of run_path (twin.py:632-704);
        ``job``: a job dict, a job YAML path or a sequence of (x, y, z) [m]."""
        return plan_path(self, job, n_steps)

    def run_path(self, job, n_steps=None, is_welding=True, interpass_steps=0):
        """Follow the job's torch path at travel speed, with interpass parking
        (twin.py:632-704); ``job`` as in ``path_positions``."""
        run_path(self, job, n_steps, is_welding, interpass_steps)

    # -- export (twin.py:701-869) --------------------------------------------
    def export_haz_vtk(self, path="haz_map.vti"):
        from .export import TIER_CORE, export_volume
        return export_volume(self, path, tiers=(TIER_CORE,), crop_liquid=False)

    def export_vtk(self, path="weld_pool.vti"):
        return self.export_vtk_full(path, tiers=(0, 3), crop_liquid=False)

    def export_vtk_full(self, path="weld_pool_full.vti", tiers=(0, 1, 2, 3), crop_liquid=False):
        from .export import TIER_MAP, export_volume
        return export_volume(self, path, tiers=tuple(TIER_MAP.get(t, t) for t in tiers),
                             crop_liquid=crop_liquid)

    def export_surface_vtk(self, path="bead_surface.vtp"):
        from .export import export_surface
        return export_surface(self, path, include_kappa=True)

    def export_tracers_vtk(self, path="tracers.vtp"):
        from .export import export_tracers
        return export_tracers(self, path)

    def export_npz(self, path="state.npz"):
        from .export import export_npz
        return export_npz(self, path)

    def export_research_bundle(self, out_dir, tag=None, tiers=(0, 1, 3), include_surface=True,
                               include_tracers=True, crop_liquid=False):
        from .export import export_research_bundle
        return export_research_bundle(self, out_dir, tag=tag, tiers=tiers,
                                      include_surface=include_surface,
                                      include_tracers=include_tracers,
                                      job_path=getattr(self, "_job_path", None),
                                      crop_liquid=crop_liquid)

    def export_research_sequence(self, *args, **kwargs):
        from .export import export_research_sequence
        return export_research_sequence(self, *args, job_path=getattr(self, "_job_path", None),
                                        **kwargs)

    # -- telemetry (twin.py:706-821) -----------------------------------------
    def telemetry_record(self):
        """Launch the pool reductions into the grid's device record (no sync);
        ``kernels.read_telemetry(grid.telem_record)`` reads it back later."""
        g = self.grid
        rec = getattr(g, "telem_record", None)
        if rec is None:
            rec = g.telem_record = kernels.telemetry_record(g.device)
        kernels.telemetry_pool(g.T, g.f_l, g.phi, g.dT_dt, g.ux, g.uy, g.uz, g.H, g.flags,
                               g.porosity_active, g.max_tracers, self.nz_solid, rec)
        return rec

    def get_telemetry(self):
        """Pool and process telemetry with the reference's keys.

        Every grid aggregate comes from one device record (two launches,
        deterministic, FP64 enthalpy sum) read back in one small copy; the
        reference's atomics, f_l slice, tracer, flags and phi copies are not
        needed.  Force diagnostics (physics/force_diagnostics.py, a telemetry-
        time re-run of each force operator) are not part of this backend."""
        g = self.grid
        r = kernels.read_telemetry(self.telemetry_record())
        if self.strict_mode:
            self._check_health()    # the telemetry read has synchronised already
        n_liquid = int(r.n_liquid)
        if n_liquid > 0:
            T_peak = float(r.T_peak)
            if r.y_min >= 0:
                pool_width_m = (r.y_max - r.y_min + 1) * g.dx
                pool_depth_m = max(0, self.nz_solid - r.z_min) * g.dx
            else:
                pool_width_m = pool_depth_m = 0.0
            pool_length_m = (float(r.i_max) - float(r.i_min) + 1.0) * g.dx
            u_max_phys = float(np.sqrt(float(r.u2_max))) * g.dx / g.dt
        else:
            T_peak = float(r.T_global)
            pool_width_m = pool_depth_m = pool_length_m = u_max_phys = 0.0
        peak_cool = float(r.peak_cool)
        n_trapped, n_active = int(r.n_tracers_trapped), int(r.n_tracers_active)
        porosity_pct = 100.0 * n_trapped / max(n_trapped + n_active, 1)
        dep_mass = self._deposited_volume_m3 * self.mat.rho
        exp_mass = expected_deposited_mass_kg(self)
        m_drop = droplet_mass_kg(self)
        exp_drop_mass = self._n_droplets_fired * m_drop
        mass_ratio = dep_mass / max(exp_drop_mass, 1e-12)
        bead_h = bead_height_m_from_k(int(r.bead_k_max), self.nz_solid, g.dx) * 1000.0
        toe_deg = 0.0
        if self.enable_wetting:
            toe_deg = toe_angle_from_column(list(r.toe_phi)[: r.toe_n],
                                            list(r.toe_flags)[: r.toe_n], int(r.toe_k0),
                                            self.contact_angle_deg, g.dx, g.FLAG_GAS)
        return {
            "step": self._step_n,
            "sim_time_ms": round(self._step_n * g.dt * 1000, 4),
            "peak_temp_K": round(T_peak, 1),
            "peak_temp_C": round(T_peak - 273.15, 1),
            "peak_cooling_rate_Ks": round(peak_cool, 1),
            "pool_width_mm": round(pool_width_m * 1000, 3),
            "pool_depth_mm": round(pool_depth_m * 1000, 3),
            "pool_length_mm": round(pool_length_m * 1000, 3),
            "n_liquid_cells": n_liquid,
            "marangoni_vel_ms": round(u_max_phys, 4),
            "material_status": self.mat.status,
            "material_name": self.mat.name,
            "heat_source": self.heat_source_name,
            "material_tables": self.use_material_tables,
            "vof_enabled": self.enable_vof,
            "travel_speed_mm_s": round(self.travel_speed_m_s * 1000, 3),
            "variable_tau": self.use_variable_tau and self.use_material_tables,
            "porosity_pct": round(porosity_pct, 3),
            "n_trapped_tracers": n_trapped,
            "window_offset_x_mm": round(self._window_offset_x_m * 1000, 3),
            "deposited_mass_g": round(dep_mass * 1000, 4),
            "expected_wire_mass_g": round(exp_mass * 1000, 4),
            "expected_drop_mass_g": round(exp_drop_mass * 1000, 4),
            "n_droplets_fired": self._n_droplets_fired,
            "droplet_mass_mg": round(m_drop * 1e6, 3),
            "droplet_transfer_mode": infer_transfer_mode(self),
            "droplet_impact_velocity_ms": round(droplet_impact_velocity_m_s(self), 4),
            "mass_balance_ratio": round(mass_ratio, 3),
            "wire_mass_flux_g_s": round(wire_mass_flux_kg_s(self) * 1000, 4),
            "T_vapor_cap_K": self.T_vapor_cap_K,
            "arc_surface_weighting": self.arc_surface_weighting,
            "enable_enthalpy_cap": self.enable_enthalpy_cap,
            "enable_wetting": self.enable_wetting,
            "enable_hydrostatic_gravity": self.enable_hydrostatic_gravity,
            "enable_bead_freeze": self.enable_bead_freeze,
            "enable_ctwd": self.enable_ctwd,
            "contact_angle_deg": round(self.contact_angle_deg, 1),
            "bead_height_mm": round(bead_h, 3),
            "toe_angle_deg": round(toe_deg, 1),
            "ctwd_mm": round(self.ctwd_m * 1000, 3),
            "T_drop_K": round(droplet_entry_temperature_K(self), 1),
            "deposition_overflow_count": self._deposition_overflow,
            "physics_tier": getattr(self, "physics_tier", "flow"),
            "strict_mode": bool(getattr(self, "strict_mode", False)),
            "arc_pressure_model": getattr(self, "arc_pressure_model", "constant"),
            "arc_pressure_peak_pa": round(arc_pressure_peak_pa(self), 1),
            "enable_lorentz": self.enable_lorentz,
            "enable_gas_shear": self.enable_gas_shear,
            "lorentz_unconverged_count": int(getattr(self, "_lorentz_unconverged", 0) or 0),
            "lorentz_unconverged_streak": int(getattr(self, "_lorentz_unconverged_streak", 0)
                                              or 0),
            "force_diagnostics": {},
            # additions: the FP64 total enthalpy and the raw pool extents
            "total_enthalpy_J": float(r.H_sum) * g.dx ** 3,
            "pool_slice_i": int(r.i_c),
        }
