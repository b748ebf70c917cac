"""CPU oracle of the whole coupled step -- TEST INFRASTRUCTURE ONLY.

``OracleTwin`` restates the reference step driver
(solvers/coupled_step.py:73-464), the twin's derived lattice scalars
(twin.py:244-274, grid.py:93-105), its reset (twin.py:486-531) and the host
droplet arithmetic (physics/deposition_balance.py:12-86,
physics/weld_forces.py:61-193, physics/electrical_stickout.py:23-36) on
numpy float32 state, calling the C oracle kernels in ``waam_oracle.c``.
It is the CPU reference for the GPU parity tests and the CPU baseline of
``bench.py``; the product never imports it.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

FLUID, SOLID, GAS, IFACE = 0, 1, 2, 4
_W = np.array([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12, dtype=np.float32)


class OracleTwin:
    """Constants or temperature tables (``tables={"cp": [(T, v), ...], ...}``),
    Gaussian2D / Goldak / conical arc, MRT, SRT or variable-tau SRT."""

    def __init__(self, nx, ny, nz, dx, mat, precision="fp32", **kw):
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be fp32 or fp64")
        self.O = O.fp64 if precision == "fp64" else O.fp32
        self.ft = self.O.dtype
        self.nx, self.ny, self.nz, self.dx = nx, ny, nz, dx
        self.mat = dict(mat)
        m = self.mat
        m.setdefault("alpha", m["k"] / (m["rho"] * m["cp"]))
        self.cfg = dict(
            arc_power_W=2800.0, arc_efficiency=0.8, T_ambient=300.0, use_srt=True,
            C_darcy=1.6e5, arc_pressure_pa=500.0, droplet_freq_hz=50.0, heat_source="gaussian2d",
            enable_vof=False, enable_csf_tension=False, enable_wetting=False,
            enable_hydrostatic_gravity=False, enable_heat_loss=False, h_conv=25.0, eps_rad=0.3,
            enable_convection=True, enable_radiation=False, enable_deposition_momentum=True,
            enable_droplet_impact_pressure=True, enable_substrate_growth=False,
            enable_bead_freeze=False, contact_angle_deg=None, deposition_superheat_K=500.0,
            deposition_footprint_sigma_scale=1.0, welding_current_A=140.0, travel_speed_m_s=0.0,
            enable_enthalpy_cap=True, T_vapor_cap_K=3200.0, arc_surface_weighting=True,
            arc_penetration_mm=2.0, wire_diameter_mm=1.2, arc_sigma_mm=2.0, bulk_tau=None,
            wire_feed_m_s=0.0, droplet_transfer_mode="auto", pulse_frequency_hz=0.0,
            droplet_size_jitter=0.12, plate_thickness_mm=None, goldak=None,
            impact_lead_angle_deg=0.0, trailing_solidify_lookback_mm=2.5,
            trailing_solidify_temp_margin_K=35.0, enable_lorentz=False, sigma_liquid_Sm=1.0e6,
            sigma_solid_Sm=1.0e5, lorentz_jacobi_iters=40, lorentz_jacobi_omega=0.85,
            lorentz_jacobi_tol=1e-4, max_tracers=64, tables=None, use_variable_tau=True,
            enable_moving_window=False, enable_recoil=False, enable_gas_shear=False,
            use_recoil_clausius_clapeyron=True, recoil_pressure_pa=5000.0, T_boiling_K=3100.0,
            P_vapor_ref_Pa=101325.0, L_vapor_J_kg=6.0e6, R_spec_vapor_J_kgK=450.0,
            gas_jet_velocity_m_s=12.0, gas_shear_coeff=1.0)
        unknown = set(kw) - set(self.cfg)
        if unknown:
            raise KeyError("unknown OracleTwin options: %s" % sorted(unknown))
        self.cfg.update(kw)
        c = self.cfg
        # grid.py:93-105
        self.dt = dx * 0.05 / 0.5
        nu_lu = (m["mu"] / m["rho"]) * self.dt / dx ** 2
        self.tau = 3.0 * nu_lu + 0.5
        # twin.py:244-274
        self.cp_rho = m["rho"] * m["cp"]
        self.L_rho = m["rho"] * m["L_fusion"]
        self.alpha_lu = m["alpha"] * self.dt / dx ** 2
        self.omega = 1.0 / self.tau
        self.omega_bulk = 1.0 / c["bulk_tau"] if c["bulk_tau"] else self.omega
        self.arc_sigma_m = c["arc_sigma_mm"] * 1e-3
        self.sigma_cells = self.arc_sigma_m / dx
        self.g_lu = 9.81 * self.dt ** 2 / dx
        scale_F = self.dt ** 2 / (m["rho"] * dx ** 2)
        self.dgamma_dT_lu = m["dgamma_dT"] * scale_F / dx
        self.gamma_lu = m["gamma_0"] * scale_F / dx
        self.force_scale = scale_F
        self._setup_tables(c["tables"])
        theta = c["contact_angle_deg"] if c["contact_angle_deg"] is not None else m.get("contact_angle_deg", 80.0)
        self.theta = math.radians(theta)
        headroom = max(6, nz // 4)
        max_solid = max(1, nz - headroom)
        t = c["plate_thickness_mm"]
        if t is not None and t > 0:
            self.nz_solid = max(1, min(int(round(t / (dx * 1000.0))), max_solid))
        else:
            self.nz_solid = max(1, min(nz // 5, max_solid))
        self.step_n = 0
        self.last_drop = 0.0
        self.n_drops = 0
        self.deposited = 0.0
        self.dir = (1.0, 0.0, 0.0)
        self.last_pos = None
        self.arc_k = None
        self.s = None
        self.lorentz_warm = False
        self.lorentz_iters = []
        self.window_offset = 0.0

    def _setup_tables(self, tables):
        """gpu_tables.py:12-80 (knot upload) and twin.py:269-273 (H_sol / H_liq
        from cp(T_solidus)); materials.py:48-58 cp_at is material_tables.py
        interp_linear."""
        m = self.mat
        tables = {k: sorted((float(a), float(b)) for a, b in v)
                  for k, v in (tables or {}).items() if v}
        self.use_tables = bool(tables)
        cols, cnt = [], []
        fb = [m["cp"], m["k"], m["mu"], m["dgamma_dT"]]
        for key, fallback in zip(("cp", "k", "mu", "dgamma_dT"), fb):
            knots = tables.get(key, [])[:8]
            t = np.zeros(8, np.float32)
            v = np.zeros(8, np.float32)
            if not knots:
                t[0], v[0] = 300.0, fallback
                n = 1
            else:
                n = len(knots)
                for q, (a, b) in enumerate(knots):
                    t[q], v[q] = a, b
            cols += [t, v]
            cnt.append(n)
        self.tab = np.concatenate(cols).astype(self.ft)
        self.cnt = np.array(cnt, np.int32)
        self.fb = np.array(fb, self.ft)

        def cp_at(T):
            knots = tables.get("cp", [])
            if not knots:
                return m["cp"]
            if T <= knots[0][0]:
                return knots[0][1]
            if T >= knots[-1][0]:
                return knots[-1][1]
            for (t0, v0), (t1, v1) in zip(knots[:-1], knots[1:]):
                if t0 <= T <= t1:
                    return v0 if t1 == t0 else v0 + (T - t0) / (t1 - t0) * (v1 - v0)
            return m["cp"]
        self.H_sol = m["rho"] * cp_at(m["T_solidus"]) * m["T_solidus"]
        self.H_liq = self.H_sol + self.L_rho

    def _refresh(self):
        """solvers/coupled_step.py:168-181 refresh_properties (use_tables = 1)."""
        s = self.s
        ref = np.array([self.cp_rho, self.alpha_lu, self.dgamma_dT_lu, self.tau], self.ft)
        self.O.call("wo_refresh_thermal_properties", s["T"], s["cp_rho_field"],
                    s["alpha_lu_field"], s["dgamma_lu_field"], s["tau_field"], s["flags"],
                    s["T"].size, self.tab, self.cnt, self.fb, ref, self.mat["rho"], self.dt,
                    self.dx, self.force_scale / self.dx, 1.0)

    def _ceiling(self):
        """solvers/coupled_step.py:17-31 _clamp_enthalpy_ceiling."""
        s, c, m = self.s, self.cfg, self.mat
        n = s["H"].size
        if self.use_tables:
            self.O.call("wo_clamp_enthalpy_ceiling_variable_cp", s["H"], s["flags"],
                        s["cp_rho_field"], n, self.H_liq, m["T_liquidus"], c["T_vapor_cap_K"])
        else:
            self.O.call("wo_clamp_enthalpy_ceiling_scalar", s["H"], s["flags"], n, self.cp_rho,
                        m["T_solidus"], m["T_liquidus"], c["T_vapor_cap_K"], self.L_rho)

    def _phase(self):
        s, m = self.s, self.mat
        n = s["H"].size
        if self.use_tables:
            self.O.call("wo_update_phase_variable_cp", s["H"], s["T"], s["f_l"],
                        s["cp_rho_field"], n, self.L_rho, m["T_solidus"], m["T_liquidus"],
                        self.H_sol, self.H_liq)
        else:
            self.O.call("wo_update_phase", s["H"], s["T"], s["f_l"], n, self.cp_rho, self.L_rho,
                        m["T_solidus"], m["T_liquidus"])

    # ---------------------------------------------------------------- state --
    def reset(self):
        # twin.py:486-531 also forgets the torch position and direction
        self.last_pos = None
        self.dir = (1.0, 0.0, 0.0)
        nx, ny, nz = self.nx, self.ny, self.nz
        sh = (nx, ny, nz)
        z = lambda: np.zeros(sh, self.ft)  # noqa: E731
        s = dict(f_a=np.zeros((19,) + sh, self.ft), f_b=np.zeros((19,) + sh, self.ft),
                 rho=z(), ux=z(), uy=z(), uz=z(), T=z(), H=z(), f_l=z(), phi=z(), phi_tmp=z(),
                 flags=np.zeros(sh, np.int32), T_max=z(), T_prev=z(), dT_dt=z(),
                 time_above_800_s=z(), time_above_1100_s=z(), time_above_solidus_s=z(),
                 Fx=z(), Fy=z(), Fz=z())
        T0 = self.cfg["T_ambient"]
        self.O.call("wo_init_grid", s["f_a"], s["rho"], s["ux"], s["uy"], s["uz"], s["T"], s["H"],
               s["f_l"], s["phi"], s["flags"], nx, ny, nz, T0, 1.0, self.cp_rho, self.nz_solid,
               0, nx, 0, ny)
        s["T_max"][...] = self.ft(T0)
        s["T_prev"][...] = self.ft(T0)
        self.O.call("wo_stream", s["f_a"], s["f_b"], s["flags"], nx, ny, nz)
        s["read_is_a"] = True
        # the property fields are zero when the grid is made and are not
        # touched by reset (grid.py:146-149, twin.py:486-531)
        for key in ("cp_rho_field", "alpha_lu_field", "dgamma_lu_field", "tau_field"):
            s[key] = self.s[key] if self.s is not None and key in self.s else z()
        self.s = s
        self._tracer_fields()
        self.lorentz_warm = False
        self.step_n = 0
        self.last_drop = 0.0
        self.n_drops = 0
        self.deposited = 0.0

    def load(self, st):
        """Adopt a state dict (numpy arrays named like the reference grid)."""
        def own(v):
            v = np.ascontiguousarray(v).copy()
            return v.astype(self.ft) if v.dtype.kind == "f" else v
        self.s = {k: (own(v) if isinstance(v, np.ndarray) else v) for k, v in st.items()}
        self.s.setdefault("phi_tmp", np.zeros_like(self.s["phi"]))
        for key in ("cp_rho_field", "alpha_lu_field", "dgamma_lu_field", "tau_field"):
            self.s.setdefault(key, np.zeros_like(self.s["phi"]))
        self.s.setdefault("read_is_a", True)
        self._tracer_fields()

    def _tracer_fields(self):
        m = int(self.cfg["max_tracers"])
        self.s.setdefault("porosity_pos", np.zeros((m, 3), self.ft))
        self.s.setdefault("porosity_active", np.zeros(m, np.int32))
        self.s.setdefault("tracer_head", np.zeros(1, np.int32))

    def fsrc(self):
        return self.s["f_a"] if self.s["read_is_a"] else self.s["f_b"]

    def fdst(self):
        return self.s["f_b"] if self.s["read_is_a"] else self.s["f_a"]

    # ------------------------------------------------------- host arithmetic --
    def _mode(self):
        c = self.cfg
        mode = str(c["droplet_transfer_mode"]).lower()
        if mode in ("globular", "spray", "pulsed"):
            return mode
        if c["pulse_frequency_hz"] > 0:
            return "pulsed"
        return "globular" if c["welding_current_A"] < 180.0 else "spray"

    def _mdot(self):
        d = self.cfg["wire_diameter_mm"] * 1e-3
        return self.mat["rho"] * math.pi * (d * 0.5) ** 2 * self.cfg["wire_feed_m_s"]

    def _period(self):
        c = self.cfg
        f = c["droplet_freq_hz"]
        base = 1.0 / max(f, 1e-9) if f > 0 else 1.0 / 50.0
        mode = self._mode()
        if mode == "globular":
            sc = 1.55
        elif mode == "spray":
            sc = 0.72
        elif mode == "pulsed":
            sc = max(0.25, min(4.0, (1.0 / max(c["pulse_frequency_hz"], 1e-9)) / base))
        else:
            sc = 1.0
        amp = max(0.0, min(c["droplet_size_jitter"], 0.35))
        jit = 1.0 + amp * math.sin(0.73 * float(self.n_drops + 1) + 0.31)
        return max(base * 0.2, base * sc * jit)

    def _drop_mass_nominal(self):
        return max(0.0, self._mdot() * max(self._period(), 0.0)) if self.cfg["droplet_freq_hz"] > 0 else 0.0

    def _impact_velocity(self, m):
        c = self.cfg
        L = 3e-3
        if c["droplet_freq_hz"] > 0 and c["wire_feed_m_s"] > 0:
            L = c["wire_feed_m_s"] / c["droplet_freq_hz"]
        v_feed = max(c["wire_feed_m_s"], 0.0)
        v_grav = math.sqrt(max(0.0, 2.0 * 9.81 * L))
        d = max(c["wire_diameter_mm"] * 1e-3, 1e-6)
        pinch = 0.35 * math.sqrt(max(c["welding_current_A"], 0.0) / 200.0) * math.sqrt(1.2e-3 / d)
        sc = {"globular": 0.78, "spray": 1.18, "pulsed": 1.05}.get(self._mode(), 1.0)
        mt = 1.0
        if m > 0:
            mt = max(0.8, min(1.25, math.sqrt(self._drop_mass_nominal() / m)))
        return min(5.0, sc * max(v_feed, v_grav + pinch) * mt)

    # ------------------------------------------------------------------ step --
    def _maybe_shift_window(self, x_world):
        """twin.py:599-631 on the oracle state."""
        s = self.s
        if x_world - self.window_offset < 0.62 * (self.nx - 8) * self.dx:
            return
        n_shift = max(8, self.nx // 10)
        self.O.call("wo_shift_simulation_window_x", s["f_a"], s["f_b"], s["T"], s["H"], s["f_l"],
                    s["phi"], s["flags"], s["T_max"], s["T_prev"], s["dT_dt"],
                    s["time_above_800_s"], s["time_above_1100_s"], s["time_above_solidus_s"],
                    s["rho"], s["ux"], s["uy"], s["uz"], s["Fx"], s["Fy"], s["Fz"],
                    s["cp_rho_field"], s["alpha_lu_field"], s["dgamma_lu_field"], s["tau_field"],
                    n_shift, self.cfg["T_ambient"], self.cp_rho, 1.0, self.nz_solid, self.nx,
                    self.ny, self.nz)
        self.window_offset += n_shift * self.dx
        pos = s["porosity_pos"]
        pos[:, 0] = pos[:, 0] - self.ft(n_shift * self.dx)

    def step(self, x, y, welding=True, z=None):
        """One step at torch position (x, y) and torch height z (None: 0, used
        for the travel direction only); with the moving window on, x is a
        world position (twin.py:533-567)."""
        if self.cfg["enable_moving_window"]:
            # the direction uses world positions, the physics the window's
            self._update_dir(x, y, z)
            self._maybe_shift_window(x)
            return self._step(x - self.window_offset, y, welding, dir_done=True)
        self._update_dir(x, y, z)
        return self._step(x, y, welding, dir_done=True)

    def _update_dir(self, x, y, z=None):
        """twin.py:540-546: the unit vector from the previous torch position."""
        z = 0.0 if z is None else float(z)
        if self.last_pos is not None:
            d = (x - self.last_pos[0], y - self.last_pos[1], z - self.last_pos[2])
            nrm = math.sqrt(sum(v * v for v in d))
            if nrm > 1e-12:
                self.dir = tuple(v / nrm for v in d)
        self.last_pos = (x, y, z)

    def _step(self, x, y, welding=True, dir_done=False):
        c, s, m = self.cfg, self.s, self.mat
        nx, ny, nz = self.nx, self.ny, self.nz
        n = nx * ny * nz
        if not dir_done:
            self._update_dir(x, y)
        self._pos = (x, y)
        arc_i, arc_j = x / self.dx, y / self.dx
        i0 = max(0, min(int(arc_i), nx - 1))
        j0 = max(0, min(int(arc_j), ny - 1))
        k = float(self.O.call("wo_surface_height_at", s["phi"], s["flags"], nx, ny, nz, i0, j0,
                         self.nz_solid))
        if k < 1.0:
            k = float(max(1, self.nz_solid - 1))
        arc_k = self.arc_k = k
        Ts, Tl = m["T_solidus"], m["T_liquidus"]
        self.O.call("wo_clear_forces", s["Fx"], s["Fy"], s["Fz"], n)
        pen = c["arc_penetration_mm"] * 1e-3 / self.dx
        en = 1 if c["arc_surface_weighting"] else 0
        cap = c["enable_enthalpy_cap"]
        if welding:
            hs = str(c["heat_source"]).lower().replace("-", "").replace("_", "")
            if hs in ("goldak", "goldak3d", "doubleellipsoid"):
                g = c["goldak"]
                sign = 1.0 if c["travel_speed_m_s"] >= 0.0 else -1.0
                self.O.call("wo_inject_goldak_heat", s["H"], s["flags"], s["f_l"], nx, ny, nz, arc_i,
                       arc_j, arc_k, c["arc_power_W"], self.dt, self.dx ** 3,
                       c["arc_efficiency"], sign, g["ff"], g["fr"], g["a_front"], g["a_rear"],
                       g["b"], g["c"], pen, en)
            elif hs in ("conical", "conicalvolume", "cone"):
                self.O.call("wo_inject_arc_heat", s["H"], s["flags"], s["f_l"], nx, ny, nz, arc_i,
                       arc_j, arc_k - 1.5, c["arc_power_W"], self.sigma_cells * 1.2, self.dt,
                       self.dx ** 3, c["arc_efficiency"], pen, en)
            else:
                self.O.call("wo_inject_arc_heat", s["H"], s["flags"], s["f_l"], nx, ny, nz, arc_i,
                       arc_j, arc_k, c["arc_power_W"], self.sigma_cells, self.dt, self.dx ** 3,
                       c["arc_efficiency"], pen, en)
            if cap:
                self._ceiling()
            self._maybe_droplet(arc_i, arc_j, arc_k)
        if self.use_tables:
            self._refresh()
            self.O.call("wo_advect_diffuse_temperature_variable", s["H"], s["T"], s["ux"],
                        s["uy"], s["uz"], s["flags"], s["alpha_lu_field"], s["cp_rho_field"],
                        nx, ny, nz, 1.0)
        else:
            self.O.call("wo_advect_diffuse_temperature", s["H"], s["T"], s["ux"], s["uy"],
                        s["uz"], s["flags"], nx, ny, nz, self.alpha_lu, 1.0, self.cp_rho)
        if c["enable_heat_loss"]:
            self.O.call("wo_apply_thermal_boundary_losses", s["H"], s["T"], s["flags"], nx, ny, nz,
                   c["T_ambient"], c["h_conv"], c["eps_rad"], int(c["enable_convection"]),
                   int(c["enable_radiation"]), self.dt, self.dx, 5.670374419e-8)
            if self.use_tables:
                self.O.call("wo_clamp_enthalpy_floor", s["H"], s["cp_rho_field"], s["flags"], n,
                            c["T_ambient"])
            else:
                self.O.call("wo_clamp_enthalpy_floor_scalar", s["H"], self.cp_rho, s["flags"], n,
                            c["T_ambient"])
        self._phase()
        if cap:
            self._ceiling()
        self._phase()
        self.O.call("wo_update_T_max", s["T"], s["T_max"], s["flags"], n)
        self.O.call("wo_update_cooling_rate", s["T"], s["T_prev"], s["dT_dt"], s["flags"], n, self.dt)
        if c["enable_vof"]:
            self.O.call("wo_advect_phi", s["phi_tmp"], s["phi"], s["ux"], s["uy"], s["uz"],
                   s["flags"], nx, ny, nz)
            s["phi"][...] = s["phi_tmp"]
            self.O.call("wo_reinitialize_phi", s["phi"], s["flags"], n)
            if c["enable_wetting"]:
                self.O.call("wo_apply_contact_angle_phi_bc", s["phi"], s["flags"], nx, ny, nz,
                       self.theta)
            self.O.call("wo_update_flags_from_phi", s["phi"], s["f_l"], s["flags"], nx, ny, nz,
                   self.nz_solid)
            self.O.call("wo_sync_phi_liquid_fraction", s["phi"], s["f_l"], s["flags"], n)
        if c["enable_csf_tension"]:
            self.O.call("wo_compute_csf_tension", s["phi"], s["flags"], s["Fx"], s["Fy"], s["Fz"], nx,
                   ny, nz, self.gamma_lu, int(c["enable_wetting"]), self.theta)
        if self.use_tables:
            self.O.call("wo_compute_marangoni_force_variable", s["T"], s["phi"], s["f_l"],
                        s["Fx"], s["Fy"], s["Fz"], s["flags"], s["dgamma_lu_field"], nx, ny, nz)
        else:
            self.O.call("wo_compute_marangoni_force", s["T"], s["phi"], s["f_l"], s["Fx"],
                        s["Fy"], s["Fz"], s["flags"], nx, ny, nz, self.dgamma_dT_lu)
        sig = self.arc_sigma_m / self.dx
        if welding and c["enable_gas_shear"]:
            # physics/weld_forces.py:126-131 gas_shear_tau_pa, 180-193
            v = c["gas_jet_velocity_m_s"]
            tau = min(0.5 * 1.6 * v * v * c["gas_shear_coeff"], 5000.0)
            self.O.call("wo_apply_gas_shear_stress", s["Fx"], s["Fy"], s["phi"], s["flags"], nx,
                        ny, nz, arc_i, arc_j, sig, tau, self.dt, self.dx, m["rho"])
        if welding:
            self.O.call("wo_apply_arc_pressure", s["Fz"], s["flags"], s["phi"], nx, ny, nz, arc_i,
                   arc_j, arc_k, self.arc_sigma_m / self.dx, c["arc_pressure_pa"], self.dt,
                   self.dx, m["rho"])
        if welding and c["enable_recoil"]:
            # physics/weld_forces.py:134-158
            if c["use_recoil_clausius_clapeyron"]:
                self.O.call("wo_apply_vapor_recoil_cc", s["Fz"], s["T"], s["phi"], s["flags"],
                            nx, ny, nz, arc_i, arc_j, sig, c["P_vapor_ref_Pa"], c["T_boiling_K"],
                            c["L_vapor_J_kg"], c["R_spec_vapor_J_kgK"], 0.54, self.dt, self.dx,
                            m["rho"])
            else:
                self.O.call("wo_apply_vapor_recoil", s["Fz"], s["T"], s["phi"], s["flags"], nx,
                            ny, nz, arc_i, arc_j, sig, c["recoil_pressure_pa"], Tl, self.dt,
                            self.dx, m["rho"])
        if c["enable_hydrostatic_gravity"]:
            self.O.call("wo_add_hydrostatic_gravity", s["Fz"], s["f_l"], s["flags"], n, 1.0, self.g_lu)
        self.O.call("wo_add_buoyancy", s["T"], s["Fz"], s["f_l"], s["flags"], n, self.g_lu,
               m["beta_T"], Tl, 1.0)
        if welding and c["enable_lorentz"]:
            self._lorentz(arc_i, arc_j, arc_k)
        self.O.call("wo_clamp_body_force_magnitude", s["Fx"], s["Fy"], s["Fz"], s["flags"], n, 0.05)
        if self.use_tables and c["use_variable_tau"]:
            self.O.call("wo_collide_srt_variable_tau", self.fsrc(), self.fdst(), s["rho"],
                        s["ux"], s["uy"], s["uz"], s["Fx"], s["Fy"], s["Fz"], s["f_l"],
                        s["flags"], s["tau_field"], n, c["C_darcy"])
        elif c["use_srt"]:
            self.O.call("wo_collide_srt", self.fsrc(), self.fdst(), s["rho"], s["ux"], s["uy"],
                   s["uz"], s["Fx"], s["Fy"], s["Fz"], s["f_l"], s["flags"], n, self.omega,
                   c["C_darcy"])
        else:
            self.O.call("wo_collide_mrt", self.fsrc(), self.fdst(), s["rho"], s["ux"], s["uy"],
                   s["uz"], s["Fx"], s["Fy"], s["Fz"], s["f_l"], s["flags"], n, self.omega,
                   self.omega_bulk, c["C_darcy"])
        self.O.call("wo_clamp_velocity_mach", s["ux"], s["uy"], s["uz"], s["flags"], n, 0.08)
        self.O.call("wo_stream", self.fdst(), self.fsrc(), s["flags"], nx, ny, nz)
        self.O.call("wo_advect_tracers", s["porosity_pos"], s["porosity_active"], s["ux"], s["uy"],
                    s["uz"], s["f_l"], s["flags"], nx, ny, nz, self.dx, int(c["max_tracers"]))
        self.O.call("wo_update_time_above_T", s["T"], s["flags"], s["time_above_800_s"],
               s["time_above_1100_s"], s["time_above_solidus_s"], n, self.dt, 800.0 + 273.15,
               1100.0 + 273.15, Ts)
        if c["enable_substrate_growth"] or c["enable_bead_freeze"]:
            if self.use_tables:
                self.O.call("wo_remelt_hot_solid", s["T"], s["H"], s["f_l"], s["phi"],
                            s["flags"], s["cp_rho_field"], n, Ts, Tl, self.L_rho)
            else:
                self.O.call("wo_remelt_hot_solid_scalar", s["T"], s["H"], s["f_l"], s["phi"],
                            s["flags"], n, self.cp_rho, Ts, Tl, self.L_rho)
            if welding and c["enable_bead_freeze"]:
                lb = max(2.0, c["trailing_solidify_lookback_mm"] / (self.dx * 1000.0))
                T_fr = Tl + c["trailing_solidify_temp_margin_K"]
                if self.use_tables:
                    self.O.call("wo_solidify_trailing_pool", s["T"], s["H"], s["f_l"], s["phi"],
                                s["flags"], s["ux"], s["uy"], s["uz"], s["cp_rho_field"], nx, ny,
                                nz, arc_i, arc_j, arc_k, self.dir[0], self.dir[1], self.dir[2],
                                lb, T_fr, Ts)
                else:
                    self.O.call("wo_solidify_trailing_pool_scalar", s["T"], s["H"], s["f_l"],
                                s["phi"], s["flags"], s["ux"], s["uy"], s["uz"], nx, ny, nz,
                                self.cp_rho, arc_i, arc_j, arc_k, self.dir[0], self.dir[1],
                                self.dir[2], lb, T_fr, Ts)
            self.O.call("wo_solidify_cooled_metal", s["T"], s["f_l"], s["phi"], s["flags"], s["ux"],
                   s["uy"], s["uz"], n, Ts, 1)
        s["read_is_a"] = not s["read_is_a"]
        self.step_n += 1

    def _lorentz(self, arc_i, arc_j, arc_k):
        """physics/weld_forces.py:196-281 on the oracle kernels."""
        import ctypes
        c, s = self.cfg, self.s
        nx, ny, nz, n = self.nx, self.ny, self.nz, self.nx * self.ny * self.nz
        sh = (nx, ny, nz)
        for f in ("phi_elec", "phi_elec_tmp", "sigma_elec", "elec_source", "Jx", "Jy", "Jz", "Bx",
                  "By", "Bz"):
            s.setdefault(f, np.zeros(sh, self.ft))
        n_bins = 64
        s.setdefault("elec_rad_bins", np.zeros((nz, n_bins), self.ft))
        I = c["welding_current_A"]
        self.O.call("wo_elec_build_sigma", s["sigma_elec"], s["f_l"], s["flags"], n,
               c["sigma_liquid_Sm"], c["sigma_solid_Sm"])
        self.O.call("wo_elec_inject_arc_source", s["elec_source"], nx, ny, nz, arc_i, arc_j, arc_k,
               self.sigma_cells, I, self.dx)
        self.O.call("wo_elec_normalize_source", s["elec_source"], n, I, self.dx)
        cold = not self.lorentz_warm
        if cold:
            s["phi_elec"][...] = 0.0
            self.lorentz_warm = True
        max_iters = max(int(c["lorentz_jacobi_iters"]), 20)
        if cold:
            nmax = max(nx, ny, nz)
            max_iters = max(max_iters, 2 * nmax * nmax)
        done = 0
        d, m = ctypes.c_double(), ctypes.c_double()
        while done < max_iters:
            for _ in range(min(10, max_iters - done)):
                self.O.call("wo_elec_jacobi_step", s["phi_elec"], s["phi_elec_tmp"], s["sigma_elec"],
                       s["elec_source"], s["flags"], nx, ny, nz, self.dx,
                       c["lorentz_jacobi_omega"], self.nz_solid)
                self.O.call("wo_elec_l1_diff", s["phi_elec_tmp"], s["phi_elec"], n, ctypes.byref(d),
                       ctypes.byref(m))
                s["phi_elec"][...] = s["phi_elec_tmp"]
                done += 1
            rel = float(self.ft(d.value)) / max(float(self.ft(m.value)), 1e-30)
            if rel < c["lorentz_jacobi_tol"]:
                break
        self.lorentz_iters.append(done)
        self.O.call("wo_elec_compute_J", s["Jx"], s["Jy"], s["Jz"], s["phi_elec"], s["sigma_elec"],
               s["flags"], nx, ny, nz, self.dx)
        bin_dr = max(float(max(nx, ny)) / (2.0 * n_bins), 0.5)
        self.O.call("wo_elec_bins", s["Jz"], s["elec_rad_bins"], nx, ny, nz, arc_i, arc_j, self.dx,
               bin_dr, n_bins)
        self.O.call("wo_elec_B_axisymmetric", s["Bx"], s["By"], s["Bz"], s["elec_rad_bins"], nx, ny,
               nz, arc_i, arc_j, self.dx, bin_dr, 4.0e-7 * math.pi, n_bins)
        self.O.call("wo_apply_lorentz_JxB", s["Fx"], s["Fy"], s["Fz"], s["Jx"], s["Jy"], s["Jz"],
               s["Bx"], s["By"], s["Bz"], s["f_l"], s["flags"], n, self.dt, self.dx,
               self.mat["rho"])

    def _maybe_droplet(self, arc_i, arc_j, arc_k):
        c, s, m = self.cfg, self.s, self.mat
        if c["droplet_freq_hz"] <= 0:
            return
        t = self.step_n * self.dt
        if t - self.last_drop < self._period():
            return
        drop_dt = t - self.last_drop
        self.last_drop = t
        mass = max(0.0, self._mdot() * max(drop_dt, 0.0))
        if mass <= 0:
            r = 3.0
        else:
            cells = mass / m["rho"] / self.dx ** 3
            r = max(1.0, min((3.0 * cells / (4.0 * math.pi)) ** (1.0 / 3.0), 10.0))
        vol = mass / m["rho"]
        T_drop = m["T_liquidus"] + c["deposition_superheat_K"]
        # solvers/coupled_step.py:120-125 (seeded by the step number, as the library does)
        self.O.call("wo_inject_tracers", s["porosity_pos"], s["porosity_active"],
                    s["tracer_head"], int(c["max_tracers"]), self._pos[0], self._pos[1],
                    float(arc_k + 1) * self.dx, float(self.sigma_cells * self.dx), 50,
                    int(self.step_n))
        r_try = max(r, self.sigma_cells * c["deposition_footprint_sigma_scale"])
        placed = 0.0
        nx, ny, nz = self.nx, self.ny, self.nz
        for _ in range(10):
            va = np.array([placed], self.ft)
            ra = np.array([placed], self.ft)
            self.O.call("wo_feed_wire_surface", self.fsrc(), s["flags"], s["f_l"], s["phi"], s["H"],
                   s["T"], s["rho"], nx, ny, nz, arc_i, arc_j, arc_k, r_try, r, vol, T_drop,
                   self.cp_rho, self.L_rho, 1.0, va, ra, self.dx ** 3)
            placed = float(ra[0])
            if placed >= vol * 0.98:
                break
            r_try = min(r_try + 1.5, 16.0)
        self.deposited += placed
        self.n_drops += 1
        if c["enable_deposition_momentum"]:
            v = self._impact_velocity(mass)
            lead = math.radians(c["impact_lead_angle_deg"])
            dxy = math.hypot(self.dir[0], self.dir[1])
            ddx, ddy = (self.dir[0] / dxy, self.dir[1] / dxy) if dxy >= 1e-9 else (1.0, 0.0)
            v_xy = min(v * 0.65, max(c["travel_speed_m_s"], abs(v) * math.tan(lead)))
            v_z = -math.sqrt(max(v * v - v_xy * v_xy, v * v * 0.2))
            k = self.dt / self.dx
            self.O.call("wo_feed_wire_momentum_impact", self.fsrc(), s["rho"], s["ux"], s["uy"],
                   s["uz"], s["flags"], s["f_l"], nx, ny, nz, arc_i, arc_j, arc_k, r,
                   v_xy * ddx * k, v_xy * ddy * k, v_z * k)
            if c["enable_droplet_impact_pressure"]:
                rm = r * self.dx
                pa = 0.5 * mass * v * v / max(math.pi * rm * rm, 1e-12) if mass > 0 else 0.0
                self.O.call("wo_apply_droplet_impact_pressure", s["Fz"], s["flags"], s["phi"],
                       s["f_l"], nx, ny, nz, arc_i, arc_j, arc_k, r, pa, self.dt, self.dx,
                       m["rho"])
