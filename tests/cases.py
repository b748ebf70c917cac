"""Kernel-level golden cases, runnable on any backend.

Each case in ``CASES`` loads ``tests/golden/k_<name>.npz`` (inputs produced by
``state_gen.seeded_state``; outputs produced by the reference's own kernels),
runs the same operation on a backend and returns the backend's outputs.  A
backend exposes the operator set of ``include/waam_b200.h`` under the
oracle's names (``wo_*`` without the prefix) and works on numpy arrays:
``OracleBackend`` calls the C oracle directly, the CUDA backend in
``tests/cuda_backend.py`` copies the arrays to the GPU and calls the C-ABI.
"""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tolerance used for every float32 field comparison:
#   |a - b| <= RTOL * |b| + RTOL * max|b over the field|
RTOL = 1e-5
# Body forces are gradients of T and phi (Marangoni, CSF).  Against the
# reference itself (numpy exp vs the shared float exp of the oracle and the
# GPU) a 1-ulp difference in H is amplified by T / (cell-to-cell dT), so the
# force fields of full-step comparisons with the REFERENCE use this bound.
# Oracle-vs-GPU comparisons use RTOL for every field.
RTOL_REF_FORCES = 5e-5
FORCE_FIELDS = ("Fx", "Fy", "Fz")


def load_case(name):
    z = np.load(os.path.join(GOLDEN, "k_%s.npz" % name))
    args = json.loads(str(z["args"]))
    fields = json.loads(str(z["fields"]))
    ins = {f: np.ascontiguousarray(z["in_" + f]) for f in fields}
    outs = {f: z["out_" + f] for f in fields}
    return args, ins, outs


def full_inputs(name):
    """All state fields for a case (fields not in the fixture come from state_gen)."""
    import state_gen

    args, ins, outs = load_case(name)
    seed_map = {"inject_goldak": 1, "thermal_s2": 2, "vof_wet": 3, "contact": 4,
                "contact_s5": 5, "forces_wet": 6, "csf": 7, "csf_wet": 8, "collide_srt": 9,
                "tail": 10, "heat_loss": 11, "surface_height": 12, "deposit": 13,
                "lorentz": 14, "tracers": 15, "refresh": 16, "thermal_var": 17, "phase_var": 18,
                "forces_var": 19, "srt_var": 20, "tail_var": 21, "shift": 24, "derived": 25,
                "weld_forces": 26, "feed_wire": 27, "feed_wire_momentum": 28}
    grids = [v.shape[-3:] for v in ins.values() if v.ndim >= 3 and v.shape[-1] != 3]
    nx, ny, nz = grids[0] if grids else (13, 11, 12)   # tracer-only cases: the kernel-case grid
    st = state_gen.seeded_state(nx, ny, nz, seed=seed_map.get(name, 0))
    st = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    st["phi_tmp"] = np.zeros_like(st["phi"])
    for f, v in ins.items():
        if f in st and f != "phi_tmp" and name not in ("reset", "shift", "weld_forces"):
            # the fixture was generated from this very seeded state
            assert np.array_equal(st[f], v), "state_gen drifted from fixture %s (%s)" % (name, f)
        st[f] = v.copy()
    return args, st, outs


def compare(name, got, want, field, rtol=None):
    rtol = RTOL if rtol is None else rtol
    want = np.asarray(want)
    got = np.asarray(got)
    assert got.shape == want.shape, (name, field, got.shape, want.shape)
    if want.dtype.kind in "iu":
        bad = np.count_nonzero(got != want)
        assert bad == 0, "%s: %s differs in %d cells" % (name, field, bad)
        return 0.0
    scale = float(np.max(np.abs(want))) if want.size else 0.0
    err = np.abs(got.astype(np.float64) - want.astype(np.float64))
    tol = rtol * np.abs(want.astype(np.float64)) + rtol * scale
    bad = np.count_nonzero(err > tol)
    assert bad == 0, "%s: %s has %d cells beyond tolerance (max err %.3e, scale %.3e)" % (
        name, field, bad, float(err.max()), scale)
    return float(err.max() / max(scale, 1e-30))


def table_arrays(a):
    """Oracle-style table arguments from a fixture's args: knots (64), counts,
    fallbacks, constants-path reference values."""
    tab = np.concatenate([np.asarray(a[key], np.float32) for key in (
        "cp_T", "cp_V", "k_T", "k_V", "mu_T", "mu_V", "dgamma_T", "dgamma_V")])
    cnt = np.array([a["n_cp"], a["n_k"], a["n_mu"], a["n_dgamma"]], np.int32)
    fb = np.array([a["cp_fallback"], a["k_fallback"], a["mu_fallback"], a["dgamma_fallback"]],
                  np.float32)
    ref = np.array([a["cp_rho_ref"], a["alpha_lu_ref"], a["dgamma_lu_ref"], a["tau_ref"]],
                   np.float32)
    return tab, cnt, fb, ref


def run_case(be, name, st, a):
    """Run case ``name`` on backend ``be`` in place on state dict ``st``."""
    nx, ny, nz = st["phi"].shape
    n = nx * ny * nz
    if name == "inject_gauss":
        be.inject_arc_heat(st["H"], st["flags"], st["f_l"], nx, ny, nz, a["arc_i"], a["arc_j"],
                           a["arc_k"], a["Q_w"], a["sigma"], a["dt"], a["dx3"], a["eta"],
                           a["pen"], a["enable"])
    elif name == "inject_goldak":
        be.inject_goldak_heat(st["H"], st["flags"], st["f_l"], nx, ny, nz, a["arc_i"], a["arc_j"],
                              a["arc_k"], a["Q_w"], a["dt"], a["dx3"], a["eta"], a["sign"],
                              a["ff"], a["fr"], a["a_front"], a["a_rear"], a["b"], a["c"],
                              a["pen"], a["enable"])
    elif name == "ceiling":
        be.clamp_enthalpy_ceiling_scalar(st["H"], st["flags"], n, a["cp_rho"], a["T_solidus"],
                                         a["T_liquidus"], a["T_cap"], a["L_rho"])
    elif name in ("thermal", "thermal_s2"):
        be.advect_diffuse_temperature(st["H"], st["T"], st["ux"], st["uy"], st["uz"], st["flags"],
                                      nx, ny, nz, a["alpha_lu"], 1.0, a["cp_rho"])
    elif name == "phase":
        be.update_phase(st["H"], st["T"], st["f_l"], n, a["cp_rho"], a["L_rho"], a["T_solidus"],
                        a["T_liquidus"])
    elif name == "tmax_cool":
        be.update_T_max(st["T"], st["T_max"], st["flags"], n)
        be.update_cooling_rate(st["T"], st["T_prev"], st["dT_dt"], st["flags"], n, a["dt"])
    elif name in ("vof", "vof_wet"):
        be.advect_phi(st["phi_tmp"], st["phi"], st["ux"], st["uy"], st["uz"], st["flags"],
                      nx, ny, nz)
        st["phi"][...] = st["phi_tmp"]
        be.reinitialize_phi(st["phi"], st["flags"], n)
        if a["wetting"]:
            be.apply_contact_angle_phi_bc(st["phi"], st["flags"], nx, ny, nz, a["theta"])
        be.update_flags_from_phi(st["phi"], st["f_l"], st["flags"], nx, ny, nz, a["nz_solid"])
        be.sync_phi_liquid_fraction(st["phi"], st["f_l"], st["flags"], n)
    elif name in ("contact", "contact_s5"):
        be.apply_contact_angle_phi_bc(st["phi"], st["flags"], nx, ny, nz, a["theta"])
    elif name in ("forces", "forces_wet"):
        be.clear_forces(st["Fx"], st["Fy"], st["Fz"], n)
        be.compute_csf_tension(st["phi"], st["flags"], st["Fx"], st["Fy"], st["Fz"], nx, ny, nz,
                               a["gamma_lu"], a["wetting"], a["theta"])
        be.compute_marangoni_force(st["T"], st["phi"], st["f_l"], st["Fx"], st["Fy"], st["Fz"],
                                   st["flags"], nx, ny, nz, a["dgamma_lu"])
        if a["welding"]:
            be.apply_arc_pressure(st["Fz"], st["flags"], st["phi"], nx, ny, nz, a["arc_i"],
                                  a["arc_j"], a["arc_k"], a["p_sigma"], a["pressure"], a["dt"],
                                  a["dx"], a["rho_phys"])
        if a["hydro"]:
            be.add_hydrostatic_gravity(st["Fz"], st["f_l"], st["flags"], n, 1.0, a["g_lu"])
        be.add_buoyancy(st["T"], st["Fz"], st["f_l"], st["flags"], n, a["g_lu"], a["beta"],
                        a["T_liquidus"], 1.0)
        be.clamp_body_force_magnitude(st["Fx"], st["Fy"], st["Fz"], st["flags"], n, a["F_cap"])
    elif name == "weld_forces":
        be.apply_gas_shear_stress(st["Fx"], st["Fy"], st["phi"], st["flags"], nx, ny, nz,
                                  a["arc_i"], a["arc_j"], a["sigma"], a["tau_pa"], a["dt"],
                                  a["dx"], a["rho_ref"])
        be.apply_vapor_recoil(st["Fz"], st["T"], st["phi"], st["flags"], nx, ny, nz, a["arc_i"],
                              a["arc_j"], a["sigma"], a["recoil_pa"], a["T_ref"], a["dt"],
                              a["dx"], a["rho_ref"])
        be.apply_vapor_recoil_cc(st["Fz"], st["T"], st["phi"], st["flags"], nx, ny, nz,
                                 a["arc_i"], a["arc_j"], a["sigma"], a["P_ref"], a["T_boil"],
                                 a["L_vap"], a["R_spec"], a["C_acc"], a["dt"], a["dx"],
                                 a["rho_ref"])
    elif name in ("csf", "csf_wet"):
        be.compute_csf_tension(st["phi"], st["flags"], st["Fx"], st["Fy"], st["Fz"], nx, ny, nz,
                               a["gamma_lu"], a["wetting"], a["theta"])
    elif name == "collide_mrt":
        be.collide_mrt(st["f_a"], st["f_b"], st["rho"], st["ux"], st["uy"], st["uz"], st["Fx"],
                       st["Fy"], st["Fz"], st["f_l"], st["flags"], n, a["omega"], a["omega_b"],
                       a["C_darcy"])
        be.clamp_velocity_mach(st["ux"], st["uy"], st["uz"], st["flags"], n, a["u_cap"])
    elif name == "collide_srt":
        be.collide_srt(st["f_a"], st["f_b"], st["rho"], st["ux"], st["uy"], st["uz"], st["Fx"],
                       st["Fy"], st["Fz"], st["f_l"], st["flags"], n, a["omega"], a["C_darcy"])
        be.clamp_velocity_mach(st["ux"], st["uy"], st["uz"], st["flags"], n, a["u_cap"])
    elif name == "stream":
        be.stream(st["f_b"], st["f_a"], st["flags"], nx, ny, nz)
    elif name == "tail":
        be.update_time_above_T(st["T"], st["flags"], st["time_above_800_s"],
                               st["time_above_1100_s"], st["time_above_solidus_s"], n, a["dt"],
                               800.0 + 273.15, 1100.0 + 273.15, a["T_solidus"])
        be.snapshot_forces(st["Fx"], st["Fy"], st["Fz"], st["Fx_snap"], st["Fy_snap"],
                           st["Fz_snap"], n)
        be.remelt_hot_solid_scalar(st["T"], st["H"], st["f_l"], st["phi"], st["flags"], n,
                                   a["cp_rho"], a["T_solidus"], a["T_liquidus"], a["L_rho"])
        d = a["dir"]
        be.solidify_trailing_pool_scalar(st["T"], st["H"], st["f_l"], st["phi"], st["flags"],
                                         st["ux"], st["uy"], st["uz"], nx, ny, nz, a["cp_rho"],
                                         a["arc_i"], a["arc_j"], a["arc_k"], d[0], d[1], d[2],
                                         a["lookback"], a["T_freeze"], a["T_solidus"])
        be.solidify_cooled_metal(st["T"], st["f_l"], st["phi"], st["flags"], st["ux"], st["uy"],
                                 st["uz"], n, a["T_solidus"], 1)
    elif name == "heat_loss":
        be.apply_thermal_boundary_losses(st["H"], st["T"], st["flags"], nx, ny, nz, a["T_amb"],
                                         a["h_conv"], a["eps_rad"], a["conv"], a["rad"], a["dt"],
                                         a["dx"], a["sigma_sb"])
        be.clamp_enthalpy_floor_scalar(st["H"], a["cp_rho"], st["flags"], n, a["T_amb"])
    elif name == "surface_height":
        got = {}
        for key in a["heights"]:
            i0, j0 = (int(v) for v in key.split("_"))
            got[key] = float(be.surface_height_at(st["phi"], st["flags"], nx, ny, nz, i0, j0,
                                                  a["nz_solid"]))
        return got
    elif name == "deposit":
        placed = []
        r_try = a["foot_r"]
        placed_real = 0.0
        for _ in range(3):
            vol, real = be.feed_wire_surface(
                st["f_a"], st["flags"], st["f_l"], st["phi"], st["H"], st["T"], st["rho"],
                nx, ny, nz, a["arc_i"], a["arc_j"], a["arc_k"], r_try, a["drop_r"],
                a["target_vol"], a["T_drop"], a["cp_rho"], a["L_rho"], 1.0, placed_real,
                placed_real, a["cell_vol"])
            placed_real = real
            placed.append([r_try, real, vol])
            r_try = min(r_try + 1.5, 16.0)
        v = a["vel"]
        be.feed_wire_momentum_impact(st["f_a"], st["rho"], st["ux"], st["uy"], st["uz"],
                                     st["flags"], st["f_l"], nx, ny, nz, a["arc_i"], a["arc_j"],
                                     a["arc_k"], a["drop_r"], v[0], v[1], v[2])
        be.apply_droplet_impact_pressure(st["Fz"], st["flags"], st["phi"], st["f_l"], nx, ny, nz,
                                         a["arc_i"], a["arc_j"], a["arc_k"], a["drop_r"],
                                         a["impact_pa"], a["dt"], a["dx"], 7800.0)
        return placed
    elif name == "feed_wire":
        acc, accs = 0.0, []
        for arc_k, drop_r in zip(a["arc_ks"], a["drop_rs"]):
            acc = be.feed_wire(st["f_a"], st["flags"], st["f_l"], st["phi"], st["H"], st["T"],
                               st["rho"], nx, ny, nz, a["arc_i"], a["arc_j"], arc_k, drop_r,
                               a["target_vol"], a["T_drop"], a["cp_rho"], a["L_rho"], a["rho0"],
                               acc, a["cell_vol"])
            accs.append(acc)
        return accs
    elif name == "feed_wire_momentum":
        be.feed_wire_momentum(st["uz"], st["flags"], st["f_l"], nx, ny, nz, a["arc_i"], a["arc_j"],
                              a["arc_k"], a["drop_r"], a["vz_lu"])
    elif name == "lorentz":
        rng = np.random.default_rng(31)
        for f in ("sigma_elec", "elec_source", "phi_elec_tmp", "Jx", "Jy", "Jz", "Bx", "By", "Bz"):
            st.setdefault(f, np.zeros((nx, ny, nz), np.float32))
        st.setdefault("phi_elec", rng.uniform(0.0, 0.05, (nx, ny, nz)).astype(np.float32))
        st.setdefault("elec_rad_bins", np.zeros((nz, a["n_bins"]), np.float32))
        be.elec_build_sigma(st["sigma_elec"], st["f_l"], st["flags"], n, a["s_liq"], a["s_sol"])
        be.elec_inject_arc_source(st["elec_source"], nx, ny, nz, a["arc_i"], a["arc_j"],
                                  a["arc_k"], a["sigma_cells"], a["current"], a["dx"])
        be.elec_normalize_source(st["elec_source"], n, a["current"], a["dx"])
        l1 = []
        for it in range(a["iters"]):
            be.elec_jacobi_step(st["phi_elec"], st["phi_elec_tmp"], st["sigma_elec"],
                                st["elec_source"], st["flags"], nx, ny, nz, a["dx"], a["omega"],
                                a["nz_solid"])
            d, m = be.elec_l1(st["phi_elec_tmp"], st["phi_elec"])
            st["phi_elec"][...] = st["phi_elec_tmp"]
            if it % 10 == 9:
                l1.append([d, m])
        be.elec_compute_J(st["Jx"], st["Jy"], st["Jz"], st["phi_elec"], st["sigma_elec"],
                          st["flags"], nx, ny, nz, a["dx"])
        be.elec_bins(st["Jz"], st["elec_rad_bins"], nx, ny, nz, a["arc_i"], a["arc_j"], a["dx"],
                     a["bin_dr"], a["n_bins"])
        be.elec_B_axisymmetric(st["Bx"], st["By"], st["Bz"], st["elec_rad_bins"], nx, ny, nz,
                               a["arc_i"], a["arc_j"], a["dx"], a["bin_dr"], a["mu0"],
                               a["n_bins"])
        be.apply_lorentz_JxB(st["Fx"], st["Fy"], st["Fz"], st["Jx"], st["Jy"], st["Jz"],
                             st["Bx"], st["By"], st["Bz"], st["f_l"], st["flags"], n, a["dt"],
                             a["dx"], a["rho_ref"])
        return l1
    elif name == "refresh":
        tab, cnt, fb, ref = table_arrays(a)
        be.refresh_thermal_properties(st["T"], st["cp_rho_field"], st["alpha_lu_field"],
                                      st["dgamma_lu_field"], st["tau_field"], st["flags"], n, tab,
                                      cnt, fb, ref, a["rho"], a["dt"], a["dx"], a["force_scale"],
                                      a["marangoni_scale"])
    elif name == "thermal_var":
        be.advect_diffuse_temperature_variable(st["H"], st["T"], st["ux"], st["uy"], st["uz"],
                                               st["flags"], st["alpha_lu_field"],
                                               st["cp_rho_field"], nx, ny, nz, 1.0)
    elif name == "phase_var":
        be.clamp_enthalpy_floor(st["H"], st["cp_rho_field"], st["flags"], n, a["T_floor"])
        for step in range(2):
            be.update_phase_variable_cp(st["H"], st["T"], st["f_l"], st["cp_rho_field"], n,
                                        a["L_rho_t"], a["T_solidus_t"], a["T_liquidus_t"],
                                        a["H_sol_t"], a["H_liq_t"])
            if step == 0:
                be.clamp_enthalpy_ceiling_variable_cp(st["H"], st["flags"], st["cp_rho_field"], n,
                                                      a["H_liq_t"], a["T_liquidus_t"],
                                                      a["T_cap_case"])
    elif name == "forces_var":
        be.clear_forces(st["Fx"], st["Fy"], st["Fz"], n)
        be.compute_marangoni_force_variable(st["T"], st["phi"], st["f_l"], st["Fx"], st["Fy"],
                                            st["Fz"], st["flags"], st["dgamma_lu_field"], nx, ny,
                                            nz)
    elif name == "srt_var":
        be.collide_srt_variable_tau(st["f_a"], st["f_b"], st["rho"], st["ux"], st["uy"],
                                    st["uz"], st["Fx"], st["Fy"], st["Fz"], st["f_l"],
                                    st["flags"], st["tau_field"], n, a["C_darcy"])
    elif name == "tail_var":
        be.remelt_hot_solid(st["T"], st["H"], st["f_l"], st["phi"], st["flags"],
                            st["cp_rho_field"], n, a["T_solidus_t"], a["T_liquidus_t"],
                            a["L_rho_t"])
        be.solidify_trailing_pool(st["T"], st["H"], st["f_l"], st["phi"], st["flags"], st["ux"],
                                  st["uy"], st["uz"], st["cp_rho_field"], nx, ny, nz, a["arc_i"],
                                  a["arc_j"], a["arc_k"], 1.0, 0.0, 0.0, a["lookback"],
                                  a["T_freeze"], a["T_solidus_t"])
    elif name == "derived":
        be.compute_curvature_field(st["phi"], st["flags"], st["kappa_field"], nx, ny, nz)
        be.compute_vorticity_magnitude(st["ux"], st["uy"], st["uz"], st["flags"],
                                       st["vorticity_mag"], nx, ny, nz, a["dt"])
    elif name == "shift":
        be.shift_simulation_window_x(
            st["f_a"], st["f_b"], st["T"], st["H"], st["f_l"], st["phi"], st["flags"],
            st["T_max"], st["T_prev"], st["dT_dt"], st["time_above_800_s"],
            st["time_above_1100_s"], st["time_above_solidus_s"], st["rho"], st["ux"], st["uy"],
            st["uz"], st["Fx"], st["Fy"], st["Fz"], st["cp_rho_field"], st["alpha_lu_field"],
            st["dgamma_lu_field"], st["tau_field"], a["n_shift"], a["T_amb"], a["cp_rho"],
            a["rho0"], a["nz_solid"], nx, ny, nz)
    elif name == "tracers":
        be.advect_tracers(st["porosity_pos"], st["porosity_active"], st["ux"], st["uy"], st["uz"],
                          st["f_l"], st["flags"], nx, ny, nz, a["dx"], a["max_tracers"])
    elif name == "reset":
        ny_ = ny
        be.init_grid(st["f_a"], st["rho"], st["ux"], st["uy"], st["uz"], st["T"], st["H"],
                     st["f_l"], st["phi"], st["flags"], nx, ny, nz, 300.0, 1.0, a["cp_rho"],
                     a["nz_solid"], 0, nx, 0, ny_)
        for f in ("T_max", "T_prev"):
            st[f][...] = np.float32(300.0)
        for f in ("dT_dt", "time_above_800_s", "Fx", "Fx_snap"):
            st[f][...] = 0.0
        be.stream(st["f_a"], st["f_b"], st["flags"], nx, ny, nz)
    else:
        raise KeyError(name)
    return None


CASES = ["inject_gauss", "inject_goldak", "ceiling", "thermal", "thermal_s2", "phase",
         "tmax_cool", "vof", "vof_wet", "contact", "contact_s5", "forces", "forces_wet",
         "weld_forces", "csf",
         "csf_wet", "collide_mrt", "collide_srt", "stream", "tail", "heat_loss",
         "surface_height", "deposit", "feed_wire", "feed_wire_momentum", "lorentz", "tracers", "refresh", "thermal_var",
         "phase_var", "forces_var", "srt_var", "tail_var", "shift", "derived", "reset"]


def check_case(be, name):
    """Run ``name`` on ``be`` and assert parity with the golden outputs."""
    a, st, outs = full_inputs(name)
    extra = run_case(be, name, st, a)
    worst = 0.0
    for f, want in outs.items():
        worst = max(worst, compare(name, st[f], want, f))
    if name == "surface_height":
        assert extra == a["heights"], (extra, a["heights"])
    if name == "lorentz":
        for got, ref in zip(extra, a["l1"]):
            for g_, r_ in zip(got, ref):
                assert abs(g_ - r_) <= RTOL * abs(r_), (extra, a["l1"])
    if name == "feed_wire":
        # the budget accumulator is float32 in both: equal to the bit
        assert [np.float32(v) for v in extra] == [np.float32(v) for v in a["vol_acc_after"]], (
            extra, a["vol_acc_after"])
    if name == "deposit":
        for got, ref in zip(extra, a["placed"]):
            assert abs(got[1] - ref[1]) <= 1e-6 * max(ref[1], 1e-30) + 1e-30, (extra, a["placed"])
    return worst


class OracleBackend:
    """Backend over the C oracle (``oracle/oracle.py``)."""

    def __init__(self):
        import sys
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        if root not in sys.path:
            sys.path.insert(0, root)
        from oracle import oracle as O
        self.O = O

    def __getattr__(self, name):
        O = self.__dict__["O"]
        fn_name = "wo_" + name
        if fn_name not in O._SIGS:
            raise AttributeError(name)

        def f(*args):
            return O.call(fn_name, *args)
        return f

    def elec_l1(self, a, b):
        import ctypes
        d, m = ctypes.c_double(), ctypes.c_double()
        self.O.call("wo_elec_l1_diff", a, b, a.size, ctypes.byref(d), ctypes.byref(m))
        return float(np.float32(d.value)), float(np.float32(m.value))

    def elec_bins(self, Jz, bins, nx, ny, nz, arc_i, arc_j, dx, bin_dr, n_bins):
        self.O.call("wo_elec_bins", Jz, bins, nx, ny, nz, arc_i, arc_j, dx, bin_dr, n_bins)

    def feed_wire(self, *args):
        args = list(args)
        acc = np.array([args[19]], dtype=np.float32)
        args[19] = acc
        self.O.call("wo_feed_wire", *args)
        return float(acc[0])

    def feed_wire_surface(self, *args):
        args = list(args)
        vol = np.array([args[20]], dtype=np.float32)
        real = np.array([args[21]], dtype=np.float32)
        args[20] = vol
        args[21] = real
        self.O.call("wo_feed_wire_surface", *args)
        return float(vol[0]), float(real[0])
