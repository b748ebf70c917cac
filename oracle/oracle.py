"""ctypes binding of the C oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/_build/libwaam_oracle.so`` (built by ``make -C oracle``) and
exposes each restated reference kernel on numpy arrays; ``fp64`` is the same
source built in double precision.  Only the parity
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libwaam_oracle.so")
LIB64_PATH = os.path.join(HERE, "_build", "libwaam_oracle64.so")

_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int32)
_f = C.c_float
_i = C.c_int
_l = C.c_int64

_SIGS = {
    "wo_init_grid": ([_F] * 9 + [_I, _i, _i, _i, _f, _f, _f, _i, _i, _i, _i, _i], None),
    "wo_clear_forces": ([_F, _F, _F, _l], None),
    "wo_inject_arc_heat": ([_F, _I, _F, _i, _i, _i] + [_f] * 9 + [_i], C.c_double),
    "wo_inject_goldak_heat": ([_F, _I, _F, _i, _i, _i] + [_f] * 15 + [_i], C.c_double),
    "wo_clamp_enthalpy_ceiling_scalar": ([_F, _I, _l, _f, _f, _f, _f, _f], None),
    "wo_advect_diffuse_temperature": ([_F, _F, _F, _F, _F, _I, _i, _i, _i, _f, _f, _f], None),
    "wo_update_phase": ([_F, _F, _F, _l, _f, _f, _f, _f], None),
    "wo_update_T_max": ([_F, _F, _I, _l], None),
    "wo_update_cooling_rate": ([_F, _F, _F, _I, _l, _f], None),
    "wo_apply_thermal_boundary_losses": ([_F, _F, _I, _i, _i, _i, _f, _f, _f, _i, _i, _f, _f, _f], None),
    "wo_clamp_enthalpy_floor_scalar": ([_F, _f, _I, _l, _f], None),
    "wo_advect_phi": ([_F, _F, _F, _F, _F, _I, _i, _i, _i], None),
    "wo_reinitialize_phi": ([_F, _I, _l], None),
    "wo_apply_contact_angle_phi_bc": ([_F, _I, _i, _i, _i, _f], None),
    "wo_update_flags_from_phi": ([_F, _F, _I, _i, _i, _i, _i], None),
    "wo_sync_phi_liquid_fraction": ([_F, _F, _I, _l], None),
    "wo_compute_csf_tension": ([_F, _I, _F, _F, _F, _i, _i, _i, _f, _i, _f], None),
    "wo_compute_marangoni_force": ([_F, _F, _F, _F, _F, _F, _I, _i, _i, _i, _f], None),
    "wo_apply_arc_pressure": ([_F, _I, _F, _i, _i, _i] + [_f] * 8, None),
    "wo_apply_gas_shear_stress": ([_F, _F, _F, _I, _i, _i, _i] + [_f] * 7, None),
    "wo_apply_vapor_recoil": ([_F, _F, _F, _I, _i, _i, _i] + [_f] * 8, None),
    "wo_apply_vapor_recoil_cc": ([_F, _F, _F, _I, _i, _i, _i] + [_f] * 11, None),
    "wo_add_hydrostatic_gravity": ([_F, _F, _I, _l, _f, _f], None),
    "wo_add_buoyancy": ([_F, _F, _F, _I, _l, _f, _f, _f, _f], None),
    "wo_clamp_body_force_magnitude": ([_F, _F, _F, _I, _l, _f], None),
    "wo_collide_mrt": ([_F] * 10 + [_I, _l, _f, _f, _f], None),
    "wo_collide_srt": ([_F] * 10 + [_I, _l, _f, _f], None),
    "wo_clamp_velocity_mach": ([_F, _F, _F, _I, _l, _f], None),
    "wo_stream": ([_F, _F, _I, _i, _i, _i], None),
    "wo_update_time_above_T": ([_F, _I, _F, _F, _F, _l, _f, _f, _f, _f], None),
    "wo_snapshot_forces": ([_F] * 6 + [_l], None),
    "wo_remelt_hot_solid_scalar": ([_F, _F, _F, _F, _I, _l, _f, _f, _f, _f], None),
    "wo_solidify_trailing_pool_scalar": ([_F, _F, _F, _F, _I, _F, _F, _F, _i, _i, _i] + [_f] * 10, None),
    "wo_solidify_cooled_metal": ([_F, _F, _F, _I, _F, _F, _F, _l, _f, _i], None),
    "wo_surface_height_at": ([_F, _I, _i, _i, _i, _i, _i, _i], C.c_float),
    "wo_feed_wire": ([_F, _I, _F, _F, _F, _F, _F, _i, _i, _i] + [_f] * 9 + [_F, _f], None),
    "wo_feed_wire_momentum": ([_F, _I, _F, _i, _i, _i] + [_f] * 5, None),
    "wo_feed_wire_surface": ([_F, _I, _F, _F, _F, _F, _F, _i, _i, _i] + [_f] * 10 + [_F, _F, _f], None),
    "wo_feed_wire_momentum_impact": ([_F, _F, _F, _F, _F, _I, _F, _i, _i, _i] + [_f] * 7, None),
    "wo_apply_droplet_impact_pressure": ([_F, _I, _F, _F, _i, _i, _i] + [_f] * 8, None),
    "wo_elec_build_sigma": ([_F, _F, _I, _l, _f, _f], None),
    "wo_elec_inject_arc_source": ([_F, _i, _i, _i] + [_f] * 6, None),
    "wo_elec_normalize_source": ([_F, _l, _f, _f], None),
    "wo_elec_jacobi_step": ([_F, _F, _F, _F, _I, _i, _i, _i, _f, _f, _i], None),
    "wo_elec_l1_diff": ([_F, _F, _l, C.POINTER(C.c_double), C.POINTER(C.c_double)], None),
    "wo_elec_compute_J": ([_F, _F, _F, _F, _F, _I, _i, _i, _i, _f], None),
    "wo_elec_bins": ([_F, _F, _i, _i, _i, _f, _f, _f, _f, _i], None),
    "wo_elec_B_axisymmetric": ([_F, _F, _F, _F, _i, _i, _i, _f, _f, _f, _f, _f, _i], None),
    "wo_apply_lorentz_JxB": ([_F] * 10 + [_I, _l, _f, _f, _f], None),
    "wo_refresh_thermal_properties": ([_F, _F, _F, _F, _F, _I, _l, _F, _I, _F, _F] + [_f] * 5,
                                      None),
    "wo_advect_diffuse_temperature_variable": ([_F] * 5 + [_I, _F, _F, _i, _i, _i, _f], None),
    "wo_update_phase_variable_cp": ([_F] * 4 + [_l] + [_f] * 5, None),
    "wo_clamp_enthalpy_ceiling_variable_cp": ([_F, _I, _F, _l, _f, _f, _f], None),
    "wo_clamp_enthalpy_floor": ([_F, _F, _I, _l, _f], None),
    "wo_compute_marangoni_force_variable": ([_F] * 6 + [_I, _F, _i, _i, _i], None),
    "wo_collide_srt_variable_tau": ([_F] * 10 + [_I, _F, _l, _f], None),
    "wo_remelt_hot_solid": ([_F] * 4 + [_I, _F, _l, _f, _f, _f], None),
    "wo_solidify_trailing_pool": ([_F] * 4 + [_I] + [_F] * 4 + [_i, _i, _i] + [_f] * 9, None),
    "wo_inject_tracers": ([_F, _I, _I, _i, _f, _f, _f, _f, _i, C.c_uint64], None),
    "wo_advect_tracers": ([_F, _I, _F, _F, _F, _F, _I, _i, _i, _i, _f, _i], None),
    "wo_shift_simulation_window_x": ([_F] * 6 + [_I] + [_F] * 17 + [_i, _f, _f, _f, _i, _i, _i,
                                                                    _i], None),
    "wo_compute_curvature_field": ([_F, _I, _F, _i, _i, _i], None),
    "wo_compute_vorticity_magnitude": ([_F, _F, _F, _I, _F, _i, _i, _i, _f], None),
    "wo_num_threads": ([], C.c_int),
    "wo_expf_array": ([_F, _F, _l], None),
    "wo_set_num_threads": ([C.c_int], None),
}

def build():
    """Compile the oracle with its Makefile (gcc; seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Oracle:
    """One build of the oracle: float32 (``libwaam_oracle.so``) or the same
    source in double precision (``libwaam_oracle64.so``, float -> double in
    every signature)."""

    def __init__(self, fp64=False):
        self.fp64 = fp64
        self.dtype = np.float64 if fp64 else np.float32
        self.path = LIB64_PATH if fp64 else LIB_PATH
        self._lib = None

    def lib(self):
        if self._lib is None:
            if not os.path.exists(self.path):
                build()
            L = C.CDLL(self.path)
            fptr, fval = (C.POINTER(C.c_double), C.c_double) if self.fp64 else (_F, _f)
            for name, (args, res) in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = [fptr if a is _F else (fval if a is _f else a) for a in args]
                fn.restype = C.c_double if (self.fp64 and res is C.c_float) else res
            self._lib = L
        return self._lib

    def _ptr(self, a):
        if a.dtype == self.dtype:
            assert a.flags.c_contiguous
            return a.ctypes.data_as(C.POINTER(C.c_double) if self.fp64 else _F)
        if a.dtype == np.int32:
            assert a.flags.c_contiguous
            return a.ctypes.data_as(_I)
        raise TypeError("oracle arrays must be %s or int32, got %s" % (
            np.dtype(self.dtype).name, a.dtype))

    def call(self, name, *args):
        """Call oracle function ``name``; numpy arrays are passed by pointer."""
        conv = [self._ptr(a) if isinstance(a, np.ndarray) else a for a in args]
        return getattr(self.lib(), name)(*conv)


fp32 = Oracle(False)
fp64 = Oracle(True)


def lib():
    return fp32.lib()


def call(name, *args):
    """Call float32 oracle function ``name``; numpy arrays are passed by pointer."""
    return fp32.call(name, *args)
