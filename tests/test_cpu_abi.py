"""C-ABI boundary checks that need no GPU: the library loads, exports every
entry point include/waam_b200.h declares, and rejects bad arguments with
WAAM_ERR_INVALID before touching the device."""
import ctypes
import re
import subprocess

import numpy as np
import pytest

from waam_solver_b200 import _native


def declared():
    return sorted(_native.parse_header())


def test_header_declares_the_operator_set():
    names = set(declared())
    for op in ("waam_collide_mrt", "waam_stream", "waam_advect_diffuse_temperature",
               "waam_inject_goldak_heat", "waam_feed_wire_surface", "waam_step_pre",
               "waam_step_main", "waam_apply_contact_angle_phi_bc"):
        assert op in names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (waam_\w+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    lib = _native.lib()
    for n in declared():
        assert getattr(lib, n) is not None


def test_abi_version_and_workspace():
    lib = _native.lib()
    assert lib.waam_abi_version() == 1
    assert lib.waam_workspace_bytes(0) >= 16384
    assert lib.waam_workspace_bytes(1000) >= 16384 + 4000
    assert lib.waam_workspace_bytes(1000) % 256 == 0


def test_ctypes_struct_layouts_match_the_library():
    lib = _native.lib()
    for which, cls in enumerate((_native.WaamFields, _native.WaamStepParams,
                                 _native.WaamMaterialTables, _native.WaamTelemetry,
                                 _native.WaamProbeSet, _native.WaamShiftPlane,
                                 _native.WaamExportChannel)):
        assert lib.waam_struct_size(which) == ctypes.sizeof(cls), cls.__name__
    assert lib.waam_struct_size(7) == 0


@pytest.mark.parametrize("call", [
    ("waam_clear_forces", (None, None, None, 10, None)),
    ("waam_stream", (None, None, None, 4, 4, 4, None)),
    ("waam_stream", (1, 1, 1, 0, 4, 4, None)),
    ("waam_update_phase", (None, 1, 1, 10, 1.0, 1.0, 1.0, 1.0, None)),
    ("waam_surface_height_at", (1, 1, 1, 4, 4, 4, 7, 0, 1, None)),
    ("waam_refresh_thermal_properties", (1, 1, 1, 1, 1, 1, 10, None, 1.0, 1.0, 1.0, 1.0, 1.0,
                                         1.0, 1.0, 1.0, 1.0, 1, None)),
    ("waam_clamp_enthalpy_floor", (1, None, 1, 10, 300.0, None)),
])
def test_invalid_arguments_are_rejected_on_the_host(call):
    name, args = call
    rc = getattr(_native.lib(), name)(*args)
    assert rc == -1
    assert _native.lib().waam_last_error()


def test_step_entry_points_reject_missing_fields():
    f = _native.WaamFields()
    p = _native.WaamStepParams()
    rc = _native.lib().waam_step_main(ctypes.byref(f), ctypes.byref(p), None, 0, None)
    assert rc == -1
    with pytest.raises(_native.WaamError):
        _native.call("waam_step_pre", ctypes.byref(f), ctypes.byref(p), None, 0, None)


def test_shared_expf_accuracy():
    """The float exponential shared by oracle and kernels is within 2 ulp of exp."""
    from oracle import oracle as O
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(-103.0, 88.0, 400_000), rng.uniform(-1, 1, 100_000),
                        np.array([0.0, -0.0, 1e-8, -1e-8, 88.7, -87.3, -100.0, -103.9],
                                 np.float64)]).astype(np.float32)
    y = np.empty_like(x)
    O.call("wo_expf_array", x, y, x.size)
    ref = np.exp(x.astype(np.float64))
    normal = ref >= np.finfo(np.float32).tiny
    ulp = np.spacing(ref.astype(np.float32)[normal]).astype(np.float64)
    err = np.abs(y[normal].astype(np.float64) - ref[normal]) / ulp
    assert err.max() <= 2.0, err.max()
    sub = ~normal
    assert np.all(np.abs(y[sub] - ref[sub]) <= 2 * 1.4e-45)
