"""Loader of the native library ``_lib/libwaam_b200.so``.

The ctypes signatures are derived from the C header ``include/waam_b200.h``
(the single definition of the ABI), so the Python host and any other FFI
binding read the same declarations.  The product path has no fallback: if
the library is missing or fails to load, every operator raises.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HEADER = os.path.join(ROOT, "include", "waam_b200.h")
LIB_PATH = os.path.join(HERE, "_lib", "libwaam_b200.so")


class WaamError(RuntimeError):
    """A native entry point returned a non-zero status."""


class WaamFields(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in (
        "f_src", "f_dst", "rho", "ux", "uy", "uz", "T", "T_next", "H", "H_next", "f_l", "phi",
        "phi_tmp", "flags", "T_max", "T_prev", "dT_dt", "t800", "t1100", "tsol", "Fx", "Fy",
        "Fz", "step_scalars")] + [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                                  ("tracer_pos", C.c_void_p), ("tracer_active", C.c_void_p),
                                  ("max_tracers", C.c_int)] + [
        (name, C.c_void_p) for name in ("cp_rho_f", "alpha_f", "dgamma_f", "tau_f", "tape_f",
                                        "tape_cells", "tape_count")] + [("tape_cap", C.c_int64)] + [
        ("lorentz_J", C.c_void_p * 3), ("lorentz_B", C.c_void_p * 3),
        ("flags_copy_w", C.c_void_p), ("flags_copy_r", C.c_void_p), ("status", C.c_void_p),
        ("tile_bits", C.c_void_p), ("tile_list", C.c_void_p), ("tile_part", C.c_void_p),
        ("flags_copy_rr", C.c_void_p), ("pop_cache_src", C.c_void_p),
        ("pop_cache_dst", C.c_void_p), ("pop_cache_stamp", C.c_void_p)]


TABLE_KNOTS = 8


class WaamMaterialTables(C.Structure):
    """gpu_tables.py MaterialGPUTables as the C struct of the header."""
    _fields_ = ([(name, C.c_float * TABLE_KNOTS) for name in (
        "cp_T", "cp_V", "k_T", "k_V", "mu_T", "mu_V", "dgamma_T", "dgamma_V")] +
        [(name, C.c_int32) for name in ("n_cp", "n_k", "n_mu", "n_dgamma")] +
        [(name, C.c_float) for name in ("cp_fallback", "k_fallback", "mu_fallback",
                                        "dgamma_fallback")])


TOE_CELLS = 16
MAX_PROBES = 64


class WaamTelemetry(C.Structure):
    """Device record of waam_telemetry_pool (see the header)."""
    _fields_ = ([(n, C.c_double) for n in ("T_global", "T_peak", "peak_cool", "u2_max", "H_sum")]
                + [(n, C.c_int64) for n in ("n_liquid", "i_sum")]
                + [(n, C.c_int32) for n in ("i_min", "i_max", "i_c", "y_min", "y_max", "z_min",
                                            "bead_k_max", "n_tracers_active",
                                            "n_tracers_trapped", "toe_k0", "toe_n")]
                + [("toe_phi", C.c_float * TOE_CELLS), ("toe_flags", C.c_int32 * TOE_CELLS)])


class WaamProbeSet(C.Structure):
    _fields_ = [("n_probes", C.c_int32), ("cell", C.c_int64 * MAX_PROBES)]


MAX_SHIFT_PLANES = 64
SHIFT_KEEP, SHIFT_CONST, SHIFT_BY_K = 0, 1, 2


class WaamShiftPlane(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("elem_bytes", C.c_int32), ("mode", C.c_int32),
                ("below", C.c_uint32), ("above", C.c_uint32)]


MAX_EXPORT_CHANNELS = 48
(EXPORT_COPY, EXPORT_COPY_I32, EXPORT_ADD, EXPORT_NEG, EXPORT_LU_VEL, EXPORT_LU_ACC, EXPORT_SPEED,
 EXPORT_ACC_MAG, EXPORT_PRESSURE, EXPORT_MUSHY) = range(10)


class WaamExportChannel(C.Structure):
    _fields_ = [("op", C.c_int32), ("a", C.c_float), ("b", C.c_float), ("c", C.c_float),
                ("src", C.c_void_p * 3)]


def _params_fields():
    """Field list of WaamStepParams, parsed from the header."""
    src = open(HEADER).read()
    body = re.search(r"typedef struct WaamStepParams \{(.*?)\} WaamStepParams;", src, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    out = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        typ, names = decl.split(None, 1)
        ctype = {"int": C.c_int, "float": C.c_float, "WaamMaterialTables": WaamMaterialTables}[typ]
        for nm in names.split(","):
            out.append((nm.strip(), ctype))
    return out


class WaamStepParams(C.Structure):
    _fields_ = _params_fields()


_CTYPES = {
    "float*": C.c_void_p, "const float*": C.c_void_p, "int32_t*": C.c_void_p,
    "const int32_t*": C.c_void_p, "void*": C.c_void_p, "float": C.c_float, "int": C.c_int,
    "int64_t": C.c_int64, "size_t": C.c_size_t, "double": C.c_double, "uint64_t": C.c_uint64,
    "const WaamFields*": C.POINTER(WaamFields),
    "const WaamStepParams*": C.POINTER(WaamStepParams), "const char*": C.c_char_p,
    "void* const*": C.c_void_p, "const WaamMaterialTables*": C.POINTER(WaamMaterialTables),
    "WaamTelemetry*": C.c_void_p, "const WaamProbeSet*": C.POINTER(WaamProbeSet),
    "const WaamShiftPlane*": C.c_void_p, "const WaamExportChannel*": C.c_void_p,
    "double*": C.c_void_p, "uint8_t*": C.c_void_p, "const uint8_t*": C.c_void_p,
    "int64_t*": C.c_void_p, "unsigned long long*": C.c_void_p,
}


def parse_header(path: str = HEADER):
    """Return {function name: (restype, [argtypes])} for every declaration."""
    src = open(path).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"typedef struct \w+ \{.*?\} \w+;", "", src, flags=re.S)
    decls = {}
    for m in re.finditer(r"(const char\*|int64_t|int|size_t)\s+(waam_\w+)\s*\(([^)]*)\)\s*;",
                         src):
        ret, name, args = m.group(1), m.group(2), m.group(3)
        types = []
        args = args.strip()
        if args and args != "void":
            for a in args.split(","):
                a = " ".join(a.split())
                typ = a.rsplit(" ", 1)[0].replace(" *", "*")
                types.append(_CTYPES[typ])
        decls[name] = (_CTYPES[ret] if ret != "int" else C.c_int, types)
    return decls


_lib = None
_lock = threading.Lock()


def lib():
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise WaamError(
                    "native library %s is missing; build it with "
                    "`python -m waam_solver_b200.build`" % LIB_PATH)
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in parse_header().items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def call(name: str, *args) -> int:
    """Call entry point ``name``; raise WaamError on a non-zero status."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        msg = lib().waam_last_error().decode(errors="replace")
        raise WaamError("%s failed (%d): %s" % (name, rc, msg))
    return rc
