"""Full-step golden cases (tests/golden/step_*.npz) for any step driver.

A fixture holds the reference twin's complete state before every step and
after the last one, the torch positions and the twin configuration
(tests/golden/make_golden.py).  ``STEP_CASES`` maps each fixture to the
options the driver needs to reproduce the same run.
"""
from __future__ import annotations

import json
import os

import numpy as np

import cases
from cases import GOLDEN, compare

FIELDS = ["rho", "ux", "uy", "uz", "T", "H", "f_l", "phi", "T_max", "T_prev", "dT_dt",
          "time_above_800_s", "time_above_1100_s", "time_above_solidus_s", "Fx", "Fy", "Fz",
          "flags", "f_a", "f_b"]

MATERIAL = dict(k=30.0, rho=7800.0, cp=680.0, T_solidus=1723.0, T_liquidus=1783.0,
                L_fusion=2.7e5, gamma_0=1.8, dgamma_dT=-4.3e-4, mu=0.0065, beta_T=1.2e-4,
                contact_angle_deg=30.0)

PROP_FIELDS = ["cp_rho_field", "alpha_lu_field", "dgamma_lu_field", "tau_field"]

# c*: constants-only material; t*: the material-table path (validated
# ER70S-6 file with cp, k, mu and Sahoo dgamma/dT tables)
STEP_CASES = ["c1_plate", "c1_seeded", "c2_drop", "c2_seeded", "t1_plate", "t1_seeded"]


def fields_for(name):
    return FIELDS + PROP_FIELDS if name.startswith("t") else FIELDS


def load_step_case(name):
    z = np.load(os.path.join(GOLDEN, "step_%s.npz" % name))
    sc = json.loads(str(z["scalars"]))
    kw = json.loads(str(z["twin_kw"]))
    n_states = max(int(k.split("_")[0][1:]) for k in z.files if k.startswith("s") and "_" in k
                   and k.split("_")[0][1:].isdigit()) + 1
    states = []
    for s in range(n_states):
        st = {f: np.ascontiguousarray(z["s%d_%s" % (s, f)]) for f in fields_for(name)}
        st["read_is_a"] = bool(z["s%d_read_is_a" % s])
        states.append(st)
    positions = [tuple(p) for p in z["positions"]]
    return sc, kw, states, positions


def driver_options(name, sc, kw):
    """Options shared by every driver for fixture ``name``."""
    opt = dict(kw)
    opt.setdefault("use_srt", False)
    opt.setdefault("enable_vof", True)
    opt.setdefault("droplet_freq_hz", 0.0)
    opt.pop("max_tracers", None)
    opt.pop("tables", None)
    extra = dict(nz_solid=sc["nz_solid"])
    if "material" in sc:
        extra["material"] = sc["material"]
    if name.startswith(("c1", "t1")):
        opt["plate_thickness_mm"] = 1.0
    else:
        opt["plate_thickness_mm"] = 0.8
        extra.update(wire_feed_m_s=0.1, droplet_transfer_mode="pulsed", pulse_frequency_hz=100.0,
                     droplet_size_jitter=0.0, goldak=sc["goldak"], last_drop=-1.0)
    return opt, extra


def material_for(name, extra):
    """(MaterialProps of the B200 twin, oracle constants dict, oracle tables)."""
    from waam_solver_b200.materials import from_constants, MaterialTables
    rec = extra.get("material")
    if rec is None:
        return (from_constants("ER70S-6-constants", MATERIAL, contact_angle_deg=30.0),
                MATERIAL, None)
    c = dict(rec["constants"])
    mat = from_constants("ER70S-6", c, contact_angle_deg=rec["contact_angle_deg"])
    mat.tables = MaterialTables(**{k: [tuple(r) for r in v] for k, v in rec["tables"].items()})
    oc = dict(c, contact_angle_deg=rec["contact_angle_deg"])
    return mat, oc, {k: [tuple(r) for r in v] for k, v in rec["tables"].items()}


def compare_state(tag, got, want, fields=FIELDS, reference=False):
    """Compare two states; ``reference=True`` when ``want`` comes from the
    reference itself (force fields then use cases.RTOL_REF_FORCES)."""
    worst = 0.0
    for f in fields:
        rtol = None
        if reference and f in cases.FORCE_FIELDS:
            rtol = max(cases.RTOL_REF_FORCES, cases.RTOL)
        worst = max(worst, compare(tag, got[f], want[f], f, rtol))
    return worst
