"""Full-size trajectory fixtures: field hashes of a bench workload every
``every`` steps from the reference reset state, computed by the CPU oracle --
the standard workload (256x128x96 D3Q19 bead-on-plate, Goldak 4 kW, 100 Hz
droplets, VOF, wetting, CSF, Marangoni, buoyancy, gravity, central-moment
MRT) and the small one (64x32x32, Gaussian 3 kW, no wire, VOF).

TEST INFRASTRUCTURE ONLY.  The GPU test (tests/test_gpu_trajectory.py)
runs the same steps through WAAMTwin and compares the hashes bit for bit::

    python tests/golden/make_trajectory.py [workload] [n_steps] [every]

(standard: about 40 minutes on 8 host cores for 10,000 steps; small: a few
seconds for 2,000).  The oracle twin is built as bench.py's CPU baseline
builds it, on the torch path of bench.path_steps.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
FIELDS = ("T", "phi", "f_l", "flags", "ux", "f_a", "f_b")


def field_hash(a):
    """First 12 hex digits of the SHA-1 of the field's float32 / int32 bytes."""
    a = np.ascontiguousarray(a)
    if a.dtype.kind == "f":
        a = a.astype(np.float32)
    return hashlib.sha1(a.tobytes()).hexdigest()[:12]


def record(step, st, drops):
    fl = st["flags"]
    rec = {"step": step, "drops": int(drops), "gas": int((fl == 2).sum()),
           "nonfinite_T": int((~np.isfinite(st["T"])).sum()),
           "read_is_a": bool(st["read_is_a"])}
    for k in FIELDS:
        rec[k] = field_hash(st[k])
    return rec


def oracle_twin(w):
    sys.path.insert(0, ROOT)
    import bench
    from oracle import oracle as O
    from oracle.oracle_step import OracleTwin
    O.lib()
    O.call("wo_set_num_threads", os.cpu_count() or 1)
    kw = bench.twin_kwargs(w)
    kw.pop("wire_diameter_mm", None)
    goldak = None
    if w.get("goldak_mm"):
        gm, dxmm = w["goldak_mm"], w["dx"] * 1e3
        goldak = dict(ff=gm["ff"], fr=gm["fr"], a_front=gm["a_front_mm"] / dxmm,
                      a_rear=gm["a_rear_mm"] / dxmm, b=gm["b_mm"] / dxmm,
                      c=gm["c_mm"] / dxmm)
    extra = {}
    if w.get("wire_feed_m_s"):
        extra = dict(wire_feed_m_s=w["wire_feed_m_s"], droplet_transfer_mode="pulsed",
                     pulse_frequency_hz=w["droplet_freq_hz"], droplet_size_jitter=0.0)
    if w.get("plate_thickness_mm"):
        extra["plate_thickness_mm"] = w["plate_thickness_mm"]
    mat = dict(bench.MATERIAL, contact_angle_deg=w.get("contact_angle_deg", 30.0))
    ot = OracleTwin(w["nx"], w["ny"], w["nz"], w["dx"], mat, goldak=goldak, **kw, **extra)
    ot.reset()
    return ot


def fixture_path(workload):
    return os.path.join(HERE, "trajectory_%s.json" % workload)


def main(workload="standard", n_steps=10000, every=500):
    sys.path.insert(0, ROOT)
    import bench
    w = dict(bench.WORKLOADS[workload])
    ot = oracle_twin(w)
    pos = bench.path_steps(w, ot.dt, n_steps)
    recs, t0 = [], time.time()
    for s in range(n_steps):
        ot.step(*pos[s])
        if (s + 1) % every == 0:
            recs.append(record(s + 1, ot.s, ot.n_drops))
            print(json.dumps(recs[-1]), "%.0f s" % (time.time() - t0), flush=True)
    with open(fixture_path(workload), "w") as fh:
        json.dump({"workload": w["workload"], "every": every, "n_steps": n_steps,
                   "generator": "CPU oracle (oracle/oracle_step.py), tests/golden/make_trajectory.py",
                   "records": recs}, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "standard",
         *(int(a) for a in sys.argv[2:4]))
