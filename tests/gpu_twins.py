"""Build B200 twins configured like the golden step fixtures (GPU tests)."""
from __future__ import annotations

import numpy as np

import steps
from waam_solver_b200 import WAAMTwin
from waam_solver_b200.physics.arc import Goldak3D


def twin_for_case(name, step_mode="fused"):
    sc, kw, states, positions = steps.load_step_case(name)
    opt, extra = steps.driver_options(name, sc, kw)
    plate = opt.pop("plate_thickness_mm")
    mat = steps.material_for(name, extra)[0]
    tw = WAAMTwin(material=mat, nx=sc["nx"], ny=sc["ny"], nz=sc["nz"], max_tracers=64,
                  step_mode=step_mode, **opt)
    tw.plate_thickness_mm = plate
    for k in ("wire_feed_m_s", "droplet_transfer_mode", "pulse_frequency_hz",
              "droplet_size_jitter"):
        if k in extra:
            setattr(tw, k, extra[k])
    if "goldak" in extra:
        gk = extra["goldak"]
        tw.arc_source = Goldak3D(ff=gk["ff"], fr=gk["fr"], a_front=gk["a_front"],
                                 a_rear=gk["a_rear"], b=gk["b"], c=gk["c"])
    tw.reset()
    assert tw.nz_solid == sc["nz_solid"]
    return tw, sc, extra, states, positions


def set_host_state(tw, name, s, extra, positions):
    import json
    z = np.load("%s/step_%s.npz" % (steps.cases.GOLDEN, name))
    log = json.loads(str(z["log"]))
    tw._step_n = s
    if s == 0:
        tw._last_droplet_time = extra.get("last_drop", 0.0)
        tw._n_droplets_fired = 0
        tw._last_torch_pos_m = None
        tw._torch_dir_xyz = (1.0, 0.0, 0.0)
    else:
        tw._last_droplet_time = log[s - 1]["last_drop"]
        tw._n_droplets_fired = log[s - 1]["droplets"]
        x, y = positions[s - 1]
        tw._last_torch_pos_m = (float(x), float(y), 0.0)
        tw._torch_dir_xyz = tuple(log[s - 1]["dir"])
    tw.invalidate()


def state_of(tw):
    st = tw.grid.state_dict()
    return st
