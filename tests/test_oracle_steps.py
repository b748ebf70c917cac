"""The oracle step driver against full reference steps (golden fixtures).

Each fixture is a short WAAMTwin.step run of the reference itself
(tests/golden/make_golden.py).  The oracle restarts from every recorded
state (with the twin's host counters at that step) and must reproduce the
next recorded state within the per-step tolerance; the whole recorded
trajectory is also replayed from the first state with a looser bound.
"""
import json

import numpy as np
import pytest

import cases
import steps
from oracle.oracle_step import OracleTwin


def make_oracle(name):
    sc, kw, states, positions = steps.load_step_case(name)
    opt, extra = steps.driver_options(name, sc, kw)
    dx = opt.pop("dx")
    host = {k: v for k, v in extra.items() if k in ("wire_feed_m_s", "droplet_transfer_mode",
                                                    "pulse_frequency_hz", "droplet_size_jitter")}
    _, mat, tables = steps.material_for(name, extra)
    ot = OracleTwin(sc["nx"], sc["ny"], sc["nz"], dx, mat, goldak=extra.get("goldak"),
                    tables=tables, **opt, **host)
    assert ot.nz_solid == sc["nz_solid"]
    return ot, sc, extra, states, positions


def host_state(name, s):
    """Host counters of the reference twin before step s."""
    z = np.load("%s/step_%s.npz" % (cases.GOLDEN, name))
    log = json.loads(str(z["log"]))
    if s == 0:
        return dict(last_drop=-1.0 if name.startswith("c2") else 0.0, n_drops=0, last_pos=None)
    pos = z["positions"][s - 1]
    return dict(last_drop=log[s - 1]["last_drop"], n_drops=log[s - 1]["droplets"],
                last_pos=(float(pos[0]), float(pos[1]), 0.0), dir=tuple(log[s - 1]["dir"]))


@pytest.mark.parametrize("name", steps.STEP_CASES)
def test_oracle_single_steps_match_reference(name):
    ot, sc, extra, states, positions = make_oracle(name)
    for k in ("alpha_lu", "omega", "gamma_lu", "dgamma_dT_lu", "g_lu", "sigma_cells"):
        assert abs(getattr(ot, k) - sc[k]) <= 1e-12 * abs(sc[k]), k
    for s in range(len(states) - 1):
        hs = host_state(name, s)
        ot.load(states[s])
        ot.step_n = s
        ot.last_drop, ot.n_drops, ot.last_pos = hs["last_drop"], hs["n_drops"], hs["last_pos"]
        if "dir" in hs:
            ot.dir = hs["dir"]
        x, y = positions[s]
        ot.step(x, y, True)
        assert ot.s["read_is_a"] == states[s + 1]["read_is_a"]
        steps.compare_state("%s step %d" % (name, s), ot.s, states[s + 1],
                            fields=steps.fields_for(name), reference=True)


@pytest.mark.parametrize("name", steps.STEP_CASES)
def test_oracle_trajectory_matches_reference(name, monkeypatch):
    ot, sc, extra, states, positions = make_oracle(name)
    ot.load(states[0])
    ot.last_drop = host_state(name, 0)["last_drop"]
    monkeypatch.setattr(cases, "RTOL", 1e-4)
    for s, (x, y) in enumerate(positions[: len(states) - 1]):
        ot.step(x, y, True)
    steps.compare_state("%s trajectory" % name, ot.s, states[-1],
                        fields=steps.fields_for(name), reference=True)


def test_trajectory_fixture_is_complete_and_consistent():
    """tests/golden/trajectory_standard.json (make_trajectory.py): one record
    every 500 steps (the small workload's every 250 through 2,000), droplets counted up by one per 100 Hz period, the state
    finite through step 9,000, and the hash helper the GPU test shares is the
    SHA-1 of the float32 bytes."""
    import hashlib
    import json
    import os
    import sys

    import numpy as np
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    from make_trajectory import FIELDS, field_hash, fixture_path
    with open(fixture_path("standard")) as fh:
        fix = json.load(fh)
    with open(fixture_path("small")) as fh:
        small = json.load(fh)
    assert [r["step"] for r in small["records"]] == list(range(250, 2001, 250))
    assert all(r["nonfinite_T"] == 0 for r in small["records"])
    recs = fix["records"]
    assert [r["step"] for r in recs] == list(range(500, fix["n_steps"] + 1, 500))
    finite = [r for r in recs if r["nonfinite_T"] == 0]
    assert finite[-1]["step"] >= 9000 and all(r["nonfinite_T"] == 0 for r in recs[:len(finite)])
    assert all(b["drops"] - a["drops"] == 1 for a, b in zip(recs, recs[1:]))
    assert all(len(r[k]) == 12 for r in recs for k in FIELDS)
    a = np.arange(10, dtype=np.float64)
    assert field_hash(a) == hashlib.sha1(a.astype(np.float32).tobytes()).hexdigest()[:12]
