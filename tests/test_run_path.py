"""run_path (twin.py:632-704): the step plan against the reference's own
run_path, which ``tests/golden/make_golden.py run_path`` ran on a recorder
object (every step call: x, y, welding, z; and the seeded torch direction)
for a job YAML with interpass parking from the argument and from the twin,
a job dict with the default step count, a shifted window and a job without
a path.  CPU: the same recorder through this package's run_path.  GPU: a
real twin following the YAML job against the oracle stepped through the
reference's recorded calls."""
import json
import os
import types

import numpy as np
import pytest

import cases
import steps

GOLDEN = cases.GOLDEN
JOB = os.path.join(GOLDEN, "job_path.yaml")


def _fixture():
    with open(os.path.join(GOLDEN, "run_path_reference.json")) as fh:
        return json.load(fh)


class Recorder:
    """The attributes run_path reads and a step that records its calls."""

    def __init__(self, nx, ny, dx, travel, interpass_attr=0, window_offset=0.0):
        self.grid = types.SimpleNamespace(nx=nx, ny=ny, dx=dx, dt=dx * 0.05 / 0.5)
        self.travel_speed_m_s = travel
        self._interpass_cooling_steps = interpass_attr
        self._window_offset_x_m = window_offset
        self._torch_dir_xyz = (1.0, 0.0, 0.0)
        self.calls = []

    def step(self, x, y, is_welding=True, torch_z_m=None):
        self.calls.append([float(x), float(y), bool(is_welding), torch_z_m])


def _job(kind):
    import yaml
    with open(JOB) as fh:
        job = yaml.safe_load(fh)
    return {"yaml": JOB, "dict": job, "empty": {"job_name": "no_path"}}[kind]


@pytest.mark.parametrize("name", sorted(_fixture()))
def test_run_path_plan_matches_reference(name):
    from waam_solver_b200.torch_path import run_path
    ref = _fixture()[name]
    rec = Recorder(ref["nx"], ref["ny"], ref["dx"], ref["travel"], ref["interpass_attr"],
                   ref["window_offset"])
    run_path(rec, _job(ref["job"]), n_steps=ref["n_steps"], interpass_steps=ref["interpass_steps"])
    assert len(rec.calls) == len(ref["calls"])
    for got, want in zip(rec.calls, ref["calls"]):
        assert got[2] == want[2]
        np.testing.assert_allclose(got[:2], want[:2], rtol=0, atol=1e-15)
        assert (got[3] is None) == (want[3] is None)
        if want[3] is not None:
            assert abs(got[3] - want[3]) <= 1e-15
    np.testing.assert_allclose(rec._torch_dir_xyz, ref["torch_dir"], rtol=0, atol=1e-15)


def test_run_path_accepts_pathlike_and_waypoint_lists(tmp_path):
    import pathlib
    from waam_solver_b200.torch_path import job_waypoints, run_path
    ref = _fixture()["yaml_interpass"]
    rec = Recorder(ref["nx"], ref["ny"], ref["dx"], ref["travel"])
    run_path(rec, pathlib.Path(JOB), n_steps=ref["n_steps"], interpass_steps=7)
    assert [c[:3] for c in rec.calls] == [c[:3] for c in ref["calls"]]
    wp = job_waypoints(JOB)
    rec2 = Recorder(ref["nx"], ref["ny"], ref["dx"], ref["travel"])
    run_path(rec2, wp, n_steps=ref["n_steps"], interpass_steps=7)
    assert rec2.calls == rec.calls
    # a CSV path next to the job file resolves relative to the job
    (tmp_path / "p.csv").write_text("x_mm,y_mm,z_mm\n3,4,0\n6,4,0\n")
    (tmp_path / "job.yaml").write_text("torch_path_csv: p.csv\n")
    assert job_waypoints(str(tmp_path / "job.yaml")) == [(0.003, 0.004, 0.0), (0.006, 0.004, 0.0)]


def test_run_path_rejects_bad_jobs(tmp_path):
    from waam_solver_b200.torch_path import job_waypoints
    with pytest.raises(FileNotFoundError):
        job_waypoints(str(tmp_path / "missing.yaml"))
    with pytest.raises(TypeError):
        job_waypoints(42)
    with pytest.raises(ValueError):
        job_waypoints([(0.001, 0.002)])
    (tmp_path / "empty.yaml").write_text("")
    assert job_waypoints(str(tmp_path / "empty.yaml")) == []


@pytest.mark.gpu
def test_run_path_yaml_job_matches_oracle():
    """A twin with the trailing-pool freeze on (it reads the torch direction)
    follows the YAML job with interpass parking; the oracle takes the
    reference's recorded step calls; the states agree."""
    import torch
    from oracle.oracle_step import OracleTwin
    from waam_solver_b200 import WAAMTwin
    from waam_solver_b200.materials import from_constants
    from waam_solver_b200.physics.arc import Goldak3D
    ref = _fixture()["yaml_interpass"]
    nx, ny, nz, dx = ref["nx"], ref["ny"], 24, ref["dx"]
    kw = dict(heat_source="goldak", arc_power_W=3000.0, arc_efficiency=0.78, droplet_freq_hz=0.0,
              use_srt=False, enable_vof=True, travel_speed_m_s=ref["travel"],
              enable_bead_freeze=True, enable_substrate_growth=True)
    gk = dict(ff=0.6, fr=1.4, a_front=4.0, a_rear=10.0, b=4.0, c=3.0)
    mat = from_constants("m", steps.MATERIAL, contact_angle_deg=30.0)
    tw = WAAMTwin(material=mat, nx=nx, ny=ny, nz=nz, dx=dx, max_tracers=64, device="cuda:0",
                  **kw)
    tw.arc_source = Goldak3D(**gk)
    tw.reset()
    ot = OracleTwin(nx, ny, nz, dx, steps.MATERIAL, goldak=gk, **kw)
    ot.reset()
    import state_gen
    st = state_gen.seeded_state(nx, ny, nz, seed=5, nz_solid=tw.nz_solid, hot=(14.0, 16.0, tw.nz_solid + 1.0))
    st = {k: v for k, v in st.items() if k != "nz_solid"}
    st["read_is_a"] = True
    tw.grid.load_state(st)
    ot.load(st)
    tw.run_path(JOB, n_steps=ref["n_steps"], interpass_steps=7)
    ot.dir = tuple(ref["torch_dir"])
    for x, y, wl, z in ref["calls"]:
        ot.step(x, y, wl, z)
    torch.cuda.synchronize()
    assert tw._step_n == len(ref["calls"])
    np.testing.assert_allclose(tw._torch_dir_xyz, ot.dir, rtol=0, atol=1e-12)
    steps.compare_state("run_path", tw.grid.state_dict(), ot.s)
