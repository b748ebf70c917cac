"""Telemetry (twin.py:706-821) against the reference's own get_telemetry on
three states (tests/golden/telemetry.npz): a seeded pool with tracers and
deposited solid, the same state without liquid, and the reset state.

CPU: the host halves (toe angle from the column, bead height from the
maximum deposited k) on the fixture arrays.  GPU: the device record
(waam_telemetry_pool) and the assembled dictionary, key by key; probes and
the CTWD update."""
import json
import math
import os

import numpy as np
import pytest

import cases
import steps

CASES = ["pool", "frozen", "reset"]
GAS, SOLID = 2, 1


def _load(name):
    z = np.load(os.path.join(cases.GOLDEN, "telemetry.npz"))
    fields = {f: np.ascontiguousarray(z["%s_%s" % (name, f)]) for f in (
        "T", "H", "f_l", "phi", "dT_dt", "ux", "uy", "uz", "flags", "porosity_active")}
    return fields, json.loads(str(z["%s_telemetry" % name])), json.loads(str(z["%s_state" % name]))


@pytest.mark.parametrize("name", CASES)
def test_host_toe_angle_and_bead_height(name):
    from waam_solver_b200.physics.bead_geometry import (bead_height_m_from_k,
                                                        toe_angle_from_column)
    f, tele, st = _load(name)
    nx, ny, nz = f["phi"].shape
    nz_solid, dx = st["nz_solid"], 2e-4
    k0, k1 = max(0, nz_solid - 1), min(nz - 1, nz_solid + 8)
    col = f["phi"][nx // 3, ny // 2, k0:k1]
    fl = f["flags"][nx // 3, ny // 2, k0:k1]
    assert round(toe_angle_from_column(col, fl, k0, 30.0, dx), 1) == tele["toe_angle_deg"]
    solid = np.argwhere(f["flags"] == SOLID)
    dep = solid[solid[:, 2] >= nz_solid][:, 2]
    k_max = int(dep.max()) if dep.size else -1
    assert round(bead_height_m_from_k(k_max, nz_solid, dx) * 1000.0, 3) == tele["bead_height_mm"]


def _twin(name):
    from waam_solver_b200 import WAAMTwin
    f, tele, st = _load(name)
    kw = dict(st["twin_kw"])
    nx, ny, nz = kw.pop("nx"), kw.pop("ny"), kw.pop("nz")
    plate = kw.pop("plate_thickness_mm")
    feed = kw.pop("wire_feed_m_s")
    mat, _, _ = steps.material_for("x", {"material": st["material"]})
    tw = WAAMTwin(material=mat, nx=nx, ny=ny, nz=nz, dx=2e-4, max_tracers=64,
                  contact_angle_deg=30.0, **kw)
    tw.plate_thickness_mm = plate
    tw.wire_feed_m_s = feed
    tw.reset()
    assert tw.nz_solid == st["nz_solid"]
    tw.grid.load_state({k: v for k, v in f.items() if k != "porosity_active"})
    import torch
    tw.grid.porosity_active.copy_(torch.from_numpy(f["porosity_active"]))
    tw._step_n = st["step"]
    tw._deposited_volume_m3 = st["deposited"]
    tw._n_droplets_fired = st["n_drops"]
    return tw, f, tele


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_telemetry_matches_reference(name):
    tw, f, want = _twin(name)
    got = tw.get_telemetry()
    for key, v in want.items():
        if key in ("material_status", "material_name", "force_diagnostics"):
            continue
        g = got[key]
        if isinstance(v, float):
            assert g == pytest.approx(v, rel=1e-9, abs=1e-12), (key, g, v)
        else:
            assert g == v, (key, g, v)
    # the FP64 enthalpy sum of the record
    assert got["total_enthalpy_J"] == pytest.approx(
        float(f["H"].astype(np.float64).sum()) * (2e-4) ** 3, rel=1e-12)


@pytest.mark.gpu
def test_gpu_telemetry_pool_reduce_buffers():
    """The reference-signature wrapper fills its 0-d buffers on the device."""
    import torch
    from waam_solver_b200 import kernels
    tw, f, want = _twin("pool")
    g = tw.grid
    bufs = [torch.zeros((), dtype=torch.int32, device="cuda")] + \
           [torch.zeros((), dtype=torch.float32, device="cuda") for _ in range(7)]
    kernels.telemetry_pool_reduce(g.T, g.f_l, g.phi, g.dT_dt, g.ux, g.uy, g.uz, *bufs)
    n, T_peak, cool, u2, i_sum, i_min, i_max, T_glob = [b.item() for b in bufs]
    liq = f["f_l"] > 0.5
    ii = np.nonzero(liq)[0]
    assert n == int(liq.sum()) == want["n_liquid_cells"]
    assert T_peak == float(f["T"][liq].max()) and T_glob == float(f["T"].max())
    assert cool == float(np.max(-f["dT_dt"][f["phi"] > 0.05]))
    assert i_sum == float(ii.sum()) and i_min == ii.min() and i_max == ii.max()
    u2_ref = (f["ux"] * f["ux"] + f["uy"] * f["uy"] + f["uz"] * f["uz"])[liq].max()
    assert u2 == float(u2_ref)


@pytest.mark.gpu
def test_gpu_probes_and_ctwd(tmp_path):
    import torch
    from waam_solver_b200.probes import ProbeRecorder
    tw, f, want = _twin("pool")
    rec = ProbeRecorder()
    rec.add_grid(9, 7, 4, tw, "center")
    rec.add_world_mm(1.0, 1.4, 0.9, tw)
    rec.add_world_mm(100.0, 0.0, 0.0, tw, "outside")
    tw.probe_recorder = rec
    for s in range(3):
        tw.step(9 * 2e-4, 7 * 2e-4, True)
    torch.cuda.synchronize()
    rows = rec.rows
    assert [r["step"] for r in rows] == [124, 125, 126]     # the fixture state is at step 123
    T = tw.grid.T.cpu().numpy()
    assert rows[-1]["center_T_K"] == round(float(T[9, 7, 4]), 2)
    i, j, k = rec.probes[1].resolve(tw)
    assert rows[-1]["probe_1_T_K"] == round(float(T[i, j, k]), 2)
    assert math.isnan(rows[-1]["outside_T_K"])
    rec.write_csv(tmp_path / "p.csv")
    assert (tmp_path / "p.csv").read_text().splitlines()[0].startswith("sim_time_ms,step,center")
    # CTWD follows the measured bead height (electrical_stickout.py:53-59)
    flags = tw.grid.flags.cpu().numpy()
    solid = np.argwhere(flags == SOLID)
    dep = solid[solid[:, 2] >= tw.nz_solid][:, 2]
    h_exp = (int(dep.max()) - tw.nz_solid + 1) * 2e-4 if dep.size else 0.0
    tw.enable_ctwd = True
    tw.layer_height_m = 0.2e-3
    tw.step(9 * 2e-4, 7 * 2e-4, True)
    h = tw._bead_height_m
    assert h == pytest.approx(h_exp, rel=1e-12) and h > 0
    assert tw.ctwd_m == pytest.approx(max(tw.ctwd_nominal_m,
                                          tw.ctwd_nominal_m + (h - tw.layer_height_m)))
