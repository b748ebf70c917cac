#!/usr/bin/env python
"""Throughput of the coupled melt-pool step on B200 (MLUPS, HBM roofline).

Workload (default): the standard-size bead-on-plate case -- 256x128x96 D3Q19
lattice, dx = 0.2 mm, constants-only ER70S-6-like steel, Goldak double
ellipsoid (a_f 3 / a_r 9 / b 3 / c 3 mm, ff 0.6 / fr 1.4), 4 kW, eta 0.78,
1.2 mm wire at 6 m/min as pulsed 100 Hz droplets, VOF with 30 deg wetting,
CSF, Marangoni, buoyancy, hydrostatic gravity, two-rate central-moment
collision, torch on a straight 40 mm line at 8 mm/s.  Synthetic inputs: the
run starts from the reference's reset state and spins up (droplets deposit a
bead) before timing.  One step = one ``WAAMTwin.step``.

``--workload large``: the large FP16-storage case -- 512x256x160 lattice,
dx = 0.15 mm, float16 population offsets, the same arc, wire and surface
physics plus the welding current's Lorentz force (140 A) and convective heat
losses, on a two-layer path of three parallel 60 mm beads (4 mm pitch, 8 mm/s;
the arc off on the moves between beads; a 5 s dwell; the second layer offset
2 mm).  ``--compare-steps N`` runs that workload N steps from reset in its own
storage and in float32 and reports remelt depth, HAZ peak temperature, pool
width / depth and peak temperature of both.

``python bench.py [--gpus N] [--steps K] [--warmup W]`` prints one JSON line.
Under torchrun every rank runs an independent replica (the step has no
cross-GPU exchange), timing is the max over ranks.
``--impl reference`` times the CPU restatement of the reference step (the
oracle, all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "standard": dict(
        workload="bead-on-plate 256x128x96 D3Q19, dx 0.2 mm, Goldak 4 kW, 100 Hz wire droplets, "
                 "VOF+wetting 30deg+CSF+Marangoni+buoyancy+gravity, central-moment MRT",
        nx=256, ny=128, nz=96, dx=2e-4, heat_source="goldak", arc_power_W=4000.0,
        arc_efficiency=0.78, goldak_mm=dict(a_front_mm=3.0, a_rear_mm=9.0, b_mm=3.0, c_mm=3.0,
                                            ff=0.6, fr=1.4),
        droplet_freq_hz=100.0, wire_feed_m_s=0.1, wire_diameter_mm=1.2, enable_vof=True,
        enable_wetting=True, contact_angle_deg=30.0, enable_csf_tension=True,
        enable_hydrostatic_gravity=True, use_srt=False, travel_speed_m_s=0.008,
        path_mm=((5.6, 12.8), (45.6, 12.8)), spinup=200),
    "small": dict(
        workload="bead-on-plate 64x32x32 D3Q19, dx 0.25 mm, Gaussian 3 kW r 3 mm, no wire, VOF, "
                 "central-moment MRT",
        nx=64, ny=32, nz=32, dx=2.5e-4, heat_source="gaussian2d", arc_power_W=3000.0,
        arc_efficiency=0.75, arc_sigma_mm=3.0, droplet_freq_hz=0.0, enable_vof=True,
        plate_thickness_mm=4.0, use_srt=False, travel_speed_m_s=0.008,
        path_mm=((4.0, 4.0), (14.0, 4.0)), spinup=200),
    "large": dict(
        workload="two-layer multi-bead 512x256x160 D3Q19, dx 0.15 mm, float16 population "
                 "storage, Goldak 4 kW, 100 Hz wire droplets, Lorentz force (140 A) + arc "
                 "pressure, convective heat losses, VOF+wetting 30deg+CSF+Marangoni+buoyancy+"
                 "gravity, central-moment MRT; 3 x 60 mm beads, pitch 4 mm, 8 mm/s, 5 s dwell, "
                 "second layer offset 2 mm",
        nx=512, ny=256, nz=160, dx=1.5e-4, heat_source="goldak", arc_power_W=4000.0,
        arc_efficiency=0.78, goldak_mm=dict(a_front_mm=3.0, a_rear_mm=9.0, b_mm=3.0, c_mm=3.0,
                                            ff=0.6, fr=1.4),
        droplet_freq_hz=100.0, wire_feed_m_s=0.1, wire_diameter_mm=1.2, enable_vof=True,
        enable_wetting=True, contact_angle_deg=30.0, enable_csf_tension=True,
        enable_hydrostatic_gravity=True, use_srt=False, travel_speed_m_s=0.008,
        enable_heat_loss=True, enable_lorentz=True, welding_current_A=140.0,
        population_dtype="float16",
        beads=dict(x0_mm=8.4, length_mm=60.0, y0_mm=15.2, pitch_mm=4.0, n=3, layers=2,
                   layer_offset_mm=2.0, dwell_s=5.0),
        path_mm=((8.4, 15.2), (68.4, 15.2)), spinup=200),
}

MATERIAL = dict(k=30.0, rho=7800.0, cp=680.0, T_solidus=1723.0, T_liquidus=1783.0,
                L_fusion=2.7e5, gamma_0=1.8, dgamma_dT=-4.3e-4, mu=0.0065, beta_T=1.2e-4)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def twin_kwargs(w):
    keys = ("heat_source", "arc_power_W", "arc_efficiency", "droplet_freq_hz", "enable_vof",
            "enable_wetting", "contact_angle_deg", "enable_csf_tension",
            "enable_hydrostatic_gravity", "use_srt", "travel_speed_m_s", "arc_sigma_mm",
            "wire_diameter_mm", "enable_heat_loss", "enable_lorentz", "welding_current_A")
    return {k: w[k] for k in keys if k in w}


def build_twin(w, device, population_dtype=None, tables=None):
    from waam_solver_b200 import WAAMTwin
    from waam_solver_b200.materials import from_constants
    from waam_solver_b200.physics.arc import goldak_from_job_mm
    mat = from_constants("ER70S-6-constants", MATERIAL, contact_angle_deg=w.get("contact_angle_deg", 30.0))
    if tables is not None:
        mat.tables = tables
    if population_dtype is None:
        population_dtype = w.get("population_dtype", "float32")
    tw = WAAMTwin(material=mat, nx=w["nx"], ny=w["ny"], nz=w["nz"], dx=w["dx"], max_tracers=1024,
                  device=device, population_dtype=population_dtype, **twin_kwargs(w))
    if w.get("plate_thickness_mm"):
        tw.plate_thickness_mm = w["plate_thickness_mm"]
    if w.get("wire_feed_m_s"):
        tw.wire_feed_m_s = w["wire_feed_m_s"]
        tw.droplet_transfer_mode = "pulsed"
        tw.pulse_frequency_hz = w["droplet_freq_hz"]
        tw.droplet_size_jitter = 0.0
    if w.get("goldak_mm"):
        tw.arc_source = goldak_from_job_mm(tw, w["goldak_mm"])
    tw.reset()
    return tw


def positions(w, dt, n, start=0):
    (x0, y0), (x1, y1) = w["path_mm"]
    L = math.hypot(x1 - x0, y1 - y0) * 1e-3
    out = []
    for s in range(start, start + n):
        d = min(s * dt * w["travel_speed_m_s"], L)
        u = d / L
        out.append((x0 * 1e-3 + u * (x1 - x0) * 1e-3, y0 * 1e-3 + u * (y1 - y0) * 1e-3))
    return out


def path_steps(w, dt, n):
    """(x, y, welding) of the first n steps.  A workload with ``beads``: bead
    after bead along +x at the travel speed with the arc on, the moves between
    beads (back to the next bead's start) at the travel speed with the arc off,
    the dwell between layers parked with the arc off."""
    b = w.get("beads")
    if not b:
        return [(x, y, True) for x, y in positions(w, dt, n)]
    v = w["travel_speed_m_s"]
    segs = []          # (x0, y0, x1, y1, duration_s, welding)
    for layer in range(b["layers"]):
        for k in range(b["n"]):
            y = (b["y0_mm"] + k * b["pitch_mm"] + layer * b["layer_offset_mm"]) * 1e-3
            x0, x1 = b["x0_mm"] * 1e-3, (b["x0_mm"] + b["length_mm"]) * 1e-3
            if segs:
                px, py = segs[-1][2], segs[-1][3]
                L = math.hypot(x0 - px, y - py)
                segs.append((px, py, x0, y, L / v, False))
            segs.append((x0, y, x1, y, (x1 - x0) / v, True))
        if layer + 1 < b["layers"]:
            px, py = segs[-1][2], segs[-1][3]
            segs.append((px, py, px, py, b["dwell_s"], False))
    out, t, si, t0 = [], 0.0, 0, 0.0
    for s in range(n):
        t = s * dt
        while si < len(segs) - 1 and t >= t0 + segs[si][4]:
            t0 += segs[si][4]
            si += 1
        x0, y0, x1, y1, dur, wl = segs[si]
        u = min(1.0, (t - t0) / dur) if dur > 0 else 1.0
        out.append((x0 + u * (x1 - x0), y0 + u * (y1 - y0), wl))
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        """Median SM clock of the samples taken under load (power draw at least
        half of the run's maximum), the maximum clock, and every throttle
        reason seen in any sample of the run."""
        rows, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm_mhz, smax, pw = float(parts[1]), float(parts[2]), float(parts[3])
            except ValueError:
                continue
            rows.append((sm_mhz, pw))
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        pmax = max((pw for _, pw in rows), default=0.0)
        load = [m for m, pw in rows if pw >= 0.5 * pmax]
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(load),
                "coverage": "the whole run: spin-up, timed steps, stage timing, end-to-end "
                            "and droplet-period timing (nvidia-smi every 200 ms)"}


def census(twin):
    import torch
    f = twin.grid.flags
    n = f.numel()
    solid = int((f == 1).sum().item())
    gas = int((f == 2).sum().item())
    return dict(n=n, solid=solid, gas=gas, fluid=n - solid - gas)


def algorithmic_bytes(c, tail_on=False, pop_bytes=4):
    """Compulsory DRAM bytes per launch of each fused stage (FP32 fields, int32
    flags), from the cell census; each field element read or written once.

    n cells, ns non-solid, ng non-gas, na active (FLUID/IFACE):
      arc        norm: flags n, f_l ng; inject: flags n, f_l ng, H r+w ng (ceiling on)
      thermal    flags, H, H_next, T_next, f_l: n; T, T_max r+w, T_prev r+w,
                 dT_dt: ng; ux, uy, uz: na
      vof_advect flags, phi, phi_tmp: n; ux, uy, uz: na
      column     phi_tmp, phi, flags r+w, f_l: n; T, 3 time-above r+w: ng; list: na
      collide    list, f_l, phi, T, flags, 19 f reads, 19 f writes, rho, u (3), F (3): na
      stream     flags: n; 19 f reads + 19 f writes: ns
    (populations of pop_bytes each: 4 for float32, 2 for the 16-bit forms)
      tail       flags: n; T, phi, f_l: ng (only when remelt / solidify run)
    Neighbour reads of the stencils are cache hits and are not counted.
    """
    n, ns, ng, na = c["n"], c["n"] - c["solid"], c["n"] - c["gas"], c["fluid"]
    return {
        "arc": 8 * n + 16 * ng,
        "thermal": 20 * n + 24 * ng + 12 * na,
        "vof_advect": 12 * n + 12 * na,
        "column": 20 * n + 28 * ng + 4 * na,
        "collide": (48 + 38 * pop_bytes) * na,
        "stream": 4 * n + 38 * pop_bytes * ns,
        "tail": (4 * n + 12 * ng) if tail_on else 0,
    }


STAGES = ["thermal", "vof_advect", "column", "collide", "stream", "tail"]


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def dist_max(x):
    """The maximum of x over the ranks (x itself without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def cpu_baseline(w, budget_s=15.0, max_steps=400):
    """The CPU oracle (C restatement, OpenMP on all host cores) on the same
    workload and state as the GPU arm: reset, the workload's spin-up steps on
    the same torch path, then as many full steps as fit the time budget."""
    from oracle.oracle_step import OracleTwin
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    O.lib()
    O.call("wo_set_num_threads", threads)
    kw = twin_kwargs(w)
    kw.pop("wire_diameter_mm", None)
    g = None
    if w.get("goldak_mm"):
        gm = w["goldak_mm"]
        dxmm = w["dx"] * 1e3
        g = dict(ff=gm["ff"], fr=gm["fr"], a_front=gm["a_front_mm"] / dxmm,
                 a_rear=gm["a_rear_mm"] / dxmm, b=gm["b_mm"] / dxmm, c=gm["c_mm"] / dxmm)
    extra = {}
    if w.get("wire_feed_m_s"):
        extra = dict(wire_feed_m_s=w["wire_feed_m_s"], droplet_transfer_mode="pulsed",
                     pulse_frequency_hz=w["droplet_freq_hz"], droplet_size_jitter=0.0)
    if w.get("plate_thickness_mm"):
        extra["plate_thickness_mm"] = w["plate_thickness_mm"]
    mat = dict(MATERIAL, contact_angle_deg=w.get("contact_angle_deg", 30.0))
    ot = OracleTwin(w["nx"], w["ny"], w["nz"], w["dx"], mat, goldak=g, **kw, **extra)
    ot.reset()
    spin = int(w["spinup"])
    pos = path_steps(w, ot.dt, spin + max_steps)
    t_spin = time.perf_counter()
    for x, y, wl in pos[:spin]:
        ot.step(x, y, wl)
    t_spin = time.perf_counter() - t_spin
    d0 = ot.n_drops
    t0 = time.perf_counter()
    n = 0
    while n < max_steps and (time.perf_counter() - t0) < budget_s:
        ot.step(*pos[spin + n])
        n += 1
    el = time.perf_counter() - t0
    cells = w["nx"] * w["ny"] * w["nz"]
    return {"value": cells * n / el / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "droplets": ot.n_drops - d0,
            "sample": "%d full steps of the %dx%dx%d workload after reset and the same %d "
                      "spin-up steps as the GPU arm (spin-up %.1f s, timed %.1f s)" % (
                          n, w["nx"], w["ny"], w["nz"], spin, t_spin, el)}


def run_reference(args, w):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    budget = max(5.0, min(60.0, 2.0 * args.steps))
    cb = cpu_baseline(w, budget_s=budget, max_steps=max(args.steps, 3))
    line = {"impl": "reference", "metric": "coupled step throughput (MLUPS)", "value": cb["value"],
            "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (reference reset state + %d spin-up steps)" % w["spinup"],
            "config": bench_config(w, world, 4, cb["droplets"]), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _time_variant(tw, w, device, K):
    """Whole-step time over K device-resident steps after the workload's
    spin-up, and the stage times of 200 instrumented steps."""
    import torch
    g = tw.grid
    pos = positions(w, g.dt, w["spinup"] + K + 204)
    s = 0
    for _ in range(w["spinup"]):
        tw.step(*pos[s], True)
        s += 1
    dev_pos = torch.tensor([[x / g.dx, y / g.dx] for x, y in pos[s:s + K]],
                           dtype=torch.float32, device=device)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(K):
        tw._device_position = dev_pos[k]
        tw.step(*pos[s], True)
        s += 1
    e1.record()
    torch.cuda.synchronize()
    tw._device_position = None
    ms = e0.elapsed_time(e1) / K
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(7)] for _ in range(200)]
    for es in evs:
        for e in es:
            e.record()
    for es in evs:
        tw._stage_events = es
        tw.step(*pos[s], True)
        s += 1
    torch.cuda.synchronize()
    tw._stage_events = None
    stages = [statistics.fmean(es[q].elapsed_time(es[q + 1]) for es in evs) for q in range(6)]
    return ms, stages


def storage_forms(w, device, K, ref_ms):
    """The same workload with 16-bit population storage (float16 / bfloat16
    offsets from the rest weights): whole-step time over K device-resident
    steps after the same spin-up, plus the stream stage alone."""
    import torch
    out = {}
    for dtype in ("float16", "bfloat16"):
        tw = build_twin(w, device, population_dtype=dtype)
        g = tw.grid
        ms, stages = _time_variant(tw, w, device, K)
        stream_ms = stages[4]
        c = census(tw)
        stream_bytes = 4 * c["n"] + 76 * (c["n"] - c["solid"])
        out[dtype] = {"value": g.n_cells / (ms * 1e-3) / 1e6, "unit": "MLUPS", "ms_per_step": ms,
                      "vs_float32": ref_ms / ms, "stream_ms": stream_ms,
                      "stream_GBps": stream_bytes / (stream_ms * 1e-3) / 1e9, "steps": K}
        del tw, g
        torch.cuda.empty_cache()
    return out


def table_material():
    """The workload's steel with temperature tables in the layout of a
    validated material file: cp, k and mu at three knots around the constants
    and the Sahoo-DebRoy dgamma/dT table (28 ppm S, 8 knots)."""
    from waam_solver_b200.materials import MaterialTables, build_sahoo_dgamma_table
    m, Tl = MATERIAL, MATERIAL["T_liquidus"]
    return MaterialTables(
        cp=[(300.0, 0.95 * m["cp"]), (1000.0, m["cp"]), (Tl, 1.06 * m["cp"])],
        k=[(300.0, 0.93 * m["k"]), (1000.0, m["k"]), (Tl, 1.13 * m["k"])],
        mu=[(300.0, 1.15 * m["mu"]), (Tl, m["mu"]), (Tl + 200.0, 0.85 * m["mu"])],
        dgamma_dT=build_sahoo_dgamma_table(28.0, Tl, max(Tl + 800.0, 2600.0), n=8))


def table_form(w, device, K, ref_ms, ref_stages):
    """The workload on the material-table path (per-cell properties refreshed
    from T inside the thermal stage, variable-tau SRT collision)."""
    import torch
    tw = build_twin(w, device, tables=table_material())
    assert tw.use_material_tables
    ms, stages = _time_variant(tw, w, device, K)
    out = {"value": tw.grid.n_cells / (ms * 1e-3) / 1e6, "unit": "MLUPS", "ms_per_step": ms,
           "vs_constants": ref_ms / ms, "thermal_ms": stages[0],
           "thermal_ms_constants": ref_stages.get("thermal"), "collide_ms": stages[3],
           "collide_ms_constants": ref_stages.get("collide"), "steps": K,
           "material": "workload constants + cp/k/mu tables (3 knots) + Sahoo dgamma/dT (8)"}
    del tw
    torch.cuda.empty_cache()
    return out


ADJOINT_C4 = dict(
    workload="differentiation 128x64x48 D3Q19, dx 0.25 mm, Goldak 3 kW (a_f 3 / a_r 9 / b 3 / c "
             "3 mm), 8 mm/s, VOF, heat losses, 2000 steps; loss: 8 surface probe traces + final "
             "smooth pool width",
    nx=128, ny=64, nz=48, dx=2.5e-4, heat_source="goldak", arc_power_W=3000.0,
    arc_efficiency=0.78, goldak_mm=dict(a_front_mm=3.0, a_rear_mm=9.0, b_mm=3.0, c_mm=3.0,
                                        ff=0.6, fr=1.4),
    droplet_freq_hz=0.0, enable_vof=True, use_srt=False, travel_speed_m_s=0.008,
    enable_heat_loss=True, steps=2000)


def _c4_problem(device, N, h_conv_scale=1.0):
    """The config-4 adjoint problem: probe targets from a run at perturbed
    parameters, the width target 0.1 mm above the base run's width."""
    import numpy as np
    from waam_solver_b200.adjoint import AdjointProblem
    w = dict(ADJOINT_C4)
    tw = build_twin(w, device)
    tw.h_conv = tw.h_conv * h_conv_scale
    g = tw.grid
    dx = g.dx
    x0, yc = 10e-3, (g.ny // 2) * dx
    pos = [(x0 + s * g.dt * w["travel_speed_m_s"], yc) for s in range(N)]
    rng = np.random.default_rng(0)
    probes = []
    for _ in range(8):
        off = rng.uniform(2e-3, 6e-3) * (1 if rng.random() < 0.5 else -1)
        probes.append((int(rng.uniform(x0 - 2e-3, x0 + 3e-3) / dx), int((yc + off) / dx),
                       tw.nz_solid - 1))
    prob = AdjointProblem(tw, pos, probes)
    base = prob.theta.copy()
    prob.forward(base * np.array([1.05, 1.2, 1.0, 1.1, 0.9, 1.1, 1.1]))
    prob.T_target = prob.T_probe.copy()
    prob.W_target, _ = prob.width()
    prob.W_target += 0.1
    prob.w_T, prob.w_W = 1e-3, 10.0
    return prob, base


FD64_FIXTURE = os.path.join(ROOT, "tests", "golden", "adjoint_fd64.npz")


def fd64_problem(device, variant):
    """The config-4 problem of ``oracle/adjoint_fd64.py`` (variant ``c4`` from
    reset, ``c4_pool`` from its seeded molten pool) on the GPU, with the FP64
    run's targets: (problem, fixture metadata, FP64 probe temperatures at the
    base parameters)."""
    import numpy as np
    from waam_solver_b200.adjoint import AdjointProblem
    z = np.load(FD64_FIXTURE)
    meta = json.loads(str(z[variant + "_meta"]))
    tw = build_twin(dict(ADJOINT_C4), device)
    g = tw.grid
    yc = (g.ny // 2) * g.dx
    if variant.split("@")[0] == "c4_pool":   # "<variant>@<step>": another difference step
        tests = os.path.join(ROOT, "tests")
        if tests not in sys.path:
            sys.path.insert(0, tests)
        import state_gen
        st = state_gen.seeded_state(g.nx, g.ny, g.nz, seed=meta["pool_seed"],
                                    nz_solid=tw.nz_solid,
                                    hot=(meta["x0"] / g.dx + 2.0, yc / g.dx, tw.nz_solid + 1.0))
        st = {k: v for k, v in st.items() if k != "nz_solid"}
        st["read_is_a"] = True
        g.load_state(st)
    pos = [(meta["x0"] + s * g.dt * meta["travel"], yc) for s in range(meta["steps"])]
    prob = AdjointProblem(tw, pos, [tuple(p) for p in meta["probes"]],
                          T_target=z[variant + "_T_target"], W_target=meta["W_target"],
                          w_T=meta["w_T"], w_W=meta["w_W"], beta=meta["beta"])
    assert np.allclose(prob.theta, meta["theta"], rtol=1e-12, atol=0.0), (prob.theta, meta)
    return prob, meta, z[variant + "_T_base"]


def adjoint_fd64(device):
    """The adjoint's gradient against central differences (relative step
    1e-3) of the FP64 oracle forward (``oracle/adjoint_fd64.py``): config 4
    from reset and from a seeded molten pool (non-zero width term)."""
    import numpy as np
    if not os.path.exists(FD64_FIXTURE):
        return None
    from waam_solver_b200.adjoint import PARAMS
    out = {}
    with np.load(FD64_FIXTURE) as z:
        variants = [k[:-5] for k in z.files if k.endswith("_meta")]
    for variant in variants:
        prob, meta, T64 = fd64_problem(device, variant)
        loss = prob.forward(prob.theta)
        grad = prob.backward()
        rel = {}
        for q, name in enumerate(PARAMS):
            if name not in meta["fd"]:
                rel[name] = {"adjoint": float(grad[q]), "fd_fp64": 0.0,
                             "note": "structural zero (nothing of this configuration reads it)"}
                continue
            f = meta["fd"][name]
            rel[name] = {"adjoint": float(grad[q]), "fd_fp64": f,
                         "rel_diff": abs(grad[q] - f) / max(abs(f), 1e-300)}
        out[variant] = {"steps": meta["steps"], "fd_step": meta["fd_step"], "loss_float32": loss,
                        "loss_fp64": meta["loss_base"], "width_mm": prob.width()[0],
                        "probe_T_max_abs_diff_vs_fp64": float(np.abs(prob.T_probe - T64).max()),
                        "gradient": rel}
        del prob
        import torch
        torch.cuda.empty_cache()
    return out


def _central_fd(prob, base, q, step):
    h = step * abs(base[q])
    tp, tm = base.copy(), base.copy()
    tp[q] += h
    tm[q] -= h
    return (prob.forward(tp) - prob.forward(tm)) / (2 * h)


def adjoint_form(device, n_steps=None, fd=True):
    """Config 4: loss + gradient with the hand-written adjoint (sqrt(N)
    checkpointing), backward time against forward time (CUDA events), and
    central finite differences (relative step 1e-3) of every parameter."""
    import torch
    from waam_solver_b200.adjoint import PARAMS
    w = dict(ADJOINT_C4)
    N = int(n_steps or w["steps"])
    prob, base = _c4_problem(device, N)
    prob.forward(base)                     # warm-up of both passes
    prob.backward()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    torch.cuda.synchronize()
    e[0].record()
    loss = prob.forward(base)
    e[1].record()
    grad = prob.backward()
    e[2].record()
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    out = {"config": w["workload"], "steps": N, "checkpoint_every": prob.K,
           "loss": loss, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
           "backward_over_forward": bwd_ms / fwd_ms,
           "gradient": {k: float(v) for k, v in zip(PARAMS, grad)}}
    if fd:
        # the specified step (1e-3 relative) and a 1e-2 one: the forward is
        # float32, so where a parameter moves the loss little the 1e-3
        # difference is dominated by rounding noise of the two forwards
        for step, key in ((1e-3, "central_fd_rel_step_1e-3"), (1e-2, "central_fd_rel_step_1e-2")):
            rel = {}
            for q, name in enumerate(PARAMS):
                if base[q] == 0.0:
                    continue
                f = _central_fd(prob, base, q, step)
                rel[name] = {"fd": f, "rel_diff": abs(grad[q] - f) / max(abs(f), 1e-300)}
            out[key] = rel
        # At h_conv 25 W/m^2K one step's convective loss from a surface cell
        # is a few float32 ULPs of its enthalpy (dt 25 us, H ~ 4e9 J/m^3, ULP
        # 256), so a 1 % change of the factor moves H_next by ~0.05 ULP and the
        # float32 forward answers it through rounding.  The same problem with
        # h_conv x1000 resolves the term: there the difference measures the
        # adjoint's heat-loss derivative itself.
        del prob
        torch.cuda.empty_cache()
        q = PARAMS.index("heat_loss_factor")
        prob, base = _c4_problem(device, N, h_conv_scale=1000.0)
        prob.forward(base)
        g_hl = float(prob.backward()[q])
        chk = {"h_conv_W_m2K": prob.tw.h_conv, "gradient": g_hl}
        for step in (1e-3, 1e-2):
            f = _central_fd(prob, base, q, step)
            chk["central_fd_rel_step_%g" % step] = {"fd": f, "rel_diff": abs(g_hl - f) / abs(f)}
        out["heat_loss_factor_at_h_conv_x1000"] = chk
    return out


def jacobi_timing(tw, reps=10):
    """The potential solve's sweep as the step runs it: 10-sweep chunks over the
    live-cell list of the twin's current state (the production entry point),
    timed with CUDA events on copies of the potential buffers."""
    import torch
    from waam_solver_b200 import kernels
    g = tw.grid
    a, b = g.phi_elec.clone(), g.phi_elec_tmp.clone()
    res, nrm = torch.zeros((), device=a.device), torch.zeros((), device=a.device)
    call = lambda: kernels.elec_jacobi_live(  # noqa: E731
        a, b, g.sigma_elec, g.elec_source, g.elec_live, g.elec_zero, g.elec_counts, g.dx,
        tw.lorentz_jacobi_omega, 10, False, g.step_scalars[0:1], tw.sigma_cells, res, nrm)
    call()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / (10 * reps)
    live = int(g.elec_counts[0].item())
    # per live cell: phi in, phi out, sigma (4 B each) and its list entry (4 B),
    # the source (4 B) inside its k slab; neighbour reads are cache hits
    nbytes = 20 * live
    return {"sweeps_per_step": int(tw._lorentz_last_iters), "live_cells": live,
            "ms_per_sweep": ms, "bytes_per_sweep": nbytes,
            "sweep_GBps": nbytes / (ms * 1e-3) / 1e9,
            "timing": "10-sweep chunks over the live-cell list of the state after the "
                      "stage-timing steps, CUDA events, %d repetitions" % reps}


def melt_metrics(tw):
    """Remelt depth, HAZ peak temperature and pool size from the step's fields.

    remelt depth: how far below the original plate top (k = nz_solid - 1) the
    metal reached the solidus (T_max >= T_s); HAZ T_max: the highest T_max in
    the substrate plane 1 mm below the deepest remelted cell; pool width /
    depth: extent of f_l > 0.5 across y and down from the top of the pool in
    the x section through the pool's centroid.  Also whether H is finite and
    the largest |rho - 1| of the FLUID/IFACE cells: the reference's LBM moves
    no populations into collided cells (streamed values land in the buffer
    the next collision overwrites), so a liquid cell under a steady force
    gathers momentum step after step and its density eventually diverges."""
    import numpy as np
    g = tw.grid
    Ts = tw.mat.T_solidus
    tmax = g.T_max.cpu().numpy().astype(np.float64)
    flags = g.flags.cpu().numpy()
    fl = g.f_l.cpu().numpy() > 0.5
    nzs = tw.nz_solid
    sub = tmax[:, :, :nzs]
    melted = np.nonzero((sub >= Ts).any(axis=(0, 1)))[0]
    k_melt = int(melted.min()) if melted.size else nzs
    depth_cells = nzs - k_melt
    k_haz = max(0, min(nzs - 1, k_melt - int(round(1e-3 / g.dx))))
    act = (flags == 0) | (flags == 4)
    rho = g.rho.cpu().numpy().astype(np.float64)
    out = {"finite": bool(np.isfinite(g.H.cpu().numpy()).all()),
           "rho_dev_max_active": float(np.abs(rho[act] - 1.0).max()) if act.any() else 0.0,
           "remelt_depth_mm": depth_cells * g.dx * 1e3, "remelt_depth_cells": depth_cells,
           "haz_plane_k": k_haz, "haz_T_max_K": float(tmax[:, :, k_haz].max()),
           "T_max_peak_K": float(tmax[flags != 2].max()) if (flags != 2).any() else None,
           "pool_width_cells": 0, "pool_depth_cells": 0,
           "H_total_J": float(g.H.double().sum().item()) * g.dx ** 3}
    if fl.any():
        ii = np.nonzero(fl)[0]
        sect = fl[int(round(ii.mean()))]
        ys, zs = np.nonzero(sect.any(axis=1))[0], np.nonzero(sect.any(axis=0))[0]
        if ys.size:
            out["pool_width_cells"] = int(ys[-1] - ys[0] + 1)
            out["pool_depth_cells"] = int(zs[-1] - zs[0] + 1)
    return out


def storage_comparison(w, device, n_steps):
    """The workload from reset for n_steps in its own population storage and
    in float32: sustained MLUPS of each run (CUDA events around all steps) and
    the melt metrics of both."""
    import torch
    out = {"steps": n_steps}
    forms = [w.get("population_dtype", "float32")]
    if forms[0] != "float32":
        forms.append("float32")
    for dtype in forms:
        tw = build_twin(w, device, population_dtype=dtype)
        g = tw.grid
        path = path_steps(w, g.dt, n_steps)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for x, y, wl in path:
            tw.step(x, y, wl)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / n_steps
        m = melt_metrics(tw)
        m.update(ms_per_step=ms, MLUPS=g.n_cells / (ms * 1e-3) / 1e6,
                 droplets=tw._n_droplets_fired, lorentz_unconverged=tw._lorentz_unconverged)
        out[dtype] = m
        del tw, g
        torch.cuda.empty_cache()
    if len(forms) == 2:
        a, b = out[forms[0]], out["float32"]
        out["difference"] = {
            "remelt_depth_cells": a["remelt_depth_cells"] - b["remelt_depth_cells"],
            "haz_T_max_rel": (a["haz_T_max_K"] - b["haz_T_max_K"]) / b["haz_T_max_K"],
            "T_max_peak_rel": (a["T_max_peak_K"] - b["T_max_peak_K"]) / b["T_max_peak_K"],
            "pool_width_cells": a["pool_width_cells"] - b["pool_width_cells"],
            "pool_depth_cells": a["pool_depth_cells"] - b["pool_depth_cells"],
            "H_total_rel": (a["H_total_J"] - b["H_total_J"]) / b["H_total_J"],
            "speedup": b["ms_per_step"] / a["ms_per_step"]}
    return out


def bench_config(w, world, pb, drops):
    """The workload record both arms print (identical keys and values)."""
    cells = w["nx"] * w["ny"] * w["nz"]
    return {"workload": w["workload"], "cells": cells, "global_batch": world,
            "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (populations %.0f MB)" % (2 * 19 * cells * pb / 1e6),
            "population_storage": "float16" if pb == 2 else "float32",
            "spinup_steps": w["spinup"], "droplets_in_timed_region": drops}


def droplet_period_steps(tw):
    """Steps per droplet of the twin's schedule (None without wire droplets)."""
    from waam_solver_b200.physics import deposition
    if tw.droplet_freq <= 0 or tw.wire_feed_m_s <= 0:
        return None
    return max(1, int(math.ceil(deposition.droplet_period_s(tw) / tw.grid.dt)))


def droplet_period_timing(tw, pos, s, period, device):
    """Whole-step time over one droplet period (the droplet step included),
    CUDA events around all steps, positions staged on the device."""
    import torch
    g = tw.grid
    dev_pos = torch.tensor([[x / g.dx, y / g.dx] for x, y, _ in pos[s:s + period]],
                           dtype=torch.float32, device=device)
    d0 = tw._n_droplets_fired
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(period):
        tw._device_position = dev_pos[k]
        tw.step(*pos[s + k])
    e1.record()
    torch.cuda.synchronize()
    tw._device_position = None
    ms = e0.elapsed_time(e1) / period
    return {"steps": period, "droplets": tw._n_droplets_fired - d0, "ms_per_step": ms,
            "value": g.n_cells / (ms * 1e-3) / 1e6, "unit": "MLUPS",
            "deposited_m3": tw._deposited_volume_m3}


def run_b200(args, w):
    import torch
    from waam_solver_b200 import _native
    world, rank, local = dist_setup()
    device = torch.device("cuda", local)
    clocks = ClockSampler(local).__enter__()     # sampled over the whole run
    tw = build_twin(w, device)
    g = tw.grid
    cells = g.n_cells
    period = droplet_period_steps(tw)
    total = (w["spinup"] + args.warmup + 2 * args.steps + min(args.steps, 400) + 4 +
             (period or 0))
    pos = path_steps(w, g.dt, total)
    lorentz = bool(w.get("enable_lorentz"))
    pb = 2 if g.population_storage else 4
    s = 0
    for _ in range(w["spinup"] + args.warmup):
        tw.step(*pos[s])
        s += 1
    torch.cuda.synchronize()

    # ---- device-resident run (value): positions staged on the device ----
    K = args.steps
    dev_pos_all = torch.tensor([[x / g.dx, y / g.dx] for x, y, _ in pos[s:s + K]],
                               dtype=torch.float32, device=device)
    dev_pos = [dev_pos_all[k] for k in range(K)]
    drops0 = tw._n_droplets_fired
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_host = time.perf_counter()
    start.record()
    for k in range(K):
        tw._device_position = dev_pos[k]
        tw.step(*pos[s])
        s += 1
    stop.record()
    host_ms = (time.perf_counter() - t_host) * 1e3 / K
    torch.cuda.synchronize()
    tw._device_position = None
    barrier()
    ms_local = start.elapsed_time(stop)
    ms = dist_max(ms_local)
    drops = tw._n_droplets_fired - drops0

    # ---- stage timing: the same step with events between the fused kernels ----
    Ks = min(K, 400)
    ev_sets = [[torch.cuda.Event(enable_timing=True) for _ in range(7)] for _ in range(Ks)]
    ev_pre = [torch.cuda.Event(enable_timing=True) for _ in range(Ks)]
    ev_lz = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
             for _ in range(Ks)]
    for es in ev_sets:
        for e in es:
            e.record()
    for es in ev_lz:
        for e in es:
            e.record()
    torch.cuda.synchronize()
    pre_steps, lz_steps = [], []
    for k in range(Ks):
        tw._stage_events = ev_sets[k]
        tw._lorentz_events = ev_lz[k] if lorentz else None
        due = tw._n_droplets_fired
        ev_pre[k].record()
        x, y, wl = pos[s]
        tw.step(x, y, wl)
        if tw._n_droplets_fired == due:
            pre_steps.append(k)     # the pre stage of droplet steps includes the deposition
        if lorentz and wl:
            lz_steps.append(k)
        s += 1
    torch.cuda.synchronize()
    tw._stage_events = None
    tw._lorentz_events = None
    stage_ms = {"pre": statistics.fmean(ev_pre[k].elapsed_time(ev_sets[k][0]) for k in pre_steps)}
    for i, name in enumerate(STAGES):
        stage_ms[name] = statistics.fmean(es[i].elapsed_time(es[i + 1]) for es in ev_sets)
    lz_info = None
    if lz_steps:
        # the potential solve runs between the column pass and the collision
        lz_ms = statistics.fmean(ev_lz[k][0].elapsed_time(ev_lz[k][1]) for k in lz_steps)
        stage_ms["lorentz_solve"] = lz_ms
        stage_ms["collide"] = statistics.fmean(
            ev_sets[k][3].elapsed_time(ev_sets[k][4]) - ev_lz[k][0].elapsed_time(ev_lz[k][1])
            for k in lz_steps)
        lz_info = jacobi_timing(tw)
    c = census(tw)
    algo = algorithmic_bytes(c, tw.enable_bead_freeze or tw.enable_substrate_growth, pb)
    hbm, hbm_src = peaks()
    dom = max(("stream", "collide", "thermal", "column", "vof_advect"),
              key=lambda k: stage_ms[k])
    dom_ms, dom_bytes, kernel = stage_ms[dom], algo[dom], "k_" + dom
    if lz_info and lz_info["ms_per_sweep"] * tw._lorentz_last_iters > dom_ms:
        dom, kernel = "jacobi", "k_elec_jacobi_live"
        dom_ms, dom_bytes = lz_info["ms_per_sweep"], lz_info["bytes_per_sweep"]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic_%s%s.json" % (
        dom, "_f16" if pb == 2 and dom in ("stream", "collide") else ""))
    if os.path.exists(tpath):
        with open(tpath) as fh:
            t = json.load(fh)
        # one capture's DRAM bytes, scaled to this census by the cells the stage touches
        per = {"stream": c["n"] - c["solid"], "collide": c["fluid"]}.get(dom, c["n"])
        traffic = t["dram_bytes"] * per / t["cells_touched"]
    step_bytes = sum(algo.values())
    from waam_solver_b200.coupled_step import _fields_cached
    lib = _native.lib()
    fl = ctypes.byref(_fields_cached(tw.grid))
    pre = lib.waam_step_launch_count(fl, tw._fused_params, 0)
    launches_graph = pre + lib.waam_step_launch_count(fl, tw._fused_params, 1)
    launches_events = pre + lib.waam_step_launch_count(fl, tw._fused_params, 2)
    if lorentz:
        # sigma + mask, source (2), the sweeps, J, bins (2), prefix, B
        launches_graph += 8 + tw._lorentz_last_iters
        launches_events += 8 + tw._lorentz_last_iters

    # ---- end-to-end run through the public API with host inputs / outputs ----
    probe = (g.nx // 2) * g.ny * g.nz + (g.ny // 2) * g.nz + tw.nz_solid - 1
    host_out = torch.zeros(K, dtype=torch.float32, pin_memory=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(K):
        tw.step(*pos[s])                 # torch position from the host (pinned H2D, 8 B)
        s += 1
        host_out[k:k + 1].copy_(g.T.view(-1)[probe:probe + 1], non_blocking=True)  # D2H, 4 B
    e1.record()
    torch.cuda.synchronize()
    barrier()
    ms_e2e = dist_max(e0.elapsed_time(e1))

    # ---- one droplet period, droplet step included (it runs eagerly and reads
    # back the placed volume); device-resident positions as for `value` ----
    drop_info = None
    if period:
        drop_info = droplet_period_timing(tw, pos, s, period, device)
        s += period
    clocks.__exit__(None, None, None)
    health = tw.health()

    value = world * cells * K / (ms * 1e-3) / 1e6
    e2e = world * cells * K / (ms_e2e * 1e-3) / 1e6
    line = {
        "metric": "coupled step throughput (MLUPS)", "value": value, "unit": "MLUPS",
        "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (reference reset state + %d spin-up steps)" % w["spinup"],
        "config": bench_config(w, world, pb, drops),
        "roofline": {"bound": "hbm", "kernel": kernel,
                     "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "peak_source": hbm_src,
                     "algorithmic_bytes_per_launch": dom_bytes},
        "stages_ms": stage_ms,
        "step_algorithmic_GBps": step_bytes / (ms / K * 1e-3) / 1e9,
        # host time of the timed loop: it blocks once the launch queue is full,
        # so it follows the device time; the enqueue work itself is ~0.03 ms
        "host_loop_ms_per_step": host_ms,
        "cell_census": c,
        "e2e": {"value": e2e, "unit": "MLUPS", "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 4},
        "gpu_launches": int(launches_graph * 2 * K + launches_events * Ks),
        "stage_timing": "events between the fused kernels over %d instrumented steps "
                        "(eager launches); value/e2e steps %s" % (
                            Ks, "run eagerly (the potential solve reads back its convergence "
                            "checks)" if lorentz else "replay CUDA graphs"),
        "clocks": clocks.summary(),
        # the fused step's health word over the whole run (non-finite enthalpy,
        # density or velocity, density out of band): the numbers above hold
        # for a state that stayed finite (the standard workload from reset
        # leaves its finite window after about 9,000 steps, oracle and GPU alike)
        "health": {"word": health["word"], "steps_run": tw._step_n,
                   "finite": not (health["nonfinite_enthalpy"] or health["nonfinite_lbm"])},
    }
    if drop_info:
        line["droplet_period"] = drop_info
    if lz_info:
        line["lorentz"] = lz_info
    standard = "beads" not in w
    if world == 1 and args.compare_steps:
        line["storage_comparison"] = storage_comparison(w, device, args.compare_steps)
    if world == 1 and standard and not args.no_precision_forms:
        line["precision_forms"] = storage_forms(w, device, min(K, 1000), ms / K)
        line["precision_forms"]["storage"] = ("headline value: float32 populations; forms: "
                                              "16-bit offsets f_q - w_q, float32 arithmetic")
        line["material_tables"] = table_form(w, device, min(K, 1000), ms / K, stage_ms)
    if world == 1 and standard and not args.no_adjoint:
        line["adjoint"] = adjoint_form(device)
        fd64 = adjoint_fd64(device)
        if fd64:
            line["adjoint"]["fd_fp64"] = fd64
    if world == 1 and standard and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def profile_run(w, n):
    """The workload's first n steps from reset, pending work flushed -- the small
    case that kernel captures under ncu select launches from (-k, -s, -c)."""
    import torch
    tw = build_twin(w, torch.device("cuda", 0))
    for x, y, welding in path_steps(w, tw.grid.dt, n):
        tw.step(x, y, welding)
    tw.grid.flush_stream()
    torch.cuda.synchronize()
    print("profile run: %d steps, %d of %d tiles worked at the last step"
          % ((n,) + tw.grid.worked_tiles()))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="standard", choices=sorted(WORKLOADS))
    ap.add_argument("--no-precision-forms", action="store_true",
                    help="skip the float16 / bfloat16 population-storage timings")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the config-4 adjoint timing and finite-difference check")
    ap.add_argument("--compare-steps", type=int, default=0,
                    help="run the workload this many steps from reset in its own population "
                         "storage and in float32; report remelt depth, HAZ T_max, pool W/D")
    ap.add_argument("--spinup", type=int, default=None,
                    help="steps run before warm-up (default: the workload's spin-up)")
    ap.add_argument("--profile", type=int, default=None, metavar="N",
                    help="run N steps of the workload from reset on cuda:0 and exit, no timing "
                         "and no JSON line (the case of the kernel captures under ncu)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    w = dict(WORKLOADS[args.workload])
    if args.spinup is not None:
        w["spinup"] = args.spinup
    if args.profile is not None:
        profile_run(w, args.profile)
    elif args.impl == "reference":
        run_reference(args, w)
    else:
        run_b200(args, w)


if __name__ == "__main__":
    main()
