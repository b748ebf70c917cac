"""Piecewise-linear torch path at constant travel speed (reference
torch_path.py:13-150): the torch sits at distance speed*t along the
polyline, parks at the last waypoint, and stays inside the domain with a
4-cell margin."""
from __future__ import annotations

import csv
import math
import os
from dataclasses import dataclass


@dataclass
class PathSegment:
    x0: float
    y0: float
    z0: float
    x1: float
    y1: float
    z1: float
    length_m: float
    cumulative_start_m: float = 0.0


def build_segments(waypoints):
    segs, cum = [], 0.0
    for (x0, y0, z0), (x1, y1, z1) in zip(waypoints[:-1], waypoints[1:]):
        length = math.sqrt((x1 - x0) ** 2 + (y1 - y0) ** 2 + (z1 - z0) ** 2)
        if length < 1e-9:
            continue
        segs.append(PathSegment(x0, y0, z0, x1, y1, z1, length, cum))
        cum += length
    return segs


def load_torch_path_csv(path):
    """Waypoints [m] from a CSV with x_mm, y_mm, z_mm columns."""
    out = []
    with open(path, newline="") as fh:
        for row in csv.DictReader(fh):
            out.append(tuple(float(row.get(a + "_mm", row.get(a, 0))) / 1000.0 for a in "xyz"))
    return out


def clamp_torch_to_domain(x_m, y_m, nx, ny, dx, margin_cells=4):
    lo_x, hi_x = margin_cells * dx, (nx - margin_cells) * dx
    lo_y, hi_y = margin_cells * dx, (ny - margin_cells) * dx
    return min(max(x_m, lo_x), hi_x), min(max(y_m, lo_y), hi_y)


class TorchPathDriver:
    def __init__(self, waypoints, travel_speed_m_s):
        self.speed = max(travel_speed_m_s, 1e-9)
        self.segments = build_segments(list(waypoints))
        self.total_length = sum(s.length_m for s in self.segments)
        self._fallback = tuple(waypoints[0]) if (not self.segments and waypoints) else (0.0, 0.0, 0.0)

    def distance_at_step(self, step, dt):
        return step * dt * self.speed

    def segment_index_at_distance(self, dist_m):
        if not self.segments:
            return 0
        d = min(dist_m, self.total_length)
        for idx, seg in enumerate(self.segments):
            if d <= seg.length_m:
                return idx
            d -= seg.length_m
        return len(self.segments) - 1

    def segment_end(self, seg_idx):
        if not self.segments or not 0 <= seg_idx < len(self.segments):
            return None
        s = self.segments[seg_idx]
        return s.x1, s.y1, s.z1

    def position_at_time(self, t):
        if not self.segments:
            return self._fallback
        d = min(t * self.speed, self.total_length)
        for s in self.segments:
            if d <= s.length_m:
                u = d / s.length_m
                return s.x0 + u * (s.x1 - s.x0), s.y0 + u * (s.y1 - s.y0), s.z0 + u * (s.z1 - s.z0)
            d -= s.length_m
        last = self.segments[-1]
        return last.x1, last.y1, last.z1

    def is_complete(self, t):
        return bool(self.segments) and self.total_length > 0.0 and \
            t * self.speed >= self.total_length - 1e-12

    def positions_for_steps(self, n_steps, dt, start_step=0):
        for step in range(start_step, start_step + n_steps):
            x, y, z = self.position_at_time(step * dt)
            yield step, x, y, z


def parse_torch_path(job, base_dir=None):
    """Waypoints [m] from a job dict (``torch_path`` list of ``{x_mm, y_mm,
    z_mm}`` or ``torch_path_csv``), job.py:9-35.  A relative CSV path is looked
    up in ``base_dir`` (the job file's folder) first, then in the working
    directory."""
    csv_ref = job.get("torch_path_csv")
    if csv_ref:
        path = str(csv_ref)
        if base_dir and not os.path.isabs(path) and os.path.exists(os.path.join(base_dir, path)):
            path = os.path.join(base_dir, path)
        return load_torch_path_csv(path)
    return [tuple(float(pt.get(a + "_mm", 0)) / 1000.0 for a in "xyz")
            for pt in (job.get("torch_path") or [])]


def load_job_config(path):
    """A job YAML file as a dict (job.py:38-49): FileNotFoundError when the
    file does not exist, {} for an empty file."""
    path = os.fspath(path)
    if not os.path.exists(path):
        raise FileNotFoundError("Job file not found: %s" % path)
    import yaml
    with open(path) as fh:
        data = yaml.safe_load(fh)
    if data is None:
        return {}
    if not isinstance(data, dict):
        raise ValueError("job file %s does not hold a mapping" % path)
    return data


def job_waypoints(job):
    """Waypoints [m] of ``run_path``'s ``job``: a job dict, a job file path
    (str or os.PathLike, loaded as twin.py:650-651 does), or a sequence of
    (x, y, z) waypoints in metres."""
    if isinstance(job, dict):
        return parse_torch_path(job)
    if isinstance(job, (str, os.PathLike)):
        path = os.fspath(job)
        return parse_torch_path(load_job_config(path),
                                base_dir=os.path.dirname(os.path.abspath(path)))
    try:
        pts = [tuple(float(v) for v in p) for p in job]
    except TypeError:
        raise TypeError("run_path: job must be a dict, a job file path or a sequence of "
                        "(x, y, z) waypoints in metres, got %s" % type(job).__name__) from None
    for p in pts:
        if len(p) != 3:
            raise ValueError("run_path: a waypoint needs (x, y, z) in metres, got %r" % (p,))
    return pts


def plan_path(twin, job, n_steps=None):
    """The step plan of run_path (twin.py:632-704): the path driver and, per
    step, (step, segment, x, y, z).  Seeds ``twin._torch_dir_xyz`` with the
    first segment's direction, as the reference does before its first step."""
    g = twin.grid
    waypoints = job_waypoints(job)
    if not waypoints:
        waypoints = [(0.01, (g.ny // 2) * g.dx, 0.0)]
    driver = TorchPathDriver(waypoints, twin.travel_speed_m_s)
    if n_steps is None:
        n_steps = max(400, int(driver.total_length / max(twin.travel_speed_m_s * g.dt, 1e-12)))
    if driver.segments:
        s0 = driver.segments[0]
        d = (s0.x1 - s0.x0, s0.y1 - s0.y0, s0.z1 - s0.z0)
        norm = math.sqrt(sum(v * v for v in d))
        if norm > 1e-12:
            twin._torch_dir_xyz = tuple(v / norm for v in d)
    out = []
    for step, x, y, z in driver.positions_for_steps(n_steps, g.dt):
        seg = driver.segment_index_at_distance(driver.distance_at_step(step, g.dt))
        out.append((step, seg, x, y, z))
    return driver, out


def run_path(twin, job, n_steps=None, is_welding=True, interpass_steps=0):
    """twin.py:632-704 on any object with ``grid``, ``travel_speed_m_s``,
    ``_interpass_cooling_steps``, ``_window_offset_x_m`` and ``step``: each
    path step clamped to the (window-shifted) domain; at every new segment,
    ``interpass`` arc-off steps parked at the end of the previous one (the
    argument, else the job's setting on the twin)."""
    driver, pos = plan_path(twin, job, n_steps)
    g = twin.grid
    interpass = (int(interpass_steps) if interpass_steps
                 else int(getattr(twin, "_interpass_cooling_steps", 0) or 0))
    prev_seg = -1

    def clamp(x, y):
        off = twin._window_offset_x_m
        cx, cy = clamp_torch_to_domain(x - off, y, g.nx, g.ny, g.dx)
        return cx + off, cy

    for step, seg, x, y, z in pos:
        if interpass > 0 and seg > prev_seg >= 0:
            park = driver.segment_end(prev_seg) or (x, y, z)
            for _ in range(interpass):
                cx, cy = clamp(park[0], park[1])
                twin.step(cx, cy, is_welding=False, torch_z_m=park[2])
        prev_seg = seg
        cx, cy = clamp(x, y)
        twin.step(cx, cy, is_welding, torch_z_m=z)
