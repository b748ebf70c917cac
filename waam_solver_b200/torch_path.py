"""Piecewise-linear torch path at constant travel speed (reference
torch_path.py:13-150): the torch sits at distance speed*t along the
polyline, parks at the last waypoint, and stays inside the domain with a
4-cell margin."""
from __future__ import annotations

import csv
import math
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


def parse_torch_path(job):
    """Waypoints [m] from a job dict (``torch_path`` list or ``torch_path_csv``)."""
    if job.get("torch_path_csv"):
        return load_torch_path_csv(job["torch_path_csv"])
    return [tuple(float(pt.get(a + "_mm", 0)) / 1000.0 for a in "xyz")
            for pt in (job.get("torch_path") or [])]
