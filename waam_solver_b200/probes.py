"""Thermocouple-style probes (reference export/probes.py:15-125).

A probe is fixed at a world position and re-resolved to a cell at every
sample (so it stays put when the window moves).  Samples are gathered on the
device into a history buffer -- one small kernel per recorded step, no host
synchronisation -- and copied to the host once, when the CSV is written or
the rows are read.
"""
from __future__ import annotations

import csv
import math
import pathlib
from dataclasses import dataclass, field

import torch

from . import kernels


@dataclass
class ProbeSpec:
    name: str
    x_m: float
    y_m: float
    z_m: float

    def resolve(self, twin):
        """export/probes.py:29-37 (truncating casts, None outside the grid)."""
        g = twin.grid
        i = int((self.x_m - twin._window_offset_x_m) / g.dx)
        j = int(self.y_m / g.dx)
        k = int(self.z_m / g.dx)
        if not (0 <= i < g.nx and 0 <= j < g.ny and 0 <= k < g.nz):
            return None
        return i, j, k


@dataclass
class ProbeRecorder:
    probes: list = field(default_factory=list)
    _steps: list = field(default_factory=list)
    _hist: object = None
    _n: int = 0

    def add_grid(self, i, j, k, twin, name=None):
        g = twin.grid
        self.probes.append(ProbeSpec(name=name or "probe_%d" % len(self.probes),
                                     x_m=(i + 0.5) * g.dx + twin._window_offset_x_m,
                                     y_m=(j + 0.5) * g.dx, z_m=(k + 0.5) * g.dx))

    def add_world_mm(self, x_mm, y_mm, z_mm, twin, name=None):
        self.probes.append(ProbeSpec(name=name or "probe_%d" % len(self.probes),
                                     x_m=x_mm / 1000.0, y_m=y_mm / 1000.0, z_m=z_mm / 1000.0))

    @classmethod
    def from_job_list(cls, entries, twin):
        rec = cls()
        for e in entries:
            name = str(e.get("name", "probe_%d" % len(rec.probes)))
            if "i" in e and "j" in e and "k" in e:
                rec.add_grid(int(e["i"]), int(e["j"]), int(e["k"]), twin, name)
            else:
                rec.add_world_mm(float(e.get("x_mm", 0)), float(e.get("y_mm", 0)),
                                 float(e.get("z_mm", 0)), twin, name)
        return rec

    def record_step(self, twin):
        """Sample T and f_l at every probe into the device history."""
        if not self.probes:
            return
        g = twin.grid
        width = 2 * len(self.probes)
        if self._hist is None or self._hist.shape[1] != width:
            self._flush_to_host()
            self._hist = torch.empty((256, width), dtype=torch.float32, device=g.device)
            self._n = 0
        if self._n == self._hist.shape[0]:
            grown = torch.empty((2 * self._n, width), dtype=torch.float32, device=g.device)
            grown[: self._n].copy_(self._hist)
            self._hist = grown
        cells = []
        for p in self.probes:
            idx = p.resolve(twin)
            cells.append(-1 if idx is None else (idx[0] * g.ny + idx[1]) * g.nz + idx[2])
        kernels.probe_sample(g.T, g.f_l, cells, self._hist[self._n])
        self._n += 1
        self._steps.append((twin._step_n, twin._step_n * g.dt * 1000.0))

    def _flush_to_host(self):
        if self._hist is None or self._n == 0:
            return
        vals = self._hist[: self._n].cpu().numpy()
        host = getattr(self, "_host_rows", [])
        start = len(host)
        for r in range(self._n):
            step, t_ms = self._steps[start + r]
            row = {"sim_time_ms": round(t_ms, 4), "step": step}
            for q, p in enumerate(self.probes):
                t, fl = float(vals[r, 2 * q]), float(vals[r, 2 * q + 1])
                row["%s_T_K" % p.name] = math.nan if math.isnan(t) else round(t, 2)
                row["%s_f_l" % p.name] = math.nan if math.isnan(fl) else round(fl, 4)
            host.append(row)
        self._host_rows = host
        self._n = 0

    @property
    def rows(self):
        """The recorded rows (export/probes.py:92-107 layout); reads the history once."""
        self._flush_to_host()
        return list(getattr(self, "_host_rows", []))

    def write_csv(self, path):
        rows = self.rows
        if not rows:
            return
        path = pathlib.Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        names = ["sim_time_ms", "step"]
        for p in self.probes:
            names += ["%s_T_K" % p.name, "%s_f_l" % p.name]
        with open(path, "w", newline="") as f:
            w = csv.DictWriter(f, fieldnames=names, extrasaction="ignore")
            w.writeheader()
            w.writerows(rows)

    def clear(self):
        self._host_rows = []
        self._steps = []
        self._n = 0
