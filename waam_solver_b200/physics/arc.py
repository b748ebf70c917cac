"""Arc heat sources (reference physics/arc.py:16-213).

Each source's ``inject`` runs the two-pass energy-normalised kernel on the
grid (weight sum, then H += eta*Q*dt*w/(sum_w*dx^3)); ``fused_terms`` gives the
same source's parameters to the fused step.
"""
from __future__ import annotations

from dataclasses import dataclass

from .. import kernels


def _pen_enable(twin):
    return twin.arc_penetration_m / twin.grid.dx, (1 if twin.arc_surface_weighting else 0)


def normalize_goldak_fractions(ff: float, fr: float):
    """Return (ff, fr) with ff + fr = 2 (Goldak double ellipsoid convention).

    A pair summing to ~1 is doubled; any other sum is rescaled to 2; a
    non-positive sum falls back to (0.6, 1.4).
    """
    total = float(ff) + float(fr)
    if total <= 1e-12:
        return 0.6, 1.4
    if abs(total - 2.0) <= 0.05:
        return float(ff), float(fr)
    if abs(total - 1.0) <= 0.05:
        return 2.0 * float(ff), 2.0 * float(fr)
    return 2.0 * float(ff) / total, 2.0 * float(fr) / total


@dataclass
class Gaussian2D:
    """Surface Gaussian with depth attenuation (kernels.py:443-510)."""

    def inject(self, twin, g, arc_i, arc_j, arc_k):
        pen, enable = _pen_enable(twin)
        kernels.inject_arc_heat(g.H, g.flags, g.phi, g.f_l, g.arc_norm_buf, arc_i, arc_j, arc_k,
                                twin.Q_w, twin.sigma_cells, g.dt, g.dx ** 3, twin.eta, pen, enable,
                                g.FLAG_SOLID, g.FLAG_GAS)

    def fused_terms(self, twin):
        return dict(arc_kind=0, arc_k_offset=0.0, sigma_heat=twin.sigma_cells)


@dataclass
class Goldak3D:
    """Goldak double ellipsoid, semi-axes in cells (kernels.py:513-622)."""

    ff: float = 0.6
    fr: float = 1.4
    a_front: float = 0.0
    a_rear: float = 0.0
    b: float = 0.0
    c: float = 0.0
    depth_front: float = 2.0
    depth_rear: float = 4.0
    sigma_scale: float = 1.0

    def resolved_axes(self, twin):
        """Axes in cells; non-positive axes come from the arc sigma / legacy depths."""
        sig = max(0.5, twin.sigma_cells * self.sigma_scale)
        a_f = self.a_front if self.a_front > 0.0 else sig
        a_r = self.a_rear if self.a_rear > 0.0 else max(sig, 2.0 * sig)
        b = self.b if self.b > 0.0 else sig
        if self.c > 0.0:
            c = self.c
        else:
            c = max(0.5, self.depth_front if self.depth_front > 0.0 else self.depth_rear)
        return a_f, a_r, b, c

    _resolved_axes = resolved_axes

    def inject(self, twin, g, arc_i, arc_j, arc_k):
        sign = 1.0 if twin.travel_speed_m_s >= 0.0 else -1.0
        pen, enable = _pen_enable(twin)
        a_f, a_r, b, c = self.resolved_axes(twin)
        kernels.inject_goldak_heat(g.H, g.flags, g.phi, g.f_l, g.arc_norm_buf, arc_i, arc_j, arc_k,
                                   twin.Q_w, g.dt, g.dx ** 3, twin.eta, sign, self.ff, self.fr,
                                   a_f, a_r, b, c, pen, enable, g.FLAG_SOLID, g.FLAG_GAS)

    def fused_terms(self, twin):
        a_f, a_r, b, c = self.resolved_axes(twin)
        return dict(arc_kind=1, arc_k_offset=0.0, sigma_heat=1.0,
                    sign=1.0 if twin.travel_speed_m_s >= 0.0 else -1.0, ff=self.ff, fr=self.fr,
                    a_f=a_f, a_r=a_r, gb=b, gc=c)


@dataclass
class ConicalVolume:
    """Widened Gaussian placed 1.5 cells below the surface (physics/arc.py:122-137)."""

    sigma_scale: float = 1.2

    def inject(self, twin, g, arc_i, arc_j, arc_k):
        pen, enable = _pen_enable(twin)
        kernels.inject_arc_heat(g.H, g.flags, g.phi, g.f_l, g.arc_norm_buf, arc_i, arc_j,
                                arc_k - 1.5, twin.Q_w, twin.sigma_cells * self.sigma_scale, g.dt,
                                g.dx ** 3, twin.eta, pen, enable, g.FLAG_SOLID, g.FLAG_GAS)

    def fused_terms(self, twin):
        return dict(arc_kind=0, arc_k_offset=-1.5, sigma_heat=twin.sigma_cells * self.sigma_scale)


def create_heat_source(name: str, **kwargs):
    key = (name or "gaussian2d").lower().replace("-", "").replace("_", "")
    if key in ("goldak", "goldak3d", "doubleellipsoid"):
        ff, fr = normalize_goldak_fractions(float(kwargs.pop("ff", 0.6)), float(kwargs.pop("fr", 1.4)))
        return Goldak3D(ff=ff, fr=fr, **kwargs)
    if key in ("conical", "conicalvolume", "cone"):
        return ConicalVolume(**kwargs)
    return Gaussian2D()


def goldak_from_job_mm(twin, goldak_cfg: dict):
    """Goldak3D with semi-axes converted from millimetres to cells.

    Keys: a_front_mm, a_rear_mm, b_mm, c_mm, ff, fr (ff+fr normalised to 2);
    legacy depth_front_mm / depth_rear_mm and sigma_scale are honoured when the
    explicit axes are absent (physics/arc.py:153-213).
    """
    cfg = goldak_cfg or {}
    dx_mm = twin.grid.dx * 1000.0
    ff, fr = normalize_goldak_fractions(float(cfg.get("ff", 0.6)), float(cfg.get("fr", 1.4)))
    sigma_scale = float(cfg.get("sigma_scale", 1.0))
    sig = max(0.5, twin.sigma_cells * sigma_scale)

    def cells(key, default=None):
        if cfg.get(key) is not None:
            return max(0.5, float(cfg[key]) / dx_mm)
        return 0.0 if default is None else max(0.5, float(default))

    a_f, a_r, b, c = cells("a_front_mm"), cells("a_rear_mm"), cells("b_mm"), cells("c_mm")
    depth_front, depth_rear = cells("depth_front_mm", 2.0), cells("depth_rear_mm", 4.0)
    if a_f <= 0.0 and a_r <= 0.0 and b <= 0.0 and c <= 0.0:
        a_f, a_r, b, c = sig, max(sig, 2.0 * sig), sig, depth_front
    elif c <= 0.0:
        c = depth_front
    return Goldak3D(ff=ff, fr=fr, a_front=a_f, a_rear=a_r, b=b, c=c, depth_front=depth_front,
                    depth_rear=depth_rear, sigma_scale=sigma_scale)


__all__ = ["Gaussian2D", "Goldak3D", "ConicalVolume", "create_heat_source",
           "goldak_from_job_mm", "normalize_goldak_fractions"]
