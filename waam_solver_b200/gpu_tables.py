"""Material property tables for the kernels (reference gpu_tables.py:12-80).

The reference uploads up to eight (T, value) knots per property to Taichi
fields.  Here the knots are kept on the host as float32 arrays and travel to
the kernels by value inside a ``WaamMaterialTables`` struct (kernel parameter
space), so a step reads no table memory and needs no upload.
"""
from __future__ import annotations

import numpy as np

from . import _native
from .materials import MaterialProps

MAX_KNOTS = _native.TABLE_KNOTS
_PROPS = (("cp", "cp"), ("k", "k"), ("mu", "mu"), ("dgamma", "dgamma_dT"))


class MaterialGPUTables:
    """Piecewise-linear material knots (at most 8 per property).

    A property without a table gets one knot (300 K, the constant), as the
    reference uploads it; knots past the eighth are dropped."""

    def __init__(self, mat: MaterialProps):
        tbl = mat.tables
        self.enabled = bool(tbl.has_any())
        self.cp_fallback = float(mat.cp)
        self.k_fallback = float(mat.k)
        self.mu_fallback = float(mat.mu)
        self.dgamma_fallback = float(mat.dgamma_dT)
        for short, attr in _PROPS:
            knots = list(getattr(tbl, attr))
            n = min(len(knots), MAX_KNOTS)
            t = np.zeros(MAX_KNOTS, np.float32)
            v = np.zeros(MAX_KNOTS, np.float32)
            if n == 0:
                t[0], v[0] = 300.0, getattr(self, short + "_fallback")
                n = 1
            else:
                for q in range(n):
                    t[q], v[q] = knots[q]
            setattr(self, short + "_T", t)
            setattr(self, short + "_V", v)
            setattr(self, "n_" + short, n)
        self.struct = self.make_struct()

    def make_struct(self) -> _native.WaamMaterialTables:
        tb = _native.WaamMaterialTables()
        for short, _ in _PROPS:
            dst_t, dst_v = getattr(tb, short + "_T"), getattr(tb, short + "_V")
            src_t, src_v = getattr(self, short + "_T"), getattr(self, short + "_V")
            for q in range(MAX_KNOTS):
                dst_t[q] = float(src_t[q])
                dst_v[q] = float(src_v[q])
            setattr(tb, "n_" + short, int(getattr(self, "n_" + short)))
            setattr(tb, short + "_fallback", getattr(self, short + "_fallback"))
        return tb
