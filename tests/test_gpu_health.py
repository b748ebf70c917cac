"""Health word of the fused step (WaamFields.status): the thermal stage and
the collision OR bits into one device word when they meet non-finite
enthalpy, density or velocity, or a density outside the twin's band; the
host reads it where it synchronises anyway.  strict_mode raises on the
non-finite bits at those points (telemetry, droplet steps), like the
reference's NaN/Inf check of its force diagnostics (twin.py:578-585).
The failures are planted in host-prepared states; nothing here faults the
GPU."""
import numpy as np
import pytest
import torch

import state_gen
from test_gpu_step import _config_twins

pytestmark = pytest.mark.gpu

SHAPE = (40, 24, 24)


def _seeded(tw, seed=3):
    st = state_gen.seeded_state(*SHAPE, seed=seed, nz_solid=tw.nz_solid)
    st = {k: v for k, v in st.items() if k != "nz_solid"}
    st["read_is_a"] = True
    return st


def _steps(tw, n, dx, y=12):
    for s in range(n):
        tw.step(0.3 * SHAPE[0] * dx + s * 1e-6, y * dx, True)
    torch.cuda.synchronize()


def test_clean_run_keeps_the_health_word_zero():
    tw, ot, dx = _config_twins("c2", *SHAPE)
    tw.grid.load_state(_seeded(tw))
    _steps(tw, 12, dx)
    h = tw.health()
    assert h["word"] == 0, h


def test_nan_enthalpy_sets_its_bit_and_strict_mode_raises_at_telemetry():
    tw, ot, dx = _config_twins("c2", *SHAPE)
    st = _seeded(tw)
    solid = np.argwhere(st["flags"] == 1)
    i, j, k = solid[len(solid) // 2]
    st["H"][i, j, k] = np.float32("nan")
    tw.grid.load_state(st)
    _steps(tw, 2, dx)
    h = tw.health()
    assert h["nonfinite_enthalpy"], h
    tw.strict_mode = True
    with pytest.raises(RuntimeError, match="NaN/Inf"):
        tw.get_telemetry()
    # cleared, it stays clear on a clean state
    tw.health(clear=True)
    tw.grid.load_state(_seeded(tw))
    _steps(tw, 2, dx)
    assert tw.health()["word"] == 0


def test_strict_mode_raises_at_a_droplet_step():
    tw, ot, dx = _config_twins("c2", *SHAPE)
    st = _seeded(tw)
    solid = np.argwhere(st["flags"] == 1)
    i, j, k = solid[len(solid) // 3]
    st["H"][i, j, k] = np.float32("nan")   # +inf would be capped by the enthalpy ceiling
    tw.grid.load_state(st)
    tw.strict_mode = True
    _steps(tw, 1, dx)                    # no droplet due: no synchronisation, no check
    tw._last_droplet_time = -1.0         # the next step deposits a droplet (reads back)
    with pytest.raises(RuntimeError, match="NaN/Inf"):
        _steps(tw, 1, dx)


def test_density_outside_the_band_sets_only_the_band_bit():
    tw, ot, dx = _config_twins("c2", *SHAPE)
    st = _seeded(tw)
    fluid = np.argwhere(st["flags"] == 0)
    i, j, k = fluid[len(fluid) // 2]
    st["f_a"][:, i, j, k] *= 3.0
    tw.grid.load_state(st)
    _steps(tw, 1, dx)
    h = tw.health()
    assert h["rho_out_of_band"] and not h["nonfinite_lbm"] and not h["nonfinite_enthalpy"], h
    tw.strict_mode = True
    tw.get_telemetry()                   # out of band is reported, not raised
