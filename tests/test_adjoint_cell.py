"""The adjoint's per-cell reverse functions (waam_adjoint_cell.h) in double
precision against central finite differences of their forward maps."""
import ctypes as C
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        import subprocess
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        L = C.CDLL(os.path.join(ROOT, "oracle", "_build", "libwaam_adjcheck.so"))
        P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        D = C.c_double
        L.wa_mrt_forward.argtypes = [P, D, D, D, D, P]
        L.wa_mrt_vjp.argtypes = [P, D, D, D, D, P, P]
        L.wa_clamp.argtypes = [P, D, P]
        L.wa_clamp_vjp.argtypes = [P, D, P, P]
        _LIB = L
    return _LIB


W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
E = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1],
              [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1], [-1, 0, -1],
              [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1], [0, -1, 1]], float)


def _state(rng, fl, u_scale=0.03):
    u = rng.uniform(-u_scale, u_scale, 3)
    rho = 1.0 + rng.normal(0, 1e-3)
    eu = E @ u
    feq = W * rho * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * u @ u)
    f = feq + rng.normal(0, 1e-4, 19)
    F = rng.normal(0, 1e-4, 3)
    return np.concatenate([f, [fl], F])


def _fd_check(fwd, vjp, x, n_out, rng, h=1e-6, rtol=1e-6):
    yb = rng.normal(size=n_out)
    xb = vjp(x, yb)
    fd = np.zeros_like(x)
    for i in range(x.size):
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd[i] = (fwd(xp) - fwd(xm)) @ yb / (2 * h)
    scale = np.abs(fd).max() + 1e-300
    assert np.max(np.abs(xb - fd)) <= rtol * scale + 1e-9 * scale, (xb, fd)


@pytest.mark.parametrize("fl,ucap,u_scale", [(1.0, 0.08, 0.03), (0.6, 0.08, 0.03),
                                             (0.3, 0.0, 0.03), (0.95, 0.02, 0.05)])
def test_mrt_vjp_matches_finite_differences(fl, ucap, u_scale):
    L = lib()
    rng = np.random.default_rng(int(fl * 100) + int(ucap * 1000))
    ws, wb, Cd = 1.0 / 0.50125, 1.0 / 0.50125, 1.6e5

    def fwd(x):
        out = np.zeros(22)
        L.wa_mrt_forward(np.ascontiguousarray(x), ws, wb, Cd, ucap, out)
        return out

    def vjp(x, yb):
        xb = np.zeros(23)
        L.wa_mrt_vjp(np.ascontiguousarray(x), ws, wb, Cd, ucap, np.ascontiguousarray(yb), xb)
        return xb

    x = _state(rng, fl, u_scale)
    # the Darcy term is stiff below fl = 1: step relative to the liquid fraction
    _fd_check(fwd, vjp, x, 22, rng, h=1e-7, rtol=2e-5)
    if ucap > 0 and u_scale > ucap:
        u = fwd(x)[19:22]
        assert np.linalg.norm(u) <= ucap * (1 + 1e-9)


def test_clamp_vjp_matches_finite_differences():
    L = lib()
    rng = np.random.default_rng(1)
    for cap in (0.5, 10.0):
        x = rng.normal(size=3)

        def fwd(v):
            y = np.zeros(3)
            L.wa_clamp(np.ascontiguousarray(v), cap, y)
            return y

        def vjp(v, yb):
            xb = np.zeros(3)
            L.wa_clamp_vjp(np.ascontiguousarray(v), cap, np.ascontiguousarray(yb), xb)
            return xb

        _fd_check(fwd, vjp, x, 3, rng)
