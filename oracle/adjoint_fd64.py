"""Central finite differences of the config-4 adjoint loss on the FP64 oracle
forward -- TEST INFRASTRUCTURE ONLY.

The CUDA adjoint (waam_solver_b200/adjoint.py) differentiates the float32
forward.  Central differences of that float32 forward at a relative step of
1e-3 are dominated by its rounding wherever a parameter moves the loss by a
few units in the last place (the heat-loss factor above all).  This script
takes the same differences on the oracle's FP64 build (``libwaam_oracle64``:
every kernel of the step in double, libm's exp), so the reference gradient
carries no float32 rounding, and writes them with the problem definition to
``tests/golden/adjoint_fd64.npz``; the GPU test and bench.py compare the
adjoint's gradient against it.

The problem restates ``bench.py``'s config-4 set-up: 128x64x48, dx 0.25 mm,
Goldak 3 kW (a_f 3 / a_r 9 / b 3 / c 3 mm, ff 0.6 / fr 1.4), eta 0.78, 8 mm/s
from x = 10 mm, VOF, central-moment collision, convective heat losses; eight
surface probes seeded with numpy's default_rng(0) at 2-6 mm from the centre
line; loss w_T sum (T - T*)^2 + w_W (W - W*)^2 with the smooth final width W
of the adjoint (dx sum_j sigmoid(beta (max_k f_l - 0.5)) on the slice through
the liquid centroid).  The targets T*, W* come from an FP64 run at the
perturbed parameters base x (1.05, 1.2, 1.0, 1.1, 0.9, 1.1, 1.1), W* = W +
0.1 mm.  Variants: ``c4`` from the reset state; ``c4_pool`` from a seeded
molten pool (tests/state_gen.py) so that the width term is not identically
zero.

    python oracle/adjoint_fd64.py c4 [steps [fd_step]]   (minutes to hours of CPU)
"""
from __future__ import annotations

import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# run as a script, this folder comes first on sys.path and its oracle.py would
# shadow the oracle package
sys.path[:] = [p for p in sys.path if os.path.abspath(p or ".") != HERE]
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle.oracle_step import OracleTwin  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "adjoint_fd64.npz")
PARAMS = ["eta", "heat_loss_factor", "arc_sigma_scale", "a_front", "a_rear", "b", "c"]
PERTURB = [1.05, 1.2, 1.0, 1.1, 0.9, 1.1, 1.1]
C4 = dict(nx=128, ny=64, nz=48, dx=2.5e-4, Q=3000.0, eta=0.78, travel=0.008, x0=10e-3,
          h_conv=25.0, arc_sigma_mm=2.0, goldak_mm=(3.0, 9.0, 3.0, 3.0), ff=0.6, fr=1.4)
W_T, W_W, BETA, W_OFFSET_MM, FD_STEP = 1e-3, 10.0, 20.0, 0.1, 1e-3
POOL_SEED = 21
MATERIAL = dict(k=30.0, rho=7800.0, cp=680.0, T_solidus=1723.0, T_liquidus=1783.0,
                L_fusion=2.7e5, gamma_0=1.8, dgamma_dT=-4.3e-4, mu=0.0065, beta_T=1.2e-4,
                contact_angle_deg=30.0)


class Problem:
    def __init__(self, variant, n_steps):
        c = C4
        self.variant, self.N = variant, int(n_steps)
        dxmm = c["dx"] * 1e3
        a_f, a_r, b, cc = (v / dxmm for v in c["goldak_mm"])
        self.base = np.array([c["eta"], 1.0, 1.0, a_f, a_r, b, cc], np.float64)
        ref = self._twin(self.base)
        self.nz_solid = ref.nz_solid
        dx = c["dx"]
        yc = (c["ny"] // 2) * dx
        self.positions = [(c["x0"] + s * ref.dt * c["travel"], yc) for s in range(self.N)]
        rng = np.random.default_rng(0)
        probes = []
        for _ in range(8):
            off = rng.uniform(2e-3, 6e-3) * (1 if rng.random() < 0.5 else -1)
            probes.append((int(rng.uniform(c["x0"] - 2e-3, c["x0"] + 3e-3) / dx),
                           int((yc + off) / dx), self.nz_solid - 1))
        self.probes = probes
        self.start = None
        if variant == "c4_pool":
            import state_gen
            st = state_gen.seeded_state(c["nx"], c["ny"], c["nz"], seed=POOL_SEED,
                                        nz_solid=self.nz_solid,
                                        hot=(c["x0"] / dx + 2.0, yc / dx, self.nz_solid + 1.0))
            self.start = {k: v for k, v in st.items() if k != "nz_solid"}
            self.start["read_is_a"] = True
        elif variant != "c4":
            raise ValueError("variant: c4 or c4_pool")

    def _twin(self, theta):
        c = C4
        ot = OracleTwin(c["nx"], c["ny"], c["nz"], c["dx"], MATERIAL, precision="fp64",
                        heat_source="goldak", arc_power_W=c["Q"], arc_efficiency=float(theta[0]),
                        goldak=dict(ff=c["ff"], fr=c["fr"], a_front=float(theta[3]),
                                    a_rear=float(theta[4]), b=float(theta[5]),
                                    c=float(theta[6])),
                        droplet_freq_hz=0.0, enable_vof=True, use_srt=False,
                        travel_speed_m_s=c["travel"], enable_heat_loss=True,
                        h_conv=c["h_conv"] * float(theta[1]), arc_sigma_mm=c["arc_sigma_mm"])
        # the sigma scale acts on the twin's sigma_cells (the adjoint's parameter);
        # nothing of this configuration reads it
        ot.sigma_cells = ot.sigma_cells * float(theta[2])
        return ot

    def forward(self, theta):
        """(probe temperatures (N, 8), smooth final width [mm]) in FP64."""
        ot = self._twin(theta)
        ot.reset()
        if self.start is not None:
            ot.load(self.start)
        c = C4
        cells = [(i, j, k) for i, j, k in self.probes]
        T = np.zeros((self.N, len(cells)))
        for n, (x, y) in enumerate(self.positions):
            ot.step(x, y, True)
            Tf = ot.s["T"]
            T[n] = [Tf[i, j, k] for i, j, k in cells]
        return T, width(ot.s["f_l"], c["dx"])

    def loss(self, T, W, T_target, W_target):
        return W_T * float(((T - T_target) ** 2).sum()) + W_W * (W - W_target) ** 2


def width(f_l, dx):
    """The adjoint's smooth width (waam_solver_b200/adjoint.py: width) on the
    slice through the liquid centroid (telemetry: round half to even of the
    mean i of f_l > 0.5, slice 0 without liquid)."""
    liq = f_l > 0.5
    n = int(liq.sum())
    ic = 0
    if n:
        ic = int(np.rint(np.nonzero(liq)[0].sum() / n))
        ic = max(0, min(f_l.shape[0] - 1, ic))
    sl = np.asarray(f_l[ic], np.float64)
    m = sl.max(axis=1)
    s = 1.0 / (1.0 + np.exp(-BETA * (m - 0.5)))
    return float(dx * 1e3 * s.sum())


def run(variant, n_steps, fd_step=FD_STEP):
    """Differences at relative step fd_step; a step other than FD_STEP is
    stored under the key ``<variant>@<fd_step>`` (a second step size shows
    how far the differences themselves depend on it)."""
    t0 = time.time()
    pb = Problem(variant, n_steps)
    key = variant if fd_step == FD_STEP else "%s@%g" % (variant, fd_step)
    T_t, W_t = pb.forward(pb.base * np.array(PERTURB))
    T0, W0 = pb.forward(pb.base)
    W_target = W0 + W_OFFSET_MM
    L0 = pb.loss(T0, W0, T_t, W_target)
    fd = {}
    for q, name in enumerate(PARAMS):
        if name == "arc_sigma_scale":
            continue    # structural zero: no kernel of this configuration reads it
        h = fd_step * abs(pb.base[q])
        tp, tm = pb.base.copy(), pb.base.copy()
        tp[q] += h
        tm[q] -= h
        Tp, Wp = pb.forward(tp)
        Tm, Wm = pb.forward(tm)
        fd[name] = (pb.loss(Tp, Wp, T_t, W_target) - pb.loss(Tm, Wm, T_t, W_target)) / (2 * h)
        print(variant, name, fd[name], "%.0f s" % (time.time() - t0), flush=True)
    meta = dict(variant=variant, steps=pb.N, params=PARAMS, theta=pb.base.tolist(),
                probes=pb.probes, x0=C4["x0"], travel=C4["travel"], w_T=W_T, w_W=W_W,
                beta=BETA, fd_step=fd_step, W_target=W_target, W_base=W0, loss_base=L0,
                fd=fd, pool_seed=POOL_SEED if variant == "c4_pool" else None,
                seconds=time.time() - t0)
    payload = {}
    if os.path.exists(OUT):
        with np.load(OUT) as z:
            payload = {k: z[k] for k in z.files}
    payload[key + "_T_target"] = T_t
    payload[key + "_T_base"] = T0
    payload[key + "_meta"] = np.array(json.dumps(meta))
    np.savez_compressed(OUT, **payload)
    print(json.dumps(meta), flush=True)


if __name__ == "__main__":
    run(sys.argv[1] if len(sys.argv) > 1 else "c4",
        int(sys.argv[2]) if len(sys.argv) > 2 else 2000,
        float(sys.argv[3]) if len(sys.argv) > 3 else FD_STEP)
