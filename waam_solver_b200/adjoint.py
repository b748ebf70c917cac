"""Hand-written adjoint of the coupled step (thermal + LBM + porosity).

Gradients of a probe-temperature and bead-width misfit with respect to the
calibration scalars (calibration.py: arc efficiency eta, heat-loss factor,
arc sigma scale) and the Goldak semi-axes (a_front, a_rear, b, c in cells),
behind ``torch.autograd.Function`` (``CoupledStepLoss``).

Forward: the twin runs the path with the fused step (CUDA graphs), records
the probe temperatures and the per-step arc scalars, and keeps a device
checkpoint of the full state every K steps (K = ceil(sqrt(N)) by default,
sqrt(N)-step checkpointing).  Backward: for each segment, newest first, the
checkpoint is restored and the K steps are recomputed eagerly with a tape
(post-injection H, the state after every step, the active cells and their
pre-collision populations, written by the collision kernel itself); then the
reverse kernels (waam_adjoint.cu) run the K steps backwards.  The VOF
interface, the flags and the active set are the forward trajectory's (a
stated approximation: their changes under a perturbation are not
differentiated).  Misfits and parameter gradients accumulate in FP64.

Supported: constant material properties, the MRT collision, float32
populations, no droplets, Lorentz force, vapour recoil, gas shear or moving
window during the differentiated run (each raises).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _native, kernels
from ._native import WaamError
from .coupled_step import _fields, step_params, upload_position

PARAMS = ("eta", "heat_loss_factor", "arc_sigma_scale", "a_front", "a_rear", "b", "c")
_FIELDS = ("f_a", "f_b", "rho", "ux", "uy", "uz", "T_max", "f_l", "phi", "flags", "T_prev",
           "dT_dt", "time_above_800_s", "time_above_1100_s", "time_above_solidus_s", "Fx", "Fy",
           "Fz", "porosity_pos", "porosity_active", "tracer_head", "step_scalars")
_HOST = ("_step_n", "_last_droplet_time", "_last_torch_pos_m", "_torch_dir_xyz",
         "_n_droplets_fired", "_deposited_volume_m3", "_deposition_overflow")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return torch.cuda.current_stream().cuda_stream


class _Checkpoint:
    """Device copy of the full twin state (every field a step reads or writes)."""

    def __init__(self, tw):
        g = tw.grid
        g.flush_stream()
        self.t = {k: getattr(g, k).clone() for k in _FIELDS}
        self.t["_H"] = [h.clone() for h in g._H]
        self.t["_T"] = [x.clone() for x in g._T]
        self.g_host = (g._read_buf is g.f_a, g._cur, getattr(g, "_forces_dirty", True),
                       getattr(g, "_tracers_live", False))
        self.host = {k: getattr(tw, k) for k in _HOST}

    def restore(self, tw):
        g = tw.grid
        g._stream_pending = False       # the checkpoint holds a streamed state
        g._collide_pending = False
        g._lag_pending = False
        g._tiles_valid = False          # the quiet-tile history is not the checkpoint's
        for k in _FIELDS:
            getattr(g, k).copy_(self.t[k])
        for dst, src in zip(g._H, self.t["_H"]):
            dst.copy_(src)
        for dst, src in zip(g._T, self.t["_T"]):
            dst.copy_(src)
        read_a, g._cur, g._forces_dirty, live = self.g_host
        g._read_buf, g._write_buf = (g.f_a, g.f_b) if read_a else (g.f_b, g.f_a)
        if live != getattr(g, "_tracers_live", False):
            g._tracers_live = live
            g.__dict__.pop("_fields_cache", None)
        for k, v in self.host.items():
            setattr(tw, k, v)


class _Tape:
    """Per-step records of one segment (device memory)."""

    def __init__(self, g, K, cap):
        n = g.n_cells
        dev = g.device
        f32 = dict(dtype=torch.float32, device=dev)
        self.K, self.cap = K, cap
        self.Hp = torch.empty((K, n), **f32)
        self.H = torch.empty((K, n), **f32)
        self.T = torch.empty((K, n), **f32)
        self.fl = torch.empty((K, n), **f32)
        self.phi = torch.empty((K, n), **f32)
        self.u = torch.empty((K, 3, n), **f32)
        self.flags = torch.empty((K, n), dtype=torch.int32, device=dev)
        self.scal = torch.empty((K, 16), **f32)
        self.tf = torch.empty((K, 19, cap), **f32)
        self.tcells = torch.empty((K, cap), dtype=torch.int32, device=dev)
        self.tcount = torch.zeros(K, dtype=torch.int32, device=dev)


def _grid_pre(g):
    """Views of the state a reverse step needs from the start of its step."""
    return dict(H=g.H.reshape(-1).clone(), T=g.T.reshape(-1).clone(),
                fl=g.f_l.reshape(-1).clone(), flags=g.flags.reshape(-1).clone(),
                u=torch.stack([g.ux.reshape(-1), g.uy.reshape(-1), g.uz.reshape(-1)]).clone())


class AdjointProblem:
    """Loss over a fixed torch path from the twin's current state.

    ``probes``: cells (i, j, k) sampled after every step; ``T_target``: (N, P)
    target temperatures; ``W_target``: final smooth pool width [mm] on the
    forward's centroid slice; loss = w_T sum (T - T*)^2 + w_W (W - W*)^2 with
    W = dx[mm] * sum_j sigmoid(beta (max_k f_l(i_c, j, k) - 0.5)).
    """

    def __init__(self, twin, positions, probes, T_target=None, W_target=None, w_T=1.0,
                 w_W=1.0, beta=20.0, checkpoint_every=None):
        self.tw = twin
        # every forward changes the twin's parameters and restores a checkpoint,
        # which drops its captured step graphs: plain launches cost less than
        # capturing them again for each forward
        twin.use_cuda_graphs = False
        self.positions = [(float(x), float(y)) for x, y in positions]
        self.N = len(self.positions)
        g = twin.grid
        self.probes = [(int(i), int(j), int(k)) for i, j, k in probes]
        self.cell_list = [(i * g.ny + j) * g.nz + k for i, j, k in self.probes]
        self.cells = torch.tensor(self.cell_list, dtype=torch.int32, device=g.device)
        self.T_target = None if T_target is None else np.asarray(T_target, np.float64)
        self.W_target = W_target
        self.w_T, self.w_W, self.beta = float(w_T), float(w_W), float(beta)
        self.K = int(checkpoint_every or max(1, math.ceil(math.sqrt(self.N))))
        self._check_supported()
        self.start = _Checkpoint(twin)
        from .physics.arc import Goldak3D
        src = twin.arc_source
        self.base = dict(h_conv=twin.h_conv, sigma_cells=twin.sigma_cells,
                         goldak=isinstance(src, Goldak3D))
        if self.base["goldak"]:
            if min(src.a_front, src.a_rear, src.b, src.c) <= 0.0:
                raise WaamError("the adjoint needs explicit Goldak semi-axes")
        self.theta = self.current_theta()

    # ---- parameters ------------------------------------------------------
    def current_theta(self):
        tw = self.tw
        src = tw.arc_source
        axes = ((src.a_front, src.a_rear, src.b, src.c) if self.base["goldak"]
                else (0.0, 0.0, 0.0, 0.0))
        return np.array([tw.eta, tw.h_conv / self.base["h_conv"] if self.base["h_conv"] else 1.0,
                         tw.sigma_cells / self.base["sigma_cells"], *axes], np.float64)

    def apply(self, theta):
        tw = self.tw
        theta = np.asarray(theta, np.float64)
        tw.eta = float(theta[0])
        tw.h_conv = self.base["h_conv"] * float(theta[1])
        tw.sigma_cells = self.base["sigma_cells"] * float(theta[2])
        if self.base["goldak"]:
            src = tw.arc_source
            src.a_front, src.a_rear, src.b, src.c = (float(v) for v in theta[3:7])
        tw.invalidate()
        tw.__dict__["_graphs"] = {}
        self.theta = theta.copy()

    def _check_supported(self):
        tw = self.tw
        bad = []
        if tw.enable_lorentz or tw.enable_recoil or tw.enable_gas_shear:
            bad.append("Lorentz / recoil / gas shear")
        if tw.enable_moving_window:
            bad.append("moving window")
        if tw.use_material_tables:
            bad.append("material tables")
        if tw.use_srt:
            bad.append("SRT collision")
        if tw.grid.population_storage:
            bad.append("16-bit populations")
        if tw.enable_substrate_growth or tw.enable_bead_freeze:
            bad.append("substrate growth / trailing freeze")
        if tw.droplet_freq > 0:
            bad.append("droplets (droplet_freq_hz > 0)")
        if tw.enable_ctwd:
            bad.append("CTWD update")
        if bad:
            raise WaamError("the adjoint does not cover: " + ", ".join(bad))

    # ---- forward -----------------------------------------------------------
    def forward(self, theta=None):
        """Run the path from the start state; returns the loss (FP64)."""
        tw = self.tw
        g = tw.grid
        if theta is not None:
            self.apply(theta)
        self.start.restore(tw)
        P = len(self.probes)
        # probe_sample writes T and f_l of every probe: row = (T0, fl0, T1, fl1, ...)
        self.hist = torch.zeros((self.N, max(2 * P, 2)), dtype=torch.float32, device=g.device)
        self.scal = torch.zeros((self.N, 16), dtype=torch.float32, device=g.device)
        self.checkpoints = {}
        for n, (x, y) in enumerate(self.positions):
            if n % self.K == 0:
                self.checkpoints[n] = _Checkpoint(tw)
            tw.step(x, y, True)
            self.scal[n].copy_(g.step_scalars)
            if P:
                kernels.probe_sample(g.T, g.f_l, self.cell_list, self.hist[n])
        self.T_probe = (self.hist[:, 0:2 * P:2].double().cpu().numpy() if P
                        else np.zeros((self.N, 0)))
        self.fl_final = g.f_l.clone()
        self.i_c = int(tw.get_telemetry()["pool_slice_i"])
        return self.loss_value()

    def loss_value(self):
        L = 0.0
        if self.T_target is not None and len(self.probes):
            L += self.w_T * float(((self.T_probe - self.T_target) ** 2).sum())
        if self.W_target is not None:
            W, _ = self.width()
            L += self.w_W * (W - self.W_target) ** 2
        self.loss = L
        return L

    def width(self):
        """Smooth final width [mm] on slice i_c and its (j, argmax k) cells."""
        g = self.tw.grid
        ic = max(self.i_c, 0)
        sl = self.fl_final[ic].double().cpu().numpy()          # (ny, nz)
        kmax = sl.argmax(axis=1)
        m = sl[np.arange(g.ny), kmax]
        s = 1.0 / (1.0 + np.exp(-self.beta * (m - 0.5)))
        dx_mm = g.dx * 1000.0
        return float(dx_mm * s.sum()), (ic, kmax, s, dx_mm)

    # ---- backward ----------------------------------------------------------
    def backward(self):
        """Gradient of the last forward's loss with respect to PARAMS."""
        tw = self.tw
        g = tw.grid
        n_cells = g.n_cells
        nx, ny, nz = g.nx, g.ny, g.nz
        dev = g.device
        f32 = dict(dtype=torch.float32, device=dev)
        lam = {"H": torch.zeros(n_cells, **f32), "Hp": torch.zeros(n_cells, **f32),
               "mu": torch.zeros(n_cells, **f32), "T": torch.zeros(n_cells, **f32),
               "fl": torch.zeros(n_cells, **f32), "u": torch.zeros((3, n_cells), **f32)}
        pops = [torch.zeros(19 * n_cells, **f32) for _ in range(3)]   # lam X, lam Y, scratch
        cap = n_cells
        ctb = torch.zeros(6 * cap, **f32)
        amap = torch.full((n_cells,), -1, dtype=torch.int32, device=dev)
        grad_h = torch.zeros(1, dtype=torch.float64, device=dev)
        inj = torch.zeros((self.N, 11), dtype=torch.float64, device=dev)
        ws = g.workspace
        P = len(self.probes)
        # probe and width adjoints
        dT = np.zeros((self.N, P))
        if self.T_target is not None and P:
            dT = 2.0 * self.w_T * (self.T_probe - self.T_target)
        dT_dev = torch.tensor(dT, dtype=torch.float32, device=dev)
        if self.W_target is not None:
            W, (ic, kmax, s, dx_mm) = self.width()
            coef = self.w_W * 2.0 * (W - self.W_target) * dx_mm * self.beta * s * (1.0 - s)
            cells = torch.tensor([(ic * ny + j) * nz + int(kmax[j]) for j in range(ny)],
                                 dtype=torch.int32, device=dev)
            _call("waam_adj_scatter_add", _ptr(lam["fl"]), _ptr(cells),
                  _ptr(torch.tensor(coef, **f32)), ny, _stream())
        tape = _Tape(g, self.K, cap)
        starts = sorted(self.checkpoints)
        for s0 in reversed(starts):
            steps = list(range(s0, min(s0 + self.K, self.N)))
            pre0 = self._record_segment(s0, steps, tape)
            for n in reversed(steps):
                slot = n - s0
                pre = pre0 if slot == 0 else dict(
                    H=tape.H[slot - 1], T=tape.T[slot - 1], fl=tape.fl[slot - 1],
                    flags=tape.flags[slot - 1], u=tape.u[slot - 1])
                if P:
                    _call("waam_adj_scatter_add", _ptr(lam["T"]), _ptr(self.cells),
                          _ptr(dT_dev[n]), P, _stream())
                pops = self._reverse_step(n, slot, pre, tape, lam, pops, ctb, amap, grad_h,
                                          inj[n], ws)
        torch.cuda.synchronize()
        return self._combine(grad_h.item(), inj.cpu().numpy())

    def _record_segment(self, s0, steps, tape):
        tw = self.tw
        g = tw.grid
        self.checkpoints[s0].restore(tw)
        pre0 = _grid_pre(g)
        tape.tcount.zero_()
        for slot, n in enumerate(steps):
            x, y = self.positions[n]
            _taped_step(tw, x, y, tape, slot)
        counts = tape.tcount[:len(steps)].cpu()
        if int(counts.min()) < 0:
            raise WaamError("adjoint tape overflow: more active cells than the tape holds")
        return pre0

    def _reverse_step(self, n, slot, pre, tape, lam, pops, ctb, amap, grad_h, inj_row, ws):
        tw = self.tw
        g = tw.grid
        nx, ny, nz = g.nx, g.ny, g.nz
        p = ctypes.byref(self._params())
        st = _stream()
        lamX, lamY, scratch = pops
        # un-swap: lam Y' = lam X_{n+1}, lam X' = lam Y_{n+1}
        lam_yp, lam_xp = lamX, lamY
        _call("waam_adj_stream", _ptr(lam_yp), _ptr(lam_xp), _ptr(scratch),
              _ptr(tape.flags[slot]), nx, ny, nz, st)
        lam_xn = scratch
        _call("waam_adj_collide", p, _ptr(tape.tf[slot]), _ptr(tape.tcells[slot]),
              _ptr(tape.tcount[slot:slot + 1]), tape.cap, _ptr(tape.phi[slot]),
              _ptr(tape.T[slot]), _ptr(tape.fl[slot]), _ptr(tape.flags[slot]),
              _ptr(tape.scal[slot]), _ptr(lam_yp), _ptr(lam_xn), _ptr(lam["u"][0]),
              _ptr(lam["u"][1]), _ptr(lam["u"][2]), _ptr(lam["fl"]), _ptr(lam["T"]), _ptr(ctb),
              _ptr(amap), nx, ny, nz, st)
        _call("waam_adj_combine", p, _ptr(lam["H"]), _ptr(lam["T"]), _ptr(lam["fl"]),
              _ptr(tape.H[slot]), _ptr(tape.flags[slot]), _ptr(tape.phi[slot]), g.n_cells, st)
        _call("waam_adj_thermal", p, _ptr(lam["H"]), _ptr(lam["Hp"]), _ptr(lam["mu"]),
              _ptr(lam["T"]), _ptr(lam["u"][0]), _ptr(lam["u"][1]), _ptr(lam["u"][2]),
              _ptr(tape.Hp[slot]), _ptr(pre["T"]), _ptr(pre["u"][0]), _ptr(pre["u"][1]),
              _ptr(pre["u"][2]), _ptr(pre["flags"]), nx, ny, nz, _ptr(grad_h), _ptr(ws),
              ws.numel(), st)
        _call("waam_adj_inject", p, _ptr(lam["H"]), _ptr(lam["Hp"]), _ptr(pre["H"]),
              _ptr(pre["fl"]), _ptr(pre["flags"]), _ptr(tape.scal[slot]), nx, ny, nz,
              _ptr(inj_row), _ptr(ws), ws.numel(), st)
        # new (lam X_n, lam Y_n, scratch)
        return [lam_xn, lam_yp, lam_xp]

    def _params(self):
        tw = self.tw
        p = tw._fused_params
        if p is None:
            p = tw._fused_params = step_params(tw)
        p.welding = 1
        p.forces_from_buffer = 0
        return p

    def _combine(self, grad_hconv, inj):
        """FP64 parameter gradients from the reverse sums (see waam_adj_inject)."""
        th = self.theta
        scal = self.scal.double().cpu().numpy()
        W, epw = scal[:, 1], scal[:, 2]
        A = inj[:, 0]
        B, D = inj[:, 1:6], inj[:, 6:11]
        ok = (W > 1e-9) & (epw > 0)
        grad = np.zeros(len(PARAMS))
        grad[0] = float(A[ok].sum()) / th[0]
        grad[1] = grad_hconv * self.base["h_conv"]
        corr = np.zeros(5)
        for q in range(5):
            corr[q] = float((B[ok, q] - D[ok, q] * A[ok] / W[ok]).sum())
        if self.base["goldak"]:
            grad[3:7] = corr[:4]
            grad[2] = 0.0           # Goldak with explicit axes does not use sigma
        else:
            tw = self.tw
            sigma_heat = tw.arc_source.fused_terms(tw)["sigma_heat"]
            grad[2] = corr[4] * sigma_heat / th[2]
        self.grad = grad
        return grad


def _call(name, *args):
    return _native.call(name, *args)


def _taped_step(tw, x, y, tape, slot):
    """One coupled step (twin.step + the fused stages, eager) that records the
    tape slot: post-injection H, the collision inputs, the state after."""
    g = tw.grid
    z_now = 0.0
    if tw._last_torch_pos_m is not None:
        px, py, pz = tw._last_torch_pos_m
        dvec = (x - px, y - py, z_now - pz)
        norm = math.sqrt(sum(v * v for v in dvec))
        if norm > 1e-12:
            tw._torch_dir_xyz = tuple(v / norm for v in dvec)
    tw._last_torch_pos_m = (x, y, z_now)
    sim_x = x - tw._window_offset_x_m - tw._sim_origin_offset_x_m
    sim_y = y - tw._sim_origin_offset_y_m
    p = tw._fused_params
    if p is None:
        p = tw._fused_params = step_params(tw)
    g.flush_stream()
    p.stream_prev = 0
    p.defer_stream = 0
    p.collide_prev = 0
    p.defer_collide = 0
    p.stream_lag = 0
    p.hold_stream = 0
    # taped steps follow checkpoint restores: every tile worked, and the next
    # fused step restarts the tile history too
    p.tile_skip = 0
    p.cache_read = 0
    p.collide_prev_cache_read = 0
    g._tiles_valid = False
    arc_i, arc_j = sim_x / g.dx, sim_y / g.dx
    p.arc_i, p.arc_j = arc_i, arc_j
    p.welding = 1
    p.forces_from_buffer = 0
    p.clear_forces = 1 if getattr(g, "_forces_dirty", True) else 0
    dx_, dy_, dz_ = tw._torch_dir_xyz
    p.dir_x, p.dir_y, p.dir_z = dx_, dy_, dz_
    f = _fields(g)
    f.tape_f = tape.tf[slot].data_ptr()
    f.tape_cells = tape.tcells[slot].data_ptr()
    f.tape_count = tape.tcount[slot:slot + 1].data_ptr()
    f.tape_cap = tape.cap
    g._pos_dst = g.step_scalars[4:6]
    upload_position(tw, arc_i, arc_j)
    ws = g.workspace
    st = _stream()
    _native.call("waam_step_pre", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(), ws.numel(), st)
    tape.Hp[slot].copy_(g.H.reshape(-1))
    _native.call("waam_step_main", ctypes.byref(f), ctypes.byref(p), ws.data_ptr(), ws.numel(),
                 st)
    g._forces_dirty = False
    g.flip_thermal()
    g.swap_buffers()
    tw._step_n += 1
    tape.H[slot].copy_(g.H.reshape(-1))
    tape.T[slot].copy_(g.T.reshape(-1))
    tape.fl[slot].copy_(g.f_l.reshape(-1))
    tape.phi[slot].copy_(g.phi.reshape(-1))
    tape.flags[slot].copy_(g.flags.reshape(-1))
    tape.u[slot, 0].copy_(g.ux.reshape(-1))
    tape.u[slot, 1].copy_(g.uy.reshape(-1))
    tape.u[slot, 2].copy_(g.uz.reshape(-1))
    tape.scal[slot].copy_(g.step_scalars)


class CoupledStepLoss(torch.autograd.Function):
    """loss = CoupledStepLoss.apply(theta, problem): theta (7,) = PARAMS."""

    @staticmethod
    def forward(ctx, theta, problem):
        ctx.problem = problem
        loss = problem.forward(theta.detach().double().cpu().numpy())
        return torch.tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        grad = ctx.problem.backward()
        return torch.as_tensor(grad, dtype=torch.float64) * grad_out, None


__all__ = ["AdjointProblem", "CoupledStepLoss", "PARAMS"]
