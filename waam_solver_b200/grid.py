"""Field store of the coupled step: the reference grid's SoA fields as torch
CUDA tensors (grid.py:37-289 of waam_twin).

Names, shapes and dtypes are the reference's: scalar fields ``(nx, ny, nz)``
float32 with k fastest, populations ``(19, nx, ny, nz)``, ``flags`` int32
with FLUID=0 / SOLID=1 / GAS=2 / IFACE=4, 0-d scratch buffers as shape-``()``
tensors.  ``f_src`` / ``f_dst`` and ``swap_buffers`` keep the reference's
ping-pong semantics.

Differences that matter to a caller:

* ``H`` and ``T`` are each backed by two tensors; the fused step writes the
  new values into the other tensor and flips the pair, so always read
  ``grid.H`` / ``grid.T`` after a step instead of holding an old reference.
* ``Fx_snap``/``Fy_snap``/``Fz_snap`` alias ``Fx``/``Fy``/``Fz`` unless the grid is
  created with ``separate_force_snapshot=True``: at every step boundary the
  reference's snapshot equals the force field (kernels.py:3338-3350).
* ``population_dtype=torch.float16`` or ``torch.bfloat16`` stores ``f_a`` /
  ``f_b`` as 16-bit offsets f_q - w_q from the rest weights (rho0 = 1); the
  kernels compute in float32.  ``populations(t)`` returns float32 f_q of
  either buffer, ``state_dict`` / ``load_state`` convert.
"""
from __future__ import annotations

import math

import torch

from . import _native

Q = 19
EX = (0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0)
EY = (0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1)
EZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1)
W = tuple([1.0 / 3.0] + [1.0 / 18.0] * 6 + [1.0 / 36.0] * 12)
OPP = (0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17)


def default_device():
    if not torch.cuda.is_available():
        raise _native.WaamError("waam_solver_b200 needs a CUDA device (B200); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


class WAAMGrid:
    FLAG_FLUID = 0
    FLAG_SOLID = 1
    FLAG_GAS = 2
    FLAG_IFACE = 4

    def __init__(self, nx, ny, nz, dx, mat, max_tracers=50_000, allocate_lorentz=False,
                 allocate_vof=False, allocate_export=False, device=None,
                 separate_force_snapshot=False, verbose=False, population_dtype=torch.float32):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx = float(dx)
        self.mat = mat
        self.max_tracers = int(max_tracers)
        # Lattice units (grid.py:93-105): u_ref 0.5 m/s <-> 0.05 lu/ts.
        self.u_ref_phys = 0.5
        self.u_ref_lu = 0.05
        self.dt = self.dx * self.u_ref_lu / self.u_ref_phys
        nu_lu = (mat.mu / mat.rho) * self.dt / (self.dx ** 2)
        self.tau = 3.0 * nu_lu + 0.5
        self.alpha_lu = mat.alpha * self.dt / (self.dx ** 2)
        self.tau_T = 3.0 * self.alpha_lu + 0.5
        # Stability checks enforced by the reference (grid.py:111-126).
        if self.tau <= 0.5:
            raise ValueError("LBM unstable: tau=%.4f <= 0.5 (nu_lu=%.3e)" % (self.tau, nu_lu))
        if self.alpha_lu > 1.0 / 6.0:
            raise ValueError("Thermal step unstable: alpha_lu=%.4f > 1/6" % self.alpha_lu)
        if verbose and self.tau < 0.505:
            print("[WAAMGrid] WARNING: tau=%.4f is marginally stable (< 0.505)" % self.tau)

        dev = torch.device(device) if device is not None else default_device()
        self.device = dev
        shape3 = (self.nx, self.ny, self.nz)
        self._shape3 = shape3
        f32 = dict(dtype=torch.float32, device=dev)

        def vol():
            return torch.zeros(shape3, **f32)

        pop_dtype = {"float32": torch.float32, "float16": torch.float16,
                     "bfloat16": torch.bfloat16}.get(population_dtype, population_dtype)
        if pop_dtype not in (torch.float32, torch.float16, torch.bfloat16):
            raise ValueError("population_dtype must be float32, float16 or bfloat16")
        self.population_dtype = pop_dtype
        self.population_storage = {torch.float32: 0, torch.float16: 1, torch.bfloat16: 2}[pop_dtype]
        self.f_a = torch.zeros((Q,) + shape3, dtype=pop_dtype, device=dev)
        self.f_b = torch.zeros((Q,) + shape3, dtype=pop_dtype, device=dev)
        self.rho = vol()
        self._T = [vol(), vol()]
        self._H = [vol(), vol()]
        self._cur = 0
        self.T_max = vol()
        self.f_l = vol()
        self.phi = vol()
        self.cp_rho_field = vol()
        self.alpha_lu_field = vol()
        self.dgamma_lu_field = vol()
        self.tau_field = vol()
        self.dT_dt = vol()
        self.T_prev = vol()
        self.time_above_800_s = vol()
        self.time_above_1100_s = vol()
        self.time_above_solidus_s = vol()
        self.ux, self.uy, self.uz = vol(), vol(), vol()
        self.Fx, self.Fy, self.Fz = vol(), vol(), vol()
        self._separate_snapshot = bool(separate_force_snapshot)
        if self._separate_snapshot:
            self._snap = (vol(), vol(), vol())
        self.flags = torch.zeros(shape3, dtype=torch.int32, device=dev)
        self.surface_k_buf = torch.zeros((), **f32)
        self.deposit_vol_buf = torch.zeros((), **f32)
        self.deposit_real_buf = torch.zeros((), **f32)
        self.arc_norm_buf = torch.zeros((), **f32)
        self.step_scalars = torch.zeros(16, **f32)
        # health word of the fused step (WAAM_HEALTH_* bits, see WAAMTwin.health)
        self.step_status = torch.zeros(1, dtype=torch.int32, device=dev)
        # quiet-tile skipping of the fused step (WaamFields.tile_*): column-chunk
        # bits then one work byte per 32 x 8 tile, the work-tile list, per-tile
        # arc weight sums; their history is valid while _tiles_valid holds
        kt, jt = (self.nz + 31) // 32, (self.ny + 7) // 8
        n_tiles = kt * jt * self.nx
        self.tile_bits = torch.zeros(kt * self.nx * self.ny + n_tiles, dtype=torch.uint8, device=dev)
        self.tile_list = torch.zeros(1 + n_tiles, dtype=torch.int32, device=dev)
        self.tile_part = torch.zeros(n_tiles, dtype=torch.float64, device=dev)
        self._tiles_valid = False
        self._n_chunk_bytes = kt * self.nx * self.ny
        self.telem_fl_slice = torch.zeros((self.ny, self.nz), **f32)
        self.porosity_pos = torch.zeros((self.max_tracers, 3), **f32)
        self.porosity_active = torch.zeros(self.max_tracers, dtype=torch.int32, device=dev)
        self.tracer_head = torch.zeros((), dtype=torch.int32, device=dev)
        self.ex = torch.tensor(EX, dtype=torch.int32, device=dev)
        self.ey = torch.tensor(EY, dtype=torch.int32, device=dev)
        self.ez = torch.tensor(EZ, dtype=torch.int32, device=dev)
        self.w = torch.tensor(W, dtype=torch.float32, device=dev)
        self.opp = torch.tensor(OPP, dtype=torch.int32, device=dev)
        n = self.nx * self.ny * self.nz
        nbytes = int(_native.lib().waam_workspace_bytes(n))
        self.workspace = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
        self._has_vof_buf = False
        self._has_lorentz = False
        self._has_export = False
        if allocate_vof:
            self.ensure_vof_buffers()
        if allocate_lorentz:
            self.ensure_lorentz_fields()
        if allocate_export:
            self.ensure_export_buffers()
        self._read_buf = self.f_a
        self._write_buf = self.f_b
        # True when F may be non-zero outside FLUID/IFACE cells (the fused step
        # then clears it; see WaamStepParams.clear_forces)
        self._forces_dirty = True

    # -- optional fields (grid.py:228-262) --------------------------------
    def ensure_vof_buffers(self):
        if not self._has_vof_buf:
            self.phi_tmp = torch.zeros(self._shape3, dtype=torch.float32, device=self.device)
            self._has_vof_buf = True

    def ensure_lorentz_fields(self):
        if self._has_lorentz:
            return
        mk = lambda: torch.zeros(self._shape3, dtype=torch.float32, device=self.device)  # noqa: E731
        self.phi_elec, self.phi_elec_tmp, self.sigma_elec, self.elec_source = mk(), mk(), mk(), mk()
        self.Jx, self.Jy, self.Jz = mk(), mk(), mk()
        self.Bx, self.By, self.Bz = mk(), mk(), mk()
        # cells the potential solve holds at 0 (GAS, grounded SOLID), one byte
        # each, and the lists of its live and newly fixed cells
        self.elec_fixed = torch.zeros(self._shape3, dtype=torch.uint8, device=self.device)
        n = self.nx * self.ny * self.nz
        self.elec_live = torch.zeros(n, dtype=torch.int32, device=self.device)
        self.elec_zero = torch.zeros(n, dtype=torch.int32, device=self.device)
        from . import _native
        m = int(_native.lib().waam_elec_counts_len(self.nx, self.ny, self.nz))
        self.elec_counts = torch.zeros(m, dtype=torch.int32, device=self.device)
        self.elec_arc_k = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.n_elec_bins = 64
        self.elec_rad_bins = torch.zeros((self.nz, self.n_elec_bins), dtype=torch.float32,
                                         device=self.device)
        # the Jacobi check's L1 change and norm, side by side so that one
        # device-to-host copy reads both
        self.elec_res_norm = torch.zeros(2, dtype=torch.float32, device=self.device)
        self.elec_res_buf = self.elec_res_norm[0]
        self.elec_norm_buf = self.elec_res_norm[1]
        self._has_lorentz = True

    def ensure_export_buffers(self):
        if not self._has_export:
            self.kappa_field = torch.zeros(self._shape3, dtype=torch.float32, device=self.device)
            self.vorticity_mag = torch.zeros(self._shape3, dtype=torch.float32, device=self.device)
            self._has_export = True

    # -- double-buffered thermal fields -----------------------------------
    @property
    def H(self):
        return self._H[self._cur]

    @property
    def T(self):
        return self._T[self._cur]

    @property
    def H_next(self):
        return self._H[1 - self._cur]

    @property
    def T_next(self):
        return self._T[1 - self._cur]

    def flip_thermal(self):
        self._cur = 1 - self._cur

    @property
    def Fx_snap(self):
        return self._snap[0] if self._separate_snapshot else self.Fx

    @property
    def Fy_snap(self):
        return self._snap[1] if self._separate_snapshot else self.Fy

    @property
    def Fz_snap(self):
        return self._snap[2] if self._separate_snapshot else self.Fz

    # -- ping-pong populations (grid.py:268-278) --------------------------
    def worked_tiles(self):
        """(worked, total) 32 x 8 tiles of the last fused step (its work bytes;
        the list count itself is zeroed for the next step).  Synchronises."""
        work = self.tile_bits[self._n_chunk_bytes:]
        return int(work.sum(dtype=torch.int64).item()), int(work.numel())

    def swap_buffers(self):
        self._read_buf, self._write_buf = self._write_buf, self._read_buf

    @property
    def f_src(self):
        """The buffer the next collision reads (runs pending step work first)."""
        self.flush_stream()
        return self._read_buf

    @property
    def f_dst(self):
        """The buffer the next collision writes (runs pending step work first)."""
        self.flush_stream()
        return self._write_buf

    # -- population storage -------------------------------------------------
    def _rest_weights(self):
        w = getattr(self, "_w_col", None)
        if w is None:
            w = self._w_col = self.w.view(Q, 1, 1, 1)
        return w

    def flush_stream(self):
        """Run the work a pipelined step left pending -- its stream, or its
        collision, tracers and stream (see coupled_step)."""
        d = self.__dict__
        if d.get("_stream_pending", False) or d.get("_collide_pending", False):
            from .coupled_step import flush_stream
            flush_stream(self)

    def populations(self, t):
        """float32 f_q of population buffer ``t`` (f_a, f_b, f_src or f_dst)."""
        self.flush_stream()
        if t.dtype == torch.float32:
            return t
        return t.float() + self._rest_weights()

    def store_populations(self, dst, f):
        """Write float32 f_q into population buffer ``dst`` in its storage."""
        self.flush_stream()
        f = torch.as_tensor(f, device=self.device).to(torch.float32).reshape(dst.shape)
        if dst.dtype == torch.float32:
            dst.copy_(f)
        else:
            dst.copy_((f - self._rest_weights()).to(dst.dtype))

    @property
    def n_cells(self):
        return self.nx * self.ny * self.nz

    def estimated_vram_mb(self):
        total = 0
        for v in vars(self).values():
            if isinstance(v, torch.Tensor):
                total += v.numel() * v.element_size()
            elif isinstance(v, list):
                total += sum(t.numel() * t.element_size() for t in v if isinstance(t, torch.Tensor))
        return total / (1024 ** 2)

    def state_dict(self):
        """Host copies of every field of the state (for checkpoints and tests)."""
        self.flush_stream()
        names = ["rho", "T", "H", "T_max", "f_l", "phi", "dT_dt", "T_prev", "time_above_800_s",
                 "time_above_1100_s", "time_above_solidus_s", "ux", "uy", "uz", "Fx", "Fy",
                 "Fz", "flags", "f_a", "f_b", "cp_rho_field", "alpha_lu_field",
                 "dgamma_lu_field", "tau_field"]
        out = {}
        for k in names:
            t = getattr(self, k)
            if k in ("f_a", "f_b"):
                t = self.populations(t)
            out[k] = t.detach().cpu().numpy()
        out["read_is_a"] = self._read_buf is self.f_a
        return out

    def load_state(self, st):
        """Inverse of state_dict (numpy arrays or tensors)."""
        self.flush_stream()
        self._forces_dirty = True
        self._tiles_valid = False
        if self._has_lorentz:
            # the potential buffers may now hold anything at fixed cells: the
            # next solve treats every fixed cell as newly fixed
            self.elec_fixed.zero_()
        for k, v in st.items():
            if k == "read_is_a":
                self._read_buf, self._write_buf = (self.f_a, self.f_b) if v else (self.f_b, self.f_a)
                continue
            if k in ("T", "H"):
                dst = getattr(self, k)
            elif not hasattr(self, k) or not isinstance(getattr(self, k), torch.Tensor):
                continue
            else:
                dst = getattr(self, k)
            if k in ("f_a", "f_b"):
                self.store_populations(dst, v)
                continue
            dst.copy_(torch.as_tensor(v).to(dst.dtype).reshape(dst.shape))


# The fields a pending collision (WaamStepParams.defer_collide) still has to
# write: reading one through the grid runs the pending work first.
_COLLIDE_OUTPUTS = ("rho", "ux", "uy", "uz", "Fx", "Fy", "Fz", "porosity_pos",
                    "porosity_active")


def _collide_output(name):
    key = "_pf_" + name

    def get(self):
        if self.__dict__.get("_collide_pending", False):
            self.flush_stream()
        return self.__dict__[key]

    def put(self, value):
        self.__dict__[key] = value

    return property(get, put, doc="%s (runs a pending collision first)" % name)


for _name in _COLLIDE_OUTPUTS:
    setattr(WAAMGrid, _name, _collide_output(_name))


# The population buffers: a pipelined step leaves its stream (and possibly its
# collision) pending, so reading f_a / f_b / f_src / f_dst through the grid
# runs that work first and the caller sees the step's streamed populations.
_POPULATIONS = ("f_a", "f_b")


def _population(name):
    key = "_pf_" + name

    def get(self):
        self.flush_stream()
        return self.__dict__[key]

    def put(self, value):
        self.__dict__[key] = value

    return property(get, put, doc="%s (runs pending step work first)" % name)


for _name in _POPULATIONS:
    setattr(WAAMGrid, _name, _population(_name))


def raw_field(g, name):
    """A field without running pending step work (the step's own use)."""
    if name in _COLLIDE_OUTPUTS or name in _POPULATIONS:
        return g.__dict__["_pf_" + name]
    if name == "f_src":
        return g._read_buf
    if name == "f_dst":
        return g._write_buf
    return getattr(g, name)


def cells_of(mm, dx):
    return max(1, int(round(mm / (dx * 1000.0))))


__all__ = ["WAAMGrid", "Q", "EX", "EY", "EZ", "W", "OPP", "cells_of", "math"]
