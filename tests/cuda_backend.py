"""Kernel-case backend over the native C ABI (GPU tests only).

Every call copies the numpy arguments to fresh CUDA tensors, calls the
``waam_*`` entry point through ctypes exactly as an FFI user would, and
copies the results back into the numpy arrays (in place), so the golden
cases in ``cases.py`` run unchanged against the CUDA kernels.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from waam_solver_b200 import _native

_WS_FUNCS = {"inject_arc_heat", "inject_goldak_heat", "advect_diffuse_temperature",
             "apply_contact_angle_phi_bc", "elec_normalize_source",
             "advect_diffuse_temperature_variable"}
_NORM_FUNCS = {"inject_arc_heat", "inject_goldak_heat"}


class CudaBackend:
    def __init__(self, device="cuda"):
        self.device = torch.device(device)
        self.launched = []

    def _up(self, a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def _run(self, name, args, n_cells):
        dev_args, back = [], []
        for a in args:
            if isinstance(a, np.ndarray):
                t = self._up(a)
                dev_args.append(t.data_ptr())
                back.append((a, t))
            else:
                dev_args.append(a)
        extra_tail = []
        norm = None
        if name in _NORM_FUNCS:
            norm = torch.zeros((), dtype=torch.float32, device=self.device)
            dev_args.insert(3, norm.data_ptr())
        if name in _WS_FUNCS:
            nbytes = int(_native.lib().waam_workspace_bytes(n_cells))
            ws = torch.zeros(nbytes, dtype=torch.uint8, device=self.device)
            extra_tail = [ws.data_ptr(), nbytes]
        stream = torch.cuda.current_stream().cuda_stream
        _native.call("waam_" + name, *(dev_args + extra_tail + [stream]))
        torch.cuda.synchronize()
        self.launched.append(name)
        for host, t in back:
            host[...] = t.cpu().numpy()
        return None if norm is None else float(norm.item())

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)

        def f(*args):
            n_cells = None
            for a in args:
                if isinstance(a, np.ndarray) and a.ndim == 3:
                    n_cells = a.size
                    break
            return self._run(name, list(args), n_cells)
        return f

    def _ws(self, n_cells):
        nbytes = int(_native.lib().waam_workspace_bytes(n_cells))
        return torch.zeros(nbytes, dtype=torch.uint8, device=self.device), nbytes

    def elec_l1(self, a, b):
        nx, ny, nz = a.shape
        ta, tb = self._up(a), self._up(b)
        d = torch.zeros((), dtype=torch.float32, device=self.device)
        m = torch.zeros((), dtype=torch.float32, device=self.device)
        ws, nbytes = self._ws(a.size)
        _native.call("waam_elec_l1_diff", ta.data_ptr(), tb.data_ptr(), d.data_ptr(),
                     m.data_ptr(), nx, ny, nz, ws.data_ptr(), nbytes,
                     torch.cuda.current_stream().cuda_stream)
        self.launched.append("elec_l1_diff")
        return float(d.item()), float(m.item())

    def elec_bins(self, Jz, bins, nx, ny, nz, arc_i, arc_j, dx, bin_dr, n_bins):
        tj, tb = self._up(Jz), self._up(bins)
        ws, nbytes = self._ws(Jz.size)
        st = torch.cuda.current_stream().cuda_stream
        _native.call("waam_elec_bin_axial_current", tj.data_ptr(), tb.data_ptr(), nx, ny, nz,
                     arc_i, arc_j, dx, bin_dr, n_bins, ws.data_ptr(), nbytes, st)
        _native.call("waam_elec_prefix_bins", tb.data_ptr(), n_bins, nz, st)
        torch.cuda.synchronize()
        self.launched.append("elec_bins")
        bins[...] = tb.cpu().numpy()

    def refresh_thermal_properties(self, T, cp_f, alpha_f, dg_f, tau_f, flags, n, tab, cnt, fb,
                                   ref, rho, dt, dx, force_scale, marangoni_scale):
        """The oracle's flat table arguments packed into a WaamMaterialTables."""
        from waam_solver_b200 import kernels
        tb = kernels.material_tables_struct(*[tab[8 * q:8 * q + 8] for q in range(8)],
                                            *[int(c) for c in cnt], *[float(v) for v in fb])
        outs = [self._up(a) for a in (cp_f, alpha_f, dg_f, tau_f)]
        tT, tf = self._up(T), self._up(flags)
        _native.call("waam_refresh_thermal_properties", tT.data_ptr(),
                     *[o.data_ptr() for o in outs], tf.data_ptr(), n, ctypes.byref(tb),
                     rho, dt, dx, force_scale, float(ref[0]), float(ref[1]), float(ref[2]),
                     float(ref[3]), marangoni_scale, 1, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        self.launched.append("refresh_thermal_properties")
        for host, t in zip((cp_f, alpha_f, dg_f, tau_f), outs):
            host[...] = t.cpu().numpy()

    def compute_vorticity_magnitude(self, ux, uy, uz, flags, vort, nx, ny, nz, dt):
        """The C entry also takes dx (unused, as in the reference)."""
        self._run("compute_vorticity_magnitude", [ux, uy, uz, flags, vort, nx, ny, nz, 0.0, dt],
                  None)

    def shift_simulation_window_x(self, *args):
        """Oracle argument order (fields, n_shift, T_amb, cp_rho, rho0, nz_solid,
        nx, ny, nz) through the reference-signature wrapper."""
        from waam_solver_b200 import kernels
        fields = list(args[:24])
        n_shift, T_amb, cp_rho, rho0, nz_solid, nx, ny, nz = args[24:]
        dev = [self._up(a) for a in fields]
        kernels.shift_simulation_window_x(n_shift, *dev, T_amb, cp_rho, rho0, nz_solid, 1, 2, 0,
                                          nx, ny, nz)
        torch.cuda.synchronize()
        self.launched.append("shift_simulation_window_x")
        for host, t in zip(fields, dev):
            host[...] = t.cpu().numpy()

    def surface_height_at(self, phi, flags, nx, ny, nz, i0, j0, nz_fallback):
        out = torch.zeros((), dtype=torch.float32, device=self.device)
        tp, tf = self._up(phi), self._up(flags)
        _native.call("waam_surface_height_at", tp.data_ptr(), tf.data_ptr(), out.data_ptr(), nx,
                     ny, nz, i0, j0, nz_fallback, torch.cuda.current_stream().cuda_stream)
        return float(out.item())

    def feed_wire(self, *args):
        """waam_feed_wire on float32 populations (storage code 0)."""
        args = list(args)
        acc = np.array([args[19]], dtype=np.float32)
        args[19] = acc
        args.insert(1, 0)
        self._run("feed_wire", args, None)
        return float(acc[0])

    def feed_wire_surface(self, *args):
        args = list(args)
        vol = np.array([args[20]], dtype=np.float32).reshape(())
        real = np.array([args[21]], dtype=np.float32).reshape(())
        va, ra = np.array(vol).reshape(1), np.array(real).reshape(1)
        args[20], args[21] = va, ra
        self._run("feed_wire_surface", args, None)
        return float(va[0]), float(ra[0])
