"""The allocation-free Goldak injection entry point, through the C ABI.

Some callers hand the library only their own input and output buffers and
cannot create device memory during a run (an FFI host with no CUDA
allocator, or a loop under a fixed device-memory budget).  For them
waam_inject_goldak_heat_noalloc keeps its reduction scratch in a static
device array.  This test checks it against the workspace entry point
(waam_inject_goldak_heat) on two calls in a row, and that oversized grids
are refused.  The file sorts last so a stop-at-first-failure run has
already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import cases
import state_gen
from waam_solver_b200 import _native

pytestmark = pytest.mark.gpu

ARGS = dict(Q_w=4000.0, dt=2e-5, dx3=8e-12, eta=0.78, sign=1.0, ff=0.6, fr=1.4, a_f=6.0,
            a_r=14.0, b=6.0, c=5.0, pen=10.0, enable=1)


def _inject(name, H, flags, f_l, norm, nx, ny, nz, arc, ws=None):
    a = ARGS
    args = [H.data_ptr(), flags.data_ptr(), f_l.data_ptr(), norm.data_ptr(), nx, ny, nz,
            arc[0], arc[1], arc[2], a["Q_w"], a["dt"], a["dx3"], a["eta"], a["sign"], a["ff"],
            a["fr"], a["a_f"], a["a_r"], a["b"], a["c"], a["pen"], a["enable"]]
    if ws is not None:
        args += [ws.data_ptr(), ws.numel()]
    args.append(torch.cuda.current_stream().cuda_stream)
    _native.call(name, *args)


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    nx, ny, nz = 72, 40, 36
    st = state_gen.seeded_state(nx, ny, nz, seed=31)
    dev = torch.device("cuda")
    flags = torch.from_numpy(st["flags"]).to(dev)
    f_l = torch.from_numpy(st["f_l"]).to(dev)
    H_ref = torch.from_numpy(st["H"]).to(dev)
    H_new = H_ref.clone()
    norm_ref = torch.zeros((), dtype=torch.float32, device=dev)
    norm_new = torch.zeros((), dtype=torch.float32, device=dev)
    ws = torch.zeros(int(_native.lib().waam_workspace_bytes(nx * ny * nz)), dtype=torch.uint8,
                     device=dev)
    for call, arc in enumerate([(30.5, 19.2, float(st["nz_solid"] + 1)),
                                (33.0, 20.7, float(st["nz_solid"]))]):
        _inject("waam_inject_goldak_heat", H_ref, flags, f_l, norm_ref, nx, ny, nz, arc, ws)
        _inject("waam_inject_goldak_heat_noalloc", H_new, flags, f_l, norm_new, nx, ny, nz, arc)
        torch.cuda.synchronize()
        assert norm_ref.item() > 0.0
        cases.compare("no-alloc call %d" % call, H_new.cpu().numpy(), H_ref.cpu().numpy(), "H")
        assert abs(norm_new.item() - norm_ref.item()) <= cases.RTOL * norm_ref.item()


def test_noalloc_rejects_grids_beyond_its_scratch():
    t = torch.zeros(8, dtype=torch.float32, device="cuda")
    fl = torch.zeros(8, dtype=torch.int32, device="cuda")
    rc = _native.lib().waam_inject_goldak_heat_noalloc(
        t.data_ptr(), fl.data_ptr(), t.data_ptr(), t.data_ptr(), 4096, 4096, 2, 1.0, 1.0, 1.0,
        1.0, 1.0, 1.0, 1.0, 1.0, 0.6, 1.4, 1.0, 1.0, 1.0, 1.0, 1.0, 1,
        torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"16777216" in _native.lib().waam_last_error()
