"""Droplet deposition: the one-CTA wavefront formulation against the serial oracle.

The reference's feed_wire_surface (kernels.py:278-400) converts gas cells
under a reserve-then-commit budget; the oracle visits them serially in
lexicographic order.  The CUDA kernel instead computes the unbudgeted
conversion set as the least solution of a recursion over the three
predecessor neighbours and keeps its first m cells.  ``model_deposit`` below
states that formulation in numpy; the CPU tests check it against the oracle
(the algorithmic claim), the GPU tests check the kernel against the oracle
bit for bit, including the footprint retry loop of
solvers/coupled_step.py:126-151, multi-word columns and the serial path for
boxes too large for shared memory.
"""
from __future__ import annotations

import numpy as np
import pytest

import state_gen
from cases import OracleBackend

GAS, FLUID, SOLID = 2, 0, 1
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32)


def _f32(x):
    return np.float32(x)


def _box(nx, ny, nz, arc_i, arc_j, arc_k, foot_r, drop_r):
    arc_i, arc_j, arc_k, foot_r, drop_r = map(_f32, (arc_i, arc_j, arc_k, foot_r, drop_r))
    sr = foot_r if foot_r > drop_r else drop_r
    i0 = max(0, int(arc_i - sr))
    i1 = min(nx, int(arc_i + sr) + 1)
    j0 = max(0, int(arc_j - sr))
    j1 = min(ny, int(arc_j + sr) + 1)
    k0 = max(0, int(arc_k - _f32(1.0)))
    k_span = max(drop_r + _f32(3.0), _f32(4.0))
    k1 = min(nz, int(arc_k + k_span) + 1)
    return (i0, i1, j0, j1, k0, k1, sr * sr, drop_r * drop_r, arc_k + drop_r + _f32(0.5))


def _metal_nb(st, i, j, k):
    flags, phi, fl = st["flags"], st["phi"], st["f_l"]
    nx, ny, nz = flags.shape
    for di, dj, dk in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
        a, b, c = i + di, j + dj, k + dk
        if 0 <= a < nx and 0 <= b < ny and 0 <= c < nz:
            if flags[a, b, c] in (FLUID, SOLID) or phi[a, b, c] > _f32(0.35) or fl[a, b, c] > _f32(0.2):
                return True
    return False


def _convert(st, cells, a):
    hdrop = _f32(a["cp_rho"]) * _f32(a["T_drop"]) + _f32(a["L_rho"])
    for (i, j, k) in cells:
        st["flags"][i, j, k] = FLUID
        st["f_l"][i, j, k] = 1.0
        st["phi"][i, j, k] = 1.0
        st["T"][i, j, k] = _f32(a["T_drop"])
        st["H"][i, j, k] = hdrop
        st["rho"][i, j, k] = 1.0
        st["f_a"][:, i, j, k] = W19 * _f32(1.0)


def model_deposit(st, a, foot_r, vol, real):
    """One feed_wire_surface call in the set formulation (numpy, small boxes)."""
    nx, ny, nz = st["flags"].shape
    i0, i1, j0, j1, k0, k1, foot2, rd2, drop_cz = _box(nx, ny, nz, a["arc_i"], a["arc_j"],
                                                       a["arc_k"], foot_r, a["drop_r"])
    arc_i, arc_j = _f32(a["arc_i"]), _f32(a["arc_j"])
    target, cv = _f32(a["target_vol"]), _f32(a["cell_vol"])
    vol, real = _f32(vol), _f32(real)
    order = [(i, j, k) for i in range(i0, i1) for j in range(j0, j1) for k in range(k0, k1)]
    E1, E2, M = set(), set(), set()
    for (i, j, k) in order:
        if st["flags"][i, j, k] != GAS:
            continue
        di, dj = _f32(i) - arc_i, _f32(j) - arc_j
        rij2 = di * di + dj * dj
        dk = _f32(k) - drop_cz
        r2 = di * di + dj * dj + dk * dk
        if not (rij2 > foot2 and r2 > rd2):
            E1.add((i, j, k))
        if not (rij2 > foot2 * _f32(1.44)):
            E2.add((i, j, k))
        if _metal_nb(st, i, j, k):
            M.add((i, j, k))

    def closure(E, seeds):
        conv = []
        cs = set()
        for (i, j, k) in order:
            if (i, j, k) in E and ((i, j, k) in seeds or (i - 1, j, k) in cs or
                                   (i, j - 1, k) in cs or (i, j, k - 1) in cs):
                cs.add((i, j, k))
                conv.append((i, j, k))
        return conv

    def spend(avail):
        nonlocal vol, real
        m = 0
        while m < avail and not (vol >= target):
            vol = vol + cv
            real = real + cv
            m += 1
        return m

    S1 = closure(E1, M)
    c1 = S1[:spend(len(S1))]
    _convert(st, c1, a)
    if not (vol >= target):
        done = set(c1)
        seeds = set(M)
        for (i, j, k) in c1:
            for d in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
                seeds.add((i + d[0], j + d[1], k + d[2]))
        S2 = closure(E2 - done, seeds)
        _convert(st, S2[:spend(len(S2))], a)
    hdrop = _f32(a["cp_rho"]) * _f32(a["T_drop"]) + _f32(a["L_rho"])
    for (i, j, k) in order:
        if st["flags"][i, j, k] != FLUID or st["f_l"][i, j, k] < _f32(0.45):
            continue
        di, dj = _f32(i) - arc_i, _f32(j) - arc_j
        if di * di + dj * dj > foot2 * _f32(1.44):
            continue
        st["T"][i, j, k] = _f32(a["T_drop"])
        st["H"][i, j, k] = hdrop
        st["rho"][i, j, k] = 1.0
        st["f_a"][:, i, j, k] = W19 * _f32(1.0)
    return float(vol), float(real)


DEP_FIELDS = ("flags", "f_l", "phi", "T", "H", "rho", "f_a")


def _state(nx, ny, nz, seed, nz_solid=None):
    st = state_gen.seeded_state(nx, ny, nz, seed=seed, nz_solid=nz_solid)
    return {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}


def _args(st, arc_i, arc_j, arc_k, drop_r, target_cells):
    m = state_gen.MATERIAL
    cell_vol = _f32(8e-12)
    return dict(arc_i=arc_i, arc_j=arc_j, arc_k=arc_k, drop_r=drop_r,
                target_vol=float(_f32(target_cells * 8e-12)), cell_vol=float(cell_vol),
                T_drop=2100.0, cp_rho=m["rho"] * m["cp"], L_rho=m["rho"] * m["L_fusion"])


def oracle_deposit(O, st, a, foot_r, vol, real):
    nx, ny, nz = st["flags"].shape
    va = np.array([vol], dtype=np.float32)
    ra = np.array([real], dtype=np.float32)
    O.call("wo_feed_wire_surface", st["f_a"], st["flags"], st["f_l"], st["phi"], st["H"], st["T"],
           st["rho"], nx, ny, nz, a["arc_i"], a["arc_j"], a["arc_k"], foot_r, a["drop_r"],
           a["target_vol"], a["T_drop"], a["cp_rho"], a["L_rho"], 1.0, va, ra, a["cell_vol"])
    return float(va[0]), float(ra[0])


def retry_radii(r_try, n=10):
    out = []
    for _ in range(n):
        out.append(r_try)
        r_try = min(r_try + 1.5, 16.0)
    return out


def oracle_droplet(O, st, a, radii, accept):
    """The host retry loop of solvers/coupled_step.py:130-151 over the oracle."""
    placed = 0.0
    vol = 0.0
    for r in radii:
        vol, placed = oracle_deposit(O, st, a, r, placed, placed)
        if placed >= accept:
            break
    return vol, placed


# (name, grid, seed, nz_solid, arc (i, j, dk above the solid), drop_r, foot_r, target cells)
CASES = [
    ("centre_cut_in_pass1", (40, 32, 24), 1, 8, (19.3, 15.6, 1.2), 3.4, 5.0, 40),
    ("centre_pass2", (40, 32, 24), 2, 8, (20.1, 16.2, 0.7), 3.0, 4.0, 400),
    ("retries_short", (40, 32, 24), 3, 8, (20.5, 15.5, 2.0), 3.8, 4.5, 5000),
    ("corner_clipped", (36, 30, 20), 4, 7, (0.6, 29.3, 1.0), 3.0, 6.0, 300),
    ("no_budget", (24, 24, 16), 5, 6, (11.0, 12.0, 1.0), 2.5, 3.0, 0),
    ("one_cell", (24, 24, 16), 6, 6, (11.5, 12.5, 1.5), 2.5, 3.0, 1),
    ("exact_fill", (30, 30, 18), 7, 6, (14.2, 15.1, 0.4), 3.1, 4.2, 57),
]


def _setup(case):
    name, (nx, ny, nz), seed, nzs, (ai, aj, dk), drop_r, foot_r, cells = case
    st = _state(nx, ny, nz, seed, nzs)
    a = _args(st, ai, aj, nzs + dk, drop_r, cells)
    return st, a, foot_r


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_set_formulation_matches_serial_oracle(case):
    """The recursion + first-m cut (numpy) equals the oracle's serial visit."""
    O = OracleBackend().O
    st, a, foot_r = _setup(case)
    st_m = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    for vol0, real0 in ((0.0, 0.0), (3 * 8e-12, 1e-11)):
        want = oracle_deposit(O, st, a, foot_r, vol0, real0)
        got = model_deposit(st_m, a, foot_r, vol0, real0)
        assert got == want
        for f in DEP_FIELDS:
            assert np.array_equal(st_m[f], st[f]), f


def _to_dev(st):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in DEP_FIELDS}


def _gpu_call(dev, a, radii, accept, vol0=0.0, real0=0.0, single=False):
    import torch
    from waam_solver_b200 import kernels
    nx, ny, nz = dev["flags"].shape
    va = torch.full((), vol0, dtype=torch.float32, device="cuda")
    ra = torch.full((), real0, dtype=torch.float32, device="cuda")
    common = (dev["f_a"], dev["flags"], dev["f_l"], dev["phi"], dev["H"], dev["T"], dev["rho"],
              a["arc_i"], a["arc_j"], a["arc_k"])
    tail = (a["drop_r"], a["target_vol"], a["T_drop"], a["cp_rho"], a["L_rho"], 1.0, va, ra,
            a["cell_vol"], GAS, FLUID, SOLID, nx, ny, nz)
    if single:
        kernels.feed_wire_surface(*common, radii[0], *tail)
    else:
        kernels.deposit_droplet(*common, radii, accept, *tail)
    torch.cuda.synchronize()
    return float(va.item()), float(ra.item())


def _check_dev(dev, st, tag):
    for f in DEP_FIELDS:
        got = dev[f].cpu().numpy()
        assert np.array_equal(got, st[f]), "%s: %s differs at %d cells" % (
            tag, f, int((got != st[f]).sum()))


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gpu_feed_wire_surface_single_attempt(case):
    O = OracleBackend().O
    st, a, foot_r = _setup(case)
    dev = _to_dev(st)
    vol0, real0 = 2 * 8e-12, 5e-12
    want = oracle_deposit(O, st, a, foot_r, vol0, real0)
    got = _gpu_call(dev, a, [foot_r], 0.0, vol0, real0, single=True)
    assert got == want
    _check_dev(dev, st, case[0])


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gpu_deposit_droplet_retry_loop(case):
    O = OracleBackend().O
    st, a, foot_r = _setup(case)
    dev = _to_dev(st)
    radii = retry_radii(foot_r)
    accept = a["target_vol"] * 0.98
    want = oracle_droplet(O, st, a, radii, accept)
    got = _gpu_call(dev, a, radii, accept)
    assert got == want
    _check_dev(dev, st, case[0])


@pytest.mark.gpu
def test_gpu_deposit_wide_box_block_wavefront():
    """Diagonals longer than a warp take the block-barrier wavefront."""
    O = OracleBackend().O
    st = _state(64, 60, 16, 11, 6)
    a = _args(st, 31.2, 29.7, 7.0, 3.0, 900)
    radii = [20.0, 21.5, 23.0]
    dev = _to_dev(st)
    want = oracle_droplet(O, st, a, radii, a["target_vol"] * 0.98)
    got = _gpu_call(dev, a, radii, a["target_vol"] * 0.98)
    assert got == want
    _check_dev(dev, st, "wide")


@pytest.mark.gpu
def test_gpu_deposit_multiword_columns():
    """Columns taller than 64 cells carry the k recursion across words."""
    O = OracleBackend().O
    st = _state(20, 20, 100, 12, 10)
    # the box spans 71 cells in k: the gas above the surface forms eligible runs
    # that cross the 64-bit word boundary
    a = _args(st, 9.5, 10.2, 11.0, 66.0, 20000)
    dev = _to_dev(st)
    before = st["flags"].copy()
    want = oracle_deposit(O, st, a, 66.0, 0.0, 0.0)
    converted = (before == GAS) & (st["flags"] == FLUID)
    assert converted[:, :, 10 + 64:].any()          # k0 = 10: bits of the second word
    got = _gpu_call(dev, a, [66.0], 0.0, single=True)
    assert got == want
    _check_dev(dev, st, "multiword")


@pytest.mark.gpu
def test_gpu_deposit_serial_path_for_large_boxes():
    """A search box beyond the shared-memory bitmasks runs the serial kernel."""
    O = OracleBackend().O
    st = _state(112, 112, 12, 13, 5)
    a = _args(st, 55.5, 56.2, 6.0, 3.0, 3000)
    dev = _to_dev(st)
    want = oracle_deposit(O, st, a, 52.0, 0.0, 0.0)
    got = _gpu_call(dev, a, [52.0], 0.0, single=True)
    assert got == want
    _check_dev(dev, st, "serial")
