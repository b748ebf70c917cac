"""The fused forms of the Lorentz solve against the reference operator sequence.

* elec_arc_source (clear + inject + normalise in two passes) against
  elec_clear_source, elec_inject_arc_source and elec_normalize_source: the same
  float expressions, the normalising sum in double in another fixed order
  (relative 1e-6);
* elec_bin_axial_current on a 512-column grid (the chunked per-warp path)
  against a float64 numpy sum of the same Jz field;
* the Jacobi sweep with the L1 check equals the plain sweep bit for bit, and
  its L1 sums match a float64 numpy sum.
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _k():
    from waam_solver_b200 import kernels
    return kernels


@pytest.mark.parametrize("shape,arc", [((40, 24, 24), (12.3, 11.7, 9.4)),
                                       ((96, 64, 80), (40.2, 30.9, 33.1)),
                                       ((30, 20, 16), (5.0, 4.0, 40.0))])
def test_arc_source_matches_operator_sequence(shape, arc):
    K = _k()
    dev = torch.device("cuda", 0)
    a = torch.full(shape, 7.0, device=dev)
    b = torch.full(shape, 7.0, device=dev)
    sigma_cells, current, dx = 6.5, 180.0, 2e-4
    K.elec_clear_source(a)
    K.elec_inject_arc_source(a, *arc, sigma_cells, current, dx, shape[2])
    K.elec_normalize_source(a, current, dx)
    K.elec_arc_source(b, *arc, sigma_cells, current, dx)
    torch.cuda.synchronize()
    an, bn = a.cpu().numpy(), b.cpu().numpy()
    assert np.array_equal(an == 0.0, bn == 0.0)
    np.testing.assert_allclose(bn, an, rtol=1e-6, atol=0.0)
    total = float((bn.astype(np.float64) * dx ** 3).sum())
    if an.any():
        assert abs(total - current) <= 1e-4 * current


def test_bins_match_float64_sum():
    K = _k()
    dev = torch.device("cuda", 0)
    nx, ny, nz, n_bins = 32, 16, 70, 64
    rng = np.random.default_rng(4)
    jz = rng.normal(0.0, 1e6, (nx, ny, nz)).astype(np.float32)
    Jz = torch.from_numpy(jz).to(dev)
    bins = torch.zeros((nz, n_bins), dtype=torch.float32, device=dev)
    arc_i, arc_j, dx = 13.4, 7.9, 2e-4
    bin_dr = max(float(max(nx, ny)) / (2.0 * n_bins), 0.5)
    K.elec_bin_axial_current(Jz, bins, arc_i, arc_j, dx, bin_dr, n_bins, nz)
    torch.cuda.synchronize()
    ref = np.zeros((nz, n_bins), np.float64)
    dx2 = np.float32(dx) * np.float32(dx)
    for i in range(nx):
        for j in range(ny):
            di = np.float32(i) - np.float32(arc_i)
            dj = np.float32(j) - np.float32(arc_j)
            r = np.sqrt(np.float32(di * di + dj * dj))
            b = min(int(r / np.float32(bin_dr)), n_bins - 1)
            ref[:, b] += (jz[i, j, :] * dx2).astype(np.float64)
    np.testing.assert_allclose(bins.cpu().numpy(), ref.astype(np.float32), rtol=1e-6,
                               atol=1e-6 * float(np.abs(ref).max()))


def test_jacobi_l1_sweep_matches_plain_sweep():
    K = _k()
    dev = torch.device("cuda", 0)
    nx, ny, nz, nzs = 64, 48, 40, 12
    rng = np.random.default_rng(8)
    flags = np.full((nx, ny, nz), 2, np.int32)
    flags[:, :, :nzs] = 1
    flags[:, :, nzs:nzs + 3] = 4
    flags[20:40, 10:30, nzs:nzs + 5] = 0
    sigma = np.where(flags == 2, 1e-8, rng.uniform(1e5, 1e6, flags.shape)).astype(np.float32)
    src = np.zeros(flags.shape, np.float32)
    src[28:34, 18:24, nzs + 1:nzs + 4] = rng.uniform(1e9, 2e9, (6, 6, 3)).astype(np.float32)
    phi = rng.uniform(0.0, 0.01, flags.shape).astype(np.float32)
    t = lambda x: torch.from_numpy(x).to(dev)  # noqa: E731
    F, S, Q, P = t(flags), t(sigma), t(src), t(phi)
    o1, o2 = torch.zeros_like(P), torch.zeros_like(P)
    diff = torch.zeros((), dtype=torch.float32, device=dev)
    norm = torch.zeros((), dtype=torch.float32, device=dev)
    K.elec_jacobi_step(P, o1, S, Q, F, 2e-4, 0.85, 2, 1, nzs, nx, ny, nz)
    K.elec_jacobi_step_l1(P, o2, S, Q, F, 2e-4, 0.85, nzs, diff, norm)
    torch.cuda.synchronize()
    a, b = o1.cpu().numpy(), o2.cpu().numpy()
    assert np.array_equal(a, b)
    d_ref = float(np.abs(b.astype(np.float64) - phi.astype(np.float64)).sum())
    n_ref = float(np.abs(phi.astype(np.float64)).sum())
    assert math.isclose(float(diff.item()), d_ref, rel_tol=1e-6)
    assert math.isclose(float(norm.item()), n_ref, rel_tol=1e-6)


@pytest.mark.parametrize("n_sweeps", [1, 4, 7])
def test_jacobi_chunk_matches_single_sweeps(n_sweeps):
    """The masked chunk (source read only inside its k slab) equals the
    reference-form sweeps bit for bit; the L1 of its last sweep matches."""
    K = _k()
    dev = torch.device("cuda", 0)
    nx, ny, nz, nzs = 48, 40, 36, 10
    rng = np.random.default_rng(12)
    flags = np.full((nx, ny, nz), 2, np.int32)
    flags[:, :, :nzs] = 1
    flags[:, :, nzs:nzs + 2] = 4
    flags[15:30, 12:28, nzs:nzs + 4] = 0
    flags[5:8, 5:8, nzs + 6] = 1          # a solid cell above nz_solid is not grounded
    fl = np.where(flags == 0, rng.uniform(0.3, 1.0, flags.shape), 0.0).astype(np.float32)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    F, FL = t(flags), t(fl)
    arc = (22.3, 19.6, float(nzs + 1))
    sigma_cells, current, dx, om = 3.5, 180.0, 2e-4, 0.85
    src = torch.zeros((nx, ny, nz), device=dev)
    K.elec_arc_source(src, *arc, sigma_cells, current, dx)
    s1, s2 = torch.zeros_like(src), torch.zeros_like(src)
    K.elec_build_sigma(s1, FL, F, 1e6, 1e5, 2)
    fixed = torch.zeros((nx, ny, nz), dtype=torch.uint8, device=dev)
    K.elec_build_sigma_mask(s2, fixed, FL, F, 1e6, 1e5, nzs)
    phi0 = rng.uniform(0.0, 0.01, (nx, ny, nz)).astype(np.float32)
    a, b = t(phi0), torch.zeros_like(src)
    d1, n1 = torch.zeros((), device=dev), torch.zeros((), device=dev)
    for s in range(n_sweeps):
        if s == n_sweeps - 1:
            K.elec_jacobi_step_l1(a, b, s1, src, F, dx, om, nzs, d1, n1)
        else:
            K.elec_jacobi_step(a, b, s1, src, F, dx, om, 2, 1, nzs, nx, ny, nz)
        a, b = b, a
    ca, cb = t(phi0), torch.zeros_like(src)
    d2, n2 = torch.zeros((), device=dev), torch.zeros((), device=dev)
    K.elec_jacobi_chunk(ca, cb, s2, src, fixed, dx, om, n_sweeps, arc[2], sigma_cells, d2, n2)
    last = cb if n_sweeps % 2 == 1 else ca
    torch.cuda.synchronize()
    assert torch.equal(s1, s2)
    assert torch.equal(a, last)
    assert math.isclose(float(d1.item()), float(d2.item()), rel_tol=1e-6)
    assert math.isclose(float(n1.item()), float(n2.item()), rel_tol=1e-6)


@pytest.mark.parametrize("shape", [(40, 32, 28, 8), (70, 80, 40, 10)])
def test_live_list_solve_matches_full_grid_sweeps(shape):
    """Three solves of 20 sweeps (chunks of 10) with the flags changing between
    them -- metal cells turning to gas and gas to metal -- on the live list and
    on full-grid sweeps: the potential in both buffers is equal bit for bit and
    the L1 sums of every chunk agree.  The second grid has more than 1024 tile
    blocks (two levels of the list's offset scan)."""
    K = _k()
    dev = torch.device("cuda", 0)
    nx, ny, nz, nzs = shape
    rng = np.random.default_rng(21)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    n = nx * ny * nz
    fixed = torch.zeros((nx, ny, nz), dtype=torch.uint8, device=dev)
    fixed_full = torch.zeros_like(fixed)
    live = torch.zeros(n, dtype=torch.int32, device=dev)
    zero = torch.zeros(n, dtype=torch.int32, device=dev)
    counts = torch.zeros(int(_native_counts_len(nx, ny, nz)), dtype=torch.int32, device=dev)
    # garbage in the buffers before the first solve (cold start zeroes only a)
    a_l, b_l = t(rng.uniform(0, 1, (nx, ny, nz)).astype(np.float32)), \
        t(rng.uniform(0, 1, (nx, ny, nz)).astype(np.float32))
    a_l.zero_()
    a_f, b_f = a_l.clone(), b_l.clone()
    sig_l, sig_f = torch.zeros_like(a_l), torch.zeros_like(a_l)
    src = torch.zeros_like(a_l)
    for solve in range(3):
        flags = np.full((nx, ny, nz), 2, np.int32)
        flags[:, :, :nzs] = 1
        flags[:, :, nzs] = 4
        x0 = 8 + 4 * solve
        flags[x0:x0 + 12, 10:22, nzs:nzs + 4 + solve] = 0
        flags[5:7, 5:7, nzs + 3] = 1
        fl = np.where(flags == 0, 0.9, 0.0).astype(np.float32)
        F, FL = t(flags), t(fl)
        arc = (x0 + 6.0, 16.0, float(nzs + 2))
        K.elec_arc_source(src, *arc, 3.0, 150.0, 2e-4)
        K.elec_prepare(sig_l, fixed, b_l, FL, F, 1e6, 1e5, nzs, live, zero, counts)
        K.elec_build_sigma_mask(sig_f, fixed_full, FL, F, 1e6, 1e5, nzs)
        for chunk in range(2):
            d1, n1 = torch.zeros((), device=dev), torch.zeros((), device=dev)
            d2, n2 = torch.zeros((), device=dev), torch.zeros((), device=dev)
            K.elec_jacobi_live(a_l, b_l, sig_l, src, live, zero, counts, 2e-4, 0.85, 10,
                               chunk == 0, torch.tensor([arc[2]], device=dev), 3.0, d1, n1)
            K.elec_jacobi_chunk(a_f, b_f, sig_f, src, fixed_full, 2e-4, 0.85, 10, arc[2], 3.0,
                                d2, n2)
            torch.cuda.synchronize()
            assert math.isclose(float(d1.item()), float(d2.item()), rel_tol=1e-6)
            assert math.isclose(float(n1.item()), float(n2.item()), rel_tol=1e-6)
        assert torch.equal(sig_l, sig_f)
        assert torch.equal(fixed, fixed_full)
        assert torch.equal(a_l, a_f), solve
        assert torch.equal(b_l, b_f), solve


def _native_counts_len(nx, ny, nz):
    from waam_solver_b200 import _native
    return _native.lib().waam_elec_counts_len(nx, ny, nz)
