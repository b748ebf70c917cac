"""Electromagnetic force of the welding current (physics/weld_forces.py:196-281).

The same sequence as the reference: conductivity map, Gaussian current source
normalised to the welding current, a warm-started damped Jacobi solve of the
electric potential with a relative-L1 convergence check every ten sweeps,
current density, axisymmetric self field from the enclosed axial current and
the f_l-weighted J x B body force added to F.

Differences of form, not of result: the potential ping-pongs between
``phi_elec`` and ``phi_elec_tmp`` instead of copying the new iterate back
(after the solve ``phi_elec`` holds the last iterate, ``phi_elec_tmp`` the one
before it); each chunk of ten sweeps is one native call whose last sweep also
computes the L1 change -- the only sweep whose L1 the reference reads; the
sweeps visit only the live cells -- those not held at 0 (GAS, grounded
SOLID), listed when the conductivity map is built -- while both buffers keep
exact zeros at the fixed cells; and clearing, injecting and normalising the
source is one call.
"""
from __future__ import annotations

import math

from .. import kernels

MU0 = 4.0e-7 * math.pi


def _jacobi_budget(twin, g, cold_start):
    max_iters = max(int(twin.lorentz_jacobi_iters), 20)
    if cold_start:
        n_max = max(g.nx, g.ny, g.nz)
        max_iters = max(max_iters, 2 * n_max * n_max)
    return max_iters


def solve_lorentz(twin, g, arc_i, arc_j, arc_k, apply_force=True, arc_k_dev=None):
    """``apply_force=False`` leaves J x B to the caller (the fused step adds it
    inside its collision, before the force clamp).  ``arc_k_dev``: the arc
    height as a one-element device tensor (the fused step's scalar), used
    instead of ``arc_k`` so that nothing is read back before the solve."""
    if not twin.enable_lorentz:
        return
    g.ensure_lorentz_fields()
    if arc_k_dev is None:
        g.elec_arc_k.fill_(float(arc_k))
        arc_k_dev = g.elec_arc_k
    # phi_elec is the first sweep's input, phi_elec_tmp its output
    kernels.elec_prepare(g.sigma_elec, g.elec_fixed, g.phi_elec_tmp, g.f_l, g.flags,
                         twin.sigma_liquid_Sm, twin.sigma_solid_Sm, twin.nz_solid, g.elec_live,
                         g.elec_zero, g.elec_counts)
    kernels.elec_arc_source_dev(g.elec_source, arc_i, arc_j, arc_k_dev, twin.sigma_cells,
                                twin.welding_current_A, g.dx)

    cold_start = not getattr(twin, "_lorentz_warm", False)
    if cold_start:
        kernels.elec_init_ground(g.phi_elec, g.flags, twin.nz_solid, g.FLAG_SOLID)
        twin._lorentz_warm = True
    max_iters = _jacobi_budget(twin, g, cold_start)
    tol = float(getattr(twin, "lorentz_jacobi_tol", 1e-4))
    check_every = 10
    converged = False
    iters_done = 0
    rel = float("inf")
    while iters_done < max_iters:
        chunk = min(check_every, max_iters - iters_done)
        kernels.elec_jacobi_live(g.phi_elec, g.phi_elec_tmp, g.sigma_elec, g.elec_source,
                                 g.elec_live, g.elec_zero, g.elec_counts, g.dx,
                                 twin.lorentz_jacobi_omega, chunk, iters_done == 0, arc_k_dev,
                                 twin.sigma_cells, g.elec_res_buf, g.elec_norm_buf)
        if chunk % 2 == 1:
            g.phi_elec, g.phi_elec_tmp = g.phi_elec_tmp, g.phi_elec
        iters_done += chunk
        res, norm = g.elec_res_norm.tolist()
        rel = res / max(norm, 1e-30)
        if rel < tol:
            converged = True
            break
    if not converged:
        twin._lorentz_unconverged = getattr(twin, "_lorentz_unconverged", 0) + 1
        twin._lorentz_unconverged_streak = getattr(twin, "_lorentz_unconverged_streak", 0) + 1
        n_bad = twin._lorentz_unconverged
        if n_bad in (1, 10, 100) or n_bad % 1000 == 0:
            print("[weld_forces] WARNING: Lorentz Jacobi hit %d iters without converging "
                  "(rel change=%.2e > %.0e); raise lorentz_jacobi_iters. (%d occurrences)"
                  % (max_iters, rel, tol, n_bad))
    else:
        twin._lorentz_unconverged_streak = 0
    twin._lorentz_last_iters = iters_done

    bin_dr_cells = max(float(max(g.nx, g.ny)) / (2.0 * g.n_elec_bins), 0.5)
    kernels.elec_fields(g.Jx, g.Jy, g.Jz, g.Bx, g.By, g.Bz, g.elec_rad_bins, g.phi_elec,
                        g.sigma_elec, g.flags, arc_i, arc_j, g.dx, bin_dr_cells, MU0,
                        g.n_elec_bins)
    if apply_force:
        kernels.apply_lorentz_JxB(g.Fx, g.Fy, g.Fz, g.Jx, g.Jy, g.Jz, g.Bx, g.By, g.Bz, g.f_l,
                                  g.flags, g.dt, g.dx, twin.mat.rho, g.FLAG_GAS)
