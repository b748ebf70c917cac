// Fused B200 pipeline of one coupled step (solvers/coupled_step.py:73-464)
// plus the column, streaming and deposition kernels shared with the
// operator API.
//
// Per step (no droplet):  surface-height -> arc weight sum -> inject + cap
// -> thermal (advect/diffuse, losses, phase, T_max, cooling rate)
// -> VOF advect+reinit -> column pass (contact angle, flags, sync, time above)
// -> forces + collide + Mach clamp -> stream -> [remelt / solidify].
#include <cmath>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

using namespace waam;

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)
constexpr int kMainEvents = 7;

// ---------------------------------------------------------------------------
// Contact-angle ghost-phi BC (kernels.py:933-991), one warp per (i, j)
// column, lanes over k.  The reference updates phi in place; its serial
// order makes cell k see the final value of cell k-1 (rule "gas above pool")
// and the ghost write of cell k-1 (rule "fluid on substrate"), while other
// columns are read before the kernel (snapshot `snap`).  The ghost write of
// cell k-1 depends only on snapshot data, so it is computed in parallel; the
// k-1 -> k dependence through the final value is resolved by a warp-wide
// fixed-point iteration, whose fixed point is the unique serial result.
// ---------------------------------------------------------------------------
struct ContactConst {
    float cos_t, sin_t, film, spread;
};

// cos/sin of the contact angle are evaluated once on the host in double and
// rounded to float (the same values the oracle uses).
__device__ __forceinline__ ContactConst contact_const(float cos_t, float sin_t) {
    ContactConst cc;
    cc.cos_t = cos_t;
    cc.sin_t = sin_t;
    cc.film = 0.5f * (1.0f - cc.cos_t);
    cc.spread = cc.film * (0.85f + 0.15f * cc.sin_t);
    return cc;
}

// Value of one non-solid cell after all rules, given the final value of the
// cell below (prev, valid only if has_prev) -- kernels.py:957-990.
__device__ __forceinline__ float contact_rules(const ContactConst& cc, float start, int flag,
                                               bool below_solid, bool any_nb, bool has_prev,
                                               float prev) {
    float v = start;
    if (below_solid && flag == GAS) {
        if (v < cc.film) v = cc.film;
    }
    if (has_prev && prev > 0.55f && flag == GAS) {
        float t = prev - cc.sin_t;
        t = fmax_(cc.film, fmin_(t, 0.95f));
        if (v < t) v = t;
    }
    if (v < 0.45f && any_nb) {
        if (v < cc.spread) v = cc.spread;
    }
    if (below_solid && v > 0.2f) {
        if (v < 0.65f) v = 0.65f;
    }
    return v;
}

// Runs the column pass for one warp; `emit(k, c, value, flag_old)` is called
// for every cell of the column (value = final phi, or snap for solid cells).
template <class Emit>
__device__ __forceinline__ void contact_column(const Dims d, const float* __restrict__ snap,
                                               const int32_t* __restrict__ flags, int i, int j,
                                               bool wetting, const ContactConst& cc, Emit emit) {
    const int lane = threadIdx.x & 31;
    int carry_flag = SOLID;      // old flag of the cell below the chunk
    float carry_final = 0.0f;    // final phi of the cell below the chunk
    float carry_ghost = -1.0f;   // ghost value written into the chunk's first cell (<0: none)
    for (int k0 = 0; k0 < d.nz; k0 += 32) {
        int k = k0 + lane;
        bool valid = k < d.nz;
        int64_t c = d.idx(i, j, valid ? k : d.nz - 1);
        float s = valid ? snap[c] : 0.0f;
        int flag = valid ? flags[c] : SOLID;
        if (!wetting) {
            if (valid) emit(k, c, s, flag);
            continue;
        }
        int flag_up = (valid && k + 1 < d.nz) ? flags[c + 1] : SOLID;
        int flag_dn = __shfl_up_sync(0xffffffffu, flag, 1);
        if (lane == 0) flag_dn = carry_flag;
        bool below_solid = k > 0 && flag_dn == SOLID;
        // neighbour columns, pre-kernel values
        bool any_nb = false;
        if (valid && flag != SOLID) {
            if (j - 1 >= 0 && snap[c - d.nz] > 0.55f) any_nb = true;
            if (j + 1 < d.ny && snap[c + d.nz] > 0.55f) any_nb = true;
            int64_t sx = (int64_t)d.ny * d.nz;
            if (i - 1 >= 0 && snap[c - sx] > 0.55f) any_nb = true;
            if (i + 1 < d.nx && snap[c + sx] > 0.55f) any_nb = true;
        }
        // ghost value this cell writes into k+1 ("fluid on substrate")
        float ghost_out = -1.0f;
        if (valid && flag != SOLID && below_solid) {
            float r1 = s;
            if (flag == GAS && r1 < cc.film) r1 = cc.film;
            if (r1 > 0.55f && k + 1 < d.nz && flag_up == GAS) {
                float g = r1 - cc.sin_t;
                ghost_out = fmax_(cc.film, fmin_(g, 0.98f));
            }
        }
        float ghost_in = __shfl_up_sync(0xffffffffu, ghost_out, 1);
        if (lane == 0) ghost_in = carry_ghost;
        float start = s;
        if (ghost_in >= 0.0f && start < ghost_in) start = ghost_in;
        bool active = valid && flag != SOLID;
        // fixed point over the chunk
        float cur = active ? contact_rules(cc, start, flag, below_solid, any_nb, false, 0.0f) : s;
        for (int it = 0; it < 34; ++it) {
            float prev = __shfl_up_sync(0xffffffffu, cur, 1);
            bool has_prev = k > 0;
            if (lane == 0) prev = carry_final;
            float nv = active ? contact_rules(cc, start, flag, below_solid, any_nb, has_prev, prev)
                              : (valid ? start : s);
            bool changed = nv != cur;
            cur = nv;
            if (!__any_sync(0xffffffffu, changed)) break;
        }
        if (valid) emit(k, c, cur, flag);
        carry_flag = __shfl_sync(0xffffffffu, flag, 31);
        carry_final = __shfl_sync(0xffffffffu, cur, 31);
        carry_ghost = __shfl_sync(0xffffffffu, ghost_out, 31);
    }
}

__global__ void k_contact_op(Dims d, const float* __restrict__ snap, float* __restrict__ phi,
                             const int32_t* __restrict__ flags, float cos_t, float sin_t) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= d.nx * d.ny) return;
    int i = warp / d.ny, j = warp % d.ny;
    ContactConst cc = contact_const(cos_t, sin_t);
    contact_column(d, snap, flags, i, j, true, cc, [&](int k, int64_t c, float v, int flag) {
        if (flag != SOLID) phi[c] = v;
    });
}

int launch_contact_columns(Dims d, const float* snap, float* phi, const int32_t* flags,
                           float theta, void* stream) {
    int64_t threads = (int64_t)d.nx * d.ny * 32;
    int blocks = (int)((threads + kThreads - 1) / kThreads);
    k_contact_op<<<blocks, kThreads, 0, STREAM(stream)>>>(d, snap, phi, flags,
                                                         (float)cos((double)theta),
                                                         (float)sin((double)theta));
    return check_launch("k_contact_op");
}

// ---------------------------------------------------------------------------
// Pull streaming (kernels.py:2971-3010): x periodic, y/z clamped, bounce-back
// from SOLID sources for non-gas cells.  One thread per cell, k fastest.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_stream(Dims d, const float* __restrict__ f_src,
                                                     float* __restrict__ f_dst,
                                                     const int32_t* __restrict__ flags) {
    const int64_t n = d.n();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int flag = flags[c];
    if (flag == SOLID) return;
    int i, j, k;
    d.ijk(c, i, j, k);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        int ni = i - ex(q);
        ni = ni < 0 ? ni + d.nx : (ni >= d.nx ? ni - d.nx : ni);
        int nj = imax(0, imin(j - ey(q), d.ny - 1));
        int nk = imax(0, imin(k - ez(q), d.nz - 1));
        int64_t s = d.idx(ni, nj, nk);
        float v;
        if (flag == GAS || flags[s] != SOLID)
            v = f_src[q * n + s];
        else
            v = f_src[opp(q) * n + c];
        f_dst[q * n + c] = v;
    }
}

int launch_stream(Dims d, const float* f_src, float* f_dst, const int32_t* flags, void* stream) {
    int64_t n = d.n();
    int blocks = (int)((n + kThreads - 1) / kThreads);
    k_stream<<<blocks, kThreads, 0, STREAM(stream)>>>(d, f_src, f_dst, flags);
    return check_launch("k_stream");
}

// ---------------------------------------------------------------------------
// Droplet deposition (kernels.py:278-400).  The reference's reserve-then-
// commit budget is order dependent; this kernel fixes the order to the serial
// lexicographic (i, j, k) one with a single thread.  The search box is at
// most (2*16+1)^2 x ~20 cells and the kernel runs once per droplet.
// ---------------------------------------------------------------------------
__device__ bool has_metal_nb(const Dims d, const float* phi, const int32_t* flags,
                             const float* f_l, int i, int j, int k) {
    const int dd[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    bool found = false;
    for (int m = 0; m < 6; ++m) {
        int ii = i + dd[m][0], jj = j + dd[m][1], kk = k + dd[m][2];
        if (ii >= 0 && jj >= 0 && kk >= 0 && ii < d.nx && jj < d.ny && kk < d.nz) {
            int64_t c = d.idx(ii, jj, kk);
            if (flags[c] == FLUID || flags[c] == SOLID)
                found = true;
            else if (phi[c] > 0.35f || f_l[c] > 0.2f)
                found = true;
        }
    }
    return found;
}

__global__ void k_deposit(Dims d, float* f_src, int32_t* flags, float* f_l, float* phi, float* H,
                          float* T, float* rho, float arc_i, float arc_j, float arc_k, float foot_r,
                          float drop_r, float target_vol, float T_drop, float cp_rho, float L_rho,
                          float rho0, float* vol_acc, float* real_acc, float cell_vol) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int64_t n = d.n();
    float sr = fmax_(foot_r, drop_r);
    int i0 = imax(0, (int)(arc_i - sr)), i1 = imin(d.nx, (int)(arc_i + sr) + 1);
    int j0 = imax(0, (int)(arc_j - sr)), j1 = imin(d.ny, (int)(arc_j + sr) + 1);
    int k0 = imax(0, (int)(arc_k - 1.0f));
    float k_span = fmax_(drop_r + 3.0f, 4.0f);
    int k1 = imin(d.nz, (int)(arc_k + k_span) + 1);
    float drop_cz = arc_k + drop_r + 0.5f;
    float rd2 = drop_r * drop_r, foot2 = sr * sr;
    float vol = *vol_acc, real = *real_acc;
    const float hdrop = cp_rho * T_drop + L_rho;
    for (int pass = 0; pass < 2; ++pass)
        for (int i = i0; i < i1; ++i)
            for (int j = j0; j < j1; ++j)
                for (int k = k0; k < k1; ++k) {
                    if (vol >= target_vol) continue;
                    int64_t c = d.idx(i, j, k);
                    if (flags[c] != GAS) continue;
                    if (!has_metal_nb(d, phi, flags, f_l, i, j, k)) continue;
                    float di = (float)i - arc_i, dj = (float)j - arc_j;
                    float rij2 = di * di + dj * dj;
                    if (pass == 0) {
                        float dk = (float)k - drop_cz;
                        float r2 = di * di + dj * dj + dk * dk;
                        if (rij2 > foot2 && r2 > rd2) continue;
                    } else if (rij2 > foot2 * 1.44f) {
                        continue;
                    }
                    float reserved = vol;
                    vol = reserved + cell_vol;
                    if (reserved >= target_vol) {
                        vol = vol - cell_vol;
                    } else {
                        flags[c] = FLUID;
                        f_l[c] = 1.0f;
                        phi[c] = 1.0f;
                        T[c] = T_drop;
                        H[c] = hdrop;
                        rho[c] = rho0;
                        for (int q = 0; q < 19; ++q) f_src[q * n + c] = wq(q) * rho0;
                        real = real + cell_vol;
                    }
                }
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                int64_t c = d.idx(i, j, k);
                if (flags[c] != FLUID || f_l[c] < 0.45f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                if (di * di + dj * dj > foot2 * 1.44f) continue;
                T[c] = T_drop;
                H[c] = hdrop;
                rho[c] = rho0;
                for (int q = 0; q < 19; ++q) f_src[q * n + c] = wq(q) * rho0;
            }
    *vol_acc = vol;
    *real_acc = real;
}

int launch_deposit(Dims d, float* f_src, int32_t* flags, float* f_l, float* phi, float* H, float* T,
                   float* rho, float arc_i, float arc_j, float arc_k, float foot_r, float drop_r,
                   float target_vol, float T_drop, float cp_rho, float L_rho, float rho0,
                   float* vol_acc, float* real_acc, float cell_vol, void* stream) {
    k_deposit<<<1, 32, 0, STREAM(stream)>>>(d, f_src, flags, f_l, phi, H, T, rho, arc_i, arc_j,
                                            arc_k, foot_r, drop_r, target_vol, T_drop, cp_rho,
                                            L_rho, rho0, vol_acc, real_acc, cell_vol);
    return check_launch("k_deposit");
}

// ---------------------------------------------------------------------------
// Fused step kernels
// ---------------------------------------------------------------------------

// Surface height at the torch column + the arc-k fallback of
// solvers/coupled_step.py:34-59 -> scalars[0].
__global__ void k_surface_arc(Dims d, const float* phi, const int32_t* flags, float* scalars,
                              int nz_solid) {
    float arc_i = scalars[kScalarArcI], arc_j = scalars[kScalarArcJ];
    int i0 = imax(0, imin((int)arc_i, d.nx - 1));
    int j0 = imax(0, imin((int)arc_j, d.ny - 1));
    int best = -1;
    for (int k = threadIdx.x; k < d.nz; k += 32) {
        int64_t c = d.idx(i0, j0, k);
        if (flags[c] != GAS && phi[c] > 0.05f) best = k;
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    if (threadIdx.x == 0) {
        int ks = best >= 0 ? best : imax(1, nz_solid - 1);
        float kf = (float)ks;
        if (kf < 1.0f) kf = (float)imax(1, nz_solid - 1);
        scalars[0] = kf;
    }
}

struct ThermalArgs {
    PhaseParams ph;
    float cpa, dt_lu, inv_dt;
    int heat_loss, conv, rad;
    float T_amb, h_conv, eps_rad, dt_phys, dx, sigma_sb, h_floor;
};

// Thermal stage for every cell: kernels.py:1611-1682 (advect/diffuse),
// 2030-2082 + 1937-1950 (losses, floor), 1519-1556 twice around the ceiling
// 1953-1984 (only the second update_phase is observable), 3016-3032 (T_max),
// 2013-2027 (cooling rate).  H and T are double-buffered so neighbour reads
// see the pre-stage values.
__global__ void __launch_bounds__(kThreads) k_thermal_fused(
    Dims d, const float* __restrict__ H, float* __restrict__ H_next, const float* __restrict__ T,
    float* __restrict__ T_next, float* __restrict__ f_l, const float* __restrict__ ux,
    const float* __restrict__ uy, const float* __restrict__ uz, const int32_t* __restrict__ flags,
    float* __restrict__ T_max, float* __restrict__ T_prev, float* __restrict__ dT_dt,
    ThermalArgs a) {
    const int64_t n = d.n();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int flag = flags[c];
    float h = H[c];
    if (flag != GAS) {
        int i, j, k;
        d.ijk(c, i, j, k);
        float u = 0.0f, v = 0.0f, w = 0.0f;
        if (flag != SOLID) {
            u = ux[c];
            v = uy[c];
            w = uz[c];
        }
        h = h + thermal_dh(d, H, T, flags, u, v, w, i, j, k, flag, h, a.cpa, a.dt_lu);
        if (a.heat_loss) {
            int ne = 0;
            if (k + 1 < d.nz && flags[c + 1] == GAS) ne++;
            if (j + 1 < d.ny && flags[c + d.nz] == GAS) ne++;
            if (j - 1 >= 0 && flags[c - d.nz] == GAS) ne++;
            int64_t sx = (int64_t)d.ny * d.nz;
            if (i + 1 < d.nx && flags[c + sx] == GAS) ne++;
            if (i - 1 >= 0 && flags[c - sx] == GAS) ne++;
            if (ne != 0) {
                float Te = fmin_(T[c], 2500.0f);
                float q = 0.0f;
                if (a.conv == 1) q += a.h_conv * (Te - a.T_amb);
                if (a.rad == 1) {
                    float t4 = Te * Te * Te * Te;
                    float a4 = a.T_amb * a.T_amb * a.T_amb * a.T_amb;
                    q += a.eps_rad * a.sigma_sb * (t4 - a4);
                }
                h -= q * (float)ne * a.dt_phys / a.dx;
            }
            if (h < a.h_floor) h = a.h_floor;
        }
        if (a.ph.cap_enabled) h = cap_h(a.ph, h);
    }
    float t, fl;
    phase(a.ph, h, t, fl);
    H_next[c] = h;
    T_next[c] = t;
    f_l[c] = fl;
    if (flag != GAS) {
        if (t > T_max[c]) T_max[c] = t;
        float tp = T_prev[c];
        dT_dt[c] = (t - tp) * a.inv_dt;
        T_prev[c] = t;
    }
}

// VOF advection + reinitialisation (kernels.py:2320-2391) -> phi_tmp.
__global__ void __launch_bounds__(kThreads) k_vof_advect(Dims d, const float* __restrict__ phi,
                                                         float* __restrict__ phi_tmp,
                                                         const float* __restrict__ ux,
                                                         const float* __restrict__ uy,
                                                         const float* __restrict__ uz,
                                                         const int32_t* __restrict__ flags) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.n()) return;
    int i, j, k;
    d.ijk(c, i, j, k);
    int flag = flags[c];
    float p = advect_phi_cell(d, phi, ux, uy, uz, flags, i, j, k, flag);
    phi_tmp[c] = reinit_phi(p, flag);
}

struct ColumnArgs {
    int vof, wetting, nz_solid;
    float cos_t, sin_t;
    float dt_phys, T800, T1100, Ts;
};

// Column pass: contact-angle BC (kernels.py:933-991) on phi_tmp, flags from
// phi (2394-2419), phi/f_l sync (3484-3504) and time-above-T (3261-3283,
// which runs after collide/stream in the reference but only reads T and the
// post-VOF flags).
__global__ void __launch_bounds__(kThreads) k_column(Dims d, const float* __restrict__ phi_tmp,
                                                     float* __restrict__ phi,
                                                     int32_t* __restrict__ flags,
                                                     float* __restrict__ f_l,
                                                     const float* __restrict__ T,
                                                     float* __restrict__ t800,
                                                     float* __restrict__ t1100,
                                                     float* __restrict__ tsol, ColumnArgs a) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= d.nx * d.ny) return;
    int i = warp / d.ny, j = warp % d.ny;
    ContactConst cc = contact_const(a.cos_t, a.sin_t);
    const float* src = a.vof ? phi_tmp : phi;
    contact_column(d, src, flags, i, j, a.vof && a.wetting, cc,
                   [&](int k, int64_t c, float v, int flag_old) {
                       int flag = flag_old;
                       if (a.vof) {
                           float fl = f_l[c];
                           flag = flag_from(v, fl, k, a.nz_solid);
                           phi[c] = v;
                           flags[c] = flag;
                           if (flag == GAS || v < 0.05f || flag == SOLID) {
                               if (fl != 0.0f) f_l[c] = 0.0f;
                           }
                       }
                       if (flag != GAS) {
                           float t = T[c];
                           if (t >= a.T800) t800[c] += a.dt_phys;
                           if (t >= a.T1100) t1100[c] += a.dt_phys;
                           if (t >= a.Ts) tsol[c] += a.dt_phys;
                       }
                   });
}

struct CollideArgs {
    ForceParams P;
    int kind, from_buffer;
    float omega, omega_b, C_darcy, u_cap;
};

// Body forces + collision + Mach clamp for FLUID/IFACE cells
// (solvers/coupled_step.py:298-402); forces stay in registers and are
// written once as the step's force field (== the reference's F_snap).
__global__ void __launch_bounds__(kThreads) k_collide_fused(
    Dims d, const float* __restrict__ f_src, float* __restrict__ f_dst, float* __restrict__ rho,
    float* __restrict__ ux, float* __restrict__ uy, float* __restrict__ uz,
    float* __restrict__ Fx, float* __restrict__ Fy, float* __restrict__ Fz,
    const float* __restrict__ phi, const float* __restrict__ T, const float* __restrict__ f_l,
    const int32_t* __restrict__ flags, const float* __restrict__ scalars, CollideArgs a) {
    const int64_t n = d.n();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int flag = flags[c];
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (a.from_buffer) {
        fx = Fx[c];
        fy = Fy[c];
        fz = Fz[c];
    }
    if (flag == SOLID || flag == GAS) {
        if (!a.from_buffer) {
            Fx[c] = 0.0f;
            Fy[c] = 0.0f;
            Fz[c] = 0.0f;
        }
        return;
    }
    int i, j, k;
    d.ijk(c, i, j, k);
    ForceParams P = a.P;
    P.arc_k = scalars[kScalarArcK];
    P.arc_i = scalars[kScalarArcI];
    P.arc_j = scalars[kScalarArcJ];
    float fl = f_l[c];
    cell_forces(d, P, phi, T, flags, i, j, k, fl, fx, fy, fz);
    float f[19], o[19];
#pragma unroll
    for (int q = 0; q < 19; ++q) f[q] = f_src[q * n + c];
    float r, u, v, w;
    if (a.kind == 0)
        collide_mrt_cell(f, fl, fx, fy, fz, a.omega, a.omega_b, a.C_darcy, o, r, u, v, w);
    else
        collide_srt_cell(f, fl, fx, fy, fz, a.omega, a.C_darcy, o, r, u, v, w);
#pragma unroll
    for (int q = 0; q < 19; ++q) f_dst[q * n + c] = o[q];
    if (a.u_cap > 0.0f) clamp_mach(u, v, w, a.u_cap);
    rho[c] = r;
    ux[c] = u;
    uy[c] = v;
    uz[c] = w;
    Fx[c] = fx;
    Fy[c] = fy;
    Fz[c] = fz;
}

struct TailArgs {
    float cp_rho, Ts, Tl, L_rho;
    int remelt, trailing, cooled;
    float arc_i, arc_j, dir_x, dir_y, dir_z, lookback, T_freeze;
};

// solvers/coupled_step.py:426-458: remelt_hot_solid_scalar (kernels.py:2489),
// solidify_trailing_pool_scalar (2573), solidify_cooled_metal (2422); all
// per cell, applied in the reference order.
__global__ void k_tail(Dims d, float* T, float* H, float* f_l, float* phi, int32_t* flags,
                       float* ux, float* uy, float* uz, const float* scalars, TailArgs a) {
    const int64_t n = d.n();
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    int flag = flags[c];
    if (a.remelt && flag == SOLID) {
        float Tc = T[c];
        if (!(Tc <= a.Ts + 5.0f)) {
            float H_sol = a.cp_rho * a.Ts;
            float fl;
            if (Tc >= a.Tl) {
                fl = 1.0f;
                H[c] = a.cp_rho * a.Tl + a.L_rho + a.cp_rho * (Tc - a.Tl);
            } else {
                fl = (Tc - a.Ts) / (a.Tl - a.Ts + 1e-6f);
                H[c] = H_sol + fl * a.L_rho;
            }
            f_l[c] = fl;
            phi[c] = 1.0f;
            flags[c] = FLUID;
            flag = FLUID;
        }
    }
    if (a.trailing && flag != GAS && !(phi[c] < 0.85f || f_l[c] < 0.05f)) {
        int i, j, k;
        d.ijk(c, i, j, k);
        float arc_k = scalars[kScalarArcK];
        float di = (float)i - scalars[kScalarArcI], dj = (float)j - scalars[kScalarArcJ];
        float dk = (float)k - arc_k;
        float proj = di * a.dir_x + dj * a.dir_y + dk * a.dir_z;
        if (!(proj > -a.lookback) && !(T[c] >= a.T_freeze)) {
            H[c] = a.cp_rho * (a.Ts - 1.0f);
            T[c] = a.Ts - 1.0f;
            f_l[c] = 0.0f;
            phi[c] = 1.0f;
            flags[c] = SOLID;
            ux[c] = uy[c] = uz[c] = 0.0f;
            flag = SOLID;
        }
    }
    if (a.cooled && flag != GAS && !(phi[c] < 0.85f)) {
        if (f_l[c] < 0.02f && T[c] < a.Ts) {
            flags[c] = SOLID;
            phi[c] = 1.0f;
            f_l[c] = 0.0f;
            ux[c] = uy[c] = uz[c] = 0.0f;
        }
    }
}

static ArcParams arc_params(const WaamStepParams* p) {
    ArcParams a{};
    a.kind = p->arc_kind;
    a.arc_i = p->arc_i;
    a.arc_j = p->arc_j;
    a.arc_k = 0.0f;  // taken from the device scalar
    a.inv2s2 = 1.0f / (2.0f * p->sigma_heat * p->sigma_heat);
    a.sign = p->sign;
    a.ff = p->ff;
    a.fr = p->fr;
    a.a_f = p->a_f;
    a.a_r = p->a_r;
    a.b = p->gb;
    a.c = p->gc;
    a.pen = p->pen;
    a.enable = p->surface_weighting;
    return a;
}

static bool fields_ok(const WaamFields* f) {
    return f && f->f_src && f->f_dst && f->rho && f->ux && f->uy && f->uz && f->T && f->T_next &&
           f->H && f->H_next && f->f_l && f->phi && f->phi_tmp && f->flags && f->T_max &&
           f->T_prev && f->dT_dt && f->t800 && f->t1100 && f->tsol && f->Fx && f->Fy && f->Fz &&
           f->step_scalars && dims_ok(f->nx, f->ny, f->nz) && f->f_src != f->f_dst &&
           f->H != f->H_next && f->T != f->T_next;
}

}  // namespace waam

extern "C" {

int waam_step_launch_count(const WaamStepParams* p, int stage) {
    if (!p) return 0;
    if (stage == 0) return p->welding ? 3 : 1;
    int n = 1 /*thermal*/ + (p->vof ? 1 : 0) + 1 /*column*/ + 1 /*collide*/ + 1 /*stream*/;
    if (p->substrate_growth || p->bead_freeze) n += 1;
    return n;
}

int waam_step_pre(const WaamFields* f, const WaamStepParams* p, void* workspace,
                  size_t workspace_bytes, void* stream) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_pre: bad fields or params");
    Dims d{f->nx, f->ny, f->nz};
    if (!workspace_ok(workspace, workspace_bytes, d.n()))
        return fail(WAAM_ERR_INVALID, "step_pre: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    k_surface_arc<<<1, 32, 0, STREAM(stream)>>>(d, f->phi, f->flags, f->step_scalars,
                                                p->nz_solid);
    int e = check_launch("k_surface_arc");
    if (e || !p->welding) return e;
    ArcParams a = arc_params(p);
    float Qe_dt = p->Q_w * p->eta * p->dt;
    k_arc_norm<<<red_blocks(d.n()), kThreads, 0, STREAM(stream)>>>(
        d, f->flags, f->f_l, a, f->step_scalars, p->arc_k_offset, Qe_dt, p->dx3, nullptr,
        f->step_scalars, ws);
    e = check_launch("k_arc_norm");
    if (e) return e;
    PhaseParams ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    k_arc_inject<<<elem_blocks(d.n()), kThreads, 0, STREAM(stream)>>>(
        d, f->H, f->flags, f->f_l, a, f->step_scalars, p->arc_k_offset, f->step_scalars,
        p->cap_enabled, ph);
    return check_launch("k_arc_inject");
}

int waam_step_main(const WaamFields* f, const WaamStepParams* p, void* workspace,
                   size_t workspace_bytes, void* stream) {
    return waam_step_main_events(f, p, workspace, workspace_bytes, nullptr, 0, stream);
}

int waam_step_main_events(const WaamFields* f, const WaamStepParams* p, void* workspace,
                          size_t workspace_bytes, void* const* events, int n_events,
                          void* stream) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_main: bad fields or params");
    if (events && n_events < kMainEvents)
        return fail(WAAM_ERR_INVALID, "step_main: need 7 events");
    auto mark = [&](int i) {
        if (events) cudaEventRecord(reinterpret_cast<cudaEvent_t>(events[i]), STREAM(stream));
    };
    Dims d{f->nx, f->ny, f->nz};
    if (!workspace_ok(workspace, workspace_bytes, d.n()))
        return fail(WAAM_ERR_INVALID, "step_main: workspace too small or misaligned");
    const int64_t n = d.n();
    const int cell_blocks = (int)((n + kThreads - 1) / kThreads);
    const int col_blocks = (int)(((int64_t)d.nx * d.ny * 32 + kThreads - 1) / kThreads);
    cudaStream_t s = STREAM(stream);

    ThermalArgs ta;
    ta.ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    ta.cpa = p->cp_rho * p->alpha_lu;
    ta.dt_lu = 1.0f;
    ta.inv_dt = 1.0f / (p->dt + 1e-12f);
    ta.heat_loss = p->heat_loss;
    ta.conv = p->conv;
    ta.rad = p->rad;
    ta.T_amb = p->T_amb;
    ta.h_conv = p->h_conv;
    ta.eps_rad = p->eps_rad;
    ta.dt_phys = p->dt;
    ta.dx = p->dx;
    ta.sigma_sb = p->sigma_sb;
    ta.h_floor = p->cp_rho * p->T_amb;
    mark(0);
    k_thermal_fused<<<cell_blocks, kThreads, 0, s>>>(d, f->H, f->H_next, f->T, f->T_next, f->f_l,
                                                     f->ux, f->uy, f->uz, f->flags, f->T_max,
                                                     f->T_prev, f->dT_dt, ta);
    int e = check_launch("k_thermal_fused");
    if (e) return e;
    mark(1);

    if (p->vof) {
        k_vof_advect<<<cell_blocks, kThreads, 0, s>>>(d, f->phi, f->phi_tmp, f->ux, f->uy, f->uz,
                                                      f->flags);
        e = check_launch("k_vof_advect");
        if (e) return e;
    }
    mark(2);
    ColumnArgs ca;
    ca.vof = p->vof;
    ca.wetting = p->wetting;
    ca.nz_solid = p->nz_solid;
    ca.cos_t = (float)cos((double)p->theta);
    ca.sin_t = (float)sin((double)p->theta);
    ca.dt_phys = p->dt;
    ca.T800 = p->T800;
    ca.T1100 = p->T1100;
    ca.Ts = p->Ts;
    k_column<<<col_blocks, kThreads, 0, s>>>(d, f->phi_tmp, f->phi, f->flags, f->f_l, f->T_next,
                                             f->t800, f->t1100, f->tsol, ca);
    e = check_launch("k_column");
    if (e) return e;
    mark(3);

    CollideArgs cl;
    ForceParams& P = cl.P;
    P.csf = p->csf;
    P.wetting = p->wetting;
    P.welding = p->welding;
    P.hydro = p->hydro;
    P.gamma_lu = p->gamma_lu;
    P.cos_t = (float)cos((double)p->theta);
    P.sin_t = (float)sin((double)p->theta);
    P.dgamma = p->dgamma_lu;
    P.arc_i = p->arc_i;
    P.arc_j = p->arc_j;
    P.arc_k = 0.0f;
    P.p_inv2s2 = 1.0f / (2.0f * p->p_sigma * p->p_sigma + 1e-6f);
    float Fphys = p->pressure / (p->rho_phys * p->dx);
    P.p_Flu = Fphys * (p->dt * p->dt) / p->dx;
    P.g_lu = p->g_lu;
    P.beta = p->beta;
    P.T_ref = p->T_ref;
    P.rho_ref = 1.0f;
    P.F_cap = p->F_cap;
    cl.kind = p->collision;
    cl.from_buffer = p->forces_from_buffer;
    cl.omega = p->omega;
    cl.omega_b = p->omega_b;
    cl.C_darcy = p->C_darcy;
    cl.u_cap = p->u_cap;
    k_collide_fused<<<cell_blocks, kThreads, 0, s>>>(d, f->f_src, f->f_dst, f->rho, f->ux, f->uy,
                                                     f->uz, f->Fx, f->Fy, f->Fz, f->phi, f->T_next,
                                                     f->f_l, f->flags, f->step_scalars, cl);
    e = check_launch("k_collide_fused");
    if (e) return e;
    mark(4);

    e = launch_stream(d, f->f_dst, f->f_src, f->flags, stream);
    if (e) return e;
    mark(5);

    if (p->substrate_growth || p->bead_freeze) {
        TailArgs t;
        t.cp_rho = p->cp_rho;
        t.Ts = p->Ts;
        t.Tl = p->Tl;
        t.L_rho = p->L_rho;
        t.remelt = 1;
        t.trailing = p->welding && p->bead_freeze;
        t.cooled = 1;
        t.arc_i = p->arc_i;
        t.arc_j = p->arc_j;
        t.dir_x = p->dir_x;
        t.dir_y = p->dir_y;
        t.dir_z = p->dir_z;
        t.lookback = p->lookback;
        t.T_freeze = p->T_freeze;
        k_tail<<<cell_blocks, kThreads, 0, s>>>(d, f->T_next, f->H_next, f->f_l, f->phi, f->flags,
                                                f->ux, f->uy, f->uz, f->step_scalars, t);
        e = check_launch("k_tail");
    }
    mark(6);
    return e;
}

}  // extern "C"
