// Reverse kernels of the coupled step (the adjoint, backward in time).
//
// The forward step n maps (H, T, f_l, u, X = f_src, Y = f_dst) to step n + 1
// (solvers/coupled_step.py:73-464; the fused pipeline of waam_fused.cu):
//   inject + ceiling:  H' = cap(H_n + S(theta))                    (non-gas)
//   thermal:           H_{n+1} = cap(floor(H' + A(H'; u_n) + D(T_n) - Q(T_n)))
//                      T_{n+1}, f_l_{n+1} = phase(H_{n+1})
//   VOF, flags:        frozen (the recorded trajectory)
//   forces + collide:  Y'[c] = C(X_n[c], f_l_{n+1}[c], F(T_{n+1}, f_l_{n+1}))
//                      and u_{n+1}[c] (Mach clamp) at the active cells
//   stream + swap:     X_{n+1} = Y', Y_{n+1} = X' with X' = stream(Y')
// The reverse step takes the adjoints of step n + 1's state to step n's in
// the opposite order.  Every kernel gathers (a thread owns its output cells
// and collects the contributions that reach them), so no floating-point
// atomics are used and the backward pass is deterministic; the parameter
// sums are FP64 with a fixed block count and a fixed combination order.
#include "../../include/waam_b200.h"
#include "waam_adjoint_cell.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

constexpr int kAdjBlocks = 592;   // fixed, so the FP64 sums never depend on the GPU
constexpr int kAdjThreads = 256;

// Adds this launch's NR sums to out[NR]: per-block totals in fixed order,
// the last block combines the partials in block order.
template <int NR>
__device__ void accumulate_sums(double (&v)[NR], Workspace ws, double* out) {
    __shared__ double sh[NR][kAdjThreads / 32];
    __shared__ bool last;
#pragma unroll
    for (int r = 0; r < NR; ++r)
        for (int o = 16; o > 0; o >>= 1) v[r] += __shfl_down_sync(0xffffffffu, v[r], o);
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int r = 0; r < NR; ++r) sh[r][warp] = v[r];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int r = 0; r < NR; ++r) {
            double t = 0.0;
            for (int w = 0; w < kAdjThreads / 32; ++w) t += sh[r][w];
            ws.partials[(int64_t)r * gridDim.x + blockIdx.x] = t;
        }
        __threadfence();
        last = atomicAdd(ws.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    if (threadIdx.x < NR) {
        const volatile double* part = ws.partials;
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += part[(int64_t)threadIdx.x * gridDim.x + b];
        out[threadIdx.x] += t;
    }
    __syncthreads();
    if (threadIdx.x == 0) *ws.counter = 0u;
}

__device__ __forceinline__ void cell_ijk(const Dims& d, int64_t c, int& i, int& j, int& k) {
    k = (int)(c % d.nz);
    const int64_t r = c / d.nz;
    j = (int)(r % d.ny);
    i = (int)(r / d.ny);
}

// ---------------------------------------------------------------------------
// Stream (kernels.py:2971-3010) transposed.  The pull writes X'[q][c] for
// every non-solid c from Y'[q][src(c, q)], or, for a non-gas c whose source
// is SOLID, from Y'[opp(q)][c].  For a source cell s the destinations that
// pulled population q from it are c = (wrap(i_s + e_x), j, k) with
// clamp(j - e_y) = j_s, clamp(k - e_z) = k_s: one cell, plus the cell itself
// on a clamped y / z face.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_adj_stream(Dims d, float* __restrict__ lam_yp,
                                                    const float* __restrict__ lam_xp,
                                                    float* __restrict__ lam_xn,
                                                    const int32_t* __restrict__ flags) {
    int i, j, k, s;
    if (!tile_cell(d, i, j, k, s)) return;
    const int64_t n = d.n();
    const int fs = flags[s];
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float acc = lam_yp[q * n + s];
        int ic = i + ex(q);
        ic = ic < 0 ? ic + d.nx : (ic >= d.nx ? ic - d.nx : ic);
        int jc[2], kc[2], nj = 0, nk = 0;
        const int j1 = j + ey(q), k1 = k + ez(q);
        if (j1 >= 0 && j1 < d.ny) jc[nj++] = j1;
        if ((ey(q) == 1 && j == 0) || (ey(q) == -1 && j == d.ny - 1)) jc[nj++] = j;
        if (k1 >= 0 && k1 < d.nz) kc[nk++] = k1;
        if ((ez(q) == 1 && k == 0) || (ez(q) == -1 && k == d.nz - 1)) kc[nk++] = k;
        for (int a = 0; a < nj; ++a)
            for (int b = 0; b < nk; ++b) {
                const int c = d.idx(ic, jc[a], kc[b]);
                const int fc = flags[c];
                if (fc == SOLID) continue;                      // not written by the stream
                if (q != 0 && fc != GAS && fs == SOLID) continue;   // bounced back instead
                acc += lam_xp[q * n + c];
            }
        // bounce-back: s (non-gas) took population opp(q) from its own Y'[q]
        if (q != 0 && fs != GAS && fs != SOLID) {
            const int qo = opp(q);
            int ni = i - ex(qo);
            ni = ni < 0 ? ni + d.nx : (ni >= d.nx ? ni - d.nx : ni);
            const int nj2 = imax(0, imin(j - ey(qo), d.ny - 1));
            const int nk2 = imax(0, imin(k - ez(qo), d.nz - 1));
            if (flags[d.idx(ni, nj2, nk2)] == SOLID) acc += lam_xp[qo * n + s];
        }
        lam_yp[q * n + s] = acc;
        lam_xn[q * n + s] = fs == SOLID ? lam_xp[q * n + s] : 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Forces + collision at the taped active cells (k_collide_list): the VJP of
// the MRT collision and the Mach clamp, then of the force clamp, hydrostatic
// and buoyancy terms (own cell) and of Marangoni (six T neighbours, kept per
// slot for the gather).  Overwritten state (Y'[c], u[c]) gets a zero adjoint.
// ---------------------------------------------------------------------------
struct AdjCollideArgs {
    ForceParams P;
    float omega, omega_b, C_darcy, u_cap;
};

__global__ void __launch_bounds__(128) k_adj_collide(
    Dims d, const float* __restrict__ tape_f, const int32_t* __restrict__ tape_cells,
    const int32_t* __restrict__ tape_count, int64_t tape_cap, const float* __restrict__ phi,
    const float* __restrict__ T, const float* __restrict__ f_l, const int32_t* __restrict__ flags,
    const float* __restrict__ scalars, float* __restrict__ lam_yp, float* __restrict__ lam_xn,
    float* __restrict__ lam_ux, float* __restrict__ lam_uy, float* __restrict__ lam_uz,
    float* __restrict__ lam_fl, float* __restrict__ lam_T, float* __restrict__ ctb,
    int32_t* __restrict__ map, AdjCollideArgs a) {
    const int cnt = *tape_count;
    const int64_t n = d.n();
    ForceParams P = a.P;
    P.arc_k = scalars[kScalarArcK];
    P.arc_i = scalars[kScalarArcI];
    P.arc_j = scalars[kScalarArcJ];
    ForceParams P0 = P;
    P0.F_cap = 0.0f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int c = tape_cells[t];
        int i, j, k;
        cell_ijk(d, c, i, j, k);
        float f[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = tape_f[(int64_t)q * tape_cap + t];
        const float fl = f_l[c];
        // pre-clamp force and the clamped force the collision saw
        float px = 0.0f, py = 0.0f, pz = 0.0f;
        cell_forces(d, P0, phi, T, flags, i, j, k, fl, px, py, pz);
        float fx = px, fy = py, fz = pz;
        if (P.F_cap > 0.0f) {
            const float mag = sqrtf(px * px + py * py + pz * pz);
            if (mag > P.F_cap) {
                const float s = P.F_cap / (mag + 1e-12f);
                fx = px * s;
                fy = py * s;
                fz = pz * s;
            }
        }
        float ob[19], fb[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            ob[q] = lam_yp[q * n + c];
            fb[q] = 0.0f;
        }
        float flb = 0.0f, fxb = 0.0f, fyb = 0.0f, fzb = 0.0f;
        waam_adj::mrt_vjp<float>(f, fl, fx, fy, fz, a.omega, a.omega_b, a.C_darcy, a.u_cap, ob,
                                 lam_ux[c], lam_uy[c], lam_uz[c], fb, flb, fxb, fyb, fzb);
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            lam_xn[q * n + c] = fb[q];
            lam_yp[q * n + c] = 0.0f;
        }
        lam_ux[c] = 0.0f;
        lam_uy[c] = 0.0f;
        lam_uz[c] = 0.0f;
        waam_adj::clamp_vjp<float>(px, py, pz, P.F_cap, fxb, fyb, fzb);
        // kernels.py:2756-2772 hydrostatic, 2729-2753 buoyancy (own cell)
        float Tb = 0.0f;
        if (P.hydro && fl > 0.0f) flb += -P.rho_ref * P.g_lu * fzb;
        if (fl > 0.0f) {
            const float gb = P.rho_ref * P.g_lu * P.beta;
            Tb += gb * fl * fzb;
            flb += gb * (T[c] - P.T_ref) * fzb;
        }
        // kernels.py:2158-2217 Marangoni (linear in the T differences)
        float cb[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (!(fl < 0.05f)) {
            const int ip = imin(i + 1, d.nx - 1), im = imax(i - 1, 0);
            const int jp = imin(j + 1, d.ny - 1), jm = imax(j - 1, 0);
            const int kp = imin(k + 1, d.nz - 1), km = imax(k - 1, 0);
            const float dx_ = 0.5f * (phi[d.idx(ip, j, k)] - phi[d.idx(im, j, k)]);
            const float dy_ = 0.5f * (phi[d.idx(i, jp, k)] - phi[d.idx(i, jm, k)]);
            const float dz_ = 0.5f * (phi[d.idx(i, j, kp)] - phi[d.idx(i, j, km)]);
            const float g = sqrtf(dx_ * dx_ + dy_ * dy_ + dz_ * dz_);
            if (!(g < 1e-6f)) {
                float txb, tyb, tzb;
                waam_adj::marangoni_t_vjp<float>(dx_ / g, dy_ / g, dz_ / g, P.dgamma * g, fxb,
                                                 fyb, fzb, txb, tyb, tzb);
                cb[0] = 0.5f * txb;
                cb[1] = -0.5f * txb;
                cb[2] = 0.5f * tyb;
                cb[3] = -0.5f * tyb;
                cb[4] = 0.5f * tzb;
                cb[5] = -0.5f * tzb;
            }
        }
#pragma unroll
        for (int s = 0; s < 6; ++s) ctb[(int64_t)t * 6 + s] = cb[s];
        lam_T[c] += Tb;
        lam_fl[c] += flb;
        map[c] = t;
    }
}

// Marangoni T contributions gathered at each cell: candidates are the cell and
// its six neighbours (whose central differences may reach it).
__global__ void __launch_bounds__(256) k_adj_forces_gather(Dims d, float* __restrict__ lam_T,
                                                           const float* __restrict__ ctb,
                                                           const int32_t* __restrict__ map) {
    int i, j, k, s;
    if (!tile_cell(d, i, j, k, s)) return;
    float acc = 0.0f;
    const int di[7] = {0, 1, -1, 0, 0, 0, 0}, dj[7] = {0, 0, 0, 1, -1, 0, 0};
    const int dk[7] = {0, 0, 0, 0, 0, 1, -1};
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        const int ic = i + di[m], jc = j + dj[m], kc = k + dk[m];
        if (ic < 0 || ic >= d.nx || jc < 0 || jc >= d.ny || kc < 0 || kc >= d.nz) continue;
        const int t = map[d.idx(ic, jc, kc)];
        if (t < 0) continue;
        const int src[6] = {d.idx(imin(ic + 1, d.nx - 1), jc, kc), d.idx(imax(ic - 1, 0), jc, kc),
                            d.idx(ic, imin(jc + 1, d.ny - 1), kc), d.idx(ic, imax(jc - 1, 0), kc),
                            d.idx(ic, jc, imin(kc + 1, d.nz - 1)), d.idx(ic, jc, imax(kc - 1, 0))};
#pragma unroll
        for (int sl = 0; sl < 6; ++sl)
            if (src[sl] == s) acc += ctb[(int64_t)t * 6 + sl];
    }
    if (acc != 0.0f) lam_T[s] += acc;
}

__global__ void k_adj_clear_map(const int32_t* __restrict__ tape_cells,
                                const int32_t* __restrict__ tape_count,
                                int32_t* __restrict__ map) {
    const int cnt = *tape_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
        map[tape_cells[t]] = -1;
}

// ---------------------------------------------------------------------------
// T_{n+1} and f_l_{n+1} are functions of H_{n+1} (kernels.py:1519-1556; f_l is
// zeroed by sync_phi_liquid_fraction, kernels.py:3484-3504, where frozen).
// ---------------------------------------------------------------------------
__global__ void k_adj_combine(float* __restrict__ lam_H, float* __restrict__ lam_T,
                              float* __restrict__ lam_fl, const float* __restrict__ H,
                              const int32_t* __restrict__ flags, const float* __restrict__ phi,
                              int64_t n, PhaseParams ph, int vof) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const float h = H[c];
        float gT, gF;
        if (h <= ph.H_sol || h >= ph.H_liq) {
            gT = 1.0f / ph.cp_rho;
            gF = 0.0f;
        } else {
            gT = (ph.Tl - ph.Ts) / ph.L_rho;
            gF = 1.0f / ph.L_rho;
        }
        const int fg = flags[c];
        if (vof && (fg == GAS || phi[c] < 0.05f || fg == SOLID)) gF = 0.0f;
        const float lt = lam_T[c], lf = lam_fl[c];
        if (lt != 0.0f || lf != 0.0f) lam_H[c] += gT * lt + gF * lf;
        lam_T[c] = 0.0f;
        lam_fl[c] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Thermal stage (k_thermal_fused) transposed.
// ---------------------------------------------------------------------------
struct AdjThermalArgs {
    PhaseParams ph;
    float cpa, dt_lu;
    int heat_loss, conv, rad, cap;
    float T_amb, h_conv, eps_rad, dt_phys, dx, sigma_sb, h_floor;
};

// Source cells and coefficients of one upwind-limited gradient of H' along
// one axis at cell c (kernels.py:1565-1608 with the masked reads of 1611-1682):
// g = sum coef[m] * H'[src[m]], m = 0..2.
__device__ __forceinline__ void grad_stencil(const Dims& d, const float* __restrict__ Hs,
                                             const int32_t* __restrict__ flags, int i, int j,
                                             int k, int axis, float u, int* src, float* coef) {
    auto clampc = [&](int o) {
        int ii = i, jj = j, kk = k;
        if (axis == 0) ii = imax(0, imin(i + o, d.nx - 1));
        if (axis == 1) jj = imax(0, imin(j + o, d.ny - 1));
        if (axis == 2) kk = imax(0, imin(k + o, d.nz - 1));
        return d.idx(ii, jj, kk);
    };
    const int c = d.idx(i, j, k);
    int cm = clampc(-1), cp = clampc(1), cmm = clampc(-2), cpp = clampc(2);
    cm = flags[cm] == GAS ? c : cm;
    cp = flags[cp] == GAS ? c : cp;
    cmm = flags[cmm] == GAS ? cm : cmm;
    cpp = flags[cpp] == GAS ? cp : cpp;
    const float qc = Hs[c], qm = Hs[cm], qp = Hs[cp], qmm = Hs[cmm], qpp = Hs[cpp];
    float d1, d2;
    int s0, s1, s2;
    float a0, a1, a2, b0, b1, b2;
    if (u > 0.0f) {
        d1 = qc - qm;
        d2 = 0.5f * (3.0f * qc - 4.0f * qm + qmm);
        s0 = c; s1 = cm; s2 = cmm;
        a0 = 1.0f; a1 = -1.0f; a2 = 0.0f;      // d1
        b0 = 1.5f; b1 = -2.0f; b2 = 0.5f;      // d2
    } else {
        d1 = qp - qc;
        d2 = 0.5f * (-3.0f * qc + 4.0f * qp - qpp);
        s0 = c; s1 = cp; s2 = cpp;
        a0 = -1.0f; a1 = 1.0f; a2 = 0.0f;
        b0 = -1.5f; b1 = 2.0f; b2 = -0.5f;
    }
    src[0] = s0;
    src[1] = s1;
    src[2] = s2;
    if (d1 * d2 > 0.0f) {
        const bool first = fabsf(d1) < fabsf(d2);
        coef[0] = first ? a0 : b0;
        coef[1] = first ? a1 : b1;
        coef[2] = first ? a2 : b2;
    } else {
        coef[0] = coef[1] = coef[2] = 0.0f;
    }
}

// Pass A: per cell, the adjoint passed through the floor / ceiling of the
// thermal update (mu), and the cell's own terms: velocity (advection), T
// (boundary loss) and the convection coefficient.
__global__ void __launch_bounds__(kAdjThreads) k_adj_thermal_mu(
    Dims d, const float* __restrict__ lam_H, float* __restrict__ mu, float* __restrict__ lam_T,
    float* __restrict__ lam_ux, float* __restrict__ lam_uy, float* __restrict__ lam_uz,
    const float* __restrict__ Hs, const float* __restrict__ T, const float* __restrict__ ux,
    const float* __restrict__ uy, const float* __restrict__ uz,
    const int32_t* __restrict__ flags, AdjThermalArgs a, Workspace ws, double* grad) {
    double sums[1] = {0.0};
    const int64_t n = d.n();
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int flag = flags[c];
        const float lh = lam_H[c];
        if (flag == GAS) {
            mu[c] = lh;
            continue;
        }
        int i, j, k;
        cell_ijk(d, c, i, j, k);
        float u = 0.0f, v = 0.0f, w = 0.0f;
        if (flag != SOLID) {
            u = ux[c];
            v = uy[c];
            w = uz[c];
        }
        const float hc = Hs[c];
        float h = hc + thermal_dh(d, Hs, T, flags, u, v, w, i, j, k, flag, hc, a.cpa, a.dt_lu);
        float dqdT = 0.0f, dqdh = 0.0f;
        bool pass = true;
        if (a.heat_loss) {
            int ne = 0;
            const int sx = d.ny * d.nz;
            if (k + 1 < d.nz && flags[c + 1] == GAS) ne++;
            if (j + 1 < d.ny && flags[c + d.nz] == GAS) ne++;
            if (j - 1 >= 0 && flags[c - d.nz] == GAS) ne++;
            if (i + 1 < d.nx && flags[c + sx] == GAS) ne++;
            if (i - 1 >= 0 && flags[c - sx] == GAS) ne++;
            if (ne != 0) {
                const float Tc = T[c];
                const float Te = fmin_(Tc, 2500.0f);
                float q = 0.0f;
                if (a.conv == 1) q += a.h_conv * (Te - a.T_amb);
                if (a.rad == 1) {
                    float t4 = Te * Te * Te * Te;
                    float a4 = a.T_amb * a.T_amb * a.T_amb * a.T_amb;
                    q += a.eps_rad * a.sigma_sb * (t4 - a4);
                }
                const float k_ne = (float)ne * a.dt_phys / a.dx;
                h -= q * (float)ne * a.dt_phys / a.dx;
                if (Tc < 2500.0f) {
                    float dq = 0.0f;
                    if (a.conv == 1) dq += a.h_conv;
                    if (a.rad == 1) dq += 4.0f * a.eps_rad * a.sigma_sb * Te * Te * Te;
                    dqdT = -dq * k_ne;
                }
                if (a.conv == 1) dqdh = -(Te - a.T_amb) * k_ne;
            }
            if (h < a.h_floor) pass = false;
            if (!pass) h = a.h_floor;
        }
        if (pass && a.cap) {
            if (h > a.ph.H_liq) {
                if (h > a.ph.cap_l) pass = false;
            } else {
                if (h > a.ph.cap_s) pass = false;
            }
        }
        const float m = pass ? lh : 0.0f;
        mu[c] = m;
        if (m == 0.0f) continue;
        if (dqdT != 0.0f) lam_T[c] += m * dqdT;
        sums[0] += (double)m * (double)dqdh;
        if (flag != SOLID) {
            // dH -= (u gx + v gy + w gz) dt
            float vel[3] = {u, v, w};
            float g3[3];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                int src[3];
                float coef[3];
                grad_stencil(d, Hs, flags, i, j, k, ax, vel[ax], src, coef);
                g3[ax] = coef[0] * Hs[src[0]] + coef[1] * Hs[src[1]] + coef[2] * Hs[src[2]];
            }
            lam_ux[c] += -m * g3[0] * a.dt_lu;
            lam_uy[c] += -m * g3[1] * a.dt_lu;
            lam_uz[c] += -m * g3[2] * a.dt_lu;
        }
    }
    accumulate_sums<1>(sums, ws, grad);
}

// Pass B: lam_Hp[s] = mu[s] + sum over the cells whose advection stencil reads
// H'[s]; lam_T[s] += the diffusion of the cells whose Laplacian reads T[s].
__global__ void __launch_bounds__(256) k_adj_thermal_gather(
    Dims d, const float* __restrict__ mu, float* __restrict__ lam_Hp, float* __restrict__ lam_T,
    const float* __restrict__ Hs, const float* __restrict__ ux, const float* __restrict__ uy,
    const float* __restrict__ uz, const int32_t* __restrict__ flags, float cpa, float dt_lu) {
    int i, j, k, s;
    if (!tile_cell(d, i, j, k, s)) return;
    float acc_h = mu[s];
    float acc_t = 0.0f;
    const int fs = flags[s];
    // advection: candidates on the three axis lines through s, offsets -2..2
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        for (int o = -2; o <= 2; ++o) {
            if (o == 0 && ax > 0) continue;        // the centre is handled with axis 0
            const int ic = i + (ax == 0 ? o : 0), jc = j + (ax == 1 ? o : 0);
            const int kc = k + (ax == 2 ? o : 0);
            if (ic < 0 || ic >= d.nx || jc < 0 || jc >= d.ny || kc < 0 || kc >= d.nz) continue;
            const int c = d.idx(ic, jc, kc);
            const int fc = flags[c];
            if (fc == GAS || fc == SOLID) continue;
            const float m = mu[c];
            if (m == 0.0f) continue;
            const float vel[3] = {ux[c], uy[c], uz[c]};
            for (int a2 = 0; a2 < 3; ++a2) {
                if (o != 0 && a2 != ax) continue;   // off-centre c reads s only along ax
                int src[3];
                float coef[3];
                grad_stencil(d, Hs, flags, ic, jc, kc, a2, vel[a2], src, coef);
                float cs = 0.0f;
#pragma unroll
                for (int sl = 0; sl < 3; ++sl)
                    if (src[sl] == s) cs += coef[sl];
                if (cs != 0.0f) acc_h += -m * vel[a2] * dt_lu * cs;
            }
        }
    }
    // diffusion: c = s (centre and fallback slots) and the six neighbours
    {
        const int di[7] = {0, 1, -1, 0, 0, 0, 0}, dj[7] = {0, 0, 0, 1, -1, 0, 0};
        const int dk[7] = {0, 0, 0, 0, 0, 1, -1};
#pragma unroll
        for (int m7 = 0; m7 < 7; ++m7) {
            const int ic = i + di[m7], jc = j + dj[m7], kc = k + dk[m7];
            if (ic < 0 || ic >= d.nx || jc < 0 || jc >= d.ny || kc < 0 || kc >= d.nz) continue;
            const int c = d.idx(ic, jc, kc);
            if (flags[c] == GAS) continue;
            const float m = mu[c];
            if (m == 0.0f) continue;
            // c's six slots: the neighbour if in range and not gas, else c itself
            float cs = m7 == 0 ? -6.0f : 0.0f;
            const int nb[6] = {d.idx(imax(0, ic - 1), jc, kc), d.idx(imin(ic + 1, d.nx - 1), jc, kc),
                               d.idx(ic, imax(0, jc - 1), kc), d.idx(ic, imin(jc + 1, d.ny - 1), kc),
                               d.idx(ic, jc, imax(0, kc - 1)), d.idx(ic, jc, imin(kc + 1, d.nz - 1))};
#pragma unroll
            for (int sl = 0; sl < 6; ++sl) {
                const int src = flags[nb[sl]] == GAS ? c : nb[sl];
                if (src == s) cs += 1.0f;
            }
            if (cs != 0.0f) acc_t += m * cpa * dt_lu * cs;
        }
    }
    (void)fs;
    lam_Hp[s] = acc_h;
    if (acc_t != 0.0f) lam_T[s] += acc_t;
}

// ---------------------------------------------------------------------------
// Arc injection + ceiling (k_arc_inject_tiles) transposed, and the parameter
// sums of the heat source: A = sum nu dh, B_p = sum nu epw wd dw/dp,
// D_p = sum wd dw/dp over the weight-sum cells, p = a_front, a_rear, b, c,
// sigma (Gaussian).  The host combines them per step with epw and W:
// dL/d eta = A / eta, dL/dp = B_p - D_p A / W.
// ---------------------------------------------------------------------------
constexpr int kInjectSums = 11;

__global__ void __launch_bounds__(kAdjThreads) k_adj_inject(
    Dims d, float* __restrict__ lam_H, const float* __restrict__ lam_Hp,
    const float* __restrict__ H, const float* __restrict__ f_l,
    const int32_t* __restrict__ flags, const float* __restrict__ scalars, ArcParams p,
    float arc_k_offset, float sigma, int welding, int cap, PhaseParams ph, Workspace ws,
    double* sums_out) {
    double sums[kInjectSums];
#pragma unroll
    for (int r = 0; r < kInjectSums; ++r) sums[r] = 0.0;
    const int64_t n = d.n();
    p.arc_k = scalars[kScalarArcK] + arc_k_offset;
    p.arc_i = scalars[kScalarArcI];
    p.arc_j = scalars[kScalarArcJ];
    const float epw = scalars[kScalarEpw];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const float lh = lam_Hp[c];
        const int flag = flags[c];
        if (!welding || flag == GAS) {
            lam_H[c] = lh;
            continue;
        }
        int i, j, k;
        cell_ijk(d, c, i, j, k);
        const float fl = f_l[c];
        const float wd = arc_weight(k, p.arc_k, fl, p.pen, p.enable);
        const bool weighted = !(wd < 1e-6f);
        float w = 0.0f;
        float dw[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        if (weighted) {
            const float di = (float)i - p.arc_i, dj = (float)j - p.arc_j, dk = (float)k - p.arc_k;
            if (p.kind == 0) {
                const float r2 = di * di + dj * dj + dk * dk * 0.25f;
                w = waam_expf(-r2 * p.inv2s2);
                dw[4] = w * r2 / (sigma * sigma * sigma);
            } else {
                w = goldak_w(di, dj, dk, p.sign, p.ff, p.fr, p.a_f, p.a_r, p.b, p.c);
                const float xt = di * p.sign;
                const bool front = xt >= 0.0f;
                const float aa = front ? p.a_f : p.a_r;
                const float ea = aa * aa + 1e-6f, eb = p.b * p.b + 1e-6f, ec = p.c * p.c + 1e-6f;
                const float da = w * 6.0f * aa * xt * xt / (ea * ea);
                dw[front ? 0 : 1] = da;
                dw[2] = w * 6.0f * p.b * dj * dj / (eb * eb);
                dw[3] = w * 6.0f * p.c * dk * dk / (ec * ec);
            }
#pragma unroll
            for (int q = 0; q < 5; ++q) sums[6 + q] += (double)(wd * dw[q]);
        }
        float dh = 0.0f;
        bool hit = false;
        if (epw > 0.0f && weighted) {
            hit = arc_cell_heat(p, epw, i, j, k, flag, fl, dh);
        }
        float h = H[c];
        if (hit) h = h + dh;
        bool pass = true;
        if (cap) {
            if (h > ph.H_liq) {
                if (h > ph.cap_l) pass = false;
            } else {
                if (h > ph.cap_s) pass = false;
            }
        }
        const float nu = pass ? lh : 0.0f;
        lam_H[c] = nu;
        if (hit && nu != 0.0f) {
            sums[0] += (double)nu * (double)dh;
#pragma unroll
            for (int q = 0; q < 5; ++q) sums[1 + q] += (double)nu * (double)(epw * wd * dw[q]);
        }
    }
    accumulate_sums<kInjectSums>(sums, ws, sums_out);
}

// lam[cells[t]] += vals[t], one thread in order (a handful of probe cells).
__global__ void k_adj_scatter_add(float* lam, const int32_t* cells, const float* vals, int count) {
    if (blockIdx.x == 0 && threadIdx.x == 0)
        for (int t = 0; t < count; ++t) lam[cells[t]] += vals[t];
}

AdjThermalArgs thermal_args(const WaamStepParams* p) {
    AdjThermalArgs a;
    a.ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    a.cpa = p->cp_rho * p->alpha_lu;
    a.dt_lu = 1.0f;
    a.heat_loss = p->heat_loss;
    a.conv = p->conv;
    a.rad = p->rad;
    a.cap = p->cap_enabled;
    a.T_amb = p->T_amb;
    a.h_conv = p->h_conv;
    a.eps_rad = p->eps_rad;
    a.dt_phys = p->dt;
    a.dx = p->dx;
    a.sigma_sb = p->sigma_sb;
    a.h_floor = p->cp_rho * p->T_amb;
    return a;
}

}  // namespace
}  // namespace waam

using namespace waam;

#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_adj_stream(float* lam_yp, const float* lam_xp, float* lam_xn, const int32_t* flags,
                    int nx, int ny, int nz, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "adj_stream: bad dims");
    REQUIRE(lam_yp && lam_xp && lam_xn && flags, "adj_stream: null field");
    REQUIRE(lam_yp != lam_xp && lam_xn != lam_xp && lam_xn != lam_yp, "adj_stream: aliasing");
    Dims d{nx, ny, nz};
    k_adj_stream<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, lam_yp, lam_xp, lam_xn,
                                                                     flags);
    return check_launch("k_adj_stream");
}

int waam_adj_collide(const WaamStepParams* p, const float* tape_f, const int32_t* tape_cells,
                     const int32_t* tape_count, int64_t tape_cap, const float* phi,
                     const float* T, const float* f_l, const int32_t* flags,
                     const float* scalars, float* lam_yp, float* lam_xn, float* lam_ux,
                     float* lam_uy, float* lam_uz, float* lam_fl, float* lam_T, float* ctb,
                     int32_t* map, int nx, int ny, int nz, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz) && p, "adj_collide: bad dims");
    REQUIRE(tape_f && tape_cells && tape_count && phi && T && f_l && flags && scalars && lam_yp &&
                lam_xn && lam_ux && lam_uy && lam_uz && lam_fl && lam_T && ctb && map,
            "adj_collide: null field");
    REQUIRE(p->collision == 0 && !p->use_tables, "adj_collide: the adjoint covers the MRT "
            "collision with constant material properties");
    AdjCollideArgs a;
    ForceParams& P = a.P;
    P.W = WeldForceParams{};
    P.csf = p->csf;
    P.wetting = p->wetting;
    P.welding = p->welding;
    P.hydro = p->hydro;
    P.gamma_lu = p->gamma_lu;
    P.cos_t = (float)cos((double)p->theta);
    P.sin_t = (float)sin((double)p->theta);
    P.dgamma = p->dgamma_lu;
    P.arc_i = P.arc_j = P.arc_k = 0.0f;
    P.p_inv2s2 = 1.0f / (2.0f * p->p_sigma * p->p_sigma + 1e-6f);
    float Fphys = p->pressure / (p->rho_phys * p->dx);
    P.p_Flu = Fphys * (p->dt * p->dt) / p->dx;
    P.g_lu = p->g_lu;
    P.beta = p->beta;
    P.T_ref = p->T_ref;
    P.rho_ref = 1.0f;
    P.F_cap = p->F_cap;
    a.omega = p->omega;
    a.omega_b = p->omega_b;
    a.C_darcy = p->C_darcy;
    a.u_cap = p->u_cap;
    Dims d{nx, ny, nz};
    k_adj_collide<<<4 * 148, 128, 0, STREAM(stream)>>>(
        d, tape_f, tape_cells, tape_count, tape_cap, phi, T, f_l, flags, scalars, lam_yp, lam_xn,
        lam_ux, lam_uy, lam_uz, lam_fl, lam_T, ctb, map, a);
    int e = check_launch("k_adj_collide");
    if (e) return e;
    k_adj_forces_gather<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, lam_T, ctb, map);
    e = check_launch("k_adj_forces_gather");
    if (e) return e;
    k_adj_clear_map<<<4 * 148, 128, 0, STREAM(stream)>>>(tape_cells, tape_count, map);
    return check_launch("k_adj_clear_map");
}

int waam_adj_combine(const WaamStepParams* p, float* lam_H, float* lam_T, float* lam_fl,
                     const float* H, const int32_t* flags, const float* phi, int64_t n,
                     void* stream) {
    REQUIRE(p && lam_H && lam_T && lam_fl && H && flags && phi, "adj_combine: null field");
    PhaseParams ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    k_adj_combine<<<elem_blocks(n), kThreads, 0, STREAM(stream)>>>(lam_H, lam_T, lam_fl, H, flags,
                                                                   phi, n, ph, p->vof);
    return check_launch("k_adj_combine");
}

int waam_adj_thermal(const WaamStepParams* p, const float* lam_H, float* lam_Hp, float* mu,
                     float* lam_T, float* lam_ux, float* lam_uy, float* lam_uz, const float* Hp,
                     const float* T, const float* ux, const float* uy, const float* uz,
                     const int32_t* flags, int nx, int ny, int nz, double* grad_hconv,
                     void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz) && p, "adj_thermal: bad dims");
    REQUIRE(lam_H && lam_Hp && mu && lam_T && lam_ux && lam_uy && lam_uz && Hp && T && ux && uy &&
                uz && flags && grad_hconv, "adj_thermal: null field");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()), "adj_thermal: workspace too small");
    AdjThermalArgs a = thermal_args(p);
    Workspace ws = Workspace::at(workspace);
    k_adj_thermal_mu<<<kAdjBlocks, kAdjThreads, 0, STREAM(stream)>>>(
        d, lam_H, mu, lam_T, lam_ux, lam_uy, lam_uz, Hp, T, ux, uy, uz, flags, a, ws, grad_hconv);
    int e = check_launch("k_adj_thermal_mu");
    if (e) return e;
    k_adj_thermal_gather<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, mu, lam_Hp, lam_T, Hp, ux, uy, uz, flags, a.cpa, a.dt_lu);
    return check_launch("k_adj_thermal_gather");
}

int waam_adj_inject(const WaamStepParams* p, float* lam_H, const float* lam_Hp, const float* H,
                    const float* f_l, const int32_t* flags, const float* scalars, int nx, int ny,
                    int nz, double* sums, void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz) && p, "adj_inject: bad dims");
    REQUIRE(lam_H && lam_Hp && H && f_l && flags && scalars && sums, "adj_inject: null field");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()), "adj_inject: workspace too small");
    static_assert(kAdjBlocks * kInjectSums <= kWsMaxPartials, "partials do not fit");
    ArcParams a{};
    a.kind = p->arc_kind;
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
    PhaseParams ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    k_adj_inject<<<kAdjBlocks, kAdjThreads, 0, STREAM(stream)>>>(
        d, lam_H, lam_Hp, H, f_l, flags, scalars, a, p->arc_k_offset, p->sigma_heat, p->welding,
        p->cap_enabled, ph, Workspace::at(workspace), sums);
    return check_launch("k_adj_inject");
}

int waam_adj_scatter_add(float* lam, const int32_t* cells, const float* vals, int count,
                         void* stream) {
    REQUIRE(lam && cells && vals && count >= 0, "adj_scatter_add: bad arguments");
    if (count == 0) return WAAM_OK;
    k_adj_scatter_add<<<1, 32, 0, STREAM(stream)>>>(lam, cells, vals, count);
    return check_launch("k_adj_scatter_add");
}

}  // extern "C"
