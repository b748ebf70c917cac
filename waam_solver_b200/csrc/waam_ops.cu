// Operator-level CUDA kernels and their C entry points (include/waam_b200.h).
//
// One kernel per reference Taichi kernel, so that the Python operator API
// (physics/*.py) can call them one by one exactly as solvers/coupled_step.py
// does.  The fused step in waam_fused.cu reuses the same device functions.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

using namespace waam;

namespace waam {

thread_local std::string g_last_error;

int fail(int code, const char* what) {
    g_last_error = what;
    return code;
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
        return WAAM_ERR_CUDA;
    }
    return WAAM_OK;
}

int elem_blocks(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > kMaxElemBlocks) b = kMaxElemBlocks;
    if (b < 1) b = 1;
    return (int)b;
}

int red_blocks(int64_t n) {
    int64_t b = (n + kThreads - 1) / kThreads;
    if (b > kRedBlocks) b = kRedBlocks;
    if (b < 1) b = 1;
    return (int)b;
}

bool dims_ok(int nx, int ny, int nz) {
    return nx > 0 && ny > 0 && nz > 0 && nx <= 65535 &&
           (int64_t)nx * ny * nz < ((int64_t)1 << 31);
}

bool workspace_ok(void* ws, size_t bytes, int64_t n) {
    return ws != nullptr && bytes >= waam_workspace_bytes(n) &&
           (reinterpret_cast<uintptr_t>(ws) % 256) == 0;
}

// ---------------------------------------------------------------------------
// Deterministic grid reduction: every block writes a double partial; the last
// block to finish sums the partials in index order.
// ---------------------------------------------------------------------------
__device__ double block_sum(double v) {
    __shared__ double sh[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    __syncthreads();
    return t;  // valid in thread 0
}

// Returns true in thread 0 of the last block; `total` then holds the sum.
__device__ bool finish_reduction(Workspace ws, double part, double& total) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        ws.partials[blockIdx.x] = part;
        __threadfence();
        unsigned prev = atomicAdd(ws.counter, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    if (threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += ((volatile double*)ws.partials)[b];
        total = t;
        *ws.counter = 0u;
    }
    return threadIdx.x == 0;
}

// Arc weight sum (pass 1 of kernels.py:443-510 / 548-622).  Writes the sum
// to norm_out (float, like the reference's 0-d field) and the energy per
// weight Q*eta*dt/(w_total*dx3) to scalars[2].
__global__ void k_arc_norm(Dims d, const int32_t* __restrict__ flags,
                           const float* __restrict__ f_l, ArcParams p, const float* arc_k_dev,
                           float arc_k_offset, float Qe_dt, float dx3, float* norm_out,
                           float* scalars, Workspace ws) {
    if (arc_k_dev) {  // fused step: arc k and torch position live in device scalars
        p.arc_k = arc_k_dev[0] + arc_k_offset;
        p.arc_i = arc_k_dev[kScalarArcI];
        p.arc_j = arc_k_dev[kScalarArcJ];
    }
    double part = 0.0;
    int64_t n = d.n();
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        int flag = flags[c];
        if (flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        part += (double)arc_cell_weight(p, i, j, k, flag, f_l[c]);
    }
    part = block_sum(part);
    double total;
    if (finish_reduction(ws, part, total)) {
        float w_total = (float)total;
        float epw = 0.0f;
        if (w_total > 1e-9f) epw = Qe_dt / (w_total * dx3);
        if (norm_out) norm_out[0] = w_total;
        scalars[1] = w_total;
        scalars[2] = epw;
    }
}

// Pass 2: H += epw * weight (non-gas cells), optionally followed by the
// enthalpy ceiling (solvers/coupled_step.py:107-108).
__global__ void k_arc_inject(Dims d, float* __restrict__ H, const int32_t* __restrict__ flags,
                             const float* __restrict__ f_l, ArcParams p, const float* arc_k_dev,
                             float arc_k_offset, const float* scalars, int cap, PhaseParams ph) {
    if (arc_k_dev) {
        p.arc_k = arc_k_dev[0] + arc_k_offset;
        p.arc_i = arc_k_dev[kScalarArcI];
        p.arc_j = arc_k_dev[kScalarArcJ];
    }
    float epw = scalars[2];
    int64_t n = d.n();
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        int flag = flags[c];
        if (flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float dh;
        bool hit = arc_cell_heat(p, epw, i, j, k, flag, f_l[c], dh);
        if (!hit && !cap) continue;
        float h = H[c];
        if (hit) h = h + dh;
        if (cap) h = cap_h(ph, h);
        H[c] = h;
    }
}

}  // namespace waam

// ---------------------------------------------------------------------------
// simple element-wise kernels
// ---------------------------------------------------------------------------
#define GRID_LOOP(c, n)                                                        \
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < (n); \
         c += (int64_t)gridDim.x * blockDim.x)

__global__ void k_init_grid(Dims d, float* f, float* rho, float* ux, float* uy, float* uz, float* T,
                            float* H, float* f_l, float* phi, int32_t* flags, float T_amb,
                            float rho0, float cp_rho, int nz_solid, int pi0, int pi1, int pj0,
                            int pj1) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int i, j, k;
        d.ijk(c, i, j, k);
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q * n + c] = wq(q) * rho0;
        rho[c] = rho0;
        ux[c] = uy[c] = uz[c] = 0.0f;
        T[c] = T_amb;
        H[c] = cp_rho * T_amb;
        f_l[c] = 0.0f;
        if (nz_solid < 0) {
            flags[c] = FLUID;
            phi[c] = 1.0f;
            f_l[c] = 1.0f;
        } else {
            bool in_plate = i >= pi0 && i < pi1 && j >= pj0 && j < pj1;
            if (in_plate && k < nz_solid) {
                phi[c] = 1.0f;
                flags[c] = SOLID;
            } else {
                phi[c] = 0.0f;
                flags[c] = GAS;
            }
        }
    }
}

__global__ void k_clear3(float* a, float* b, float* c3, int64_t n) {
    GRID_LOOP(c, n) { a[c] = b[c] = c3[c] = 0.0f; }
}

__global__ void k_ceiling(float* H, const int32_t* flags, int64_t n, PhaseParams ph) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        float h = H[c];
        float h2 = cap_h(ph, h);
        if (h2 != h) H[c] = h2;
    }
}

__global__ void k_copy(float* dst, const float* src, int64_t n) {
    GRID_LOOP(c, n) { dst[c] = src[c]; }
}

// cp_f / alpha_f non-null: the cell's own rho*cp and alpha_lu (kernels.py:1775-1836)
__global__ void k_thermal_op(Dims d, float* H, const float* Hs, const float* T, const float* ux,
                             const float* uy, const float* uz, const int32_t* flags, float cpa,
                             float dt, const float* cp_f, const float* alpha_f) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float Hc = Hs[c];
        float u = 0.0f, v = 0.0f, w = 0.0f;
        if (flag != SOLID) {
            u = ux[c];
            v = uy[c];
            w = uz[c];
        }
        const float cpa_c = cp_f ? cp_f[c] * alpha_f[c] : cpa;
        float dH = thermal_dh(d, Hs, T, flags, u, v, w, i, j, k, flag, Hc, cpa_c, dt);
        H[c] = Hc + dH;
    }
}

__global__ void k_phase(const float* H, float* T, float* f_l, int64_t n, PhaseParams ph) {
    GRID_LOOP(c, n) {
        float t, fl;
        phase(ph, H[c], t, fl);
        T[c] = t;
        f_l[c] = fl;
    }
}

__global__ void k_tmax(const float* T, float* T_max, const int32_t* flags, int64_t n) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        float t = T[c];
        if (t > T_max[c]) T_max[c] = t;
    }
}

__global__ void k_cooling(const float* T, float* T_prev, float* dT_dt, const int32_t* flags,
                          int64_t n, float inv_dt) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        float t = T[c];
        dT_dt[c] = (t - T_prev[c]) * inv_dt;
        T_prev[c] = t;
    }
}

__device__ __forceinline__ float heat_loss_dh(const Dims d, const float* T, const int32_t* flags,
                                              int i, int j, int k, float T_amb, float h_conv,
                                              float eps_rad, int conv, int rad, float dt, float dx,
                                              float sigma_sb, bool& any) {
    int ne = 0;
    if (k + 1 < d.nz && flags[d.idx(i, j, k + 1)] == GAS) ne++;
    if (j + 1 < d.ny && flags[d.idx(i, j + 1, k)] == GAS) ne++;
    if (j - 1 >= 0 && flags[d.idx(i, j - 1, k)] == GAS) ne++;
    if (i + 1 < d.nx && flags[d.idx(i + 1, j, k)] == GAS) ne++;
    if (i - 1 >= 0 && flags[d.idx(i - 1, j, k)] == GAS) ne++;
    any = ne != 0;
    if (!any) return 0.0f;
    float Te = fmin_(T[d.idx(i, j, k)], 2500.0f);
    float q = 0.0f;
    if (conv == 1) q += h_conv * (Te - T_amb);
    if (rad == 1) {
        float t4 = Te * Te * Te * Te;
        float a4 = T_amb * T_amb * T_amb * T_amb;
        q += eps_rad * sigma_sb * (t4 - a4);
    }
    return q * (float)ne * dt / dx;
}

__global__ void k_heat_loss(Dims d, float* H, const float* T, const int32_t* flags, float T_amb,
                            float h_conv, float eps_rad, int conv, int rad, float dt, float dx,
                            float sigma_sb) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        bool any;
        float q = heat_loss_dh(d, T, flags, i, j, k, T_amb, h_conv, eps_rad, conv, rad, dt, dx,
                               sigma_sb, any);
        if (any) H[c] -= q;
    }
}

__global__ void k_floor(float* H, float h_min, const int32_t* flags, int64_t n) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        if (H[c] < h_min) H[c] = h_min;
    }
}

__global__ void k_floor_var(float* H, const float* cp_f, const int32_t* flags, int64_t n,
                            float T_floor) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        const float h_min = cp_f[c] * T_floor;
        if (H[c] < h_min) H[c] = h_min;
    }
}

__global__ void k_refresh(const float* T, float* cp_f, float* alpha_f, float* dg_f, float* tau_f,
                          const int32_t* flags, int64_t n, WaamMaterialTables tb, TableConsts k) {
    GRID_LOOP(c, n) {
        const CellProps p = refresh_cell(tb, k, flags[c], T[c]);
        cp_f[c] = p.cp_rho;
        alpha_f[c] = p.alpha;
        dg_f[c] = p.dgamma;
        tau_f[c] = p.tau;
    }
}

__global__ void k_phase_var(const float* H, float* T, float* f_l, const float* cp_f, int64_t n,
                            VarPhase vp) {
    GRID_LOOP(c, n) {
        float t, fl;
        phase_var(vp, cp_f[c], H[c], t, fl);
        f_l[c] = fl;
        T[c] = t;
    }
}

__global__ void k_ceiling_var(float* H, const int32_t* flags, const float* cp_f, int64_t n,
                              VarPhase vp) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        const float h = H[c];
        const float h2 = cap_h_var(vp, cp_f[c], h);
        if (h2 != h) H[c] = h2;
    }
}

__global__ void k_advect_phi(Dims d, float* phi_dst, const float* phi, const float* ux,
                             const float* uy, const float* uz, const int32_t* flags) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int i, j, k;
        d.ijk(c, i, j, k);
        phi_dst[c] = advect_phi_cell(d, phi, ux, uy, uz, flags, i, j, k, flags[c]);
    }
}

__global__ void k_reinit(float* phi, const int32_t* flags, int64_t n) {
    GRID_LOOP(c, n) { phi[c] = reinit_phi(phi[c], flags[c]); }
}

__global__ void k_flags(Dims d, const float* phi, const float* f_l, int32_t* flags, int nz_solid) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int k = (int)(c % d.nz);
        flags[c] = flag_from(phi[c], f_l[c], k, nz_solid);
    }
}

__global__ void k_sync(const float* phi, float* f_l, const int32_t* flags, int64_t n) {
    GRID_LOOP(c, n) {
        int fl = flags[c];
        if (fl == GAS || phi[c] < 0.05f || fl == SOLID) f_l[c] = 0.0f;
    }
}

__global__ void k_csf(Dims d, const float* phi, const int32_t* flags, float* Fx, float* Fy,
                      float* Fz, ForceParams P) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        ForceParams Q = P;
        Q.welding = 0;
        Q.hydro = 0;
        Q.F_cap = 0.0f;
        // CSF only: disable the Marangoni / buoyancy branches via fl = 0.
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        cell_forces(d, Q, phi, nullptr, flags, i, j, k, 0.0f, fx, fy, fz);
        if (fx != 0.0f || fy != 0.0f || fz != 0.0f) {
            Fx[c] += fx;
            Fy[c] += fy;
            Fz[c] += fz;
        }
    }
}

// dg_f non-null: the cell's own dgamma (kernels.py:2221-2269)
__global__ void k_marangoni(Dims d, const float* T, const float* phi, const float* f_l, float* Fx,
                            float* Fy, float* Fz, const int32_t* flags, float dgamma,
                            const float* dg_f) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float fl = f_l[c];
        if (fl < 0.05f) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        int ip = imin(i + 1, d.nx - 1), im = imax(i - 1, 0);
        int jp = imin(j + 1, d.ny - 1), jm = imax(j - 1, 0);
        int kp = imin(k + 1, d.nz - 1), km = imax(k - 1, 0);
        float dx_ = 0.5f * (phi[d.idx(ip, j, k)] - phi[d.idx(im, j, k)]);
        float dy_ = 0.5f * (phi[d.idx(i, jp, k)] - phi[d.idx(i, jm, k)]);
        float dz_ = 0.5f * (phi[d.idx(i, j, kp)] - phi[d.idx(i, j, km)]);
        float g = sqrtf(dx_ * dx_ + dy_ * dy_ + dz_ * dz_);
        if (g < 1e-6f) continue;
        float nxn = dx_ / g, nyn = dy_ / g, nzn = dz_ / g;
        float tx = 0.5f * (T[d.idx(ip, j, k)] - T[d.idx(im, j, k)]);
        float ty = 0.5f * (T[d.idx(i, jp, k)] - T[d.idx(i, jm, k)]);
        float tz = 0.5f * (T[d.idx(i, j, kp)] - T[d.idx(i, j, km)]);
        float nd = nxn * tx + nyn * ty + nzn * tz;
        float sx = tx - nd * nxn, sy = ty - nd * nyn, sz = tz - nd * nzn;
        float scale = (dg_f ? dg_f[c] : dgamma) * g;
        Fx[c] += scale * sx;
        Fy[c] += scale * sy;
        Fz[c] += scale * sz;
    }
}

// kernels.py:1094-1141 apply_gas_shear_stress / 995-1091 apply_vapor_recoil(_cc)
__global__ void k_gas_shear(Dims d, float* Fx, float* Fy, const int32_t* flags, const float* phi,
                            float arc_i, float arc_j, WeldForceParams W) {
    GRID_LOOP(c, d.n()) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float fx = Fx[c], fy = Fy[c];
        gas_shear_cell(d, phi, i, j, k, arc_i, arc_j, W, fx, fy);
        Fx[c] = fx;
        Fy[c] = fy;
    }
}

__global__ void k_recoil(Dims d, float* Fz, const float* T, const int32_t* flags, const float* phi,
                         float arc_i, float arc_j, WeldForceParams W) {
    GRID_LOOP(c, d.n()) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float fz = Fz[c];
        recoil_cell(d, phi, T[c], i, j, k, arc_i, arc_j, W, fz);
        Fz[c] = fz;
    }
}

__global__ void k_arc_pressure(Dims d, float* Fz, const int32_t* flags, const float* phi,
                               float arc_i, float arc_j, float arc_k, float inv2s2, float Flu) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float dpz = phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))];
        if (fabsf(dpz) > 0.05f) {
            float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
            float r2 = di * di + dj * dj + dk * dk * 0.1f;
            Fz[c] += -Flu * waam_expf(-r2 * inv2s2);
        }
    }
}

__global__ void k_hydro(float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                        float rho_ref, float g_lu) {
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float fl = f_l[c];
        if (fl > 0.0f) Fz[c] += -rho_ref * g_lu * fl;
    }
}

__global__ void k_buoy(const float* T, float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                       float g_lu, float beta, float T_ref, float rho_ref) {
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float fl = f_l[c];
        if (fl > 0.0f) Fz[c] += rho_ref * g_lu * beta * (T[c] - T_ref) * fl;
    }
}

__global__ void k_clamp_force(float* Fx, float* Fy, float* Fz, const int32_t* flags, int64_t n,
                              float F_max) {
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float fx = Fx[c], fy = Fy[c], fz = Fz[c];
        float mag = sqrtf(fx * fx + fy * fy + fz * fz);
        if (mag > F_max) {
            float s = F_max / (mag + 1e-12f);
            Fx[c] = fx * s;
            Fy[c] = fy * s;
            Fz[c] = fz * s;
        }
    }
}

template <int KIND>
__global__ void k_collide(const float* __restrict__ f_src, float* __restrict__ f_dst, float* rho,
                          float* ux, float* uy, float* uz, const float* Fx, const float* Fy,
                          const float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                          float omega_s, float omega_b, float C_darcy, const float* tau_f) {
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float f[19], o[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) f[q] = f_src[q * n + c];
        float r, u, v, w;
        if (KIND == 0)
            collide_mrt_cell(f, f_l[c], Fx[c], Fy[c], Fz[c], omega_s, omega_b, C_darcy, o, r, u, v,
                             w);
        else
            // tau_f non-null: omega = 1 / (tau + 1e-6) per cell (kernels.py:2889-2965)
            collide_srt_cell(f, f_l[c], Fx[c], Fy[c], Fz[c],
                             tau_f ? 1.0f / (tau_f[c] + 1e-6f) : omega_s, C_darcy, o, r, u, v, w);
#pragma unroll
        for (int q = 0; q < 19; ++q) f_dst[q * n + c] = o[q];
        rho[c] = r;
        ux[c] = u;
        uy[c] = v;
        uz[c] = w;
    }
}

__global__ void k_clamp_vel(float* ux, float* uy, float* uz, const int32_t* flags, int64_t n,
                            float umax) {
    GRID_LOOP(c, n) {
        int flag = flags[c];
        if (flag == SOLID || flag == GAS) continue;
        float u = ux[c], v = uy[c], w = uz[c];
        float mag = sqrtf(u * u + v * v + w * w);
        if (mag > umax) {
            float s = umax / (mag + 1e-12f);
            ux[c] = u * s;
            uy[c] = v * s;
            uz[c] = w * s;
        }
    }
}

__global__ void k_time_above(const float* T, const int32_t* flags, float* t800, float* t1100,
                             float* tsol, int64_t n, float dt, float T800, float T1100, float Tsol) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        float t = T[c];
        if (t >= T800) t800[c] += dt;
        if (t >= T1100) t1100[c] += dt;
        if (t >= Tsol) tsol[c] += dt;
    }
}

__global__ void k_snapshot(const float* Fx, const float* Fy, const float* Fz, float* Sx, float* Sy,
                           float* Sz, int64_t n) {
    GRID_LOOP(c, n) {
        Sx[c] = Fx[c];
        Sy[c] = Fy[c];
        Sz[c] = Fz[c];
    }
}

// cp_f non-null: the cell's own rho*cp (kernels.py:2454-2485)
__global__ void k_remelt(const float* T, float* H, float* f_l, float* phi, int32_t* flags, int64_t n,
                         float cp_rho_c, float Ts, float Tl, float L_rho, const float* cp_f) {
    GRID_LOOP(c, n) {
        if (flags[c] != SOLID) continue;
        float Tc = T[c];
        if (Tc <= Ts + 5.0f) continue;
        const float cp_rho = cp_f ? cp_f[c] : cp_rho_c;
        float H_sol = cp_rho * Ts;
        float fl;
        if (Tc >= Tl) {
            fl = 1.0f;
            H[c] = cp_rho * Tl + L_rho + cp_rho * (Tc - Tl);
        } else {
            fl = (Tc - Ts) / (Tl - Ts + 1e-6f);
            H[c] = H_sol + fl * L_rho;
        }
        f_l[c] = fl;
        phi[c] = 1.0f;
        flags[c] = FLUID;
    }
}

__global__ void k_trailing(Dims d, float* T, float* H, float* f_l, float* phi, int32_t* flags,
                           float* ux, float* uy, float* uz, float cp_rho, float arc_i, float arc_j,
                           float arc_k, float dir_x, float dir_y, float dir_z, float lookback,
                           float T_freeze, float Ts, const float* cp_f) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        if (phi[c] < 0.85f || f_l[c] < 0.05f) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
        float proj = di * dir_x + dj * dir_y + dk * dir_z;
        if (proj > -lookback) continue;
        if (T[c] >= T_freeze) continue;
        // cp_f non-null: the cell's own rho*cp (kernels.py:2524-2570)
        H[c] = (cp_f ? cp_f[c] : cp_rho) * (Ts - 1.0f);
        T[c] = Ts - 1.0f;
        f_l[c] = 0.0f;
        phi[c] = 1.0f;
        flags[c] = SOLID;
        ux[c] = uy[c] = uz[c] = 0.0f;
    }
}

__global__ void k_cooled(const float* T, float* f_l, float* phi, int32_t* flags, float* ux,
                         float* uy, float* uz, int64_t n, float Ts, int zero_velocity) {
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        if (phi[c] < 0.85f) continue;
        if (f_l[c] < 0.02f && T[c] < Ts) {
            flags[c] = SOLID;
            phi[c] = 1.0f;
            f_l[c] = 0.0f;
            if (zero_velocity == 1) ux[c] = uy[c] = uz[c] = 0.0f;
        }
    }
}

// Highest metal cell of column (i0, j0): one warp scans the column.
__global__ void k_surface_height(Dims d, const float* phi, const int32_t* flags, float* out, int i0,
                                 int j0, int nz_fallback) {
    int best = -1;
    for (int k = threadIdx.x; k < d.nz; k += 32) {
        int64_t c = d.idx(i0, j0, k);
        if (flags[c] != GAS && phi[c] > 0.05f) best = k;
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    if (threadIdx.x == 0) {
        int ks = imax(1, nz_fallback - 1);
        if (best >= 0) ks = best;
        out[0] = (float)ks;
    }
}

__global__ void k_momentum_impact(Dims d, void* f_src, int storage, const float* rho, float* ux,
                                  float* uy, float* uz, const int32_t* flags, const float* f_l,
                                  float arc_i, float arc_j, float arc_k, float drop_r, float vx,
                                  float vy, float vz, int i0, int i1, int j0, int j1, int k0,
                                  int k1) {
    int64_t n = d.n();
    int ni = i1 - i0, nj = j1 - j0, nk = k1 - k0;
    int64_t m = (int64_t)ni * nj * nk;
    float drop_cz = arc_k + drop_r + 1.0f;
    float u2 = vx * vx + vy * vy + vz * vz;
    GRID_LOOP(t, m) {
        int k = k0 + (int)(t % nk);
        int j = j0 + (int)((t / nk) % nj);
        int i = i0 + (int)(t / ((int64_t)nk * nj));
        int64_t c = d.idx(i, j, k);
        if (flags[c] == GAS) continue;
        if (f_l[c] < 0.45f) continue;
        float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - drop_cz;
        float r2 = di * di + dj * dj + dk * dk;
        float rij2 = di * di + dj * dj;
        bool in_drop = r2 <= drop_r * drop_r || (rij2 <= drop_r * drop_r && (float)k >= arc_k + 1.0f);
        if (!in_drop) continue;
        float rl = rho[c];
        ux[c] = vx;
        uy[c] = vy;
        uz[c] = vz;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            float eu = (float)ex(q) * vx + (float)ey(q) * vy + (float)ez(q) * vz;
            pop_store(f_src, q * n + c, q,
                      wq(q) * rl * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2), storage);
        }
    }
}

// Block-wide exclusive scan of one 0/1 value per thread (blockDim.x a multiple
// of 32, at most 1024); returns the thread's prefix, *total the block's sum.
__device__ __forceinline__ unsigned block_scan01(unsigned v, unsigned* total) {
    __shared__ unsigned warp_sum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, v != 0u);
    const unsigned in_warp = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) warp_sum[warp] = __popc(m);
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    unsigned before = 0, all = 0;
    for (int w = 0; w < nw; ++w) {
        const unsigned s = warp_sum[w];
        before += w < warp ? s : 0u;
        all += s;
    }
    __syncthreads();   // warp_sum is reused by the next call
    *total = all;
    return before + in_warp;
}

// kernels.py:177-242 feed_wire: in the box around the arc, a GAS cell inside
// the droplet sphere or the column above the arc becomes liquid metal while
// the volume budget lasts.  Serially (lexicographic i, j, k) each eligible
// cell is taken while the float32 accumulator is below the target, so the
// cells taken are the first `take` eligible cells in that order: one thread
// replays the accumulation to find `take`, then the block converts the first
// `take` eligible cells chunk by chunk with a block scan.  One CTA.
__global__ void __launch_bounds__(1024) k_feed_wire(
    Dims d, void* f_src, int storage, int32_t* flags, float* f_l, float* phi, float* H, float* T,
    float* rho, float arc_i, float arc_j, float arc_k, float drop_r, float search_r,
    float target_vol, float T_drop, float cp_rho, float L_rho, float rho0, float* vol_acc,
    float cell_vol, int i0, int i1, int j0, int j1, int k0, int k1) {
    const int nj = j1 - j0, nk = k1 - k0;
    const int64_t m = (int64_t)(i1 - i0) * nj * nk;
    const int64_t n = d.n();
    const float drop_cz = arc_k + drop_r + 1.0f;
    auto cell_of = [&](int64_t t) -> int64_t {
        const int k = k0 + (int)(t % nk);
        const int j = j0 + (int)((t / nk) % nj);
        const int i = i0 + (int)(t / ((int64_t)nk * nj));
        return d.idx(i, j, k);
    };
    auto eligible = [&](int64_t t) -> bool {
        const int k = k0 + (int)(t % nk);
        const int j = j0 + (int)((t / nk) % nj);
        const int i = i0 + (int)(t / ((int64_t)nk * nj));
        const float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - drop_cz;
        const float r2 = di * di + dj * dj + dk * dk;
        const float rij2 = di * di + dj * dj;
        const bool in_sphere = r2 <= drop_r * drop_r;
        const bool in_column = rij2 <= search_r * search_r && (float)k >= arc_k + 1.0f;
        return (in_sphere || in_column) && flags[d.idx(i, j, k)] == GAS;
    };
    __shared__ unsigned s_take;
    unsigned total = 0, local = 0;
    for (int64_t t = threadIdx.x; t < m; t += blockDim.x) local += eligible(t) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    __shared__ unsigned warp_tot[32];
    if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = local;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += warp_tot[w];
        float acc = *vol_acc;
        unsigned take = 0;
        while (take < total && acc < target_vol) {
            acc = acc + cell_vol;
            ++take;
        }
        *vol_acc = acc;
        s_take = take;
    }
    __syncthreads();
    const unsigned take = s_take;
    unsigned base = 0;
    for (int64_t t0 = 0; t0 < m && base < take; t0 += blockDim.x) {
        const int64_t t = t0 + threadIdx.x;
        const bool e = t < m && eligible(t);
        unsigned chunk = 0;
        const unsigned rank = block_scan01(e ? 1u : 0u, &chunk);
        if (e && base + rank < take) {
            const int64_t c = cell_of(t);
            flags[c] = FLUID;
            f_l[c] = 1.0f;
            phi[c] = 1.0f;
            T[c] = T_drop;
            H[c] = cp_rho * T_drop + L_rho;
            rho[c] = rho0;
#pragma unroll
            for (int q = 0; q < 19; ++q) pop_store(f_src, q * n + c, q, wq(q) * rho0, storage);
        }
        base += chunk;
    }
}

// kernels.py:644-676 feed_wire_momentum: downward droplet momentum for the
// liquid (f_l >= 0.5), non-gas cells of the column under the droplet.
__global__ void k_feed_wire_momentum(Dims d, float* uz, const int32_t* flags, const float* f_l,
                                     float arc_i, float arc_j, float drop_r, float vz_lu, int i0,
                                     int i1, int j0, int j1, int k0, int k1) {
    const int nj = j1 - j0, nk = k1 - k0;
    const int64_t m = (int64_t)(i1 - i0) * nj * nk;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int k = k0 + (int)(t % nk);
        const int j = j0 + (int)((t / nk) % nj);
        const int i = i0 + (int)(t / ((int64_t)nk * nj));
        const int64_t c = d.idx(i, j, k);
        if (flags[c] == GAS) continue;
        if (f_l[c] < 0.5f) continue;
        const float di = (float)i - arc_i, dj = (float)j - arc_j;
        if (di * di + dj * dj <= drop_r * drop_r) uz[c] = fmin_(uz[c] + vz_lu, 0.15f);
    }
}

__global__ void k_impact_pressure(Dims d, float* Fz, const int32_t* flags, const float* phi,
                                  const float* f_l, float arc_i, float arc_j, float arc_k,
                                  float drop_r, float inv2s2, float Flu) {
    int64_t n = d.n();
    GRID_LOOP(c, n) {
        if (flags[c] == GAS) continue;
        if (f_l[c] < 0.25f && phi[c] < 0.25f) continue;
        int i, j, k;
        d.ijk(c, i, j, k);
        float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
        float r2 = di * di + dj * dj + dk * dk;
        if (r2 > drop_r * drop_r * 4.0f) continue;
        Fz[c] += -Flu * waam_expf(-r2 * inv2s2);
    }
}

// ---------------------------------------------------------------------------
// C entry points
// ---------------------------------------------------------------------------
#define STREAM(s) reinterpret_cast<cudaStream_t>(s)
#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)
#define EW(kernel, n, stream, ...)                                                       \
    do {                                                                                 \
        if ((n) <= 0) return waam::fail(WAAM_ERR_INVALID, #kernel ": empty grid");       \
        kernel<<<waam::elem_blocks(n), waam::kThreads, 0, STREAM(stream)>>>(__VA_ARGS__); \
        return waam::check_launch(#kernel);                                              \
    } while (0)

extern "C" {

const char* waam_last_error(void) { return waam::g_last_error.c_str(); }

int waam_abi_version(void) { return 1; }

size_t waam_workspace_bytes(int64_t n) { return waam::ws_total_bytes(n); }

size_t waam_struct_size(int which) {
    switch (which) {
        case 0: return sizeof(WaamFields);
        case 1: return sizeof(WaamStepParams);
        case 2: return sizeof(WaamMaterialTables);
        case 3: return sizeof(WaamTelemetry);
        case 4: return sizeof(WaamProbeSet);
        case 5: return sizeof(WaamShiftPlane);
        case 6: return sizeof(WaamExportChannel);
        default: return 0;
    }
}

int waam_init_grid(float* f, float* rho, float* ux, float* uy, float* uz, float* T, float* H,
                   float* f_l, float* phi, int32_t* flags, int nx, int ny, int nz, float T_amb,
                   float rho0, float cp_rho, int nz_solid, int pi0, int pi1, int pj0, int pj1,
                   void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "init_grid: bad dims");
    REQUIRE(f && rho && ux && uy && uz && T && H && f_l && phi && flags, "init_grid: null field");
    Dims d{nx, ny, nz};
    EW(k_init_grid, d.n(), stream, d, f, rho, ux, uy, uz, T, H, f_l, phi, flags, T_amb, rho0,
       cp_rho, nz_solid, pi0, pi1, pj0, pj1);
}

int waam_clear_forces(float* Fx, float* Fy, float* Fz, int64_t n, void* stream) {
    REQUIRE(Fx && Fy && Fz, "clear_forces: null field");
    EW(k_clear3, n, stream, Fx, Fy, Fz, n);
}

static int inject_common(float* H, const int32_t* flags, const float* f_l, float* norm_buf, Dims d,
                         ArcParams p, float Qe_dt, float dx3, void* workspace, size_t wsb,
                         void* stream) {
    REQUIRE(dims_ok(d.nx, d.ny, d.nz), "inject: bad dims");
    REQUIRE(H && flags && f_l, "inject: null field");
    REQUIRE(waam::workspace_ok(workspace, wsb, d.n()), "inject: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    int rb = waam::red_blocks(d.n());
    k_arc_norm<<<rb, kThreads, 0, STREAM(stream)>>>(d, flags, f_l, p, nullptr, 0.0f, Qe_dt, dx3,
                                                    norm_buf, ws.scalars, ws);
    int e = waam::check_launch("k_arc_norm");
    if (e) return e;
    PhaseParams dummy{};
    k_arc_inject<<<waam::elem_blocks(d.n()), kThreads, 0, STREAM(stream)>>>(
        d, H, flags, f_l, p, nullptr, 0.0f, ws.scalars, 0, dummy);
    return waam::check_launch("k_arc_inject");
}

int waam_inject_arc_heat(float* H, const int32_t* flags, const float* f_l, float* norm_buf,
                         int nx, int ny, int nz, float arc_i, float arc_j, float arc_k, float Q_w,
                         float sigma, float dt, float dx3, float eta, float pen, int enable,
                         void* workspace, size_t workspace_bytes, void* stream) {
    ArcParams p{};
    p.kind = 0;
    p.arc_i = arc_i;
    p.arc_j = arc_j;
    p.arc_k = arc_k;
    p.inv2s2 = 1.0f / (2.0f * sigma * sigma);
    p.pen = pen;
    p.enable = enable;
    float Qe_dt = Q_w * eta * dt;
    return inject_common(H, flags, f_l, norm_buf, Dims{nx, ny, nz}, p, Qe_dt, dx3, workspace,
                         workspace_bytes, stream);
}

int waam_inject_goldak_heat(float* H, const int32_t* flags, const float* f_l, float* norm_buf,
                            int nx, int ny, int nz, float arc_i, float arc_j, float arc_k,
                            float Q_w, float dt, float dx3, float eta, float sign, float ff,
                            float fr, float a_f, float a_r, float b, float c, float pen,
                            int enable, void* workspace, size_t workspace_bytes, void* stream) {
    ArcParams p{};
    p.kind = 1;
    p.arc_i = arc_i;
    p.arc_j = arc_j;
    p.arc_k = arc_k;
    p.sign = sign;
    p.ff = ff;
    p.fr = fr;
    p.a_f = a_f;
    p.a_r = a_r;
    p.b = b;
    p.c = c;
    p.pen = pen;
    p.enable = enable;
    float Qe_dt = Q_w * eta * dt;
    return inject_common(H, flags, f_l, norm_buf, Dims{nx, ny, nz}, p, Qe_dt, dx3, workspace,
                         workspace_bytes, stream);
}

int waam_clamp_enthalpy_ceiling_scalar(float* H, const int32_t* flags, int64_t n, float cp_rho,
                                       float Ts, float Tl, float T_cap, float L_rho,
                                       void* stream) {
    REQUIRE(H && flags, "ceiling: null field");
    EW(k_ceiling, n, stream, H, flags, n, make_phase(cp_rho, L_rho, Ts, Tl, T_cap, 1));
}

int waam_advect_diffuse_temperature(float* H, const float* T, const float* ux, const float* uy,
                                    const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                    float alpha_lu, float dt, float cp_rho, void* workspace,
                                    size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "thermal: bad dims");
    REQUIRE(H && T && ux && uy && uz && flags, "thermal: null field");
    Dims d{nx, ny, nz};
    REQUIRE(waam::workspace_ok(workspace, workspace_bytes, d.n()), "thermal: workspace too small");
    float* Hs = Workspace::at(workspace).field;
    int b = waam::elem_blocks(d.n());
    k_copy<<<b, kThreads, 0, STREAM(stream)>>>(Hs, H, d.n());
    int e = waam::check_launch("k_copy");
    if (e) return e;
    float cpa = cp_rho * alpha_lu;
    k_thermal_op<<<b, kThreads, 0, STREAM(stream)>>>(d, H, Hs, T, ux, uy, uz, flags, cpa, dt,
                                                     nullptr, nullptr);
    return waam::check_launch("k_thermal_op");
}

int waam_update_phase(const float* H, float* T, float* f_l, int64_t n, float cp_rho, float L_rho,
                      float Ts, float Tl, void* stream) {
    REQUIRE(H && T && f_l, "update_phase: null field");
    EW(k_phase, n, stream, H, T, f_l, n, make_phase(cp_rho, L_rho, Ts, Tl, 0.0f, 0));
}

int waam_update_T_max(const float* T, float* T_max, const int32_t* flags, int64_t n,
                      void* stream) {
    REQUIRE(T && T_max && flags, "update_T_max: null field");
    EW(k_tmax, n, stream, T, T_max, flags, n);
}

int waam_update_cooling_rate(const float* T, float* T_prev, float* dT_dt, const int32_t* flags,
                             int64_t n, float dt_phys, void* stream) {
    REQUIRE(T && T_prev && dT_dt && flags, "update_cooling_rate: null field");
    float inv_dt = 1.0f / (dt_phys + 1e-12f);
    EW(k_cooling, n, stream, T, T_prev, dT_dt, flags, n, inv_dt);
}

int waam_apply_thermal_boundary_losses(float* H, const float* T, const int32_t* flags, int nx,
                                       int ny, int nz, float T_amb, float h_conv, float eps_rad,
                                       int conv, int rad, float dt, float dx, float sigma_sb,
                                       void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "heat_loss: bad dims");
    REQUIRE(H && T && flags, "heat_loss: null field");
    Dims d{nx, ny, nz};
    EW(k_heat_loss, d.n(), stream, d, H, T, flags, T_amb, h_conv, eps_rad, conv, rad, dt, dx,
       sigma_sb);
}

int waam_clamp_enthalpy_floor_scalar(float* H, float cp_rho, const int32_t* flags, int64_t n,
                                     float T_floor, void* stream) {
    REQUIRE(H && flags, "floor: null field");
    float h_min = cp_rho * T_floor;
    EW(k_floor, n, stream, H, h_min, flags, n);
}

int waam_advect_phi(float* phi_dst, const float* phi_src, const float* ux, const float* uy,
                    const float* uz, const int32_t* flags, int nx, int ny, int nz, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "advect_phi: bad dims");
    REQUIRE(phi_dst && phi_src && ux && uy && uz && flags, "advect_phi: null field");
    REQUIRE(phi_dst != phi_src, "advect_phi: phi_dst must not alias phi_src");
    Dims d{nx, ny, nz};
    EW(k_advect_phi, d.n(), stream, d, phi_dst, phi_src, ux, uy, uz, flags);
}

int waam_reinitialize_phi(float* phi, const int32_t* flags, int64_t n, void* stream) {
    REQUIRE(phi && flags, "reinitialize_phi: null field");
    EW(k_reinit, n, stream, phi, flags, n);
}

int waam_apply_contact_angle_phi_bc(float* phi, const int32_t* flags, int nx, int ny, int nz,
                                    float theta, void* workspace, size_t workspace_bytes,
                                    void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "contact_bc: bad dims");
    REQUIRE(phi && flags, "contact_bc: null field");
    Dims d{nx, ny, nz};
    REQUIRE(waam::workspace_ok(workspace, workspace_bytes, d.n()), "contact_bc: workspace too small");
    float* snap = Workspace::at(workspace).field;
    k_copy<<<waam::elem_blocks(d.n()), kThreads, 0, STREAM(stream)>>>(snap, phi, d.n());
    int e = waam::check_launch("k_copy");
    if (e) return e;
    return waam::launch_contact_columns(d, snap, phi, flags, theta, stream);
}

int waam_update_flags_from_phi(const float* phi, const float* f_l, int32_t* flags, int nx, int ny,
                               int nz, int nz_solid, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "update_flags: bad dims");
    REQUIRE(phi && f_l && flags, "update_flags: null field");
    Dims d{nx, ny, nz};
    EW(k_flags, d.n(), stream, d, phi, f_l, flags, nz_solid);
}

int waam_sync_phi_liquid_fraction(const float* phi, float* f_l, const int32_t* flags, int64_t n,
                                  void* stream) {
    REQUIRE(phi && f_l && flags, "sync_phi: null field");
    EW(k_sync, n, stream, phi, f_l, flags, n);
}

int waam_compute_csf_tension(const float* phi, const int32_t* flags, float* Fx, float* Fy,
                             float* Fz, int nx, int ny, int nz, float gamma_lu, int wetting,
                             float theta, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "csf: bad dims");
    REQUIRE(phi && flags && Fx && Fy && Fz, "csf: null field");
    Dims d{nx, ny, nz};
    ForceParams P{};
    P.csf = 1;
    P.wetting = wetting;
    P.gamma_lu = gamma_lu;
    P.cos_t = (float)cos((double)theta);
    P.sin_t = (float)sin((double)theta);
    EW(k_csf, d.n(), stream, d, phi, flags, Fx, Fy, Fz, P);
}

int waam_compute_marangoni_force(const float* T, const float* phi, const float* f_l, float* Fx,
                                 float* Fy, float* Fz, const int32_t* flags, int nx, int ny,
                                 int nz, float dgamma, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "marangoni: bad dims");
    REQUIRE(T && phi && f_l && Fx && Fy && Fz && flags, "marangoni: null field");
    Dims d{nx, ny, nz};
    EW(k_marangoni, d.n(), stream, d, T, phi, f_l, Fx, Fy, Fz, flags, dgamma, nullptr);
}

int waam_apply_gas_shear_stress(float* Fx, float* Fy, const float* phi, const int32_t* flags,
                                int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                                float tau_peak_pa, float dt, float dx, float rho_ref,
                                void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "gas_shear: bad dims");
    REQUIRE(Fx && Fy && flags && phi, "gas_shear: null field");
    Dims d{nx, ny, nz};
    WeldForceParams W = weld_force_params(1, tau_peak_pa, 0, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f,
                                          0.0f, sigma, dt, dx, rho_ref);
    EW(k_gas_shear, d.n(), stream, d, Fx, Fy, flags, phi, arc_i, arc_j, W);
}

int waam_apply_vapor_recoil(float* Fz, const float* T, const float* phi, const int32_t* flags,
                            int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                            float recoil_pa, float T_ref, float dt, float dx, float rho_ref,
                            void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "vapor_recoil: bad dims");
    REQUIRE(Fz && T && flags && phi, "vapor_recoil: null field");
    Dims d{nx, ny, nz};
    WeldForceParams W = weld_force_params(0, 0.0f, 1, recoil_pa, T_ref, 0.0f, 0.0f, 0.0f, 0.0f,
                                          0.0f, sigma, dt, dx, rho_ref);
    EW(k_recoil, d.n(), stream, d, Fz, T, flags, phi, arc_i, arc_j, W);
}

int waam_apply_vapor_recoil_cc(float* Fz, const float* T, const float* phi, const int32_t* flags,
                               int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                               float P_ref, float T_boil, float L_vap, float R_spec, float C_acc,
                               float dt, float dx, float rho_ref, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "vapor_recoil_cc: bad dims");
    REQUIRE(Fz && T && flags && phi, "vapor_recoil_cc: null field");
    Dims d{nx, ny, nz};
    WeldForceParams W = weld_force_params(0, 0.0f, 2, 0.0f, 0.0f, P_ref, T_boil, L_vap, R_spec,
                                          C_acc, sigma, dt, dx, rho_ref);
    EW(k_recoil, d.n(), stream, d, Fz, T, flags, phi, arc_i, arc_j, W);
}

int waam_apply_arc_pressure(float* Fz, const int32_t* flags, const float* phi, int nx, int ny,
                            int nz, float arc_i, float arc_j, float arc_k, float sigma,
                            float pressure, float dt, float dx, float rho_ref, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "arc_pressure: bad dims");
    REQUIRE(Fz && flags && phi, "arc_pressure: null field");
    Dims d{nx, ny, nz};
    float inv2s2 = 1.0f / (2.0f * sigma * sigma + 1e-6f);
    float Fphys = pressure / (rho_ref * dx);
    float Flu = Fphys * (dt * dt) / dx;
    EW(k_arc_pressure, d.n(), stream, d, Fz, flags, phi, arc_i, arc_j, arc_k, inv2s2, Flu);
}

int waam_add_hydrostatic_gravity(float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                                 float rho_ref, float g_lu, void* stream) {
    REQUIRE(Fz && f_l && flags, "hydrostatic: null field");
    EW(k_hydro, n, stream, Fz, f_l, flags, n, rho_ref, g_lu);
}

int waam_add_buoyancy(const float* T, float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                      float g_lu, float beta, float T_ref, float rho_ref, void* stream) {
    REQUIRE(T && Fz && f_l && flags, "buoyancy: null field");
    EW(k_buoy, n, stream, T, Fz, f_l, flags, n, g_lu, beta, T_ref, rho_ref);
}

int waam_clamp_body_force_magnitude(float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                    int64_t n, float F_max, void* stream) {
    REQUIRE(Fx && Fy && Fz && flags, "clamp_force: null field");
    EW(k_clamp_force, n, stream, Fx, Fy, Fz, flags, n, F_max);
}

int waam_collide_mrt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                     const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                     const int32_t* flags, int64_t n, float omega_s, float omega_b,
                     float C_darcy, void* stream) {
    REQUIRE(f_src && f_dst && rho && ux && uy && uz && Fx && Fy && Fz && f_l && flags,
            "collide_mrt: null field");
    REQUIRE(f_src != f_dst, "collide_mrt: f_src must not alias f_dst");
    EW(k_collide<0>, n, stream, f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, n, omega_s,
       omega_b, C_darcy, nullptr);
}

int waam_collide_srt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                     const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                     const int32_t* flags, int64_t n, float omega, float C_darcy, void* stream) {
    REQUIRE(f_src && f_dst && rho && ux && uy && uz && Fx && Fy && Fz && f_l && flags,
            "collide_srt: null field");
    REQUIRE(f_src != f_dst, "collide_srt: f_src must not alias f_dst");
    EW(k_collide<1>, n, stream, f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, n, omega,
       0.0f, C_darcy, nullptr);
}

int waam_clamp_velocity_mach(float* ux, float* uy, float* uz, const int32_t* flags, int64_t n,
                             float u_max, void* stream) {
    REQUIRE(ux && uy && uz && flags, "clamp_velocity: null field");
    EW(k_clamp_vel, n, stream, ux, uy, uz, flags, n, u_max);
}

int waam_stream(const float* f_src, float* f_dst, const int32_t* flags, int nx, int ny, int nz,
                void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "stream: bad dims");
    REQUIRE(f_src && f_dst && flags, "stream: null field");
    REQUIRE(f_src != f_dst, "stream: f_src must not alias f_dst");
    return waam::launch_stream(Dims{nx, ny, nz}, f_src, f_dst, flags, stream);
}

int waam_update_time_above_T(const float* T, const int32_t* flags, float* t800, float* t1100,
                             float* tsol, int64_t n, float dt, float T800, float T1100, float Tsol,
                             void* stream) {
    REQUIRE(T && flags && t800 && t1100 && tsol, "time_above: null field");
    EW(k_time_above, n, stream, T, flags, t800, t1100, tsol, n, dt, T800, T1100, Tsol);
}

int waam_snapshot_forces(const float* Fx, const float* Fy, const float* Fz, float* Sx, float* Sy,
                         float* Sz, int64_t n, void* stream) {
    REQUIRE(Fx && Fy && Fz && Sx && Sy && Sz, "snapshot_forces: null field");
    EW(k_snapshot, n, stream, Fx, Fy, Fz, Sx, Sy, Sz, n);
}

int waam_remelt_hot_solid_scalar(const float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                 int64_t n, float cp_rho, float Ts, float Tl, float L_rho,
                                 void* stream) {
    REQUIRE(T && H && f_l && phi && flags, "remelt: null field");
    EW(k_remelt, n, stream, T, H, f_l, phi, flags, n, cp_rho, Ts, Tl, L_rho, nullptr);
}

int waam_solidify_trailing_pool_scalar(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                       float* ux, float* uy, float* uz, int nx, int ny, int nz,
                                       float cp_rho, float arc_i, float arc_j, float arc_k,
                                       float dir_x, float dir_y, float dir_z, float lookback,
                                       float T_freeze, float Ts, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "trailing: bad dims");
    REQUIRE(T && H && f_l && phi && flags && ux && uy && uz, "trailing: null field");
    Dims d{nx, ny, nz};
    EW(k_trailing, d.n(), stream, d, T, H, f_l, phi, flags, ux, uy, uz, cp_rho, arc_i, arc_j, arc_k,
       dir_x, dir_y, dir_z, lookback, T_freeze, Ts, nullptr);
}

static bool tables_ok(const WaamMaterialTables* t) {
    const int32_t cnt[4] = {t->n_cp, t->n_k, t->n_mu, t->n_dgamma};
    for (int q = 0; q < 4; ++q)
        if (cnt[q] < 0 || cnt[q] > WAAM_TABLE_KNOTS) return false;
    return true;
}

int waam_refresh_thermal_properties(const float* T, float* cp_rho_f, float* alpha_f,
                                    float* dgamma_f, float* tau_f, const int32_t* flags, int64_t n,
                                    const WaamMaterialTables* tables, float rho, float dt,
                                    float dx, float force_scale, float cp_rho_ref,
                                    float alpha_lu_ref, float dgamma_lu_ref, float tau_ref,
                                    float marangoni_scale, int use_tables, void* stream) {
    REQUIRE(T && cp_rho_f && alpha_f && dgamma_f && tau_f && flags, "refresh: null field");
    REQUIRE(use_tables != 1 || (tables && tables_ok(tables)), "refresh: bad tables");
    WaamMaterialTables tb{};
    if (tables) tb = *tables;
    TableConsts k{rho, dt, dx, force_scale, marangoni_scale, cp_rho_ref, alpha_lu_ref,
                  dgamma_lu_ref, tau_ref, use_tables};
    EW(k_refresh, n, stream, T, cp_rho_f, alpha_f, dgamma_f, tau_f, flags, n, tb, k);
}

int waam_advect_diffuse_temperature_variable(float* H, const float* T, const float* ux,
                                             const float* uy, const float* uz,
                                             const int32_t* flags, const float* alpha_f,
                                             const float* cp_rho_f, int nx, int ny, int nz,
                                             float dt, void* workspace, size_t workspace_bytes,
                                             void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "thermal_variable: bad dims");
    REQUIRE(H && T && ux && uy && uz && flags && alpha_f && cp_rho_f,
            "thermal_variable: null field");
    Dims d{nx, ny, nz};
    REQUIRE(waam::workspace_ok(workspace, workspace_bytes, d.n()),
            "thermal_variable: workspace too small");
    float* Hs = Workspace::at(workspace).field;
    int b = waam::elem_blocks(d.n());
    k_copy<<<b, kThreads, 0, STREAM(stream)>>>(Hs, H, d.n());
    int e = waam::check_launch("k_copy");
    if (e) return e;
    k_thermal_op<<<b, kThreads, 0, STREAM(stream)>>>(d, H, Hs, T, ux, uy, uz, flags, 0.0f, dt,
                                                     cp_rho_f, alpha_f);
    return waam::check_launch("k_thermal_op");
}

int waam_update_phase_variable_cp(const float* H, float* T, float* f_l, const float* cp_rho_f,
                                  int64_t n, float L_rho, float T_solidus, float T_liquidus,
                                  float H_sol, float H_liq, void* stream) {
    REQUIRE(H && T && f_l && cp_rho_f, "phase_variable: null field");
    VarPhase vp{H_sol, H_liq, L_rho, T_solidus, T_liquidus, 0.0f};
    EW(k_phase_var, n, stream, H, T, f_l, cp_rho_f, n, vp);
}

int waam_clamp_enthalpy_ceiling_variable_cp(float* H, const int32_t* flags, const float* cp_rho_f,
                                            int64_t n, float H_liq, float T_liquidus,
                                            float T_cap, void* stream) {
    REQUIRE(H && flags && cp_rho_f, "ceiling_variable: null field");
    VarPhase vp{0.0f, H_liq, 0.0f, 0.0f, T_liquidus, T_cap};
    EW(k_ceiling_var, n, stream, H, flags, cp_rho_f, n, vp);
}

int waam_clamp_enthalpy_floor(float* H, const float* cp_rho_f, const int32_t* flags, int64_t n,
                              float T_floor, void* stream) {
    REQUIRE(H && cp_rho_f && flags, "floor: null field");
    EW(k_floor_var, n, stream, H, cp_rho_f, flags, n, T_floor);
}

int waam_compute_marangoni_force_variable(const float* T, const float* phi, const float* f_l,
                                          float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                          const float* dgamma_f, int nx, int ny, int nz,
                                          void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "marangoni_variable: bad dims");
    REQUIRE(T && phi && f_l && Fx && Fy && Fz && flags && dgamma_f,
            "marangoni_variable: null field");
    Dims d{nx, ny, nz};
    EW(k_marangoni, d.n(), stream, d, T, phi, f_l, Fx, Fy, Fz, flags, 0.0f, dgamma_f);
}

int waam_collide_srt_variable_tau(const float* f_src, float* f_dst, float* rho, float* ux,
                                  float* uy, float* uz, const float* Fx, const float* Fy,
                                  const float* Fz, const float* f_l, const int32_t* flags,
                                  const float* tau_f, int64_t n, float C_darcy, void* stream) {
    REQUIRE(f_src && f_dst && rho && ux && uy && uz && Fx && Fy && Fz && f_l && flags && tau_f,
            "collide_srt_variable_tau: null field");
    REQUIRE(f_src != f_dst, "collide_srt_variable_tau: f_src must not alias f_dst");
    EW(k_collide<1>, n, stream, f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, n, 0.0f,
       0.0f, C_darcy, tau_f);
}

int waam_remelt_hot_solid(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                          const float* cp_rho_f, int64_t n, float T_solidus, float T_liquidus,
                          float L_rho, void* stream) {
    REQUIRE(T && H && f_l && phi && flags && cp_rho_f, "remelt: null field");
    EW(k_remelt, n, stream, T, H, f_l, phi, flags, n, 0.0f, T_solidus, T_liquidus, L_rho,
       cp_rho_f);
}

int waam_solidify_trailing_pool(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                float* ux, float* uy, float* uz, const float* cp_rho_f, int nx,
                                int ny, int nz, float arc_i, float arc_j, float arc_k, float dir_x,
                                float dir_y, float dir_z, float lookback, float T_freeze,
                                float T_solidus, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "trailing: bad dims");
    REQUIRE(T && H && f_l && phi && flags && ux && uy && uz && cp_rho_f,
            "trailing: null field");
    Dims d{nx, ny, nz};
    EW(k_trailing, d.n(), stream, d, T, H, f_l, phi, flags, ux, uy, uz, 0.0f, arc_i, arc_j, arc_k,
       dir_x, dir_y, dir_z, lookback, T_freeze, T_solidus, cp_rho_f);
}

int waam_solidify_cooled_metal(const float* T, float* f_l, float* phi, int32_t* flags, float* ux,
                               float* uy, float* uz, int64_t n, float Ts, int zero_velocity,
                               void* stream) {
    REQUIRE(T && f_l && phi && flags && ux && uy && uz, "solidify_cooled: null field");
    EW(k_cooled, n, stream, T, f_l, phi, flags, ux, uy, uz, n, Ts, zero_velocity);
}

int waam_surface_height_at(const float* phi, const int32_t* flags, float* out, int nx, int ny,
                           int nz, int i0, int j0, int nz_fallback, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "surface_height: bad dims");
    REQUIRE(phi && flags && out, "surface_height: null field");
    REQUIRE(i0 >= 0 && i0 < nx && j0 >= 0 && j0 < ny, "surface_height: column out of range");
    k_surface_height<<<1, 32, 0, STREAM(stream)>>>(Dims{nx, ny, nz}, phi, flags, out, i0, j0,
                                                   nz_fallback);
    return waam::check_launch("k_surface_height");
}

int waam_feed_wire_surface(float* f_src, int32_t* flags, float* f_l, float* phi, float* H, float* T,
                           float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                           float arc_k, float foot_r, float drop_r, float target_vol, float T_drop,
                           float cp_rho, float L_rho, float rho0, float* vol_acc, float* real_acc,
                           float cell_vol, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "feed_wire_surface: bad dims");
    REQUIRE(f_src && flags && f_l && phi && H && T && rho && vol_acc && real_acc,
            "feed_wire_surface: null field");
    return waam::launch_deposit(Dims{nx, ny, nz}, f_src, waam::kStoreF32, flags, f_l, phi, H, T,
                                rho, arc_i, arc_j, arc_k, &foot_r, 1, 0.0, drop_r, target_vol,
                                T_drop, cp_rho, L_rho, rho0, vol_acc, real_acc, cell_vol, stream);
}

int waam_deposit_droplet(void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi,
                         float* H, float* T, float* rho, int nx, int ny, int nz, float arc_i,
                         float arc_j, float arc_k, const float* foot_radii, int n_tries,
                         double accept_volume, float drop_r, float target_vol, float T_drop,
                         float cp_rho, float L_rho, float rho0, float* vol_acc, float* real_acc,
                         float cell_vol, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "deposit_droplet: bad dims");
    REQUIRE(f_src && flags && f_l && phi && H && T && rho && vol_acc && real_acc,
            "deposit_droplet: null field");
    REQUIRE(foot_radii && n_tries >= 1 && n_tries <= WAAM_DEPOSIT_MAX_TRIES,
            "deposit_droplet: need 1..WAAM_DEPOSIT_MAX_TRIES footprint radii");
    return waam::launch_deposit(Dims{nx, ny, nz}, f_src, f_storage, flags, f_l, phi, H, T, rho,
                                arc_i, arc_j, arc_k, foot_radii, n_tries, accept_volume, drop_r,
                                target_vol, T_drop, cp_rho, L_rho, rho0, vol_acc, real_acc,
                                cell_vol, stream);
}

int waam_feed_wire_momentum_impact_stored(void* f_src, int f_storage, const float* rho, float* ux,
                                          float* uy, float* uz, const int32_t* flags,
                                          const float* f_l, int nx, int ny, int nz, float arc_i,
                                          float arc_j, float arc_k, float drop_r, float vx,
                                          float vy, float vz, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "momentum_impact: bad dims");
    REQUIRE(f_src && rho && ux && uy && uz && flags && f_l, "momentum_impact: null field");
    REQUIRE(f_storage >= waam::kStoreF32 && f_storage <= waam::kStoreBF16,
            "momentum_impact: f_storage must be 0, 1 or 2");
    Dims d{nx, ny, nz};
    int i0 = imax(0, (int)(arc_i - drop_r * 2.5f)), i1 = imin(nx, (int)(arc_i + drop_r * 2.5f) + 1);
    int j0 = imax(0, (int)(arc_j - drop_r * 2.5f)), j1 = imin(ny, (int)(arc_j + drop_r * 2.5f) + 1);
    int k0 = imax(0, (int)arc_k), k1 = imin(nz, (int)(arc_k + drop_r * 3.0f) + 1);
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) return WAAM_OK;
    int64_t m = (int64_t)(i1 - i0) * (j1 - j0) * (k1 - k0);
    k_momentum_impact<<<waam::elem_blocks(m), kThreads, 0, STREAM(stream)>>>(
        d, f_src, f_storage, rho, ux, uy, uz, flags, f_l, arc_i, arc_j, arc_k, drop_r, vx, vy, vz,
        i0, i1, j0, j1, k0, k1);
    return waam::check_launch("k_momentum_impact");
}

int waam_feed_wire_momentum_impact(float* f_src, const float* rho, float* ux, float* uy, float* uz,
                                   const int32_t* flags, const float* f_l, int nx, int ny, int nz,
                                   float arc_i, float arc_j, float arc_k, float drop_r, float vx,
                                   float vy, float vz, void* stream) {
    return waam_feed_wire_momentum_impact_stored(f_src, waam::kStoreF32, rho, ux, uy, uz, flags,
                                                 f_l, nx, ny, nz, arc_i, arc_j, arc_k, drop_r, vx,
                                                 vy, vz, stream);
}

int waam_feed_wire(void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi, float* H,
                   float* T, float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                   float arc_k, float drop_r, float target_vol, float T_drop, float cp_rho,
                   float L_rho, float rho0, float* vol_acc, float cell_vol, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "feed_wire: bad dims");
    REQUIRE(f_src && flags && f_l && phi && H && T && rho && vol_acc, "feed_wire: null field");
    REQUIRE(f_storage >= waam::kStoreF32 && f_storage <= waam::kStoreBF16,
            "feed_wire: f_storage must be 0, 1 or 2");
    REQUIRE(std::isfinite(arc_i) && std::isfinite(arc_j) && std::isfinite(arc_k) &&
                std::isfinite(drop_r) && drop_r >= 0.0f && fabsf(arc_i) < 1e7f &&
                fabsf(arc_j) < 1e7f && fabsf(arc_k) < 1e7f && drop_r < 1e6f,
            "feed_wire: arc position or droplet radius out of range");
    // kernels.py:211-217: the search box (ti.cast truncates toward zero)
    const float search_r = fmax_(drop_r * 2.5f, drop_r + 2.0f);
    const int i0 = imax(0, (int)(arc_i - search_r)), i1 = imin(nx, (int)(arc_i + search_r) + 1);
    const int j0 = imax(0, (int)(arc_j - search_r)), j1 = imin(ny, (int)(arc_j + search_r) + 1);
    const int k0 = imax(0, (int)(arc_k + 1.0f)), k1 = imin(nz, (int)(arc_k + search_r * 3.0f) + 1);
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) return WAAM_OK;
    k_feed_wire<<<1, 1024, 0, STREAM(stream)>>>(Dims{nx, ny, nz}, f_src, f_storage, flags, f_l,
                                                 phi, H, T, rho, arc_i, arc_j, arc_k, drop_r,
                                                 search_r, target_vol, T_drop, cp_rho, L_rho,
                                                 rho0, vol_acc, cell_vol, i0, i1, j0, j1, k0, k1);
    return waam::check_launch("k_feed_wire");
}

int waam_feed_wire_momentum(float* uz, const int32_t* flags, const float* f_l, int nx, int ny,
                            int nz, float arc_i, float arc_j, float arc_k, float drop_r,
                            float vz_lu, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "feed_wire_momentum: bad dims");
    REQUIRE(uz && flags && f_l, "feed_wire_momentum: null field");
    REQUIRE(std::isfinite(arc_i) && std::isfinite(arc_j) && std::isfinite(arc_k) &&
                std::isfinite(drop_r) && fabsf(arc_i) < 1e7f && fabsf(arc_j) < 1e7f &&
                fabsf(arc_k) < 1e7f && fabsf(drop_r) < 1e6f,
            "feed_wire_momentum: arc position or droplet radius out of range");
    // kernels.py:662-667
    const int i0 = imax(0, (int)(arc_i - drop_r)), i1 = imin(nx, (int)(arc_i + drop_r) + 1);
    const int j0 = imax(0, (int)(arc_j - drop_r)), j1 = imin(ny, (int)(arc_j + drop_r) + 1);
    const int k0 = imax(0, (int)arc_k), k1 = imin(nz, (int)(arc_k + drop_r * 2.0f) + 1);
    if (i1 <= i0 || j1 <= j0 || k1 <= k0) return WAAM_OK;
    const int64_t m = (int64_t)(i1 - i0) * (j1 - j0) * (k1 - k0);
    k_feed_wire_momentum<<<waam::elem_blocks(m), kThreads, 0, STREAM(stream)>>>(
        Dims{nx, ny, nz}, uz, flags, f_l, arc_i, arc_j, drop_r, vz_lu, i0, i1, j0, j1, k0, k1);
    return waam::check_launch("k_feed_wire_momentum");
}

int waam_apply_droplet_impact_pressure(float* Fz, const int32_t* flags, const float* phi,
                                       const float* f_l, int nx, int ny, int nz, float arc_i,
                                       float arc_j, float arc_k, float drop_r, float impact_pa,
                                       float dt, float dx, float rho_ref, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "impact_pressure: bad dims");
    REQUIRE(Fz && flags && phi && f_l, "impact_pressure: null field");
    Dims d{nx, ny, nz};
    float inv2s2 = 1.0f / (2.0f * drop_r * drop_r + 1e-6f);
    float Fphys = impact_pa / (rho_ref * dx);
    float Flu = Fphys * dt * dt / dx;
    EW(k_impact_pressure, d.n(), stream, d, Fz, flags, phi, f_l, arc_i, arc_j, arc_k, drop_r,
       inv2s2, Flu);
}

}  // extern "C"
