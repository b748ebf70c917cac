// Shared device code for the B200 coupled melt-pool step.
//
// Layout (identical to the reference grid, grid.py:128-206): scalar fields are
// (nx, ny, nz) row-major with k fastest; D3Q19 populations are (19, nx, ny, nz)
// with one contiguous plane per direction; flags are int32 with FLUID=0,
// SOLID=1, GAS=2, IFACE=4.  Every device function keeps the reference's
// float32 expression order (left-to-right Python/Taichi evaluation) and the
// library is compiled with -fmad=false, so a result differs from a serial
// float32 run of the reference only through expf/sinf/cosf rounding and the
// order of global sums.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "../../include/waam_b200.h"
#include "waam_expf.h"

namespace waam {

constexpr int FLUID = 0;
constexpr int SOLID = 1;
constexpr int GAS = 2;
constexpr int IFACE = 4;

__host__ __device__ constexpr int ex(int q) {
    return q == 1 || q == 7 || q == 9 || q == 11 || q == 13 ? 1
         : (q == 2 || q == 8 || q == 10 || q == 12 || q == 14 ? -1 : 0);
}
__host__ __device__ constexpr int ey(int q) {
    return q == 3 || q == 7 || q == 10 || q == 15 || q == 17 ? 1
         : (q == 4 || q == 8 || q == 9 || q == 16 || q == 18 ? -1 : 0);
}
__host__ __device__ constexpr int ez(int q) {
    return q == 5 || q == 11 || q == 14 || q == 15 || q == 18 ? 1
         : (q == 6 || q == 12 || q == 13 || q == 16 || q == 17 ? -1 : 0);
}
__host__ __device__ constexpr int opp(int q) { return q == 0 ? 0 : (q & 1 ? q + 1 : q - 1); }
// kernels.py:45-50: Python 1/3, 1/18, 1/36 rounded to float32.
__host__ __device__ constexpr float wq(int q) {
    return q == 0 ? 0.333333343f : (q < 7 ? 0.0555555560f : 0.0277777780f);
}

// Population storage.  kStoreF32 keeps f_q; kStoreF16 / kStoreBF16 keep the
// offset f_q - w_q (rho0 = 1) in 16 bits, rounded to nearest, and every
// kernel computes in float on w_q + offset.
enum PopStorage { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2 };

template <int S>
struct Pop;
template <>
struct Pop<kStoreF32> {
    typedef float T;
    __device__ static __forceinline__ float get(T v, int) { return v; }
    __device__ static __forceinline__ T put(float f, int) { return f; }
};
template <>
struct Pop<kStoreF16> {
    typedef __half T;
    __device__ static __forceinline__ float get(T v, int q) { return wq(q) + __half2float(v); }
    __device__ static __forceinline__ T put(float f, int q) { return __float2half_rn(f - wq(q)); }
};
template <>
struct Pop<kStoreBF16> {
    typedef __nv_bfloat16 T;
    __device__ static __forceinline__ float get(T v, int q) {
        return wq(q) + __bfloat162float(v);
    }
    __device__ static __forceinline__ T put(float f, int q) {
        return __float2bfloat16_rn(f - wq(q));
    }
};

// Store one population value at element index idx in any storage (for the
// sparse writers: deposition, droplet impact).
__device__ __forceinline__ void pop_store(void* f, size_t idx, int q, float v, int storage) {
    if (storage == kStoreF16)
        static_cast<__half*>(f)[idx] = Pop<kStoreF16>::put(v, q);
    else if (storage == kStoreBF16)
        static_cast<__nv_bfloat16*>(f)[idx] = Pop<kStoreBF16>::put(v, q);
    else
        static_cast<float*>(f)[idx] = v;
}

// Grids are limited to fewer than 2^31 cells (checked on the host), so a cell
// index fits an int; population offsets q*n + c are formed in 64 bits.
struct Dims {
    int nx, ny, nz;
    __host__ __device__ int64_t n() const { return (int64_t)nx * ny * nz; }
    __host__ __device__ int idx(int i, int j, int k) const { return (i * ny + j) * nz + k; }
    __device__ void ijk(int64_t c, int& i, int& j, int& k) const {
        k = (int)(c % nz);
        int64_t r = c / nz;
        j = (int)(r % ny);
        i = (int)(r / ny);
    }
};

__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ float fmin_(float a, float b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ float fmax_(float a, float b) { return a > b ? a : b; }

// kernels.py:406-437 arc_deposition_weight
__device__ __forceinline__ float arc_weight(int k, float arc_k, float fl, float pen, int enable) {
    float w = 1.0f;
    if (enable == 1) {
        if (fl > 0.55f) {
            w = 1.0f;
        } else {
            float dz = arc_k - (float)k;
            if (dz < -0.5f) {
                w = 0.0f;
            } else {
                float depth = fmax_(0.0f, dz);
                float inv_pen = 1.0f / (pen + 1e-6f);
                w = waam_expf(-depth * inv_pen);
            }
        }
    }
    return w;
}

// kernels.py:513-545 _goldak_pdf_weight
__device__ __forceinline__ float goldak_w(float di, float dj, float dk, float sign, float ff,
                                          float fr, float a_f, float a_r, float b, float c) {
    const float eps = 1e-6f;
    float xt = di * sign;
    bool front = xt >= 0.0f;
    float a = front ? a_f : a_r;
    float frac = front ? ff : fr;
    return frac * waam_expf(-3.0f * ((xt * xt) / (a * a + eps) + (dj * dj) / (b * b + eps) +
                                (dk * dk) / (c * c + eps)));
}

// Arc heat source parameters (physics/arc.py:59-137; kernels.py:443-622).
struct ArcParams {
    int kind;          // 0 = Gaussian2D / conical, 1 = Goldak double ellipsoid
    float arc_i, arc_j, arc_k;
    float inv2s2;      // Gaussian: 1 / (2 sigma^2)
    float sign, ff, fr, a_f, a_r, b, c;  // Goldak
    float pen;
    int enable;
};

// The spatial factor of one cell's arc weight (the Gaussian exponential or the
// Goldak pdf), before the depth weight.
__device__ __forceinline__ float arc_cell_shape(const ArcParams& p, int i, int j, int k) {
    float di = (float)i - p.arc_i, dj = (float)j - p.arc_j, dk = (float)k - p.arc_k;
    if (p.kind == 0) {
        float r2 = di * di + dj * dj + dk * dk * 0.25f;
        return waam_expf(-r2 * p.inv2s2);
    }
    return goldak_w(di, dj, dk, p.sign, p.ff, p.fr, p.a_f, p.a_r, p.b, p.c);
}

// Weight of one cell before normalisation (0 for skipped cells).
__device__ __forceinline__ float arc_cell_weight(const ArcParams& p, int i, int j, int k, int flag,
                                                 float fl) {
    if (flag == GAS) return 0.0f;
    float wd = arc_weight(k, p.arc_k, fl, p.pen, p.enable);
    if (wd < 1e-6f) return 0.0f;
    float di = (float)i - p.arc_i, dj = (float)j - p.arc_j, dk = (float)k - p.arc_k;
    if (p.kind == 0) {
        float r2 = di * di + dj * dj + dk * dk * 0.25f;
        return waam_expf(-r2 * p.inv2s2) * wd;
    }
    float w = goldak_w(di, dj, dk, p.sign, p.ff, p.fr, p.a_f, p.a_r, p.b, p.c);
    return w * wd;
}

// Enthalpy added to one cell: epw * exp(...) * w_dep (Gaussian) or
// epw * w * w_dep (Goldak), reference order.  Returns -1 marker via ok=false
// when the reference skips the cell.
__device__ __forceinline__ bool arc_cell_heat(const ArcParams& p, float epw, int i, int j, int k,
                                              int flag, float fl, float& dh) {
    if (epw <= 0.0f || flag == GAS) return false;
    float wd = arc_weight(k, p.arc_k, fl, p.pen, p.enable);
    if (wd < 1e-6f) return false;
    float di = (float)i - p.arc_i, dj = (float)j - p.arc_j, dk = (float)k - p.arc_k;
    if (p.kind == 0) {
        float r2 = di * di + dj * dj + dk * dk * 0.25f;
        dh = epw * waam_expf(-r2 * p.inv2s2) * wd;
    } else {
        float w = goldak_w(di, dj, dk, p.sign, p.ff, p.fr, p.a_f, p.a_r, p.b, p.c);
        dh = epw * w * wd;
    }
    return true;
}

// Thermal material constants (twin.py:244-274; kernels.py:1519-1556, 1953-1984).
struct PhaseParams {
    float cp_rho, L_rho, Ts, Tl;
    float H_sol, H_liq, cap_l, cap_s;  // derived in reference order
    int cap_enabled;
};

__host__ inline PhaseParams make_phase(float cp_rho, float L_rho, float Ts, float Tl, float T_cap,
                                       int cap_enabled) {
    PhaseParams p;
    p.cp_rho = cp_rho;
    p.L_rho = L_rho;
    p.Ts = Ts;
    p.Tl = Tl;
    p.H_sol = cp_rho * Ts;
    p.H_liq = p.H_sol + L_rho;
    p.cap_l = p.H_liq + cp_rho * (T_cap - Tl);
    p.cap_s = cp_rho * T_cap;
    p.cap_enabled = cap_enabled;
    return p;
}

// ---- temperature-dependent material tables (kernels.py:1686-2010) ----

// Constants of the property refresh (kernels.py:1710-1772): the values of
// SOLID / GAS cells (and of every cell without tables) and the unit factors.
struct TableConsts {
    float rho, dt, dx, force_scale, marangoni_scale;
    float cp_rho_ref, alpha_ref, dgamma_ref, tau_ref;
    int use_tables;
};

// Phase constants of the table path (twin.py:271-273): H_sol, H_liq come
// from cp(T_solidus), not from the per-cell rho*cp.
struct VarPhase {
    float H_sol, H_liq, L_rho, Ts, Tl, T_cap;
};

// kernels.py:1686-1707 lookup_table_1d: clamped to the end knots, linear
// inside; where knots repeat, the last segment containing T wins.  Every
// index is a compile-time constant, so the knots stay in parameter space.
__device__ __forceinline__ float table_lookup(float T, const float (&t)[WAAM_TABLE_KNOTS],
                                              const float (&v)[WAAM_TABLE_KNOTS], int n,
                                              float fallback) {
    float result = fallback;
    if (n > 0) {
        float t_last = t[0], v_last = v[0];
#pragma unroll
        for (int q = 1; q < WAAM_TABLE_KNOTS; ++q) {
            if (q == n - 1) {
                t_last = t[q];
                v_last = v[q];
            }
        }
        if (T <= t[0]) {
            result = v[0];
        } else if (T >= t_last) {
            result = v_last;
        } else {
#pragma unroll
            for (int idx = 0; idx < WAAM_TABLE_KNOTS - 1; ++idx) {
                if (idx < n - 1) {
                    const float t0 = t[idx], t1 = t[idx + 1];
                    if (T >= t0 && T <= t1) {
                        const float w = (T - t0) / (t1 - t0 + 1e-8f);
                        result = v[idx] + w * (v[idx + 1] - v[idx]);
                    }
                }
            }
        }
    }
    return result;
}

struct CellProps {
    float cp_rho, alpha, dgamma, tau;
};

// kernels.py:1710-1772 refresh_thermal_properties for one cell
__device__ __forceinline__ CellProps refresh_cell(const WaamMaterialTables& tb,
                                                  const TableConsts& k, int flag, float T) {
    CellProps p;
    if (flag == SOLID || flag == GAS) {
        p.cp_rho = k.cp_rho_ref;
        p.alpha = k.alpha_ref;
        p.dgamma = k.dgamma_ref;
        p.tau = k.tau_ref;
    } else if (k.use_tables == 1) {
        const float cp = table_lookup(T, tb.cp_T, tb.cp_V, tb.n_cp, tb.cp_fallback);
        const float kv = table_lookup(T, tb.k_T, tb.k_V, tb.n_k, tb.k_fallback);
        const float mu = table_lookup(T, tb.mu_T, tb.mu_V, tb.n_mu, tb.mu_fallback);
        const float dg = table_lookup(T, tb.dgamma_T, tb.dgamma_V, tb.n_dgamma,
                                      tb.dgamma_fallback);
        const float alpha_phys = kv / (k.rho * cp + 1e-9f);
        const float nu_phys = mu / (k.rho + 1e-9f);
        const float nu_lu = nu_phys * k.dt / (k.dx * k.dx);
        p.cp_rho = k.rho * cp;
        p.alpha = alpha_phys * k.dt / (k.dx * k.dx);
        p.dgamma = dg * k.force_scale * k.marangoni_scale;
        p.tau = 3.0f * nu_lu + 0.5f;
    } else {
        p.cp_rho = k.cp_rho_ref;
        p.alpha = k.alpha_ref;
        p.dgamma = k.dgamma_ref * k.marangoni_scale;
        p.tau = k.tau_ref;
    }
    return p;
}

// kernels.py:1988-2010 clamp_enthalpy_ceiling_variable_cp (one non-gas cell)
__device__ __forceinline__ float cap_h_var(const VarPhase& p, float cp_r, float h) {
    const float cap_l = p.H_liq + cp_r * (p.T_cap - p.Tl);
    const float cap_s = cp_r * p.T_cap;
    if (h > p.H_liq) {
        if (h > cap_l) h = cap_l;
    } else {
        if (h > cap_s) h = cap_s;
    }
    return h;
}

// kernels.py:1839-1863 update_phase_variable_cp (one cell)
__device__ __forceinline__ void phase_var(const VarPhase& p, float cp, float h, float& T,
                                          float& fl) {
    if (h <= p.H_sol) {
        fl = 0.0f;
        T = h / (cp + 1e-9f);
    } else if (h >= p.H_liq) {
        fl = 1.0f;
        T = p.Tl + (h - p.H_liq) / (cp + 1e-9f);
    } else {
        const float f = (h - p.H_sol) / p.L_rho;
        fl = f;
        T = p.Ts + f * (p.Tl - p.Ts);
    }
}

// kernels.py:1953-1984 clamp_enthalpy_ceiling_scalar (one cell, non-gas)
__device__ __forceinline__ float cap_h(const PhaseParams& p, float h) {
    if (h > p.H_liq) {
        if (h > p.cap_l) h = p.cap_l;
    } else {
        if (h > p.cap_s) h = p.cap_s;
    }
    return h;
}

// kernels.py:1519-1556 update_phase (one cell)
__device__ __forceinline__ void phase(const PhaseParams& p, float h, float& T, float& fl) {
    if (h <= p.H_sol) {
        fl = 0.0f;
        T = h / p.cp_rho;
    } else if (h >= p.H_liq) {
        fl = 1.0f;
        T = p.Tl + (h - p.H_liq) / p.cp_rho;
    } else {
        float f = (h - p.H_sol) / p.L_rho;
        fl = f;
        T = p.Ts + f * (p.Tl - p.Ts);
    }
}

// kernels.py:1565-1608 _minmod / _limited_upwind_grad
__device__ __forceinline__ float minmod(float a, float b) {
    float out = 0.0f;
    if (a * b > 0.0f) out = fabsf(a) < fabsf(b) ? a : b;
    return out;
}
__device__ __forceinline__ float upwind_grad(float u, float qmm, float qm, float qc, float qp,
                                             float qpp) {
    if (u > 0.0f) {
        float d1 = qc - qm;
        float d2 = 0.5f * (3.0f * qc - 4.0f * qm + qmm);
        return minmod(d1, d2);
    }
    float d1 = qp - qc;
    float d2 = 0.5f * (-3.0f * qc + 4.0f * qp - qpp);
    return minmod(d1, d2);
}

// Enthalpy change of one non-gas cell (kernels.py:1611-1682).  `Hs` is the
// snapshot H (pre-kernel values), `T` the temperature field.
__device__ __forceinline__ float thermal_dh(const Dims d, const float* __restrict__ Hs,
                                            const float* __restrict__ T,
                                            const int32_t* __restrict__ flags, float u, float v,
                                            float w, int i, int j, int k, int flag, float Hc,
                                            float cpa, float dt) {
    auto masked = [&](const float* f, int ii, int jj, int kk, float fb) {
        ii = imax(0, imin(ii, d.nx - 1));
        jj = imax(0, imin(jj, d.ny - 1));
        kk = imax(0, imin(kk, d.nz - 1));
        int c = d.idx(ii, jj, kk);
        float val = f[c];
        if (flags[c] == GAS) val = fb;
        return val;
    };
    float Tc = T[d.idx(i, j, k)];
    float Tim = masked(T, i - 1, j, k, Tc);
    float Tip = masked(T, i + 1, j, k, Tc);
    float Tjm = masked(T, i, j - 1, k, Tc);
    float Tjp = masked(T, i, j + 1, k, Tc);
    float Tkm = masked(T, i, j, k - 1, Tc);
    float Tkp = masked(T, i, j, k + 1, Tc);
    float lap = Tip + Tim + Tjp + Tjm + Tkp + Tkm - 6.0f * Tc;
    float dH = cpa * lap * dt;
    if (flag != SOLID) {
        float Him = masked(Hs, i - 1, j, k, Hc);
        float Hip = masked(Hs, i + 1, j, k, Hc);
        float Himm = masked(Hs, i - 2, j, k, Him);
        float Hipp = masked(Hs, i + 2, j, k, Hip);
        float Hjm = masked(Hs, i, j - 1, k, Hc);
        float Hjp = masked(Hs, i, j + 1, k, Hc);
        float Hjmm = masked(Hs, i, j - 2, k, Hjm);
        float Hjpp = masked(Hs, i, j + 2, k, Hjp);
        float Hkm = masked(Hs, i, j, k - 1, Hc);
        float Hkp = masked(Hs, i, j, k + 1, Hc);
        float Hkmm = masked(Hs, i, j, k - 2, Hkm);
        float Hkpp = masked(Hs, i, j, k + 2, Hkp);
        float gx = upwind_grad(u, Himm, Him, Hc, Hip, Hipp);
        float gy = upwind_grad(v, Hjmm, Hjm, Hc, Hjp, Hjpp);
        float gz = upwind_grad(w, Hkmm, Hkm, Hc, Hkp, Hkpp);
        dH -= (u * gx + v * gy + w * gz) * dt;
    }
    return dH;
}

// thermal_dh with neighbour offsets instead of clamped coordinates (same
// values): a neighbour outside the domain clamps to the cell itself
// (non-gas: the centre value) and a second neighbour outside it to the first
// one.  Every value and its flag are loaded unconditionally and the GAS
// fallback is applied afterwards, so no load waits on another.  Tc = T[c].
__device__ __forceinline__ float thermal_dh_offsets(const Dims& d, const float* __restrict__ Hs,
                                                    const float* __restrict__ T,
                                                    const int32_t* __restrict__ flags, float u,
                                                    float v, float w, int i, int j, int k, int c,
                                                    int flag, float Hc, float Tc, float cpa,
                                                    float dt) {
    const int sx = d.ny * d.nz, sy = d.nz;
    const int cxm = i > 0 ? c - sx : c, cxp = i < d.nx - 1 ? c + sx : c;
    const int cym = j > 0 ? c - sy : c, cyp = j < d.ny - 1 ? c + sy : c;
    const int czm = k > 0 ? c - 1 : c, czp = k < d.nz - 1 ? c + 1 : c;
    const bool gxm = flags[cxm] == GAS, gxp = flags[cxp] == GAS, gym = flags[cym] == GAS;
    const bool gyp = flags[cyp] == GAS, gzm = flags[czm] == GAS, gzp = flags[czp] == GAS;
    const float tim = T[cxm], tip = T[cxp], tjm = T[cym], tjp = T[cyp], tkm = T[czm], tkp = T[czp];
    const float Tim = gxm ? Tc : tim, Tip = gxp ? Tc : tip;
    const float Tjm = gym ? Tc : tjm, Tjp = gyp ? Tc : tjp;
    const float Tkm = gzm ? Tc : tkm, Tkp = gzp ? Tc : tkp;
    float lap = Tip + Tim + Tjp + Tjm + Tkp + Tkm - 6.0f * Tc;
    float dH = cpa * lap * dt;
    if (flag != SOLID) {
        const int cxmm = i >= 2 ? c - 2 * sx : cxm, cxpp = i <= d.nx - 3 ? c + 2 * sx : cxp;
        const int cymm = j >= 2 ? c - 2 * sy : cym, cypp = j <= d.ny - 3 ? c + 2 * sy : cyp;
        const int czmm = k >= 2 ? c - 2 : czm, czpp = k <= d.nz - 3 ? c + 2 : czp;
        const float him = Hs[cxm], hip = Hs[cxp], hjm = Hs[cym], hjp = Hs[cyp];
        const float hkm = Hs[czm], hkp = Hs[czp];
        const float himm = Hs[cxmm], hipp = Hs[cxpp], hjmm = Hs[cymm], hjpp = Hs[cypp];
        const float hkmm = Hs[czmm], hkpp = Hs[czpp];
        const bool gxmm = flags[cxmm] == GAS, gxpp = flags[cxpp] == GAS;
        const bool gymm = flags[cymm] == GAS, gypp = flags[cypp] == GAS;
        const bool gzmm = flags[czmm] == GAS, gzpp = flags[czpp] == GAS;
        const float Him = gxm ? Hc : him, Hip = gxp ? Hc : hip;
        const float Hjm = gym ? Hc : hjm, Hjp = gyp ? Hc : hjp;
        const float Hkm = gzm ? Hc : hkm, Hkp = gzp ? Hc : hkp;
        const float Himm = gxmm ? Him : himm, Hipp = gxpp ? Hip : hipp;
        const float Hjmm = gymm ? Hjm : hjmm, Hjpp = gypp ? Hjp : hjpp;
        const float Hkmm = gzmm ? Hkm : hkmm, Hkpp = gzpp ? Hkp : hkpp;
        float gx = upwind_grad(u, Himm, Him, Hc, Hip, Hipp);
        float gy = upwind_grad(v, Hjmm, Hjm, Hc, Hjp, Hjpp);
        float gz = upwind_grad(w, Hkmm, Hkm, Hc, Hkp, Hkpp);
        dH -= (u * gx + v * gy + w * gz) * dt;
    }
    return dH;
}

// kernels.py:2275-2317 _vof_face_flux
__device__ __forceinline__ float vof_flux(const Dims d, const float* __restrict__ phi,
                                          const float* __restrict__ vel,
                                          const int32_t* __restrict__ flags, int i0, int j0,
                                          int k0, int i1, int j1, int k1) {
    float flux = 0.0f;
    // x is periodic: i0, i1 lie in [-1, nx]
    int ii0 = i0 < 0 ? i0 + d.nx : (i0 >= d.nx ? i0 - d.nx : i0);
    int ii1 = i1 < 0 ? i1 + d.nx : (i1 >= d.nx ? i1 - d.nx : i1);
    bool in0 = j0 >= 0 && k0 >= 0 && j0 < d.ny && k0 < d.nz;
    bool in1 = j1 >= 0 && k1 >= 0 && j1 < d.ny && k1 < d.nz;
    if (in0 && in1) {
        int c0 = d.idx(ii0, j0, k0), c1 = d.idx(ii1, j1, k1);
        int fl0 = flags[c0], fl1 = flags[c1];
        if (fl0 != SOLID && fl1 != SOLID) {
            float u0 = 0.0f, u1 = 0.0f;
            if (fl0 != GAS) u0 = vel[c0];
            if (fl1 != GAS) u1 = vel[c1];
            float uf = 0.5f * (u0 + u1);
            flux = uf > 0.0f ? uf * phi[c0] : uf * phi[c1];
        }
    }
    return flux;
}

// kernels.py:2320-2361 advect_phi for one cell
__device__ __forceinline__ float advect_phi_cell(const Dims d, const float* __restrict__ phi,
                                                 const float* __restrict__ ux,
                                                 const float* __restrict__ uy,
                                                 const float* __restrict__ uz,
                                                 const int32_t* __restrict__ flags, int i, int j,
                                                 int k, int flag) {
    int64_t c = d.idx(i, j, k);
    if (flag == SOLID) return phi[c];
    float fe = vof_flux(d, phi, ux, flags, i, j, k, i + 1, j, k);
    float fw = vof_flux(d, phi, ux, flags, i - 1, j, k, i, j, k);
    float fn = vof_flux(d, phi, uy, flags, i, j, k, i, j + 1, k);
    float fs = vof_flux(d, phi, uy, flags, i, j - 1, k, i, j, k);
    float ft = vof_flux(d, phi, uz, flags, i, j, k, i, j, k + 1);
    float fb = vof_flux(d, phi, uz, flags, i, j, k - 1, i, j, k);
    return phi[c] - (fe - fw) - (fn - fs) - (ft - fb);
}

// kernels.py:2364-2391 reinitialize_phi for one cell
__device__ __forceinline__ float reinit_phi(float p, int flag) {
    if (flag == SOLID) return 1.0f;
    if (flag == GAS) return p < 1e-6f ? 0.0f : fmin_(1.0f, p);
    return fmax_(0.0f, fmin_(1.0f, p));
}

// kernels.py:2394-2419 update_flags_from_phi for one cell
__device__ __forceinline__ int flag_from(float p, float fl, int k, int nz_solid) {
    if (k < nz_solid) return SOLID;
    if (p > 0.85f && fl < 0.05f) return SOLID;
    if (p > 0.55f && fl > 0.1f) return FLUID;
    if (p < 0.05f) return GAS;
    return IFACE;
}

// kernels.py:770-796 _phi_unit_normal_at
__device__ __forceinline__ void phi_normal(const Dims d, const float* __restrict__ phi, int i, int j,
                                           int k, float& nx_, float& ny_, float& nz_, float& g) {
    float dpx = 0.5f * (phi[d.idx(imin(i + 1, d.nx - 1), j, k)] - phi[d.idx(imax(i - 1, 0), j, k)]);
    float dpy = 0.5f * (phi[d.idx(i, imin(j + 1, d.ny - 1), k)] - phi[d.idx(i, imax(j - 1, 0), k)]);
    float dpz = 0.5f * (phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))]);
    float gm = sqrtf(dpx * dpx + dpy * dpy + dpz * dpz);
    nx_ = ny_ = nz_ = 0.0f;
    if (gm >= 1e-6f) {
        nx_ = dpx / gm;
        ny_ = dpy / gm;
        nz_ = dpz / gm;
    }
    g = gm;
}

// kernels.py:800-855 _brackbill_curvature_at: kappa = -div(n) of the unit
// normals of the six neighbours (the centre normal where a neighbour has no
// gradient); g0 = |grad phi| at the cell.  kappa = 0 when g0 < 1e-6.
__device__ __forceinline__ float brackbill_kappa(const Dims d, const float* __restrict__ phi,
                                                 int i, int j, int k, float& g0) {
    const float eps = 1e-6f;
    float n0x, n0y, n0z;
    phi_normal(d, phi, i, j, k, n0x, n0y, n0z, g0);
    float kappa = 0.0f;
    if (g0 >= eps) {
        float a, b, gp, gm, gp2, gm2, gp3, gm3, nxp, nxm, nyp, nym, nzp, nzm;
        phi_normal(d, phi, imin(i + 1, d.nx - 1), j, k, nxp, a, b, gp);
        phi_normal(d, phi, imax(i - 1, 0), j, k, nxm, a, b, gm);
        phi_normal(d, phi, i, imin(j + 1, d.ny - 1), k, a, nyp, b, gp2);
        phi_normal(d, phi, i, imax(j - 1, 0), k, a, nym, b, gm2);
        phi_normal(d, phi, i, j, imin(k + 1, d.nz - 1), a, b, nzp, gp3);
        phi_normal(d, phi, i, j, imax(k - 1, 0), a, b, nzm, gm3);
        if (gp < eps) nxp = n0x;
        if (gm < eps) nxm = n0x;
        if (gp2 < eps) nyp = n0y;
        if (gm2 < eps) nym = n0y;
        if (gp3 < eps) nzp = n0z;
        if (gm3 < eps) nzm = n0z;
        float div_n = 0.5f * (nxp - nxm) + 0.5f * (nyp - nym) + 0.5f * (nzp - nzm);
        kappa = -div_n;
    }
    return kappa;
}

// Force parameters (solvers/coupled_step.py:298-362)
// Shielding-gas shear and vapour recoil (kernels.py:995-1141): the constants
// the reference computes per kernel call, prepared on the host in its float
// order.  recoil: 0 off, 1 the T-ratio form, 2 the Clausius-Clapeyron form.
struct WeldForceParams {
    int gas_shear;
    float gs_tau, gs_scale, gs_inv2s2;        // tau_peak, F(1 Pa), 1 / (2 sigma^2 + eps)
    int recoil;
    float rc_inv2s2;
    float rc_Fpeak, rc_Tref;                  // T-ratio form: F_peak_lu, T_ref
    float rc_LR, rc_invTb, rc_Tboil, rc_CP;   // CC form: L / (R + eps), 1 / (T_boil + eps),
    float rc_rhodx, rc_dt, rc_dx;             //   T_boil, C_acc * P_ref, rho * dx, dt, dx
};

// The constants in the reference's float order (kernels.py:1015, 1033-1035,
// 1072-1086, 1117-1119).
__host__ inline WeldForceParams weld_force_params(int gas_shear, float tau_peak_pa, int recoil,
                                                  float recoil_pa, float T_ref, float P_ref,
                                                  float T_boil, float L_vap, float R_spec,
                                                  float C_acc, float sigma, float dt, float dx,
                                                  float rho_ref) {
    const float eps = 1e-6f;
    WeldForceParams W{};
    W.gas_shear = gas_shear;
    W.gs_tau = tau_peak_pa;
    W.gs_scale = 1.0f / (rho_ref * dx) * dt * dt / dx;
    W.gs_inv2s2 = 1.0f / (2.0f * sigma * sigma + eps);
    W.recoil = recoil;
    W.rc_inv2s2 = W.gs_inv2s2;
    W.rc_Fpeak = (recoil_pa / (rho_ref * dx)) * dt * dt / dx;
    W.rc_Tref = T_ref;
    W.rc_LR = L_vap / (R_spec + eps);
    W.rc_invTb = 1.0f / (T_boil + eps);
    W.rc_Tboil = T_boil;
    W.rc_CP = C_acc * P_ref;
    W.rc_rhodx = rho_ref * dx;
    W.rc_dt = dt;
    W.rc_dx = dx;
    return W;
}

// kernels.py:1094-1141 apply_gas_shear_stress for one non-solid non-gas cell.
__device__ __forceinline__ void gas_shear_cell(const Dims& d, const float* __restrict__ phi,
                                               int i, int j, int k, float arc_i, float arc_j,
                                               const WeldForceParams& W, float& fx, float& fy) {
    const float eps = 1e-6f;
    const float dpx = 0.5f * (phi[d.idx(imin(i + 1, d.nx - 1), j, k)] - phi[d.idx(imax(i - 1, 0), j, k)]);
    const float dpy = 0.5f * (phi[d.idx(i, imin(j + 1, d.ny - 1), k)] - phi[d.idx(i, imax(j - 1, 0), k)]);
    const float dpz = 0.5f * (phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))]);
    const float gmag = sqrtf(dpx * dpx + dpy * dpy + dpz * dpz);
    if (gmag < 0.08f) return;
    const float di = (float)i - arc_i, dj = (float)j - arc_j;
    const float r2 = di * di + dj * dj;
    const float r = sqrtf(r2 + eps);
    const float rx = di / r, ry = dj / r;
    const float nxn = dpx / gmag, nyn = dpy / gmag;
    const float rdotn = rx * nxn + ry * nyn;
    float tx = rx - rdotn * nxn, ty = ry - rdotn * nyn;
    const float tmag = sqrtf(tx * tx + ty * ty + eps);
    tx = tx / tmag;
    ty = ty / tmag;
    const float tau = W.gs_tau * waam_expf(-r2 * W.gs_inv2s2);
    const float Fmag = tau * W.gs_scale;
    fx += Fmag * tx;
    fy += Fmag * ty;
}

// kernels.py:995-1028 (recoil 1) and 1046-1091 (recoil 2) for one non-solid
// non-gas cell with temperature Tc.
__device__ __forceinline__ void recoil_cell(const Dims& d, const float* __restrict__ phi, float Tc,
                                            int i, int j, int k, float arc_i, float arc_j,
                                            const WeldForceParams& W, float& fz) {
    const float eps = 1e-6f;
    const float dpz = phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))];
    if (fabsf(dpz) < 0.05f) return;
    const float di = (float)i - arc_i, dj = (float)j - arc_j;
    const float r2 = di * di + dj * dj;
    if (W.recoil == 1) {
        const float t_ratio = fmin_(Tc / (W.rc_Tref + eps), 3.0f);
        fz += -W.rc_Fpeak * t_ratio * waam_expf(-r2 * W.rc_inv2s2);
    } else {
        if (Tc <= W.rc_Tboil) return;
        float ex = W.rc_LR * (W.rc_invTb - 1.0f / (Tc + eps));
        ex = fmin_(ex, 12.0f);
        const float P_vap = W.rc_CP * waam_expf(ex);
        const float F_peak = P_vap / W.rc_rhodx * W.rc_dt * W.rc_dt / W.rc_dx;
        fz += -F_peak * waam_expf(-r2 * W.rc_inv2s2);
    }
}

struct ForceParams {
    WeldForceParams W;
    int csf, wetting, welding, hydro;
    float gamma_lu, cos_t, sin_t;
    float dgamma;
    float arc_i, arc_j, arc_k, p_inv2s2, p_Flu;
    float g_lu, beta, T_ref, rho_ref;
    float F_cap;
};

// Body force of one non-solid non-gas cell (CSF -> Marangoni -> gas shear ->
// arc pressure -> recoil -> hydrostatic -> buoyancy -> clamp), accumulated on (fx, fy, fz) in the
// reference order (solvers/coupled_step.py:298-362).
__device__ __forceinline__ void cell_forces(const Dims d, const ForceParams& P,
                                            const float* __restrict__ phi,
                                            const float* __restrict__ T,
                                            const int32_t* __restrict__ flags, int i, int j, int k,
                                            float fl, float& fx, float& fy, float& fz) {
    const float eps = 1e-6f;
    int64_t c = d.idx(i, j, k);
    // kernels.py:858-926 compute_csf_tension
    if (P.csf && !(i < 1 || j < 1 || k < 1 || i > d.nx - 2 || j > d.ny - 2 || k > d.nz - 2)) {
        float g0;
        const float kappa = brackbill_kappa(d, phi, i, j, k, g0);
        float gmag = g0;
        if (gmag >= eps) {
            float dpx = 0.5f * (phi[d.idx(imin(i + 1, d.nx - 1), j, k)] - phi[d.idx(imax(i - 1, 0), j, k)]);
            float dpy = 0.5f * (phi[d.idx(i, imin(j + 1, d.ny - 1), k)] - phi[d.idx(i, imax(j - 1, 0), k)]);
            float dpz = 0.5f * (phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))]);
            float sx = P.gamma_lu * kappa * dpx;
            float sy = P.gamma_lu * kappa * dpy;
            float sz = P.gamma_lu * kappa * dpz;
            if (P.wetting != 0) {
                float wx = 0.0f, wy = 0.0f, wz = 0.0f;
                int has_wall = 0;
                if (i > 0 && flags[d.idx(i - 1, j, k)] == SOLID) { wx += 1.0f; has_wall = 1; }
                if (i < d.nx - 1 && flags[d.idx(i + 1, j, k)] == SOLID) { wx -= 1.0f; has_wall = 1; }
                if (j > 0 && flags[d.idx(i, j - 1, k)] == SOLID) { wy += 1.0f; has_wall = 1; }
                if (j < d.ny - 1 && flags[d.idx(i, j + 1, k)] == SOLID) { wy -= 1.0f; has_wall = 1; }
                if (k > 0 && flags[d.idx(i, j, k - 1)] == SOLID) { wz += 1.0f; has_wall = 1; }
                if (k < d.nz - 1 && flags[d.idx(i, j, k + 1)] == SOLID) { wz -= 1.0f; has_wall = 1; }
                float wmag = sqrtf(wx * wx + wy * wy + wz * wz);
                if (wmag > 1e-8f) {
                    wx /= wmag;
                    wy /= wmag;
                    wz /= wmag;
                }
                if (has_wall != 0) {
                    float nxn = dpx / gmag, nyn = dpy / gmag, nzn = dpz / gmag;
                    // kernels.py:723-766 _correct_normal_contact_angle
                    float dot = nxn * wx + nyn * wy + nzn * wz;
                    float tx = nxn - dot * wx, ty = nyn - dot * wy, tz = nzn - dot * wz;
                    float tmag = sqrtf(tx * tx + ty * ty + tz * tz);
                    float ncx = 0.0f, ncy = 0.0f, ncz = 0.0f;
                    if (tmag > 1e-8f) {
                        ncx = P.cos_t * wx + P.sin_t * tx / tmag;
                        ncy = P.cos_t * wy + P.sin_t * ty / tmag;
                        ncz = P.cos_t * wz + P.sin_t * tz / tmag;
                    } else if (fabsf(wz) > 0.5f) {
                        ncx = P.sin_t; ncy = 0.0f; ncz = P.cos_t;
                    } else if (fabsf(wx) > 0.5f) {
                        ncx = P.cos_t; ncy = P.sin_t; ncz = 0.0f;
                    } else {
                        ncx = P.cos_t * wx + P.sin_t; ncy = P.cos_t * wy; ncz = P.cos_t * wz;
                    }
                    float cmag = sqrtf(ncx * ncx + ncy * ncy + ncz * ncz);
                    if (cmag > 1e-8f) {
                        ncx /= cmag;
                        ncy /= cmag;
                        ncz /= cmag;
                    }
                    sx = P.gamma_lu * kappa * ncx * gmag;
                    sy = P.gamma_lu * kappa * ncy * gmag;
                    sz = P.gamma_lu * kappa * ncz * gmag;
                }
            }
            fx += sx;
            fy += sy;
            fz += sz;
        }
    }
    // kernels.py:2158-2217 compute_marangoni_force
    if (!(fl < 0.05f)) {
        int ip = imin(i + 1, d.nx - 1), im = imax(i - 1, 0);
        int jp = imin(j + 1, d.ny - 1), jm = imax(j - 1, 0);
        int kp = imin(k + 1, d.nz - 1), km = imax(k - 1, 0);
        float dx_ = 0.5f * (phi[d.idx(ip, j, k)] - phi[d.idx(im, j, k)]);
        float dy_ = 0.5f * (phi[d.idx(i, jp, k)] - phi[d.idx(i, jm, k)]);
        float dz_ = 0.5f * (phi[d.idx(i, j, kp)] - phi[d.idx(i, j, km)]);
        float g = sqrtf(dx_ * dx_ + dy_ * dy_ + dz_ * dz_);
        if (!(g < 1e-6f)) {
            float nxn = dx_ / g, nyn = dy_ / g, nzn = dz_ / g;
            float tx = 0.5f * (T[d.idx(ip, j, k)] - T[d.idx(im, j, k)]);
            float ty = 0.5f * (T[d.idx(i, jp, k)] - T[d.idx(i, jm, k)]);
            float tz = 0.5f * (T[d.idx(i, j, kp)] - T[d.idx(i, j, km)]);
            float nd = nxn * tx + nyn * ty + nzn * tz;
            float sx = tx - nd * nxn, sy = ty - nd * nyn, sz = tz - nd * nzn;
            float scale = P.dgamma * g;
            fx += scale * sx;
            fy += scale * sy;
            fz += scale * sz;
        }
    }
    // physics/weld_forces.py:161-193 apply_gas_shear (solvers/coupled_step.py:325-326)
    if (P.welding && P.W.gas_shear) gas_shear_cell(d, phi, i, j, k, P.arc_i, P.arc_j, P.W, fx, fy);
    // kernels.py:3038-3083 apply_arc_pressure
    if (P.welding) {
        float dpz = phi[d.idx(i, j, imin(k + 1, d.nz - 1))] - phi[d.idx(i, j, imax(k - 1, 0))];
        if (fabsf(dpz) > 0.05f) {
            float di = (float)i - P.arc_i, dj = (float)j - P.arc_j, dk = (float)k - P.arc_k;
            float r2 = di * di + dj * dj + dk * dk * 0.1f;
            fz += -P.p_Flu * waam_expf(-r2 * P.p_inv2s2);
        }
    }
    // physics/weld_forces.py:137-158 apply_recoil (solvers/coupled_step.py:334)
    if (P.welding && P.W.recoil) recoil_cell(d, phi, T[c], i, j, k, P.arc_i, P.arc_j, P.W, fz);
    // kernels.py:2756-2772 add_hydrostatic_gravity
    if (P.hydro && fl > 0.0f) fz += -P.rho_ref * P.g_lu * fl;
    // kernels.py:2729-2753 add_buoyancy
    if (fl > 0.0f) fz += P.rho_ref * P.g_lu * P.beta * (T[c] - P.T_ref) * fl;
    // kernels.py:3286-3309 clamp_body_force_magnitude
    if (P.F_cap > 0.0f) {
        float mag = sqrtf(fx * fx + fy * fy + fz * fz);
        if (mag > P.F_cap) {
            float s = P.F_cap / (mag + 1e-12f);
            fx = fx * s;
            fy = fy * s;
            fz = fz * s;
        }
    }
}

// cell_forces with every stencil value requested before any is used: the six
// face neighbours of phi, T and flags (clamped at the domain faces, as
// cell_forces clamps them) and, for a CSF cell, the twelve further phi
// values the six neighbour normals of its curvature need.  The expressions,
// operands and order are cell_forces' own, so the forces are identical; the
// loads no longer wait on the branches that consume them (one memory round
// trip instead of one per force term).  c = d.idx(i, j, k).
__device__ __forceinline__ void cell_forces_preloaded(const Dims d, const ForceParams& P,
                                                      const float* __restrict__ phi,
                                                      const float* __restrict__ T,
                                                      const int32_t* __restrict__ flags, int i,
                                                      int j, int k, int c, float fl, float& fx,
                                                      float& fy, float& fz) {
    const float eps = 1e-6f;
    const int sx = d.ny * d.nz, sy = d.nz;
    // face neighbours, clamped to the domain (imin / imax of cell_forces)
    const int cxm = i > 0 ? c - sx : c, cxp = i < d.nx - 1 ? c + sx : c;
    const int cym = j > 0 ? c - sy : c, cyp = j < d.ny - 1 ? c + sy : c;
    const int czm = k > 0 ? c - 1 : c, czp = k < d.nz - 1 ? c + 1 : c;
    const float Pxm = phi[cxm], Pxp = phi[cxp], Pym = phi[cym], Pyp = phi[cyp];
    const float Pzm = phi[czm], Pzp = phi[czp];
    const float Txm = T[cxm], Txp = T[cxp], Tym = T[cym], Typ = T[cyp], Tzm = T[czm], Tzp = T[czp];
    const float Tc = T[c];
    const bool csf = P.csf && !(i < 1 || j < 1 || k < 1 || i > d.nx - 2 || j > d.ny - 2 ||
                                k > d.nz - 2);
    // the curvature's second ring (CSF cells are interior: the first ring is
    // unclamped, the second clamps at the domain faces)
    float P0 = 0.0f, Pxpp = 0.0f, Pxmm = 0.0f, Pypp = 0.0f, Pymm = 0.0f, Pzpp = 0.0f, Pzmm = 0.0f;
    float Pxpyp = 0.0f, Pxpym = 0.0f, Pxmyp = 0.0f, Pxmym = 0.0f, Pxpzp = 0.0f, Pxpzm = 0.0f;
    float Pxmzp = 0.0f, Pxmzm = 0.0f, Pypzp = 0.0f, Pypzm = 0.0f, Pymzp = 0.0f, Pymzm = 0.0f;
    int fxm = FLUID, fxp = FLUID, fym = FLUID, fyp = FLUID, fzm = FLUID, fzp = FLUID;
    if (csf) {
        P0 = phi[c];
        Pxpp = phi[i + 2 <= d.nx - 1 ? c + 2 * sx : c + sx];
        Pxmm = phi[i - 2 >= 0 ? c - 2 * sx : c - sx];
        Pypp = phi[j + 2 <= d.ny - 1 ? c + 2 * sy : c + sy];
        Pymm = phi[j - 2 >= 0 ? c - 2 * sy : c - sy];
        Pzpp = phi[k + 2 <= d.nz - 1 ? c + 2 : c + 1];
        Pzmm = phi[k - 2 >= 0 ? c - 2 : c - 1];
        Pxpyp = phi[c + sx + sy];
        Pxpym = phi[c + sx - sy];
        Pxmyp = phi[c - sx + sy];
        Pxmym = phi[c - sx - sy];
        Pxpzp = phi[c + sx + 1];
        Pxpzm = phi[c + sx - 1];
        Pxmzp = phi[c - sx + 1];
        Pxmzm = phi[c - sx - 1];
        Pypzp = phi[c + sy + 1];
        Pypzm = phi[c + sy - 1];
        Pymzp = phi[c - sy + 1];
        Pymzm = phi[c - sy - 1];
        if (P.wetting != 0) {
            fxm = flags[c - sx];
            fxp = flags[c + sx];
            fym = flags[c - sy];
            fyp = flags[c + sy];
            fzm = flags[c - 1];
            fzp = flags[c + 1];
        }
    }
    // kernels.py:858-926 compute_csf_tension
    if (csf) {
        // _phi_unit_normal_at of the cell and of its six neighbours (phi_normal)
        auto gmag3 = [](float a, float b, float cc) { return sqrtf(a * a + b * b + cc * cc); };
        const float d0x = 0.5f * (Pxp - Pxm), d0y = 0.5f * (Pyp - Pym), d0z = 0.5f * (Pzp - Pzm);
        const float g0 = gmag3(d0x, d0y, d0z);
        float kappa = 0.0f;
        if (g0 >= eps) {
            const float n0x = d0x / g0, n0y = d0y / g0, n0z = d0z / g0;
            // x neighbours: x component of their normal
            float ax = 0.5f * (Pxpp - P0), ay = 0.5f * (Pxpyp - Pxpym), az = 0.5f * (Pxpzp - Pxpzm);
            float g = gmag3(ax, ay, az);
            const float nxp = g < eps ? n0x : ax / g;
            ax = 0.5f * (P0 - Pxmm); ay = 0.5f * (Pxmyp - Pxmym); az = 0.5f * (Pxmzp - Pxmzm);
            g = gmag3(ax, ay, az);
            const float nxm = g < eps ? n0x : ax / g;
            // y neighbours: y component
            ax = 0.5f * (Pxpyp - Pxmyp); ay = 0.5f * (Pypp - P0); az = 0.5f * (Pypzp - Pypzm);
            g = gmag3(ax, ay, az);
            const float nyp = g < eps ? n0y : ay / g;
            ax = 0.5f * (Pxpym - Pxmym); ay = 0.5f * (P0 - Pymm); az = 0.5f * (Pymzp - Pymzm);
            g = gmag3(ax, ay, az);
            const float nym = g < eps ? n0y : ay / g;
            // z neighbours: z component
            ax = 0.5f * (Pxpzp - Pxmzp); ay = 0.5f * (Pypzp - Pymzp); az = 0.5f * (Pzpp - P0);
            g = gmag3(ax, ay, az);
            const float nzp = g < eps ? n0z : az / g;
            ax = 0.5f * (Pxpzm - Pxmzm); ay = 0.5f * (Pypzm - Pymzm); az = 0.5f * (P0 - Pzmm);
            g = gmag3(ax, ay, az);
            const float nzm = g < eps ? n0z : az / g;
            const float div_n = 0.5f * (nxp - nxm) + 0.5f * (nyp - nym) + 0.5f * (nzp - nzm);
            kappa = -div_n;
        }
        const float gmag = g0;
        if (gmag >= eps) {
            const float dpx = 0.5f * (Pxp - Pxm), dpy = 0.5f * (Pyp - Pym), dpz = 0.5f * (Pzp - Pzm);
            float sx_ = P.gamma_lu * kappa * dpx;
            float sy_ = P.gamma_lu * kappa * dpy;
            float sz_ = P.gamma_lu * kappa * dpz;
            if (P.wetting != 0) {
                float wx = 0.0f, wy = 0.0f, wz = 0.0f;
                int has_wall = 0;
                if (fxm == SOLID) { wx += 1.0f; has_wall = 1; }
                if (fxp == SOLID) { wx -= 1.0f; has_wall = 1; }
                if (fym == SOLID) { wy += 1.0f; has_wall = 1; }
                if (fyp == SOLID) { wy -= 1.0f; has_wall = 1; }
                if (fzm == SOLID) { wz += 1.0f; has_wall = 1; }
                if (fzp == SOLID) { wz -= 1.0f; has_wall = 1; }
                float wmag = sqrtf(wx * wx + wy * wy + wz * wz);
                if (wmag > 1e-8f) {
                    wx /= wmag;
                    wy /= wmag;
                    wz /= wmag;
                }
                if (has_wall != 0) {
                    float nxn = dpx / gmag, nyn = dpy / gmag, nzn = dpz / gmag;
                    // kernels.py:723-766 _correct_normal_contact_angle
                    float dot = nxn * wx + nyn * wy + nzn * wz;
                    float tx = nxn - dot * wx, ty = nyn - dot * wy, tz = nzn - dot * wz;
                    float tmag = sqrtf(tx * tx + ty * ty + tz * tz);
                    float ncx = 0.0f, ncy = 0.0f, ncz = 0.0f;
                    if (tmag > 1e-8f) {
                        ncx = P.cos_t * wx + P.sin_t * tx / tmag;
                        ncy = P.cos_t * wy + P.sin_t * ty / tmag;
                        ncz = P.cos_t * wz + P.sin_t * tz / tmag;
                    } else if (fabsf(wz) > 0.5f) {
                        ncx = P.sin_t; ncy = 0.0f; ncz = P.cos_t;
                    } else if (fabsf(wx) > 0.5f) {
                        ncx = P.cos_t; ncy = P.sin_t; ncz = 0.0f;
                    } else {
                        ncx = P.cos_t * wx + P.sin_t; ncy = P.cos_t * wy; ncz = P.cos_t * wz;
                    }
                    float cmag = sqrtf(ncx * ncx + ncy * ncy + ncz * ncz);
                    if (cmag > 1e-8f) {
                        ncx /= cmag;
                        ncy /= cmag;
                        ncz /= cmag;
                    }
                    sx_ = P.gamma_lu * kappa * ncx * gmag;
                    sy_ = P.gamma_lu * kappa * ncy * gmag;
                    sz_ = P.gamma_lu * kappa * ncz * gmag;
                }
            }
            fx += sx_;
            fy += sy_;
            fz += sz_;
        }
    }
    // kernels.py:2158-2217 compute_marangoni_force
    if (!(fl < 0.05f)) {
        float dx_ = 0.5f * (Pxp - Pxm);
        float dy_ = 0.5f * (Pyp - Pym);
        float dz_ = 0.5f * (Pzp - Pzm);
        float g = sqrtf(dx_ * dx_ + dy_ * dy_ + dz_ * dz_);
        if (!(g < 1e-6f)) {
            float nxn = dx_ / g, nyn = dy_ / g, nzn = dz_ / g;
            float tx = 0.5f * (Txp - Txm);
            float ty = 0.5f * (Typ - Tym);
            float tz = 0.5f * (Tzp - Tzm);
            float nd = nxn * tx + nyn * ty + nzn * tz;
            float sx_ = tx - nd * nxn, sy_ = ty - nd * nyn, sz_ = tz - nd * nzn;
            float scale = P.dgamma * g;
            fx += scale * sx_;
            fy += scale * sy_;
            fz += scale * sz_;
        }
    }
    // physics/weld_forces.py:161-193 apply_gas_shear (solvers/coupled_step.py:325-326)
    if (P.welding && P.W.gas_shear) gas_shear_cell(d, phi, i, j, k, P.arc_i, P.arc_j, P.W, fx, fy);
    // kernels.py:3038-3083 apply_arc_pressure
    if (P.welding) {
        float dpz = Pzp - Pzm;
        if (fabsf(dpz) > 0.05f) {
            float di = (float)i - P.arc_i, dj = (float)j - P.arc_j, dk = (float)k - P.arc_k;
            float r2 = di * di + dj * dj + dk * dk * 0.1f;
            fz += -P.p_Flu * waam_expf(-r2 * P.p_inv2s2);
        }
    }
    // physics/weld_forces.py:137-158 apply_recoil (solvers/coupled_step.py:334)
    if (P.welding && P.W.recoil) recoil_cell(d, phi, Tc, i, j, k, P.arc_i, P.arc_j, P.W, fz);
    // kernels.py:2756-2772 add_hydrostatic_gravity
    if (P.hydro && fl > 0.0f) fz += -P.rho_ref * P.g_lu * fl;
    // kernels.py:2729-2753 add_buoyancy
    if (fl > 0.0f) fz += P.rho_ref * P.g_lu * P.beta * (Tc - P.T_ref) * fl;
    // kernels.py:3286-3309 clamp_body_force_magnitude
    if (P.F_cap > 0.0f) {
        float mag = sqrtf(fx * fx + fy * fy + fz * fz);
        if (mag > P.F_cap) {
            float s_ = P.F_cap / (mag + 1e-12f);
            fx = fx * s_;
            fy = fy * s_;
            fz = fz * s_;
        }
    }
}

// cumulant_kernel.py:28-209 collide_mrt for one cell: f (19 pre-collision
// populations) -> out (19 post-collision), macroscopic rho/u.
__device__ __forceinline__ void collide_mrt_cell(const float* f, float fl, float fx, float fy,
                                                 float fz, float omega_s, float omega_b,
                                                 float C_darcy, float* out, float& r, float& u,
                                                 float& v, float& w) {
    const float cs2 = 1.0f / 3.0f, eps = 1.0e-6f;
    const float w0 = 0.333333343f, w1 = 0.0555555560f, w2 = 0.0277777780f;
    r = f[0];
#pragma unroll
    for (int q = 1; q < 19; ++q) r = r + f[q];
    float inv_rho = 1.0f / (r + eps);
    float jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
    float jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
    float jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
    float uxr = (jx + 0.5f * fx) * inv_rho;
    float uyr = (jy + 0.5f * fy) * inv_rho;
    float uzr = (jz + 0.5f * fz) * inv_rho;
    float om = 1.0f - fl;
    float ck = 1.0f + C_darcy * (om * om) / (fl * fl * fl + eps);
    u = uxr / ck;
    v = uyr / ck;
    w = uzr / ck;
    float Pxx = f[1] + f[2] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14];
    float Pyy = f[3] + f[4] + f[7] + f[8] + f[9] + f[10] + f[15] + f[16] + f[17] + f[18];
    float Pzz = f[5] + f[6] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    float Pxy = f[7] + f[8] - f[9] - f[10];
    float Pxz = f[11] + f[12] - f[13] - f[14];
    float Pyz = f[15] + f[16] - f[17] - f[18];
    float kxx = Pxx - r * u * u, kyy = Pyy - r * v * v, kzz = Pzz - r * w * w;
    float kxy = Pxy - r * u * v, kxz = Pxz - r * u * w, kyz = Pyz - r * v * w;
    float km = (kxx + kyy + kzz) / 3.0f;
    float kmp = km - omega_b * (km - r * cs2);
    float kxxp = kmp + (1.0f - omega_s) * (kxx - km);
    float kyyp = kmp + (1.0f - omega_s) * (kyy - km);
    float kzzp = kmp + (1.0f - omega_s) * (kzz - km);
    float kxyp = kxy - omega_s * kxy;
    float kxzp = kxz - omega_s * kxz;
    float kyzp = kyz - omega_s * kyz;
    float u2 = u * u + v * v + w * w;
    float uF = u * fx + v * fy + w * fz;
    float ax = kxxp - r * cs2, ay = kyyp - r * cs2, az = kzzp - r * cs2;
    float r3 = r * 3.0f, r9h = r * 3.0f * 3.0f * 0.5f, rd = r * 0.5f * 3.0f * u2;
    float oms = 1.0f - 0.5f * omega_s;
    float Kxy = ax + ay, Kxz = ax + az, Kyz = ay + az;
    float txy = 2.0f * kxyp, txz = 2.0f * kxzp, tyz = 2.0f * kyzp;
    float bxy = -2.0f * kxyp, bxz = -2.0f * kxzp, byz = -2.0f * kyzp;
#define WAAM_FEQ(Q, WQ, EU, FE, K)                                                   \
    {                                                                                \
        float eu_ = (EU), fe_ = (FE);                                                \
        float feq_ = WQ * (r + r3 * eu_ + r9h * eu_ * eu_ - rd + 4.5f * (K));       \
        float s_ = WQ * oms * (3.0f * fe_ + 9.0f * fe_ * eu_ - 3.0f * uF);           \
        out[Q] = feq_ + s_;                                                          \
    }
    WAAM_FEQ(0, w0, 0.0f, 0.0f, 0.0f)
    WAAM_FEQ(1, w1, u, fx, ax)
    WAAM_FEQ(2, w1, -u, -fx, ax)
    WAAM_FEQ(3, w1, v, fy, ay)
    WAAM_FEQ(4, w1, -v, -fy, ay)
    WAAM_FEQ(5, w1, w, fz, az)
    WAAM_FEQ(6, w1, -w, -fz, az)
    WAAM_FEQ(7, w2, u + v, fx + fy, Kxy + txy)
    WAAM_FEQ(8, w2, -u + -v, -fx + -fy, Kxy + txy)
    WAAM_FEQ(9, w2, u + -v, fx + -fy, Kxy + bxy)
    WAAM_FEQ(10, w2, -u + v, -fx + fy, Kxy + bxy)
    WAAM_FEQ(11, w2, u + w, fx + fz, Kxz + txz)
    WAAM_FEQ(12, w2, -u + -w, -fx + -fz, Kxz + txz)
    WAAM_FEQ(13, w2, u + -w, fx + -fz, Kxz + bxz)
    WAAM_FEQ(14, w2, -u + w, -fx + fz, Kxz + bxz)
    WAAM_FEQ(15, w2, v + w, fy + fz, Kyz + tyz)
    WAAM_FEQ(16, w2, -v + -w, -fy + -fz, Kyz + tyz)
    WAAM_FEQ(17, w2, v + -w, fy + -fz, Kyz + byz)
    WAAM_FEQ(18, w2, -v + w, -fy + fz, Kyz + byz)
#undef WAAM_FEQ
}

// kernels.py:2778-2885 collide_srt for one cell
__device__ __forceinline__ void collide_srt_cell(const float* f, float fl, float fx, float fy,
                                                 float fz, float omega, float C_darcy, float* out,
                                                 float& r, float& u, float& v, float& w) {
    const float eps = 1e-6f;
    r = 0.0f;
    float jx = 0.0f, jy = 0.0f, jz = 0.0f;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float fq = f[q];
        r += fq;
        jx += fq * (float)ex(q);
        jy += fq * (float)ey(q);
        jz += fq * (float)ez(q);
    }
    float inv_r = 1.0f / (r + eps);
    float uxr = jx * inv_r + 0.5f * fx * inv_r;
    float uyr = jy * inv_r + 0.5f * fy * inv_r;
    float uzr = jz * inv_r + 0.5f * fz * inv_r;
    float om = 1.0f - fl;
    float ck = 1.0f + C_darcy * (om * om) / (fl * fl * fl + eps);
    u = uxr / ck;
    v = uyr / ck;
    w = uzr / ck;
    float u2 = u * u + v * v + w * w;
#pragma unroll
    for (int q = 0; q < 19; ++q) {
        float eu = (float)ex(q) * u + (float)ey(q) * v + (float)ez(q) * w;
        float wqq = wq(q);
        float feq = wqq * r * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
        float Fe = (float)ex(q) * fx + (float)ey(q) * fy + (float)ez(q) * fz;
        float S = wqq * (1.0f - 0.5f * omega) *
                  (3.0f * Fe + 9.0f * (eu * Fe) - 3.0f * (u * fx + v * fy + w * fz));
        out[q] = f[q] - omega * (f[q] - feq) + S;
    }
}

// kernels.py:3312-3335 clamp_velocity_mach for one cell
__device__ __forceinline__ void clamp_mach(float& u, float& v, float& w, float umax) {
    float mag = sqrtf(u * u + v * v + w * w);
    if (mag > umax) {
        float s = umax / (mag + 1e-12f);
        u = u * s;
        v = v * s;
        w = w * s;
    }
}

}  // namespace waam
