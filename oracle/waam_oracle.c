/* CPU oracle for the waam_twin coupled melt-pool step -- TEST INFRASTRUCTURE.
 *
 * Plain float32 C restatement of the reference's Taichi kernels.  Each
 * function cites the reference file:line it follows and keeps the
 * reference's expression order (left-to-right float32 evaluation), so that
 * with -ffp-contract=off it reproduces a serial float32 execution of the
 * reference source up to the rounding of exp/sin/cos.  Parallel loops
 * (OpenMP) are used only where every cell writes only itself.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef WAAM_ORACLE_FP64
/* FP64 build (make fp64): every float of this file and of waam_oracle.h is a
 * double and the exponential is the C library's -- the double-precision run
 * that the reduced-precision population storage is measured against. */
#define float double
#define sqrtf sqrt
#define fabsf fabs
#define waam_expf exp
#include "waam_oracle.h"
#else
#include "waam_oracle.h"
/* The same float exponential the CUDA kernels use (Cody-Waite + Taylor), so
 * that exp rounding does not blur the oracle/GPU comparison. */
#include "../waam_solver_b200/csrc/waam_expf.h"
#endif

#define FLUID 0
#define SOLID 1
#define GAS 2
#define IFACE 4

static const int EX[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
static const int EY[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
static const int EZ[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int OPP[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
/* kernels.py:45-50: Python floats 1/3, 1/18, 1/36 rounded to float32. */
static float WQ(int q) { return q == 0 ? (float)(1.0 / 3.0) : (q < 7 ? (float)(1.0 / 18.0) : (float)(1.0 / 36.0)); }

#define IX(i, j, k) (((int64_t)(i) * ny + (j)) * nz + (k))

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline float fminf_(float a, float b) { return a < b ? a : b; }
static inline float fmaxf_(float a, float b) { return a > b ? a : b; }

/* Exposes the shared exponential for accuracy tests. */
void wo_expf_array(const float* x, float* y, int64_t n) {
    for (int64_t i = 0; i < n; ++i) y[i] = waam_expf(x[i]);
}

int wo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void wo_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* kernels.py:62-120 init_grid */
void wo_init_grid(float* f, float* rho, float* ux, float* uy, float* uz, float* T, float* H,
                  float* f_l, float* phi, int32_t* flags, int nx, int ny, int nz, float T_amb,
                  float rho0, float cp_rho, int nz_solid, int pi0, int pi1, int pj0, int pj1) {
    int64_t n = (int64_t)nx * ny * nz;
    for (int q = 0; q < 19; ++q)
        for (int64_t c = 0; c < n; ++c) f[q * n + c] = WQ(q) * rho0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
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
                    int in_plate = i >= pi0 && i < pi1 && j >= pj0 && j < pj1;
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

/* kernels.py:161-170 clear_forces */
void wo_clear_forces(float* Fx, float* Fy, float* Fz, int64_t n) {
    memset(Fx, 0, n * sizeof(float));
    memset(Fy, 0, n * sizeof(float));
    memset(Fz, 0, n * sizeof(float));
}

/* kernels.py:406-437 arc_deposition_weight */
static float arc_weight(int k, float arc_k, float fl, float pen, int enable) {
    float w = 1.0f;
    if (enable == 1) {
        if (fl > 0.55f) {
            w = 1.0f;
        } else {
            float dz = arc_k - (float)k;
            if (dz < -0.5f) {
                w = 0.0f;
            } else {
                float depth = fmaxf_(0.0f, dz);
                float inv_pen = 1.0f / (pen + 1e-6f);
                w = waam_expf(-depth * inv_pen);
            }
        }
    }
    return w;
}

/* kernels.py:443-510 inject_arc_heat (Gaussian2D, physics/arc.py:63-72).
 * The weight sum is accumulated in double (the reference's float atomic sum
 * has no defined order).  Returns the weight sum. */
double wo_inject_arc_heat(float* H, const int32_t* flags, const float* f_l, int nx, int ny, int nz,
                          float arc_i, float arc_j, float arc_k, float Q_w, float sigma, float dt,
                          float dx3, float eta, float pen, int enable) {
    float inv2s2 = 1.0f / (2.0f * sigma * sigma);
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                float wd = arc_weight(k, arc_k, f_l[c], pen, enable);
                if (wd < 1e-6f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float r2 = di * di + dj * dj + dk * dk * 0.25f;
                acc += (double)(waam_expf(-r2 * inv2s2) * wd);
            }
    float w_total = (float)acc;
    float epw = 0.0f;
    if (w_total > 1e-9f) epw = Q_w * eta * dt / (w_total * dx3);
    if (epw <= 0.0f) return acc;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                float wd = arc_weight(k, arc_k, f_l[c], pen, enable);
                if (wd < 1e-6f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float r2 = di * di + dj * dj + dk * dk * 0.25f;
                H[c] += epw * waam_expf(-r2 * inv2s2) * wd;
            }
    return acc;
}

/* kernels.py:513-545 _goldak_pdf_weight */
static float goldak_w(float di, float dj, float dk, float sign, float ff, float fr, float a_f,
                      float a_r, float b, float c) {
    const float eps = 1e-6f;
    float xt = di * sign;
    int front = xt >= 0.0f;
    float a = front ? a_f : a_r;
    float frac = front ? ff : fr;
    return frac * waam_expf(-3.0f * ((xt * xt) / (a * a + eps) + (dj * dj) / (b * b + eps) +
                                (dk * dk) / (c * c + eps)));
}

/* kernels.py:548-622 inject_goldak_heat (physics/arc.py:106-119) */
double wo_inject_goldak_heat(float* H, const int32_t* flags, const float* f_l, int nx, int ny,
                             int nz, float arc_i, float arc_j, float arc_k, float Q_w, float dt,
                             float dx3, float eta, float sign, float ff, float fr, float a_f,
                             float a_r, float b, float c, float pen, int enable) {
    double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t cc = IX(i, j, k);
                if (flags[cc] == GAS) continue;
                float wd = arc_weight(k, arc_k, f_l[cc], pen, enable);
                if (wd < 1e-6f) continue;
                float w = goldak_w((float)i - arc_i, (float)j - arc_j, (float)k - arc_k, sign, ff,
                                   fr, a_f, a_r, b, c);
                acc += (double)(w * wd);
            }
    float w_total = (float)acc;
    float epw = 0.0f;
    if (w_total > 1e-9f) epw = Q_w * eta * dt / (w_total * dx3);
    if (epw <= 0.0f) return acc;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t cc = IX(i, j, k);
                if (flags[cc] == GAS) continue;
                float wd = arc_weight(k, arc_k, f_l[cc], pen, enable);
                if (wd < 1e-6f) continue;
                float w = goldak_w((float)i - arc_i, (float)j - arc_j, (float)k - arc_k, sign, ff,
                                   fr, a_f, a_r, b, c);
                H[cc] += epw * w * wd;
            }
    return acc;
}

/* kernels.py:1953-1984 clamp_enthalpy_ceiling_scalar */
void wo_clamp_enthalpy_ceiling_scalar(float* H, const int32_t* flags, int64_t n, float cp_rho,
                                      float Ts, float Tl, float T_cap, float L_rho) {
    float H_sol = cp_rho * Ts;
    float H_liq = H_sol + L_rho;
    float cap_l = H_liq + cp_rho * (T_cap - Tl);
    float cap_s = cp_rho * T_cap;
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        float h = H[c];
        if (h > H_liq) {
            if (h > cap_l) H[c] = cap_l;
        } else {
            if (h > cap_s) H[c] = cap_s;
        }
    }
}

/* kernels.py:1565-1571 _minmod */
static inline float minmod(float a, float b) {
    float out = 0.0f;
    if (a * b > 0.0f) out = fabsf(a) < fabsf(b) ? a : b;
    return out;
}

/* kernels.py:1593-1608 _limited_upwind_grad */
static inline float upwind_grad(float u, float qmm, float qm, float qc, float qp, float qpp) {
    if (u > 0.0f) {
        float d1 = qc - qm;
        float d2 = 0.5f * (3.0f * qc - 4.0f * qm + qmm);
        return minmod(d1, d2);
    }
    float d1 = qp - qc;
    float d2 = 0.5f * (-3.0f * qc + 4.0f * qp - qpp);
    return minmod(d1, d2);
}

/* kernels.py:1574-1590 _masked_at */
static inline float masked(const float* fld, const int32_t* flags, int nx, int ny, int nz, int i,
                           int j, int k, float fallback) {
    int ii = imax(0, imin(i, nx - 1)), jj = imax(0, imin(j, ny - 1)), kk = imax(0, imin(k, nz - 1));
    int64_t c = IX(ii, jj, kk);
    float v = fld[c];
    if (flags[c] == GAS) v = fallback;
    return v;
}

/* kernels.py:1611-1682 advect_diffuse_temperature, snapshot semantics on H */
static void advect_diffuse_impl(float* H, const float* T, const float* ux, const float* uy,
                                const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                float alpha_lu, float dt, float cp_rho, const float* alpha_f,
                                const float* cp_f);

void wo_advect_diffuse_temperature(float* H, const float* T, const float* ux, const float* uy,
                                   const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                   float alpha_lu, float dt, float cp_rho) {
    advect_diffuse_impl(H, T, ux, uy, uz, flags, nx, ny, nz, alpha_lu, dt, cp_rho, NULL, NULL);
}

/* kernels.py:1775-1836 advect_diffuse_temperature_variable: the same scheme
 * with the cell's own cp*rho and alpha_lu */
void wo_advect_diffuse_temperature_variable(float* H, const float* T, const float* ux,
                                            const float* uy, const float* uz,
                                            const int32_t* flags, const float* alpha_f,
                                            const float* cp_f, int nx, int ny, int nz, float dt) {
    advect_diffuse_impl(H, T, ux, uy, uz, flags, nx, ny, nz, 0.0f, dt, 0.0f, alpha_f, cp_f);
}

static void advect_diffuse_impl(float* H, const float* T, const float* ux, const float* uy,
                                const float* uz, const int32_t* flags, int nx, int ny, int nz,
                                float alpha_lu, float dt, float cp_rho, const float* alpha_f,
                                const float* cp_f) {
    int64_t n = (int64_t)nx * ny * nz;
    float* H0 = (float*)malloc(n * sizeof(float));
    memcpy(H0, H, n * sizeof(float));
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                int flag = flags[c];
                if (flag == GAS) continue;
                float Tc = T[c], Hc = H0[c];
                float Tim = masked(T, flags, nx, ny, nz, i - 1, j, k, Tc);
                float Tip = masked(T, flags, nx, ny, nz, i + 1, j, k, Tc);
                float Tjm = masked(T, flags, nx, ny, nz, i, j - 1, k, Tc);
                float Tjp = masked(T, flags, nx, ny, nz, i, j + 1, k, Tc);
                float Tkm = masked(T, flags, nx, ny, nz, i, j, k - 1, Tc);
                float Tkp = masked(T, flags, nx, ny, nz, i, j, k + 1, Tc);
                float lap = Tip + Tim + Tjp + Tjm + Tkp + Tkm - 6.0f * Tc;
                float cr = cp_f ? cp_f[c] : cp_rho, al = alpha_f ? alpha_f[c] : alpha_lu;
                float dH = cr * al * lap * dt;
                if (flag != SOLID) {
                    float u = ux[c], v = uy[c], w = uz[c];
                    float Him = masked(H0, flags, nx, ny, nz, i - 1, j, k, Hc);
                    float Hip = masked(H0, flags, nx, ny, nz, i + 1, j, k, Hc);
                    float Himm = masked(H0, flags, nx, ny, nz, i - 2, j, k, Him);
                    float Hipp = masked(H0, flags, nx, ny, nz, i + 2, j, k, Hip);
                    float Hjm = masked(H0, flags, nx, ny, nz, i, j - 1, k, Hc);
                    float Hjp = masked(H0, flags, nx, ny, nz, i, j + 1, k, Hc);
                    float Hjmm = masked(H0, flags, nx, ny, nz, i, j - 2, k, Hjm);
                    float Hjpp = masked(H0, flags, nx, ny, nz, i, j + 2, k, Hjp);
                    float Hkm = masked(H0, flags, nx, ny, nz, i, j, k - 1, Hc);
                    float Hkp = masked(H0, flags, nx, ny, nz, i, j, k + 1, Hc);
                    float Hkmm = masked(H0, flags, nx, ny, nz, i, j, k - 2, Hkm);
                    float Hkpp = masked(H0, flags, nx, ny, nz, i, j, k + 2, Hkp);
                    float gx = upwind_grad(u, Himm, Him, Hc, Hip, Hipp);
                    float gy = upwind_grad(v, Hjmm, Hjm, Hc, Hjp, Hjpp);
                    float gz = upwind_grad(w, Hkmm, Hkm, Hc, Hkp, Hkpp);
                    dH -= (u * gx + v * gy + w * gz) * dt;
                }
                H[c] = Hc + dH;
            }
    free(H0);
}

/* kernels.py:1519-1556 update_phase */
void wo_update_phase(const float* H, float* T, float* f_l, int64_t n, float cp_rho, float L_rho,
                     float Ts, float Tl) {
    float H_sol = cp_rho * Ts;
    float H_liq = H_sol + L_rho;
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        float h = H[c];
        if (h <= H_sol) {
            f_l[c] = 0.0f;
            T[c] = h / cp_rho;
        } else if (h >= H_liq) {
            f_l[c] = 1.0f;
            T[c] = Tl + (h - H_liq) / cp_rho;
        } else {
            float fl = (h - H_sol) / L_rho;
            f_l[c] = fl;
            T[c] = Ts + fl * (Tl - Ts);
        }
    }
}

/* kernels.py:3016-3032 update_T_max */
void wo_update_T_max(const float* T, float* T_max, const int32_t* flags, int64_t n) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        if (T[c] > T_max[c]) T_max[c] = T[c];
    }
}

/* kernels.py:2013-2027 update_cooling_rate */
void wo_update_cooling_rate(const float* T, float* T_prev, float* dT_dt, const int32_t* flags,
                            int64_t n, float dt_phys) {
    float inv_dt = 1.0f / (dt_phys + 1e-12f);
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        dT_dt[c] = (T[c] - T_prev[c]) * inv_dt;
        T_prev[c] = T[c];
    }
}

/* kernels.py:2030-2082 apply_thermal_boundary_losses */
void wo_apply_thermal_boundary_losses(float* H, const float* T, const int32_t* flags, int nx,
                                      int ny, int nz, float T_amb, float h_conv, float eps_rad,
                                      int conv, int rad, float dt, float dx, float sigma_sb) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                int ne = 0;
                if (k + 1 < nz && flags[IX(i, j, k + 1)] == GAS) ne++;
                if (j + 1 < ny && flags[IX(i, j + 1, k)] == GAS) ne++;
                if (j - 1 >= 0 && flags[IX(i, j - 1, k)] == GAS) ne++;
                if (i + 1 < nx && flags[IX(i + 1, j, k)] == GAS) ne++;
                if (i - 1 >= 0 && flags[IX(i - 1, j, k)] == GAS) ne++;
                if (ne == 0) continue;
                float Te = fminf_(T[c], 2500.0f);
                float q = 0.0f;
                if (conv == 1) q += h_conv * (Te - T_amb);
                if (rad == 1) {
                    float t4 = Te * Te * Te * Te;
                    float a4 = T_amb * T_amb * T_amb * T_amb;
                    q += eps_rad * sigma_sb * (t4 - a4);
                }
                H[c] -= q * (float)ne * dt / dx;
            }
}

/* kernels.py:1937-1950 clamp_enthalpy_floor_scalar */
void wo_clamp_enthalpy_floor_scalar(float* H, float cp_rho, const int32_t* flags, int64_t n,
                                    float T_floor) {
    float h_min = cp_rho * T_floor;
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        if (H[c] < h_min) H[c] = h_min;
    }
}

/* kernels.py:2275-2317 _vof_face_flux */
static inline float vof_flux(const float* phi, const float* vel, const int32_t* flags, int nx,
                             int ny, int nz, int i0, int j0, int k0, int i1, int j1, int k1) {
    float flux = 0.0f;
    int ii0 = (i0 + nx) % nx, ii1 = (i1 + nx) % nx;
    int in0 = j0 >= 0 && k0 >= 0 && j0 < ny && k0 < nz;
    int in1 = j1 >= 0 && k1 >= 0 && j1 < ny && k1 < nz;
    if (in0 && in1) {
        int64_t c0 = IX(ii0, j0, k0), c1 = IX(ii1, j1, k1);
        int fl0 = flags[c0], fl1 = flags[c1];
        if (fl0 != SOLID && fl1 != SOLID) {
            float u0 = 0.0f, u1 = 0.0f;
            if (fl0 != GAS) u0 = vel[c0];
            if (fl1 != GAS) u1 = vel[c1];
            float uf = 0.5f * (u0 + u1);
            if (uf > 0.0f)
                flux = uf * phi[c0];
            else
                flux = uf * phi[c1];
        }
    }
    return flux;
}

/* kernels.py:2320-2361 advect_phi */
void wo_advect_phi(float* phi_dst, const float* phi_src, const float* ux, const float* uy,
                   const float* uz, const int32_t* flags, int nx, int ny, int nz) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID) {
                    phi_dst[c] = phi_src[c];
                    continue;
                }
                float fe = vof_flux(phi_src, ux, flags, nx, ny, nz, i, j, k, i + 1, j, k);
                float fw = vof_flux(phi_src, ux, flags, nx, ny, nz, i - 1, j, k, i, j, k);
                float fn = vof_flux(phi_src, uy, flags, nx, ny, nz, i, j, k, i, j + 1, k);
                float fs = vof_flux(phi_src, uy, flags, nx, ny, nz, i, j - 1, k, i, j, k);
                float ft = vof_flux(phi_src, uz, flags, nx, ny, nz, i, j, k, i, j, k + 1);
                float fb = vof_flux(phi_src, uz, flags, nx, ny, nz, i, j, k - 1, i, j, k);
                phi_dst[c] = phi_src[c] - (fe - fw) - (fn - fs) - (ft - fb);
            }
}

/* kernels.py:2364-2391 reinitialize_phi */
void wo_reinitialize_phi(float* phi, const int32_t* flags, int64_t n) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        int flag = flags[c];
        if (flag == SOLID) {
            phi[c] = 1.0f;
        } else if (flag == GAS) {
            if (phi[c] < 1e-6f)
                phi[c] = 0.0f;
            else
                phi[c] = fminf_(1.0f, phi[c]);
        } else {
            float p = phi[c];
            phi[c] = fmaxf_(0.0f, fminf_(1.0f, p));
        }
    }
}

/* kernels.py:933-991 apply_contact_angle_phi_bc.  Sequential in k inside a
 * column; reads of other columns see the pre-kernel snapshot. */
void wo_apply_contact_angle_phi_bc(float* phi, const int32_t* flags, int nx, int ny, int nz,
                                   float theta) {
    int64_t n = (int64_t)nx * ny * nz;
    float* P0 = (float*)malloc(n * sizeof(float));
    memcpy(P0, phi, n * sizeof(float));
    float cos_t = (float)cos((double)theta), sin_t = (float)sin((double)theta);
    float film = 0.5f * (1.0f - cos_t);
    float spread = film * (0.85f + 0.15f * sin_t);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID) continue;
                int below_solid = k > 0 && flags[IX(i, j, k - 1)] == SOLID;
                if (below_solid && flags[c] == GAS) {
                    if (phi[c] < film) phi[c] = film;
                }
                if (below_solid && phi[c] > 0.55f) {
                    if (k + 1 < nz && flags[IX(i, j, k + 1)] == GAS) {
                        float g = phi[c] - sin_t;
                        g = fmaxf_(film, fminf_(g, 0.98f));
                        if (phi[IX(i, j, k + 1)] < g) phi[IX(i, j, k + 1)] = g;
                    }
                }
                if (k > 0 && phi[IX(i, j, k - 1)] > 0.55f && flags[c] == GAS) {
                    float t = phi[IX(i, j, k - 1)] - sin_t;
                    t = fmaxf_(film, fminf_(t, 0.95f));
                    if (phi[c] < t) phi[c] = t;
                }
                if (phi[c] < 0.45f) {
                    for (int d = -1; d <= 1; d += 2) {
                        int jj = j + d;
                        if (jj >= 0 && jj < ny && P0[IX(i, jj, k)] > 0.55f)
                            if (phi[c] < spread) phi[c] = spread;
                    }
                    for (int d = -1; d <= 1; d += 2) {
                        int ii = i + d;
                        if (ii >= 0 && ii < nx && P0[IX(ii, j, k)] > 0.55f)
                            if (phi[c] < spread) phi[c] = spread;
                    }
                }
                if (below_solid && phi[c] > 0.2f) {
                    if (phi[c] < 0.65f) phi[c] = 0.65f;
                }
            }
    free(P0);
}

/* kernels.py:2394-2419 update_flags_from_phi */
void wo_update_flags_from_phi(const float* phi, const float* f_l, int32_t* flags, int nx, int ny,
                              int nz, int nz_solid) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (k < nz_solid) {
                    flags[c] = SOLID;
                    continue;
                }
                float p = phi[c], fl = f_l[c];
                if (p > 0.85f && fl < 0.05f)
                    flags[c] = SOLID;
                else if (p > 0.55f && fl > 0.1f)
                    flags[c] = FLUID;
                else if (p < 0.05f)
                    flags[c] = GAS;
                else
                    flags[c] = IFACE;
            }
}

/* kernels.py:3484-3504 sync_phi_liquid_fraction */
void wo_sync_phi_liquid_fraction(const float* phi, float* f_l, const int32_t* flags, int64_t n) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        int fl = flags[c];
        if (fl == GAS || phi[c] < 0.05f)
            f_l[c] = 0.0f;
        else if (fl == SOLID)
            f_l[c] = 0.0f;
    }
}

/* kernels.py:770-796 _phi_unit_normal_at */
static inline void phi_normal(const float* phi, int nx, int ny, int nz, int i, int j, int k,
                              float* nxn, float* nyn, float* nzn, float* g) {
    float dpx = 0.5f * (phi[IX(imin(i + 1, nx - 1), j, k)] - phi[IX(imax(i - 1, 0), j, k)]);
    float dpy = 0.5f * (phi[IX(i, imin(j + 1, ny - 1), k)] - phi[IX(i, imax(j - 1, 0), k)]);
    float dpz = 0.5f * (phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))]);
    float gm = sqrtf(dpx * dpx + dpy * dpy + dpz * dpz);
    *nxn = *nyn = *nzn = 0.0f;
    if (gm >= 1e-6f) {
        *nxn = dpx / gm;
        *nyn = dpy / gm;
        *nzn = dpz / gm;
    }
    *g = gm;
}

/* kernels.py:800-855 _brackbill_curvature_at: -div of the neighbours' unit
 * normals (the centre normal where a neighbour has no gradient) */
static float brackbill_kappa(const float* phi, int nx, int ny, int nz, int i, int j, int k,
                             float* g0) {
    const float eps = 1e-6f;
    float n0x, n0y, n0z;
    phi_normal(phi, nx, ny, nz, i, j, k, &n0x, &n0y, &n0z, g0);
    float kappa = 0.0f;
    if (*g0 >= eps) {
        float a, b, gp, gm, gp2, gm2, gp3, gm3, nxp, nxm, nyp, nym, nzp, nzm;
        phi_normal(phi, nx, ny, nz, imin(i + 1, nx - 1), j, k, &nxp, &a, &b, &gp);
        phi_normal(phi, nx, ny, nz, imax(i - 1, 0), j, k, &nxm, &a, &b, &gm);
        phi_normal(phi, nx, ny, nz, i, imin(j + 1, ny - 1), k, &a, &nyp, &b, &gp2);
        phi_normal(phi, nx, ny, nz, i, imax(j - 1, 0), k, &a, &nym, &b, &gm2);
        phi_normal(phi, nx, ny, nz, i, j, imin(k + 1, nz - 1), &a, &b, &nzp, &gp3);
        phi_normal(phi, nx, ny, nz, i, j, imax(k - 1, 0), &a, &b, &nzm, &gm3);
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

/* kernels.py:858-926 compute_csf_tension (+ 681-855 helpers) */
void wo_compute_csf_tension(const float* phi, const int32_t* flags, float* Fx, float* Fy,
                            float* Fz, int nx, int ny, int nz, float gamma_lu, int wetting,
                            float theta) {
    const float eps = 1e-6f;
    float cos_t = (float)cos((double)theta), sin_t = (float)sin((double)theta);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                if (i < 1 || j < 1 || k < 1 || i > nx - 2 || j > ny - 2 || k > nz - 2) continue;
                float g0;
                float kappa = brackbill_kappa(phi, nx, ny, nz, i, j, k, &g0);
                float gmag = g0;
                if (gmag < eps) continue;
                float dpx = 0.5f * (phi[IX(imin(i + 1, nx - 1), j, k)] - phi[IX(imax(i - 1, 0), j, k)]);
                float dpy = 0.5f * (phi[IX(i, imin(j + 1, ny - 1), k)] - phi[IX(i, imax(j - 1, 0), k)]);
                float dpz = 0.5f * (phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))]);
                float fx = gamma_lu * kappa * dpx;
                float fy = gamma_lu * kappa * dpy;
                float fz = gamma_lu * kappa * dpz;
                if (wetting != 0) {
                    float wx = 0.0f, wy = 0.0f, wz = 0.0f;
                    int has_wall = 0;
                    if (i > 0 && flags[IX(i - 1, j, k)] == SOLID) { wx += 1.0f; has_wall = 1; }
                    if (i < nx - 1 && flags[IX(i + 1, j, k)] == SOLID) { wx -= 1.0f; has_wall = 1; }
                    if (j > 0 && flags[IX(i, j - 1, k)] == SOLID) { wy += 1.0f; has_wall = 1; }
                    if (j < ny - 1 && flags[IX(i, j + 1, k)] == SOLID) { wy -= 1.0f; has_wall = 1; }
                    if (k > 0 && flags[IX(i, j, k - 1)] == SOLID) { wz += 1.0f; has_wall = 1; }
                    if (k < nz - 1 && flags[IX(i, j, k + 1)] == SOLID) { wz -= 1.0f; has_wall = 1; }
                    float wmag = sqrtf(wx * wx + wy * wy + wz * wz);
                    if (wmag > 1e-8f) {
                        wx /= wmag;
                        wy /= wmag;
                        wz /= wmag;
                    }
                    if (has_wall != 0) {
                        float nxn = dpx / gmag, nyn = dpy / gmag, nzn = dpz / gmag;
                        /* kernels.py:723-766 _correct_normal_contact_angle */
                        float dot = nxn * wx + nyn * wy + nzn * wz;
                        float tx = nxn - dot * wx, ty = nyn - dot * wy, tz = nzn - dot * wz;
                        float tmag = sqrtf(tx * tx + ty * ty + tz * tz);
                        float ncx = 0.0f, ncy = 0.0f, ncz = 0.0f;
                        if (tmag > 1e-8f) {
                            ncx = cos_t * wx + sin_t * tx / tmag;
                            ncy = cos_t * wy + sin_t * ty / tmag;
                            ncz = cos_t * wz + sin_t * tz / tmag;
                        } else {
                            if (fabsf(wz) > 0.5f) {
                                ncx = sin_t; ncy = 0.0f; ncz = cos_t;
                            } else if (fabsf(wx) > 0.5f) {
                                ncx = cos_t; ncy = sin_t; ncz = 0.0f;
                            } else {
                                ncx = cos_t * wx + sin_t; ncy = cos_t * wy; ncz = cos_t * wz;
                            }
                        }
                        float cmag = sqrtf(ncx * ncx + ncy * ncy + ncz * ncz);
                        if (cmag > 1e-8f) {
                            ncx /= cmag;
                            ncy /= cmag;
                            ncz /= cmag;
                        }
                        fx = gamma_lu * kappa * ncx * gmag;
                        fy = gamma_lu * kappa * ncy * gmag;
                        fz = gamma_lu * kappa * ncz * gmag;
                    }
                }
                Fx[c] += fx;
                Fy[c] += fy;
                Fz[c] += fz;
            }
}

/* kernels.py:2158-2217 compute_marangoni_force */
static void marangoni_impl(const float* T, const float* phi, const float* f_l, float* Fx,
                           float* Fy, float* Fz, const int32_t* flags, int nx, int ny, int nz,
                           float dgamma, const float* dg_f);

void wo_compute_marangoni_force(const float* T, const float* phi, const float* f_l, float* Fx,
                                float* Fy, float* Fz, const int32_t* flags, int nx, int ny, int nz,
                                float dgamma) {
    marangoni_impl(T, phi, f_l, Fx, Fy, Fz, flags, nx, ny, nz, dgamma, NULL);
}

/* kernels.py:2221-2269 compute_marangoni_force_variable (per-cell dgamma) */
void wo_compute_marangoni_force_variable(const float* T, const float* phi, const float* f_l,
                                         float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                         const float* dg_f, int nx, int ny, int nz) {
    marangoni_impl(T, phi, f_l, Fx, Fy, Fz, flags, nx, ny, nz, 0.0f, dg_f);
}

static void marangoni_impl(const float* T, const float* phi, const float* f_l, float* Fx,
                           float* Fy, float* Fz, const int32_t* flags, int nx, int ny, int nz,
                           float dgamma, const float* dg_f) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                if (f_l[c] < 0.05f) continue;
                int ip = imin(i + 1, nx - 1), im = imax(i - 1, 0);
                int jp = imin(j + 1, ny - 1), jm = imax(j - 1, 0);
                int kp = imin(k + 1, nz - 1), km = imax(k - 1, 0);
                float dx_ = 0.5f * (phi[IX(ip, j, k)] - phi[IX(im, j, k)]);
                float dy_ = 0.5f * (phi[IX(i, jp, k)] - phi[IX(i, jm, k)]);
                float dz_ = 0.5f * (phi[IX(i, j, kp)] - phi[IX(i, j, km)]);
                float g = sqrtf(dx_ * dx_ + dy_ * dy_ + dz_ * dz_);
                if (g < 1e-6f) continue;
                float nxn = dx_ / g, nyn = dy_ / g, nzn = dz_ / g;
                float tx = 0.5f * (T[IX(ip, j, k)] - T[IX(im, j, k)]);
                float ty = 0.5f * (T[IX(i, jp, k)] - T[IX(i, jm, k)]);
                float tz = 0.5f * (T[IX(i, j, kp)] - T[IX(i, j, km)]);
                float nd = nxn * tx + nyn * ty + nzn * tz;
                float sx = tx - nd * nxn, sy = ty - nd * nyn, sz = tz - nd * nzn;
                float scale = (dg_f ? dg_f[c] : dgamma) * g;
                Fx[c] += scale * sx;
                Fy[c] += scale * sy;
                Fz[c] += scale * sz;
            }
}

/* kernels.py:3038-3083 apply_arc_pressure */
void wo_apply_arc_pressure(float* Fz, const int32_t* flags, const float* phi, int nx, int ny,
                           int nz, float arc_i, float arc_j, float arc_k, float sigma,
                           float pressure, float dt, float dx, float rho_ref) {
    float inv2s2 = 1.0f / (2.0f * sigma * sigma + 1e-6f);
    float Fphys = pressure / (rho_ref * dx);
    float Flu = Fphys * (dt * dt) / dx;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                float dpz = phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))];
                if (fabsf(dpz) > 0.05f) {
                    float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                    float r2 = di * di + dj * dj + dk * dk * 0.1f;
                    Fz[c] += -Flu * waam_expf(-r2 * inv2s2);
                }
            }
}

/* kernels.py:1094-1141 apply_gas_shear_stress (arc_k is not used there) */
void wo_apply_gas_shear_stress(float* Fx, float* Fy, const float* phi, const int32_t* flags,
                               int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                               float tau_peak_pa, float dt, float dx, float rho_ref) {
    const float eps = 1e-6f;
    const float inv2s2 = 1.0f / (2.0f * sigma * sigma + eps);
    const float F_scale = 1.0f / (rho_ref * dx) * dt * dt / dx;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                float dpx = 0.5f * (phi[IX(imin(i + 1, nx - 1), j, k)] - phi[IX(imax(i - 1, 0), j, k)]);
                float dpy = 0.5f * (phi[IX(i, imin(j + 1, ny - 1), k)] - phi[IX(i, imax(j - 1, 0), k)]);
                float dpz = 0.5f * (phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))]);
                float gmag = sqrtf(dpx * dpx + dpy * dpy + dpz * dpz);
                if (gmag < 0.08f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                float r2 = di * di + dj * dj;
                float r = sqrtf(r2 + eps);
                float rx = di / r, ry = dj / r;
                float nxn = dpx / gmag, nyn = dpy / gmag;
                float rdotn = rx * nxn + ry * nyn;
                float tx = rx - rdotn * nxn, ty = ry - rdotn * nyn;
                float tmag = sqrtf(tx * tx + ty * ty + eps);
                tx = tx / tmag;
                ty = ty / tmag;
                float tau = tau_peak_pa * waam_expf(-r2 * inv2s2);
                float Fmag = tau * F_scale;
                Fx[c] += Fmag * tx;
                Fy[c] += Fmag * ty;
            }
}

/* kernels.py:995-1028 apply_vapor_recoil (T-ratio form) */
void wo_apply_vapor_recoil(float* Fz, const float* T, const float* phi, const int32_t* flags,
                           int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                           float recoil_pa, float T_ref, float dt, float dx, float rho_ref) {
    const float eps = 1e-6f;
    const float inv2s2 = 1.0f / (2.0f * sigma * sigma + eps);
    const float F_peak = (recoil_pa / (rho_ref * dx)) * dt * dt / dx;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                float dpz = phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))];
                if (fabsf(dpz) < 0.05f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                float r2 = di * di + dj * dj;
                float t_ratio = fminf_(T[c] / (T_ref + eps), 3.0f);
                Fz[c] += -F_peak * t_ratio * waam_expf(-r2 * inv2s2);
            }
}

/* kernels.py:1046-1091 apply_vapor_recoil_clausius_clapeyron */
void wo_apply_vapor_recoil_cc(float* Fz, const float* T, const float* phi, const int32_t* flags,
                              int nx, int ny, int nz, float arc_i, float arc_j, float sigma,
                              float P_ref, float T_boil, float L_vap, float R_spec, float C_acc,
                              float dt, float dx, float rho_ref) {
    const float eps = 1e-6f;
    const float inv2s2 = 1.0f / (2.0f * sigma * sigma + eps);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == SOLID || flags[c] == GAS) continue;
                float dpz = phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))];
                if (fabsf(dpz) < 0.05f) continue;
                float Tc = T[c];
                if (Tc <= T_boil) continue;
                float ex = (L_vap / (R_spec + eps)) * (1.0f / (T_boil + eps) - 1.0f / (Tc + eps));
                ex = fminf_(ex, 12.0f);
                float P_vap = C_acc * P_ref * waam_expf(ex);
                float F_peak = P_vap / (rho_ref * dx) * dt * dt / dx;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                float r2 = di * di + dj * dj;
                Fz[c] += -F_peak * waam_expf(-r2 * inv2s2);
            }
}

/* kernels.py:2756-2772 add_hydrostatic_gravity */
void wo_add_hydrostatic_gravity(float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                                float rho_ref, float g_lu) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
        float fl = f_l[c];
        if (fl > 0.0f) Fz[c] += -rho_ref * g_lu * fl;
    }
}

/* kernels.py:2729-2753 add_buoyancy */
void wo_add_buoyancy(const float* T, float* Fz, const float* f_l, const int32_t* flags, int64_t n,
                     float g_lu, float beta, float T_ref, float rho_ref) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
        float fl = f_l[c];
        if (fl > 0.0f) Fz[c] += rho_ref * g_lu * beta * (T[c] - T_ref) * fl;
    }
}

/* kernels.py:3286-3309 clamp_body_force_magnitude */
void wo_clamp_body_force_magnitude(float* Fx, float* Fy, float* Fz, const int32_t* flags,
                                   int64_t n, float F_max) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
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

/* cumulant_kernel.py:28-209 collide_mrt: two-rate central-moment collision
 * with Guo forcing and Carman-Kozeny damping. */
void wo_collide_mrt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                    const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                    const int32_t* flags, int64_t n, float omega_s, float omega_b,
                    float C_darcy) {
    const float cs2 = 1.0f / 3.0f, eps = 1.0e-6f;
    const float w0 = 0.3333333333f, w1 = 0.0555555556f, w2 = 0.0277777778f;
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
        float fl = f_l[c], fx = Fx[c], fy = Fy[c], fz = Fz[c];
        float f[19];
        for (int q = 0; q < 19; ++q) f[q] = f_src[q * n + c];
        float r = f[0];
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
        float u = uxr / ck, v = uyr / ck, w = uzr / ck;
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
        float om_s = 1.0f - 0.5f * omega_s;
        for (int q = 0; q < 19; ++q) {
            float eu, Fe, K, wq;
            switch (q) {
                case 0: eu = 0.0f; Fe = 0.0f; K = 0.0f; wq = w0; break;
                case 1: eu = u; Fe = fx; K = ax; wq = w1; break;
                case 2: eu = -u; Fe = -fx; K = ax; wq = w1; break;
                case 3: eu = v; Fe = fy; K = ay; wq = w1; break;
                case 4: eu = -v; Fe = -fy; K = ay; wq = w1; break;
                case 5: eu = w; Fe = fz; K = az; wq = w1; break;
                case 6: eu = -w; Fe = -fz; K = az; wq = w1; break;
                case 7: eu = u + v; Fe = fx + fy; K = ax + ay + 2.0f * kxyp; wq = w2; break;
                case 8: eu = -u + -v; Fe = -fx + -fy; K = ax + ay + 2.0f * kxyp; wq = w2; break;
                case 9: eu = u + -v; Fe = fx + -fy; K = ax + ay + -2.0f * kxyp; wq = w2; break;
                case 10: eu = -u + v; Fe = -fx + fy; K = ax + ay + -2.0f * kxyp; wq = w2; break;
                case 11: eu = u + w; Fe = fx + fz; K = ax + az + 2.0f * kxzp; wq = w2; break;
                case 12: eu = -u + -w; Fe = -fx + -fz; K = ax + az + 2.0f * kxzp; wq = w2; break;
                case 13: eu = u + -w; Fe = fx + -fz; K = ax + az + -2.0f * kxzp; wq = w2; break;
                case 14: eu = -u + w; Fe = -fx + fz; K = ax + az + -2.0f * kxzp; wq = w2; break;
                case 15: eu = v + w; Fe = fy + fz; K = ay + az + 2.0f * kyzp; wq = w2; break;
                case 16: eu = -v + -w; Fe = -fy + -fz; K = ay + az + 2.0f * kyzp; wq = w2; break;
                case 17: eu = v + -w; Fe = fy + -fz; K = ay + az + -2.0f * kyzp; wq = w2; break;
                default: eu = -v + w; Fe = -fy + fz; K = ay + az + -2.0f * kyzp; wq = w2; break;
            }
            float feq = wq * (r + r3 * eu + r9h * eu * eu - rd + 4.5f * K);
            float S = wq * om_s * (3.0f * Fe + 9.0f * Fe * eu - 3.0f * uF);
            f_dst[q * n + c] = feq + S;
        }
        rho[c] = r;
        ux[c] = u;
        uy[c] = v;
        uz[c] = w;
    }
}

/* kernels.py:2778-2885 collide_srt (BGK + Guo + Carman-Kozeny) */
static void collide_srt_impl(const float* f_src, float* f_dst, float* rho, float* ux, float* uy,
                             float* uz, const float* Fx, const float* Fy, const float* Fz,
                             const float* f_l, const int32_t* flags, int64_t n, float omega_c,
                             float C_darcy, const float* tau_f);

void wo_collide_srt(const float* f_src, float* f_dst, float* rho, float* ux, float* uy, float* uz,
                    const float* Fx, const float* Fy, const float* Fz, const float* f_l,
                    const int32_t* flags, int64_t n, float omega, float C_darcy) {
    collide_srt_impl(f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, n, omega, C_darcy,
                     NULL);
}

/* kernels.py:2889-2965 collide_srt_variable_tau: omega = 1/(tau + 1e-6) per cell */
void wo_collide_srt_variable_tau(const float* f_src, float* f_dst, float* rho, float* ux,
                                 float* uy, float* uz, const float* Fx, const float* Fy,
                                 const float* Fz, const float* f_l, const int32_t* flags,
                                 const float* tau_f, int64_t n, float C_darcy) {
    collide_srt_impl(f_src, f_dst, rho, ux, uy, uz, Fx, Fy, Fz, f_l, flags, n, 0.0f, C_darcy,
                     tau_f);
}

static void collide_srt_impl(const float* f_src, float* f_dst, float* rho, float* ux, float* uy,
                             float* uz, const float* Fx, const float* Fy, const float* Fz,
                             const float* f_l, const int32_t* flags, int64_t n, float omega_c,
                             float C_darcy, const float* tau_f) {
    const float eps = 1e-6f;
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
        float fl = f_l[c];
        float omega = tau_f ? 1.0f / (tau_f[c] + eps) : omega_c;
        float r = 0.0f, jx = 0.0f, jy = 0.0f, jz = 0.0f;
        for (int q = 0; q < 19; ++q) {
            float fq = f_src[q * n + c];
            r += fq;
            jx += fq * (float)EX[q];
            jy += fq * (float)EY[q];
            jz += fq * (float)EZ[q];
        }
        float inv_r = 1.0f / (r + eps);
        float fx = Fx[c], fy = Fy[c], fz = Fz[c];
        float uxr = jx * inv_r + 0.5f * fx * inv_r;
        float uyr = jy * inv_r + 0.5f * fy * inv_r;
        float uzr = jz * inv_r + 0.5f * fz * inv_r;
        float om = 1.0f - fl;
        float ck = 1.0f + C_darcy * (om * om) / (fl * fl * fl + eps);
        float u = uxr / ck, v = uyr / ck, w = uzr / ck;
        float u2 = u * u + v * v + w * w;
        for (int q = 0; q < 19; ++q) {
            float eu = (float)EX[q] * u + (float)EY[q] * v + (float)EZ[q] * w;
            float wq = WQ(q);
            float feq = wq * r * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
            float Fe = (float)EX[q] * fx + (float)EY[q] * fy + (float)EZ[q] * fz;
            float S = wq * (1.0f - 0.5f * omega) *
                      (3.0f * Fe + 9.0f * (eu * Fe) - 3.0f * (u * fx + v * fy + w * fz));
            float fs = f_src[q * n + c];
            f_dst[q * n + c] = fs - omega * (fs - feq) + S;
        }
        rho[c] = r;
        ux[c] = u;
        uy[c] = v;
        uz[c] = w;
    }
}

/* kernels.py:3312-3335 clamp_velocity_mach */
void wo_clamp_velocity_mach(float* ux, float* uy, float* uz, const int32_t* flags, int64_t n,
                            float u_max) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) continue;
        float vx = ux[c], vy = uy[c], vz = uz[c];
        float mag = sqrtf(vx * vx + vy * vy + vz * vz);
        if (mag > u_max) {
            float s = u_max / (mag + 1e-12f);
            ux[c] = vx * s;
            uy[c] = vy * s;
            uz[c] = vz * s;
        }
    }
}

/* kernels.py:2971-3010 stream (pull; bounce-back from SOLID for non-gas
 * cells; x periodic; y, z clamped) */
void wo_stream(const float* f_src, float* f_dst, const int32_t* flags, int nx, int ny, int nz) {
    int64_t n = (int64_t)nx * ny * nz;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                int flag = flags[c];
                if (flag == SOLID) continue;
                for (int q = 0; q < 19; ++q) {
                    int ni = (i - EX[q] + nx) % nx;
                    int nj = imax(0, imin(j - EY[q], ny - 1));
                    int nk = imax(0, imin(k - EZ[q], nz - 1));
                    int64_t s = IX(ni, nj, nk);
                    if (flag == GAS)
                        f_dst[q * n + c] = f_src[q * n + s];
                    else if (flags[s] == SOLID)
                        f_dst[q * n + c] = f_src[OPP[q] * n + c];
                    else
                        f_dst[q * n + c] = f_src[q * n + s];
                }
            }
}

/* kernels.py:3261-3283 update_time_above_T */
void wo_update_time_above_T(const float* T, const int32_t* flags, float* t800, float* t1100,
                            float* tsol, int64_t n, float dt, float T800, float T1100, float Tsol) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        float t = T[c];
        if (t >= T800) t800[c] += dt;
        if (t >= T1100) t1100[c] += dt;
        if (t >= Tsol) tsol[c] += dt;
    }
}

/* kernels.py:3338-3350 snapshot_forces */
void wo_snapshot_forces(const float* Fx, const float* Fy, const float* Fz, float* Sx, float* Sy,
                        float* Sz, int64_t n) {
    memcpy(Sx, Fx, n * sizeof(float));
    memcpy(Sy, Fy, n * sizeof(float));
    memcpy(Sz, Fz, n * sizeof(float));
}

/* kernels.py:2489-2520 remelt_hot_solid_scalar */
void wo_remelt_hot_solid_scalar(const float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                int64_t n, float cp_rho, float Ts, float Tl, float L_rho) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] != SOLID) continue;
        float Tc = T[c];
        if (Tc <= Ts + 5.0f) continue;
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

/* kernels.py:2573-2617 solidify_trailing_pool_scalar */
void wo_solidify_trailing_pool_scalar(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                                      float* ux, float* uy, float* uz, int nx, int ny, int nz,
                                      float cp_rho, float arc_i, float arc_j, float arc_k,
                                      float dir_x, float dir_y, float dir_z, float lookback,
                                      float T_freeze, float Ts) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                if (phi[c] < 0.85f || f_l[c] < 0.05f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float proj = di * dir_x + dj * dir_y + dk * dir_z;
                if (proj > -lookback) continue;
                if (T[c] >= T_freeze) continue;
                H[c] = cp_rho * (Ts - 1.0f);
                T[c] = Ts - 1.0f;
                f_l[c] = 0.0f;
                phi[c] = 1.0f;
                flags[c] = SOLID;
                ux[c] = uy[c] = uz[c] = 0.0f;
            }
}

/* kernels.py:2422-2450 solidify_cooled_metal (physics/free_surface.py:73-91) */
void wo_solidify_cooled_metal(const float* T, float* f_l, float* phi, int32_t* flags, float* ux,
                              float* uy, float* uz, int64_t n, float Ts, int zero_velocity) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
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

/* kernels.py:625-641 surface_height_at */
float wo_surface_height_at(const float* phi, const int32_t* flags, int nx, int ny, int nz, int i0,
                           int j0, int nz_fallback) {
    (void)nx;
    int ks = imax(1, nz_fallback - 1);
    for (int k = 0; k < nz; ++k) {
        int64_t c = IX(i0, j0, k);
        if (flags[c] != GAS && phi[c] > 0.05f) ks = k;
    }
    return (float)ks;
}

/* kernels.py:245-275 _has_metal_neighbor */
static int has_metal_nb(const float* phi, const int32_t* flags, const float* f_l, int nx, int ny,
                        int nz, int i, int j, int k) {
    static const int d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    int found = 0;
    for (int m = 0; m < 6; ++m) {
        int ii = i + d[m][0], jj = j + d[m][1], kk = k + d[m][2];
        if (ii >= 0 && jj >= 0 && kk >= 0 && ii < nx && jj < ny && kk < nz) {
            int64_t c = IX(ii, jj, kk);
            if (flags[c] == FLUID || flags[c] == SOLID)
                found = 1;
            else if (phi[c] > 0.35f || f_l[c] > 0.2f)
                found = 1;
        }
    }
    return found;
}

static void deposit_cell(float* f_src, int32_t* flags, float* f_l, float* phi, float* H, float* T,
                         float* rho, int64_t n, int64_t c, float T_drop, float cp_rho, float L_rho,
                         float rho0) {
    flags[c] = FLUID;
    f_l[c] = 1.0f;
    phi[c] = 1.0f;
    T[c] = T_drop;
    H[c] = cp_rho * T_drop + L_rho;
    rho[c] = rho0;
    for (int q = 0; q < 19; ++q) f_src[q * n + c] = WQ(q) * rho0;
}

/* kernels.py:177-242 feed_wire -- serial lexicographic order of the
 * reserve-then-commit budget over the droplet sphere and the column above
 * the arc. */
void wo_feed_wire(float* f_src, int32_t* flags, float* f_l, float* phi, float* H, float* T,
                  float* rho, int nx, int ny, int nz, float arc_i, float arc_j, float arc_k,
                  float drop_r, float target_vol, float T_drop, float cp_rho, float L_rho,
                  float rho0, float* vol_acc, float cell_vol) {
    int64_t n = (int64_t)nx * ny * nz;
    float search_r = fmaxf_(drop_r * 2.5f, drop_r + 2.0f);
    int i0 = imax(0, (int)(arc_i - search_r)), i1 = imin(nx, (int)(arc_i + search_r) + 1);
    int j0 = imax(0, (int)(arc_j - search_r)), j1 = imin(ny, (int)(arc_j + search_r) + 1);
    int k0 = imax(0, (int)(arc_k + 1.0f)), k1 = imin(nz, (int)(arc_k + search_r * 3.0f) + 1);
    float drop_cz = arc_k + drop_r + 1.0f;
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                if (*vol_acc >= target_vol) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - drop_cz;
                float r2 = di * di + dj * dj + dk * dk;
                float rij2 = di * di + dj * dj;
                int in_sphere = r2 <= drop_r * drop_r;
                int in_column = rij2 <= search_r * search_r && (float)k >= arc_k + 1.0f;
                int64_t c = IX(i, j, k);
                if (!((in_sphere || in_column) && flags[c] == GAS)) continue;
                float reserved = *vol_acc;
                *vol_acc = reserved + cell_vol;
                if (reserved >= target_vol)
                    *vol_acc = *vol_acc - cell_vol;
                else
                    deposit_cell(f_src, flags, f_l, phi, H, T, rho, n, c, T_drop, cp_rho, L_rho,
                                 rho0);
            }
}

/* kernels.py:644-676 feed_wire_momentum */
void wo_feed_wire_momentum(float* uz, const int32_t* flags, const float* f_l, int nx, int ny,
                           int nz, float arc_i, float arc_j, float arc_k, float drop_r,
                           float vz_lu) {
    int i0 = imax(0, (int)(arc_i - drop_r)), i1 = imin(nx, (int)(arc_i + drop_r) + 1);
    int j0 = imax(0, (int)(arc_j - drop_r)), j1 = imin(ny, (int)(arc_j + drop_r) + 1);
    int k0 = imax(0, (int)arc_k), k1 = imin(nz, (int)(arc_k + drop_r * 2.0f) + 1);
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                if (f_l[c] < 0.5f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                if (di * di + dj * dj <= drop_r * drop_r) uz[c] = fminf_(uz[c] + vz_lu, 0.15f);
            }
}

/* kernels.py:278-400 feed_wire_surface -- serial lexicographic order of the
 * reserve-then-commit budget. */
void wo_feed_wire_surface(float* f_src, int32_t* flags, float* f_l, float* phi, float* H,
                          float* T, float* rho, int nx, int ny, int nz, float arc_i, float arc_j,
                          float arc_k, float foot_r, float drop_r, float target_vol, float T_drop,
                          float cp_rho, float L_rho, float rho0, float* vol_acc, float* real_acc,
                          float cell_vol) {
    int64_t n = (int64_t)nx * ny * nz;
    float sr = fmaxf_(foot_r, drop_r);
    int i0 = imax(0, (int)(arc_i - sr)), i1 = imin(nx, (int)(arc_i + sr) + 1);
    int j0 = imax(0, (int)(arc_j - sr)), j1 = imin(ny, (int)(arc_j + sr) + 1);
    int k0 = imax(0, (int)(arc_k - 1.0f));
    float k_span = fmaxf_(drop_r + 3.0f, 4.0f);
    int k1 = imin(nz, (int)(arc_k + k_span) + 1);
    float drop_cz = arc_k + drop_r + 0.5f;
    float rd2 = drop_r * drop_r, foot2 = sr * sr;
    for (int pass = 0; pass < 2; ++pass)
        for (int i = i0; i < i1; ++i)
            for (int j = j0; j < j1; ++j)
                for (int k = k0; k < k1; ++k) {
                    if (*vol_acc >= target_vol) continue;
                    int64_t c = IX(i, j, k);
                    if (flags[c] != GAS) continue;
                    if (!has_metal_nb(phi, flags, f_l, nx, ny, nz, i, j, k)) continue;
                    float di = (float)i - arc_i, dj = (float)j - arc_j;
                    float rij2 = di * di + dj * dj;
                    if (pass == 0) {
                        float dk = (float)k - drop_cz;
                        float r2 = di * di + dj * dj + dk * dk;
                        if (rij2 > foot2 && r2 > rd2) continue;
                    } else {
                        if (rij2 > foot2 * 1.44f) continue;
                    }
                    float reserved = *vol_acc;
                    *vol_acc = reserved + cell_vol;
                    if (reserved >= target_vol) {
                        *vol_acc = *vol_acc - cell_vol;
                    } else {
                        deposit_cell(f_src, flags, f_l, phi, H, T, rho, n, c, T_drop, cp_rho,
                                     L_rho, rho0);
                        *real_acc = *real_acc + cell_vol;
                    }
                }
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] != FLUID || f_l[c] < 0.45f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                if (di * di + dj * dj > foot2 * 1.44f) continue;
                T[c] = T_drop;
                H[c] = cp_rho * T_drop + L_rho;
                rho[c] = rho0;
                for (int q = 0; q < 19; ++q) f_src[q * n + c] = WQ(q) * rho0;
            }
}

/* kernels.py:1176-1233 feed_wire_momentum_impact */
void wo_feed_wire_momentum_impact(float* f_src, const float* rho, float* ux, float* uy, float* uz,
                                  const int32_t* flags, const float* f_l, int nx, int ny, int nz,
                                  float arc_i, float arc_j, float arc_k, float drop_r, float vx,
                                  float vy, float vz) {
    int64_t n = (int64_t)nx * ny * nz;
    int i0 = imax(0, (int)(arc_i - drop_r * 2.5f)), i1 = imin(nx, (int)(arc_i + drop_r * 2.5f) + 1);
    int j0 = imax(0, (int)(arc_j - drop_r * 2.5f)), j1 = imin(ny, (int)(arc_j + drop_r * 2.5f) + 1);
    int k0 = imax(0, (int)arc_k), k1 = imin(nz, (int)(arc_k + drop_r * 3.0f) + 1);
    float drop_cz = arc_k + drop_r + 1.0f;
    float u2 = vx * vx + vy * vy + vz * vz;
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                if (f_l[c] < 0.45f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - drop_cz;
                float r2 = di * di + dj * dj + dk * dk;
                float rij2 = di * di + dj * dj;
                int in_drop = r2 <= drop_r * drop_r ||
                              (rij2 <= drop_r * drop_r && (float)k >= arc_k + 1.0f);
                if (!in_drop) continue;
                float rl = rho[c];
                ux[c] = vx;
                uy[c] = vy;
                uz[c] = vz;
                for (int q = 0; q < 19; ++q) {
                    float eu = (float)EX[q] * vx + (float)EY[q] * vy + (float)EZ[q] * vz;
                    f_src[q * n + c] = WQ(q) * rl * (1.0f + 3.0f * eu + 4.5f * eu * eu - 1.5f * u2);
                }
            }
}

/* kernels.py:1142-1173 apply_droplet_impact_pressure (+ 1032-1035) */
void wo_apply_droplet_impact_pressure(float* Fz, const int32_t* flags, const float* phi,
                                      const float* f_l, int nx, int ny, int nz, float arc_i,
                                      float arc_j, float arc_k, float drop_r, float impact_pa,
                                      float dt, float dx, float rho_ref) {
    float inv2s2 = 1.0f / (2.0f * drop_r * drop_r + 1e-6f);
    float Fphys = impact_pa / (rho_ref * dx);
    float Flu = Fphys * dt * dt / dx;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                if (f_l[c] < 0.25f && phi[c] < 0.25f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float r2 = di * di + dj * dj + dk * dk;
                if (r2 > drop_r * drop_r * 4.0f) continue;
                Fz[c] += -Flu * waam_expf(-r2 * inv2s2);
            }
}

/* ---------------- Lorentz (kernels.py:1236-1513) ---------------- */

/* kernels.py:1237-1251 elec_build_sigma */
void wo_elec_build_sigma(float* sigma, const float* f_l, const int32_t* flags, int64_t n,
                         float s_liq, float s_sol) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS)
            sigma[c] = 1e-8f;
        else if (f_l[c] > 0.55f)
            sigma[c] = s_liq;
        else
            sigma[c] = s_sol;
    }
}

/* kernels.py:1255-1284 elec_clear_source + elec_inject_arc_source */
void wo_elec_inject_arc_source(float* src, int nx, int ny, int nz, float arc_i, float arc_j,
                               float arc_k, float sigma_cells, float current, float dx) {
    const float eps = 1e-6f;
    float inv2s2 = 1.0f / (2.0f * sigma_cells * sigma_cells + eps);
    float cell_vol = dx * dx * dx;
    int kmax = imin(nz, (int)(arc_k + sigma_cells * 4.0f) + 1);
    int kmin = imax(0, (int)(arc_k - sigma_cells));
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                src[c] = 0.0f;
                if (k < kmin || k > kmax) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float r2 = di * di + dj * dj + 0.25f * dk * dk;
                float wgt = waam_expf(-r2 * inv2s2);
                src[c] = current * wgt / (cell_vol + eps);
            }
}

/* kernels.py:1287-1300 elec_normalize_source (sum accumulated in double) */
void wo_elec_normalize_source(float* src, int64_t n, float current, float dx) {
    float cell_vol = dx * dx * dx;
    double tot = 0.0;
#pragma omp parallel for reduction(+ : tot)
    for (int64_t c = 0; c < n; ++c) tot += (double)(src[c] * cell_vol);
    float total = (float)tot;
    float scale = current / fmaxf_(total, 1e-12f);
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) src[c] *= scale;
}

static inline float sig_at(const float* s, int nx, int ny, int nz, int i, int j, int k) {
    return s[IX(imax(0, imin(nx - 1, i)), imax(0, imin(ny - 1, j)), imax(0, imin(nz - 1, k)))];
}

/* kernels.py:1314-1354 elec_jacobi_step */
void wo_elec_jacobi_step(const float* phi_in, float* phi_out, const float* sigma,
                         const float* src, const int32_t* flags, int nx, int ny, int nz, float dx,
                         float omega_j, int nz_solid) {
    const float eps = 1e-12f;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) { phi_out[c] = 0.0f; continue; }
                if (k <= nz_solid && flags[c] == SOLID) { phi_out[c] = 0.0f; continue; }
                float sp = sig_at(sigma, nx, ny, nz, i + 1, j, k);
                float sm = sig_at(sigma, nx, ny, nz, i - 1, j, k);
                float sn = sig_at(sigma, nx, ny, nz, i, j + 1, k);
                float ss = sig_at(sigma, nx, ny, nz, i, j - 1, k);
                float st = sig_at(sigma, nx, ny, nz, i, j, k + 1);
                float sb = sig_at(sigma, nx, ny, nz, i, j, k - 1);
                float denom = sp + sm + sn + ss + st + sb + eps;
                float nb = sp * phi_in[IX(imin(i + 1, nx - 1), j, k)] +
                           sm * phi_in[IX(imax(i - 1, 0), j, k)] +
                           sn * phi_in[IX(i, imin(j + 1, ny - 1), k)] +
                           ss * phi_in[IX(i, imax(j - 1, 0), k)] +
                           st * phi_in[IX(i, j, imin(k + 1, nz - 1))] +
                           sb * phi_in[IX(i, j, imax(k - 1, 0))];
                float pn = (nb + src[c] * dx * dx) / denom;
                phi_out[c] = (1.0f - omega_j) * phi_in[c] + omega_j * pn;
            }
}

/* kernels.py:1387-1398 elec_l1_diff (double accumulation) */
void wo_elec_l1_diff(const float* a, const float* b, int64_t n, double* diff, double* norm) {
    double d = 0.0, m = 0.0;
#pragma omp parallel for reduction(+ : d, m)
    for (int64_t c = 0; c < n; ++c) {
        d += (double)fabsf(a[c] - b[c]);
        m += (double)fabsf(b[c]);
    }
    *diff = d;
    *norm = m;
}

/* kernels.py:1358-1383 elec_compute_J */
void wo_elec_compute_J(float* Jx, float* Jy, float* Jz, const float* phi, const float* sigma,
                       const int32_t* flags, int nx, int ny, int nz, float dx) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) { Jx[c] = Jy[c] = Jz[c] = 0.0f; continue; }
                float sg = sigma[c];
                float ddx = (phi[IX(imin(i + 1, nx - 1), j, k)] - phi[IX(imax(i - 1, 0), j, k)]) / (2.0f * dx);
                float ddy = (phi[IX(i, imin(j + 1, ny - 1), k)] - phi[IX(i, imax(j - 1, 0), k)]) / (2.0f * dx);
                float ddz = (phi[IX(i, j, imin(k + 1, nz - 1))] - phi[IX(i, j, imax(k - 1, 0))]) / (2.0f * dx);
                Jx[c] = -sg * ddx;
                Jy[c] = -sg * ddy;
                Jz[c] = -sg * ddz;
            }
}

/* kernels.py:1402-1434 elec_bin_axial_current + elec_prefix_bins.  Bin
 * sums accumulated in double per z slab, then prefix-summed in float. */
void wo_elec_bins(const float* Jz, float* bins, int nx, int ny, int nz, float arc_i, float arc_j,
                  float dx, float bin_dr, int n_bins) {
    double* acc = (double*)calloc((size_t)nz * n_bins, sizeof(double));
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            float di = (float)i - arc_i, dj = (float)j - arc_j;
            float r = sqrtf(di * di + dj * dj);
            int b = imin((int)(r / bin_dr), n_bins - 1);
            for (int k = 0; k < nz; ++k) acc[(size_t)k * n_bins + b] += (double)(Jz[IX(i, j, k)] * dx * dx);
        }
    for (int k = 0; k < nz; ++k) {
        float a = 0.0f;
        for (int b = 0; b < n_bins; ++b) {
            a += (float)acc[(size_t)k * n_bins + b];
            bins[(size_t)k * n_bins + b] = a;
        }
    }
    free(acc);
}

/* kernels.py:1438-1475 elec_B_axisymmetric */
void wo_elec_B_axisymmetric(float* Bx, float* By, float* Bz, const float* bins, int nx, int ny,
                            int nz, float arc_i, float arc_j, float dx, float bin_dr, float mu0,
                            int n_bins) {
    const float pi = 3.14159265358979323846f;
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                float di = (float)i - arc_i, dj = (float)j - arc_j;
                float rc = sqrtf(di * di + dj * dj);
                Bx[c] = By[c] = Bz[c] = 0.0f;
                if (rc > 1e-3f) {
                    int b = imin((int)(rc / bin_dr), n_bins - 1);
                    float I = bins[(size_t)k * n_bins + b];
                    float rm = rc * dx;
                    float Bt = mu0 * I / (2.0f * pi * rm);
                    Bx[c] = -Bt * dj / rc;
                    By[c] = Bt * di / rc;
                }
            }
}

/* kernels.py:1479-1513 apply_lorentz_JxB */
void wo_apply_lorentz_JxB(float* Fx, float* Fy, float* Fz, const float* Jx, const float* Jy,
                          const float* Jz, const float* Bx, const float* By, const float* Bz,
                          const float* f_l, const int32_t* flags, int64_t n, float dt, float dx,
                          float rho_ref) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS || f_l[c] < 0.05f) continue;
        float jx = Jx[c], jy = Jy[c], jz = Jz[c], bx = Bx[c], by = By[c], bz = Bz[c];
        float fxp = jy * bz - jz * by, fyp = jz * bx - jx * bz, fzp = jx * by - jy * bx;
        float flw = fminf_(1.0f, f_l[c]);
        float scale = flw * dt * dt / (rho_ref * dx);
        Fx[c] += fxp * scale;
        Fy[c] += fyp * scale;
        Fz[c] += fzp * scale;
    }
}

/* ---------------- tracers (kernels.py:3182-3255) ---------------- */

static uint64_t wo_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static float wo_uniform01(uint64_t seed, uint64_t index, int component) {
    uint64_t h = wo_mix64(seed ^ wo_mix64(index * 2ull + (uint64_t)component));
    return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);
}

void wo_inject_tracers(float* pos, int32_t* active, int32_t* head, int max_tracers, float arc_x,
                       float arc_y, float arc_z, float sigma_m, int spawn_count, uint64_t seed) {
    int base = *head;
    for (int t = 0; t < spawn_count; ++t) {
        uint64_t index = (uint64_t)(uint32_t)base + (uint64_t)t;
        int slot = (int)(index % (uint64_t)max_tracers);
        active[slot] = 1;
        float rdx = (wo_uniform01(seed, index, 0) * 2.0f - 1.0f) * sigma_m;
        float rdy = (wo_uniform01(seed, index, 1) * 2.0f - 1.0f) * sigma_m;
        pos[3 * slot + 0] = arc_x + rdx;
        pos[3 * slot + 1] = arc_y + rdy;
        pos[3 * slot + 2] = arc_z;
    }
    *head = base + spawn_count;
}

void wo_advect_tracers(float* pos, int32_t* active, const float* ux, const float* uy,
                       const float* uz, const float* f_l, const int32_t* flags, int nx, int ny,
                       int nz, float dx, int max_tracers) {
    for (int p = 0; p < max_tracers; ++p) {
        if (active[p] != 1) continue;
        int i = (int)(pos[3 * p] / dx), j = (int)(pos[3 * p + 1] / dx), k = (int)(pos[3 * p + 2] / dx);
        if (i < 0 || i >= nx || j < 0 || j >= ny || k < 0 || k >= nz) { active[p] = 0; continue; }
        int64_t c = IX(i, j, k);
        if (flags[c] == GAS) { active[p] = 0; continue; }
        if (f_l[c] < 0.05f || flags[c] == SOLID) { active[p] = 2; continue; }
        pos[3 * p] = pos[3 * p] + ux[c] * dx;
        pos[3 * p + 1] = pos[3 * p + 1] + uy[c] * dx;
        pos[3 * p + 2] = pos[3 * p + 2] + uz[c] * dx;
    }
}

/* ---------------- material-table path (kernels.py:1686-2010, 2454-2570) ---------------- */

/* kernels.py:1686-1707 lookup_table_1d (the last matching segment wins) */
static float lookup_1d(float T, const float* t, const float* v, int n, float fallback) {
    float result = fallback;
    if (n > 0) {
        if (T <= t[0]) {
            result = v[0];
        } else if (T >= t[n - 1]) {
            result = v[n - 1];
        } else {
            for (int idx = 0; idx < 7; ++idx) {
                if (idx < n - 1) {
                    float t0 = t[idx], t1 = t[idx + 1];
                    if (T >= t0 && T <= t1) {
                        float w = (T - t0) / (t1 - t0 + 1e-8f);
                        result = v[idx] + w * (v[idx + 1] - v[idx]);
                    }
                }
            }
        }
    }
    return result;
}

/* kernels.py:1710-1772 refresh_thermal_properties (use_tables = 1).  tab holds
 * cp_T, cp_V, k_T, k_V, mu_T, mu_V, dgamma_T, dgamma_V (8 knots each), cnt the
 * four knot counts, fb the four fallbacks, ref cp_rho, alpha_lu, dgamma_lu,
 * tau of the constants path. */
void wo_refresh_thermal_properties(const float* T, float* cp_f, float* alpha_f, float* dg_f,
                                   float* tau_f, const int32_t* flags, int64_t n,
                                   const float* tab, const int32_t* cnt, const float* fb,
                                   const float* ref, float rho, float dt, float dx,
                                   float force_scale, float marangoni_scale) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == SOLID || flags[c] == GAS) {
            cp_f[c] = ref[0];
            alpha_f[c] = ref[1];
            dg_f[c] = ref[2];
            tau_f[c] = ref[3];
            continue;
        }
        float Tc = T[c];
        float cp = lookup_1d(Tc, tab + 0, tab + 8, cnt[0], fb[0]);
        float kv = lookup_1d(Tc, tab + 16, tab + 24, cnt[1], fb[1]);
        float mu = lookup_1d(Tc, tab + 32, tab + 40, cnt[2], fb[2]);
        float dg = lookup_1d(Tc, tab + 48, tab + 56, cnt[3], fb[3]);
        float cp_r = rho * cp;
        float alpha_phys = kv / (rho * cp + 1e-9f);
        float nu_phys = mu / (rho + 1e-9f);
        float nu_lu = nu_phys * dt / (dx * dx);
        cp_f[c] = cp_r;
        alpha_f[c] = alpha_phys * dt / (dx * dx);
        dg_f[c] = dg * force_scale * marangoni_scale;
        tau_f[c] = 3.0f * nu_lu + 0.5f;
    }
}

/* kernels.py:1839-1863 update_phase_variable_cp */
void wo_update_phase_variable_cp(const float* H, float* T, float* f_l, const float* cp_f,
                                 int64_t n, float L_rho, float Ts, float Tl, float H_sol,
                                 float H_liq) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        float h = H[c], cp = cp_f[c];
        if (h <= H_sol) {
            f_l[c] = 0.0f;
            T[c] = h / (cp + 1e-9f);
        } else if (h >= H_liq) {
            f_l[c] = 1.0f;
            T[c] = Tl + (h - H_liq) / (cp + 1e-9f);
        } else {
            float fl = (h - H_sol) / L_rho;
            f_l[c] = fl;
            T[c] = Ts + fl * (Tl - Ts);
        }
    }
}

/* kernels.py:1988-2010 clamp_enthalpy_ceiling_variable_cp */
void wo_clamp_enthalpy_ceiling_variable_cp(float* H, const int32_t* flags, const float* cp_f,
                                           int64_t n, float H_liq, float Tl, float T_cap) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        float cp_r = cp_f[c];
        float cap_l = H_liq + cp_r * (T_cap - Tl);
        float cap_s = cp_r * T_cap;
        float h = H[c];
        if (h > H_liq) {
            if (h > cap_l) H[c] = cap_l;
        } else {
            if (h > cap_s) H[c] = cap_s;
        }
    }
}

/* kernels.py:1922-1935 clamp_enthalpy_floor (per-cell cp*rho) */
void wo_clamp_enthalpy_floor(float* H, const float* cp_f, const int32_t* flags, int64_t n,
                             float T_floor) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] == GAS) continue;
        float h_min = cp_f[c] * T_floor;
        if (H[c] < h_min) H[c] = h_min;
    }
}

/* kernels.py:2454-2485 remelt_hot_solid (per-cell cp*rho) */
void wo_remelt_hot_solid(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                         const float* cp_f, int64_t n, float Ts, float Tl, float L_rho) {
#pragma omp parallel for
    for (int64_t c = 0; c < n; ++c) {
        if (flags[c] != SOLID) continue;
        float Tc = T[c];
        if (Tc <= Ts + 5.0f) continue;
        float cp_r = cp_f[c];
        float H_sol = cp_r * Ts;
        float fl;
        if (Tc >= Tl) {
            fl = 1.0f;
            H[c] = cp_r * Tl + L_rho + cp_r * (Tc - Tl);
        } else {
            fl = (Tc - Ts) / (Tl - Ts + 1e-6f);
            H[c] = H_sol + fl * L_rho;
        }
        f_l[c] = fl;
        phi[c] = 1.0f;
        flags[c] = FLUID;
    }
}

/* kernels.py:2524-2570 solidify_trailing_pool (per-cell cp*rho) */
void wo_solidify_trailing_pool(float* T, float* H, float* f_l, float* phi, int32_t* flags,
                               float* ux, float* uy, float* uz, const float* cp_f, int nx, int ny,
                               int nz, float arc_i, float arc_j, float arc_k, float dir_x,
                               float dir_y, float dir_z, float lookback, float T_freeze,
                               float Ts) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                if (flags[c] == GAS) continue;
                if (phi[c] < 0.85f || f_l[c] < 0.05f) continue;
                float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
                float proj = di * dir_x + dj * dir_y + dk * dir_z;
                if (proj > -lookback) continue;
                if (T[c] >= T_freeze) continue;
                float cp_r = cp_f[c];
                H[c] = cp_r * (Ts - 1.0f);
                T[c] = Ts - 1.0f;
                f_l[c] = 0.0f;
                phi[c] = 1.0f;
                flags[c] = SOLID;
                ux[c] = 0.0f;
                uy[c] = 0.0f;
                uz[c] = 0.0f;
            }
}

/* kernels.py:2620-2723 shift_simulation_window_x: every field moves n_shift
 * cells towards i = 0 (ascending serial copy per (j, k) column), the right
 * strip i >= nx - n_shift becomes ambient plate / gas at rest; the property
 * fields are moved but not reset. */
void wo_shift_simulation_window_x(float* f_a, float* f_b, float* T, float* H, float* f_l,
                                  float* phi, int32_t* flags, float* T_max, float* T_prev,
                                  float* dT_dt, float* t800, float* t1100, float* tsol,
                                  float* rho, float* ux, float* uy, float* uz, float* Fx,
                                  float* Fy, float* Fz, float* cp_f, float* alpha_f,
                                  float* dg_f, float* tau_f, int n_shift, float T_amb,
                                  float cp_rho, float rho0, int nz_solid, int nx, int ny,
                                  int nz) {
    int64_t n = (int64_t)nx * ny * nz;
    float* fl32[] = {T, H, f_l, phi, T_max, T_prev, dT_dt, t800, t1100, tsol, rho,
                     ux, uy, uz, Fx, Fy, Fz, cp_f, alpha_f, dg_f, tau_f};
    const int nf = (int)(sizeof(fl32) / sizeof(fl32[0]));
    for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx - n_shift; ++i) {
                int64_t d = IX(i, j, k), s = IX(i + n_shift, j, k);
                for (int q = 0; q < nf; ++q) fl32[q][d] = fl32[q][s];
                flags[d] = flags[s];
                for (int q = 0; q < 19; ++q) {
                    f_a[q * n + d] = f_a[q * n + s];
                    f_b[q * n + d] = f_b[q * n + s];
                }
            }
    int i0 = nx - n_shift;
    for (int i = i0 < 0 ? 0 : i0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                T[c] = T_amb;
                H[c] = cp_rho * T_amb;
                f_l[c] = 0.0f;
                rho[c] = rho0;
                ux[c] = uy[c] = uz[c] = 0.0f;
                Fx[c] = Fy[c] = Fz[c] = 0.0f;
                T_prev[c] = T_amb;
                dT_dt[c] = 0.0f;
                T_max[c] = T_amb;
                t800[c] = t1100[c] = tsol[c] = 0.0f;
                if (k < nz_solid) {
                    flags[c] = SOLID;
                    phi[c] = 1.0f;
                } else {
                    flags[c] = GAS;
                    phi[c] = 0.0f;
                }
                for (int q = 0; q < 19; ++q) {
                    float feq = WQ(q) * rho0;
                    f_a[q * n + c] = feq;
                    f_b[q * n + c] = feq;
                }
            }
}

/* kernels.py:3354-3376 compute_curvature_field */
void wo_compute_curvature_field(const float* phi, const int32_t* flags, float* kappa, int nx,
                                int ny, int nz) {
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                kappa[c] = 0.0f;
                if (flags[c] == GAS) continue;
                if (i < 1 || j < 1 || k < 1 || i > nx - 2 || j > ny - 2 || k > nz - 2) continue;
                float g0;
                float kv = brackbill_kappa(phi, nx, ny, nz, i, j, k, &g0);
                if (g0 >= 1e-6f) kappa[c] = kv;
            }
}

/* kernels.py:3379-3418 compute_vorticity_magnitude */
void wo_compute_vorticity_magnitude(const float* ux, const float* uy, const float* uz,
                                    const int32_t* flags, float* vort, int nx, int ny, int nz,
                                    float dt) {
    const float scale = 1.0f / (dt + 1e-12f);
#pragma omp parallel for collapse(2)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                int64_t c = IX(i, j, k);
                vort[c] = 0.0f;
                if (flags[c] == GAS) continue;
                int ip = imin(i + 1, nx - 1), im = imax(i - 1, 0);
                int jp = imin(j + 1, ny - 1), jm = imax(j - 1, 0);
                int kp = imin(k + 1, nz - 1), km = imax(k - 1, 0);
                float duz_dy = 0.5f * (uz[IX(i, jp, k)] - uz[IX(i, jm, k)]);
                float duy_dz = 0.5f * (uy[IX(i, j, kp)] - uy[IX(i, j, km)]);
                float dux_dz = 0.5f * (ux[IX(i, j, kp)] - ux[IX(i, j, km)]);
                float duz_dx = 0.5f * (uz[IX(ip, j, k)] - uz[IX(im, j, k)]);
                float duy_dx = 0.5f * (uy[IX(ip, j, k)] - uy[IX(im, j, k)]);
                float dux_dy = 0.5f * (ux[IX(i, jp, k)] - ux[IX(i, jm, k)]);
                float wx = (duz_dy - duy_dz) * scale;
                float wy = (dux_dz - duz_dx) * scale;
                float wz = (duy_dx - dux_dy) * scale;
                vort[c] = sqrtf(wx * wx + wy * wy + wz * wz);
            }
}
