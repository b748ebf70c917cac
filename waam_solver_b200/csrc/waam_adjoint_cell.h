// Per-cell reverse-mode derivatives of the coupled step (hand-written).
//
// Each *_vjp function returns the vector-Jacobian product of one cell's
// forward map: given the adjoints of the outputs it accumulates the adjoints
// of the inputs.  The forward maps are restated here as templates (float on
// the device, with the same expression order as the production kernels, and
// double on the host, where the tests compare every product with central
// finite differences).  Branches (clamps, the Darcy / Marangoni thresholds)
// take the side the forward took.
//
// Forward maps (cumulant_kernel.py:28-209, kernels.py:2158-2217, 2729-2772,
// 3286-3335):
//   mrt_forward: 19 populations, liquid fraction, body force -> 19
//     post-collision populations and the velocity, then the Mach clamp of the
//     stored velocity;
//   clamp_vjp: y = x * cap / (|x| + 1e-12) when |x| > cap (force and Mach
//     clamps).
#pragma once

#ifdef __CUDACC__
#define WAAM_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#define WAAM_HD inline
#endif

namespace waam_adj {

WAAM_HD float sqrt_(float x) { return sqrtf(x); }
WAAM_HD double sqrt_(double x) { return sqrt(x); }

WAAM_HD int cx(int q) {
    return q == 1 || q == 7 || q == 9 || q == 11 || q == 13 ? 1
         : (q == 2 || q == 8 || q == 10 || q == 12 || q == 14 ? -1 : 0);
}
WAAM_HD int cy(int q) {
    return q == 3 || q == 7 || q == 10 || q == 15 || q == 17 ? 1
         : (q == 4 || q == 8 || q == 9 || q == 16 || q == 18 ? -1 : 0);
}
WAAM_HD int cz(int q) {
    return q == 5 || q == 11 || q == 14 || q == 15 || q == 18 ? 1
         : (q == 6 || q == 12 || q == 13 || q == 16 || q == 17 ? -1 : 0);
}

// Central-moment MRT collision (cumulant_kernel.py:28-209), the production
// kernel's expression order.  out: post-collision populations; u, v, w: the
// velocity before the Mach clamp.
template <class F>
WAAM_HD void mrt_forward(const F* f, F fl, F fx, F fy, F fz, F omega_s, F omega_b, F C_darcy,
                         F* out, F& r, F& u, F& v, F& w) {
    const F cs2 = F(1) / F(3), eps = F(1.0e-6);
    const F w0 = F(0.333333343f), w1 = F(0.0555555560f), w2 = F(0.0277777780f);
    r = f[0];
    for (int q = 1; q < 19; ++q) r = r + f[q];
    F inv_rho = F(1) / (r + eps);
    F jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
    F jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
    F jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
    F uxr = (jx + F(0.5) * fx) * inv_rho;
    F uyr = (jy + F(0.5) * fy) * inv_rho;
    F uzr = (jz + F(0.5) * fz) * inv_rho;
    F om = F(1) - fl;
    F ck = F(1) + C_darcy * (om * om) / (fl * fl * fl + eps);
    u = uxr / ck;
    v = uyr / ck;
    w = uzr / ck;
    F Pxx = f[1] + f[2] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14];
    F Pyy = f[3] + f[4] + f[7] + f[8] + f[9] + f[10] + f[15] + f[16] + f[17] + f[18];
    F Pzz = f[5] + f[6] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    F Pxy = f[7] + f[8] - f[9] - f[10];
    F Pxz = f[11] + f[12] - f[13] - f[14];
    F Pyz = f[15] + f[16] - f[17] - f[18];
    F kxx = Pxx - r * u * u, kyy = Pyy - r * v * v, kzz = Pzz - r * w * w;
    F kxy = Pxy - r * u * v, kxz = Pxz - r * u * w, kyz = Pyz - r * v * w;
    F km = (kxx + kyy + kzz) / F(3);
    F kmp = km - omega_b * (km - r * cs2);
    F kxxp = kmp + (F(1) - omega_s) * (kxx - km);
    F kyyp = kmp + (F(1) - omega_s) * (kyy - km);
    F kzzp = kmp + (F(1) - omega_s) * (kzz - km);
    F kxyp = kxy - omega_s * kxy;
    F kxzp = kxz - omega_s * kxz;
    F kyzp = kyz - omega_s * kyz;
    F u2 = u * u + v * v + w * w;
    F uF = u * fx + v * fy + w * fz;
    F ax = kxxp - r * cs2, ay = kyyp - r * cs2, az = kzzp - r * cs2;
    F r3 = r * F(3), r9h = r * F(3) * F(3) * F(0.5), rd = r * F(0.5) * F(3) * u2;
    F oms = F(1) - F(0.5) * omega_s;
    F K[19];
    K[0] = F(0);
    K[1] = K[2] = ax;
    K[3] = K[4] = ay;
    K[5] = K[6] = az;
    K[7] = K[8] = (ax + ay) + F(2) * kxyp;
    K[9] = K[10] = (ax + ay) + F(-2) * kxyp;
    K[11] = K[12] = (ax + az) + F(2) * kxzp;
    K[13] = K[14] = (ax + az) + F(-2) * kxzp;
    K[15] = K[16] = (ay + az) + F(2) * kyzp;
    K[17] = K[18] = (ay + az) + F(-2) * kyzp;
    for (int q = 0; q < 19; ++q) {
        const F wq = q == 0 ? w0 : (q < 7 ? w1 : w2);
        const F eu = q == 0 ? F(0) : F(cx(q)) * u + F(cy(q)) * v + F(cz(q)) * w;
        const F fe = q == 0 ? F(0) : F(cx(q)) * fx + F(cy(q)) * fy + F(cz(q)) * fz;
        F feq = wq * (r + r3 * eu + r9h * eu * eu - rd + F(4.5) * K[q]);
        F s = wq * oms * (F(3) * fe + F(9) * fe * eu - F(3) * uF);
        out[q] = feq + s;
    }
}

// Reverse of y = x * cap / (|x| + 1e-12) for |x| > cap (identity otherwise).
template <class F>
WAAM_HD void clamp_vjp(F x, F y, F z, F cap, F& xb, F& yb, F& zb) {
    if (!(cap > F(0))) return;
    const F m = sqrt_(x * x + y * y + z * z);
    if (!(m > cap)) return;
    const F den = m + F(1e-12);
    const F s = cap / den;
    const F dot = x * xb + y * yb + z * zb;
    const F k = -cap / (den * den) * dot / m;
    const F nx = s * xb + k * x, ny = s * yb + k * y, nz = s * zb + k * z;
    xb = nx;
    yb = ny;
    zb = nz;
}

// Vector-Jacobian product of mrt_forward followed by the Mach clamp of the
// stored velocity (kernels.py:3312-3335, limit ucap when > 0).
//   ob: adjoint of out[19]; usb, vsb, wsb: adjoint of the stored velocity;
//   fb[19], flb, fxb, fyb, fzb: accumulated (+=).
template <class F>
WAAM_HD void mrt_vjp(const F* f, F fl, F fx, F fy, F fz, F omega_s, F omega_b, F C_darcy, F ucap,
                     const F* ob, F usb, F vsb, F wsb, F* fb, F& flb, F& fxb, F& fyb, F& fzb) {
    const F cs2 = F(1) / F(3), eps = F(1.0e-6);
    const F w0 = F(0.333333343f), w1 = F(0.0555555560f), w2 = F(0.0277777780f);
    // ---- forward intermediates ----
    F r = f[0];
    for (int q = 1; q < 19; ++q) r = r + f[q];
    F inv_rho = F(1) / (r + eps);
    F jx = f[1] - f[2] + f[7] - f[8] + f[9] - f[10] + f[11] - f[12] + f[13] - f[14];
    F jy = f[3] - f[4] + f[7] - f[8] - f[9] + f[10] + f[15] - f[16] + f[17] - f[18];
    F jz = f[5] - f[6] + f[11] - f[12] - f[13] + f[14] + f[15] - f[16] - f[17] + f[18];
    F uxr = (jx + F(0.5) * fx) * inv_rho;
    F uyr = (jy + F(0.5) * fy) * inv_rho;
    F uzr = (jz + F(0.5) * fz) * inv_rho;
    F om = F(1) - fl;
    F den = fl * fl * fl + eps;
    F ck = F(1) + C_darcy * (om * om) / den;
    F u = uxr / ck, v = uyr / ck, w = uzr / ck;
    F Pxx = f[1] + f[2] + f[7] + f[8] + f[9] + f[10] + f[11] + f[12] + f[13] + f[14];
    F Pyy = f[3] + f[4] + f[7] + f[8] + f[9] + f[10] + f[15] + f[16] + f[17] + f[18];
    F Pzz = f[5] + f[6] + f[11] + f[12] + f[13] + f[14] + f[15] + f[16] + f[17] + f[18];
    F Pxy = f[7] + f[8] - f[9] - f[10];
    F Pxz = f[11] + f[12] - f[13] - f[14];
    F Pyz = f[15] + f[16] - f[17] - f[18];
    F kxx = Pxx - r * u * u, kyy = Pyy - r * v * v, kzz = Pzz - r * w * w;
    F kxy = Pxy - r * u * v, kxz = Pxz - r * u * w, kyz = Pyz - r * v * w;
    F kxyp = kxy - omega_s * kxy, kxzp = kxz - omega_s * kxz, kyzp = kyz - omega_s * kyz;
    F u2 = u * u + v * v + w * w;
    F r3 = r * F(3), r9h = r * F(3) * F(3) * F(0.5);
    F oms = F(1) - F(0.5) * omega_s;
    (void)kxyp;
    (void)kxzp;
    (void)kyzp;
    // ---- reverse ----
    // Mach clamp of the stored velocity: adjoint of the unclamped velocity
    F ub = usb, vb = vsb, wb = wsb;
    clamp_vjp(u, v, w, ucap, ub, vb, wb);
    F rb = F(0), r3b = F(0), r9hb = F(0), rdb = F(0), uFb = F(0);
    F axb = F(0), ayb = F(0), azb = F(0), kxypb = F(0), kxzpb = F(0), kyzpb = F(0);
    for (int q = 0; q < 19; ++q) {
        const F wq = q == 0 ? w0 : (q < 7 ? w1 : w2);
        const F ex_ = F(cx(q)), ey_ = F(cy(q)), ez_ = F(cz(q));
        const F eu = q == 0 ? F(0) : ex_ * u + ey_ * v + ez_ * w;
        const F fe = q == 0 ? F(0) : ex_ * fx + ey_ * fy + ez_ * fz;
        const F Ab = ob[q] * wq, Bb = ob[q] * wq * oms;
        rb += Ab;
        r3b += Ab * eu;
        r9hb += Ab * eu * eu;
        rdb -= Ab;
        const F Kb = F(4.5) * Ab;
        const F eub = Ab * (r3 + F(2) * r9h * eu) + Bb * (F(9) * fe);
        const F feb = Bb * (F(3) + F(9) * eu);
        uFb -= F(3) * Bb;
        if (q > 0) {
            ub += eub * ex_;
            vb += eub * ey_;
            wb += eub * ez_;
            fxb += feb * ex_;
            fyb += feb * ey_;
            fzb += feb * ez_;
        }
        switch (q) {
            case 1: case 2: axb += Kb; break;
            case 3: case 4: ayb += Kb; break;
            case 5: case 6: azb += Kb; break;
            case 7: case 8: axb += Kb; ayb += Kb; kxypb += F(2) * Kb; break;
            case 9: case 10: axb += Kb; ayb += Kb; kxypb -= F(2) * Kb; break;
            case 11: case 12: axb += Kb; azb += Kb; kxzpb += F(2) * Kb; break;
            case 13: case 14: axb += Kb; azb += Kb; kxzpb -= F(2) * Kb; break;
            case 15: case 16: ayb += Kb; azb += Kb; kyzpb += F(2) * Kb; break;
            case 17: case 18: ayb += Kb; azb += Kb; kyzpb -= F(2) * Kb; break;
            default: break;
        }
    }
    // r3 = 3 r, r9h = 4.5 r, rd = 1.5 r u2, uF = u.F
    rb += F(3) * r3b + F(4.5) * r9hb + F(1.5) * u2 * rdb;
    F u2b = F(1.5) * r * rdb;
    ub += uFb * fx;
    vb += uFb * fy;
    wb += uFb * fz;
    fxb += uFb * u;
    fyb += uFb * v;
    fzb += uFb * w;
    ub += F(2) * u * u2b;
    vb += F(2) * v * u2b;
    wb += F(2) * w * u2b;
    // a = kp - r cs2
    F kxxpb = axb, kyypb = ayb, kzzpb = azb;
    rb -= cs2 * (axb + ayb + azb);
    // off-diagonal relaxation
    F kxyb = (F(1) - omega_s) * kxypb, kxzb = (F(1) - omega_s) * kxzpb;
    F kyzb = (F(1) - omega_s) * kyzpb;
    // diagonal relaxation: kpp = kmp + (1 - ws)(k - km)
    F kmpb = kxxpb + kyypb + kzzpb;
    F kxxb = (F(1) - omega_s) * kxxpb, kyyb = (F(1) - omega_s) * kyypb;
    F kzzb = (F(1) - omega_s) * kzzpb;
    F kmb = -(F(1) - omega_s) * (kxxpb + kyypb + kzzpb);
    // kmp = km - wb (km - r cs2)
    kmb += (F(1) - omega_b) * kmpb;
    rb += omega_b * cs2 * kmpb;
    // km = (kxx + kyy + kzz) / 3
    kxxb += kmb / F(3);
    kyyb += kmb / F(3);
    kzzb += kmb / F(3);
    // central moments
    rb -= u * u * kxxb + v * v * kyyb + w * w * kzzb + u * v * kxyb + u * w * kxzb + v * w * kyzb;
    ub -= F(2) * r * u * kxxb + r * v * kxyb + r * w * kxzb;
    vb -= F(2) * r * v * kyyb + r * u * kxyb + r * w * kyzb;
    wb -= F(2) * r * w * kzzb + r * u * kxzb + r * v * kyzb;
    const F Pxxb = kxxb, Pyyb = kyyb, Pzzb = kzzb, Pxyb = kxyb, Pxzb = kxzb, Pyzb = kyzb;
    // u = ur / ck
    F uxrb = ub / ck, uyrb = vb / ck, uzrb = wb / ck;
    F ckb = -(ub * uxr + vb * uyr + wb * uzr) / (ck * ck);
    // ck = 1 + C om^2 / (fl^3 + eps)
    flb += ckb * C_darcy * (F(-2) * om * den - om * om * F(3) * fl * fl) / (den * den);
    // ur = (j + F/2) * inv_rho
    F jxb = uxrb * inv_rho, jyb = uyrb * inv_rho, jzb = uzrb * inv_rho;
    fxb += F(0.5) * uxrb * inv_rho;
    fyb += F(0.5) * uyrb * inv_rho;
    fzb += F(0.5) * uzrb * inv_rho;
    F invb = uxrb * (jx + F(0.5) * fx) + uyrb * (jy + F(0.5) * fy) + uzrb * (jz + F(0.5) * fz);
    rb -= invb * inv_rho * inv_rho;
    // linear moments of f
    for (int q = 0; q < 19; ++q) {
        const int a = cx(q), b = cy(q), c = cz(q);
        F g = rb + F(a) * jxb + F(b) * jyb + F(c) * jzb;
        g += F(a * a) * Pxxb + F(b * b) * Pyyb + F(c * c) * Pzzb;
        g += F(a * b) * Pxyb + F(a * c) * Pxzb + F(b * c) * Pyzb;
        fb[q] += g;
    }
}

// Marangoni force of one cell (kernels.py:2158-2217, inside cell_forces) is
// linear in T: F = dgamma * g * (I - n n^T) t with t the half central
// differences of T along x, y, z.  Reverse: the adjoint of t.
template <class F>
WAAM_HD void marangoni_t_vjp(F nxn, F nyn, F nzn, F scale, F fxb, F fyb, F fzb, F& txb, F& tyb,
                             F& tzb) {
    const F nd = nxn * fxb + nyn * fyb + nzn * fzb;
    txb = scale * (fxb - nd * nxn);
    tyb = scale * (fyb - nd * nyn);
    tzb = scale * (fzb - nd * nzn);
}

}  // namespace waam_adj
