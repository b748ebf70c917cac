// Host instantiations of the per-cell reverse functions of the adjoint
// (waam_solver_b200/csrc/waam_adjoint_cell.h) in double precision, so the
// tests can compare every vector-Jacobian product with central finite
// differences of the matching forward map.  TEST INFRASTRUCTURE ONLY.
#include "../waam_solver_b200/csrc/waam_adjoint_cell.h"

extern "C" {

// in[23] = f[19], fl, fx, fy, fz; out[22] = post-collision f[19], stored u, v, w
// (after the Mach clamp with limit ucap)
void wa_mrt_forward(const double* in, double ws, double wb, double C, double ucap, double* out) {
    double r, u, v, w;
    waam_adj::mrt_forward<double>(in, in[19], in[20], in[21], in[22], ws, wb, C, out, r, u, v, w);
    if (ucap > 0) {
        double m = sqrt(u * u + v * v + w * w);
        if (m > ucap) {
            double s = ucap / (m + 1e-12);
            u *= s;
            v *= s;
            w *= s;
        }
    }
    out[19] = u;
    out[20] = v;
    out[21] = w;
}

// outb[22] -> inb[23]
void wa_mrt_vjp(const double* in, double ws, double wb, double C, double ucap, const double* outb,
                double* inb) {
    for (int q = 0; q < 23; ++q) inb[q] = 0.0;
    waam_adj::mrt_vjp<double>(in, in[19], in[20], in[21], in[22], ws, wb, C, ucap, outb,
                              outb[19], outb[20], outb[21], inb, inb[19], inb[20], inb[21],
                              inb[22]);
}

void wa_clamp(const double* x, double cap, double* y) {
    double m = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    double s = m > cap ? cap / (m + 1e-12) : 1.0;
    for (int q = 0; q < 3; ++q) y[q] = x[q] * s;
}

void wa_clamp_vjp(const double* x, double cap, const double* yb, double* xb) {
    xb[0] = yb[0];
    xb[1] = yb[1];
    xb[2] = yb[2];
    waam_adj::clamp_vjp<double>(x[0], x[1], x[2], cap, xb[0], xb[1], xb[2]);
}

}  // extern "C"
