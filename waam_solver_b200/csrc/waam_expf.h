/* Single-precision exponential shared by the CUDA kernels and the CPU oracle.
 *
 * Method: Cody-Waite argument reduction x = n*ln2 + r with ln2 split into a
 * short high part (exact products n*ln2_hi for |n| < 256) and a low part,
 * then e^r for |r| <= ln2/2 from the degree-7 Taylor polynomial in Horner
 * form (truncation error < 0.2 ulp), then an exact scaling by 2^n built from
 * the exponent bits (two-step scaling for subnormal results).  Every
 * operation is a plain IEEE float add/multiply, so hosts compiled with
 * -ffp-contract=off and devices compiled with -fmad=false produce
 * bit-identical results.  Accuracy against double-precision exp is checked
 * by the oracle tests (max error <= 2 ulp over the float range).
 */
#ifndef WAAM_EXPF_H
#define WAAM_EXPF_H
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define WAAM_HD __host__ __device__ __forceinline__
#else
#define WAAM_HD static inline
#endif

WAAM_HD float waam_pow2i(int e) {
    /* 2^e for e in [-126, 127] */
    uint32_t bits = (uint32_t)(e + 127) << 23;
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
}

WAAM_HD float waam_expf(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return 1.0f / 0.0f;
    if (x < -103.972084f) return 0.0f;
    const float inv_ln2 = 1.44269502f;
    const float ln2_hi = 0.693145752f;   /* 0x3F317200: low 9 mantissa bits zero */
    const float ln2_lo = 1.42860677e-06f; /* ln2 - ln2_hi */
    float t = x * inv_ln2;
    float fn = t >= 0.0f ? (float)(int)(t + 0.5f) : -(float)(int)(0.5f - t);
    int n = (int)fn;
    float r = (x - fn * ln2_hi) - fn * ln2_lo;
    float p = 1.98412698e-04f;           /* 1/5040 */
    p = p * r + 1.38888889e-03f;         /* 1/720 */
    p = p * r + 8.33333377e-03f;         /* 1/120 */
    p = p * r + 4.16666679e-02f;         /* 1/24 */
    p = p * r + 1.66666672e-01f;         /* 1/6 */
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    if (n > 127) return p * waam_pow2i(127) * waam_pow2i(n - 127);
    if (n < -126) return p * waam_pow2i(n + 64) * waam_pow2i(-64);
    return p * waam_pow2i(n);
}

#endif
