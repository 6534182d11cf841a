/*
 * lumen_expf.h - the exponential used by every alpha, activation and
 * sigmoid evaluation on the render path, as one host/device function.
 *
 * Why a project-written exp: compositing skips a splat when
 * opacity * exp(-power) < 1/255 and stops a pixel when the transmittance
 * crosses a threshold. Those decisions flip on a one-ulp difference in exp,
 * and they decide the per-pixel contributor counts, which must agree bit for
 * bit between the CUDA kernels and the CPU restatement they are tested
 * against. Both therefore compile this one function. It uses only IEEE
 * operations whose results are fully specified (fmaf, rintf, float multiply,
 * integer bit assembly), so host and device produce identical bits.
 *
 * Method (Cody & Waite, "Software Manual for the Elementary Functions",
 * 1980): x = k*ln2 + r with k the integer nearest x*log2(e) and |r| about
 * ln2/2, where ln2 is split into a short high part (exact when multiplied by
 * any |k| < 256) and a low correction, so r is formed with two fused
 * multiply-adds. k is rounded by adding 1.5 * 2^23 inside a fused
 * multiply-add (the sum's low mantissa bits then hold k, read back as an
 * integer without a conversion instruction). e^r is the degree-7 Taylor
 * polynomial of the exponential (coefficients 1/n!), evaluated in Horner
 * form; for |r| <= 0.35 its truncation error is below 6e-9 relative. The
 * result is scaled by 2^k assembled in the exponent field, in two steps near
 * the overflow and underflow ends.
 * Accuracy: within 2 ulp of the true exponential over [-103, 88.7].
 */
#ifndef LUMEN_EXPF_H
#define LUMEN_EXPF_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define LUMEN_HD __host__ __device__ __forceinline__
#else
#define LUMEN_HD static inline
#endif

LUMEN_HD float lumen_bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof(f));
    return f;
#endif
}

/* 2^k for k in [-126, 127], assembled in the exponent field. */
LUMEN_HD float lumen_pow2i(int k) {
    return lumen_bits_to_float((uint32_t)(k + 127) << 23);
}

LUMEN_HD int lumen_float_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_int(f);
#else
    int u;
    memcpy(&u, &f, sizeof(u));
    return u;
#endif
}

/* The reduction and polynomial: p = e^r and ki with e^x = p * 2^ki; also
 * the bits of t = x*log2(e) + 1.5*2^23, which are 0x4B400000 + ki. */
LUMEN_HD float lumen_expf_reduced(float x, int* ki_out, uint32_t* tbits_out) {
    /* ln 2 = LN2_HI + LN2_LO; LN2_HI = 0x3F317200 has 16 significant bits. */
    const float LN2_HI = 0.693145751953125f;
    const float LN2_LO = 1.42860682030941723e-6f;
    const float LOG2E = 1.44269504088896341f;
    const float SHIFTER = 12582912.0f;       /* 1.5 * 2^23, bits 0x4B400000 */
    const float t = fmaf(x, LOG2E, SHIFTER);
    const float k = t - SHIFTER;             /* exact: the nearest integer to x*log2(e) */
    const int ki = lumen_float_bits(t) - 0x4B400000;
    float r = fmaf(-k, LN2_HI, x);
    r = fmaf(-k, LN2_LO, r);
    /* Taylor coefficients 1/n!, n = 7 .. 0 */
    float p = 1.98412698412698413e-4f;       /* 1/5040 */
    p = fmaf(p, r, 1.38888888888888889e-3f); /* 1/720  */
    p = fmaf(p, r, 8.33333333333333333e-3f); /* 1/120  */
    p = fmaf(p, r, 4.16666666666666667e-2f); /* 1/24   */
    p = fmaf(p, r, 1.66666666666666667e-1f); /* 1/6    */
    p = fmaf(p, r, 0.5f);                    /* 1/2    */
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    *ki_out = ki;
    *tbits_out = (uint32_t)lumen_float_bits(t);
    return p;
}

/* e^x for x in [-87, 0], where 2^ki is a normal number: the same result as
 * lumen_expf without its range checks (used where the argument is known to
 * lie in [-4.5, 0]). */
LUMEN_HD float lumen_expf_core(float x) {
    int ki;
    uint32_t tb;
    const float p = lumen_expf_reduced(x, &ki, &tb);
    /* 2^ki = bits (ki + 127) << 23 = (tb << 23) + (127 << 23) mod 2^32, as
     * 0x4B400000 << 23 vanishes mod 2^32: one integer multiply-add */
    return p * lumen_bits_to_float(tb * 8388608u + 0x3F800000u);
}

LUMEN_HD float lumen_expf(float x) {
    if (!(x == x)) return x;                 /* NaN */
    if (x > 88.72283935546875f) return INFINITY;
    if (x < -103.97208404541015625f) return 0.0f;
    int ki;
    uint32_t tb;
    const float p = lumen_expf_reduced(x, &ki, &tb);
    if (ki > 127) return (p * lumen_pow2i(ki - 1)) * 2.0f;
    if (ki < -126) return (p * lumen_pow2i(ki + 64)) * lumen_pow2i(-64);
    return p * lumen_pow2i(ki);
}

#endif /* LUMEN_EXPF_H */
