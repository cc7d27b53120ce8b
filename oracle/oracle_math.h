/*
 * oracle_math.h -- deterministic single-precision sin, cos, exp, log, pow.
 *
 * TEST INFRASTRUCTURE (part of the CPU oracle).
 *
 * The reference calls sinf/cosf/sincosf/expf/logf/powf/rsqrtf in its path loop
 * (vector.cuh:271-283, sample.cuh:63-108, nee.cuh:290-297, render.cuh:58-73,
 * config.cuh:3).  Their last-ulp results differ between the host libm, CUDA's
 * accurate functions and the -use_fast_math intrinsics the reference is built
 * with, so a bit-exact CPU/GPU comparison needs one fixed definition.  These
 * functions are that definition, written from the published textbook method:
 *   - sin/cos: Cody-Waite reduction by pi/2 with a three-part split of pi/2
 *     (Cody & Waite, "Software Manual for the Elementary Functions", 1980),
 *     then the Taylor series of sin to x^11 and of cos to x^10 on [-pi/4, pi/4];
 *   - exp: reduction by ln 2 (two-part split), Taylor series to r^8, scaling by
 *     2^k with ldexpf;
 *   - log: frexp into m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1))
 *     by its series to s^11, plus e * ln 2;
 *   - pow(x, y) = exp(y log x) for x > 0;
 *   - rsqrt(x) = 1 / sqrt(x) with IEEE division and square root.
 * Every step is an IEEE-754 operation with round-to-nearest (explicit fmaf
 * where a fused multiply-add is meant), so the CUDA build of the same method
 * (compiled with --fmad=false) returns the same bits.  The coefficients are
 * 1/n! and 1/n rounded to float.  Accuracy is a few ulp for |x| < 1e5.
 */
#ifndef APERTURE_ORACLE_MATH_H
#define APERTURE_ORACLE_MATH_H

#include <math.h>

static inline void om_sincosf(float x, float* s, float* c)
{
    if (!(fabsf(x) < 1.0e5f)) {
        if (isnan(x) || isinf(x)) { *s = NAN; *c = NAN; return; }
    }
    const float k = rintf(x * 0x1.45f306p-1f);               /* x * 2/pi */
    float r = fmaf(-k, 0x1.921fb6p+0f, x);                    /* pi/2 hi  */
    r = fmaf(-k, -0x1.777a5cp-25f, r);                        /* pi/2 mid */
    r = fmaf(-k, -0x1.ee59dap-50f, r);                        /* pi/2 lo  */
    const float z = r * r;
    float ps = fmaf(z, -0x1.ae6456p-26f, 0x1.71de3ap-19f);    /* -1/11!, 1/9! */
    ps = fmaf(z, ps, -0x1.a01a02p-13f);                       /* -1/7! */
    ps = fmaf(z, ps, 0x1.111112p-7f);                         /*  1/5! */
    ps = fmaf(z, ps, -0x1.555556p-3f);                        /* -1/3! */
    const float sr = fmaf(r * z, ps, r);
    float pc = fmaf(z, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);    /* -1/10!, 1/8! */
    pc = fmaf(z, pc, -0x1.6c16c2p-10f);                       /* -1/6! */
    pc = fmaf(z, pc, 0x1.555556p-5f);                         /*  1/4! */
    pc = fmaf(z, pc, -0.5f);                                  /* -1/2! */
    const float cr = fmaf(z, pc, 1.0f);
    const int q = (int)((long long)k & 3);
    switch (q) {
    case 0: *s = sr;  *c = cr;  break;
    case 1: *s = cr;  *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
    }
}

static inline float om_sinf(float x) { float s, c; om_sincosf(x, &s, &c); return s; }
static inline float om_cosf(float x) { float s, c; om_sincosf(x, &s, &c); return c; }
static inline float om_tanf(float x) { float s, c; om_sincosf(x, &s, &c); return s / c; }

static inline float om_expf(float x)
{
    if (isnan(x)) return x;
    if (x > 88.72f) return INFINITY;
    if (x < -103.98f) return 0.0f;
    const float k = rintf(x * 0x1.715476p+0f);                /* x * log2(e) */
    float r = fmaf(-k, 0x1.62e430p-1f, x);                    /* ln2 hi */
    r = fmaf(-k, -0x1.05c610p-29f, r);                        /* ln2 lo */
    float p = 0x1.a01a02p-16f;                                /* 1/8! */
    p = fmaf(p, r, 0x1.a01a02p-13f);                          /* 1/7! */
    p = fmaf(p, r, 0x1.6c16c2p-10f);                          /* 1/6! */
    p = fmaf(p, r, 0x1.111112p-7f);                           /* 1/5! */
    p = fmaf(p, r, 0x1.555556p-5f);                           /* 1/4! */
    p = fmaf(p, r, 0x1.555556p-3f);                           /* 1/3! */
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return ldexpf(p, (int)k);
}

static inline float om_logf(float x)
{
    if (isnan(x) || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (isinf(x)) return x;
    int e;
    float m = frexpf(x, &e);                                  /* m in [0.5, 1) */
    if (m < 0x1.6a09e6p-1f) { m = m * 2.0f; e = e - 1; }      /* sqrt(1/2) */
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = fmaf(z, 0x1.745d18p-4f, 0x1.c71c72p-4f);        /* 1/11, 1/9 */
    p = fmaf(z, p, 0x1.24924ap-3f);                           /* 1/7 */
    p = fmaf(z, p, 0x1.99999ap-3f);                           /* 1/5 */
    p = fmaf(z, p, 0x1.555556p-2f);                           /* 1/3 */
    const float t = 2.0f * s;
    const float logm = fmaf(t * z, p, t);
    const float ef = (float)e;
    return fmaf(ef, 0x1.62e430p-1f, fmaf(ef, -0x1.05c610p-29f, logm));
}

static inline float om_powf(float x, float y)
{
    if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    if (x == 1.0f || y == 0.0f) return 1.0f;
    if (x < 0.0f || isnan(x) || isnan(y)) return NAN;
    return om_expf(y * om_logf(x));
}

static inline float om_rsqrtf(float x) { return 1.0f / sqrtf(x); }

#endif /* APERTURE_ORACLE_MATH_H */
