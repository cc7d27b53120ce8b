// spectral.cuh -- hero-wavelength spectral rendering: wavelength sampling,
// CIE 1931 / D65 weights and the reference's RGB -> spectrum upsampling through
// its tabulated basis network (core/spectrum/*).
//
// Tables (colour matching functions, D65, network weights) are the reference's
// data, supplied at run time through ar_scene_set_spectral.  The two lookup
// tables the path loop reads -- a wavelength table of 840 x 4 values and an
// RGB table of res^3 x 4 values -- are built on the GPU by k_lut_lambda /
// k_lut_rgb from those weights (PrecomputeLambdaLUTKernel /
// PrecomputeRGBLUTKernel, spectrum_lut.cuh:12-58).
//
// Arithmetic follows the reference's expressions: explicit fmaf where it uses
// fmaf / __fmaf_rn (network layers, LUT accumulation, inverse normal CDF),
// otherwise no contraction; sin/cos/exp/log are this project's fixed functions
// (detmath.h), erfc is the rational approximation of Numerical Recipes
// (Press et al., 2nd ed., sec. 6.2, fractional error < 1.2e-7).
#pragma once

#include "detmath.h"

namespace ar {

constexpr int kSpecKernel = 4;         // spectrum::query::KERNEL
constexpr int kSpecWidth = 32;         // spectrum::query::WIDTH
constexpr int kSpecBlocks = 7;         // residual blocks per network
constexpr int kLambdaLutRes = 840;     // SPECTRUM_LAMBDA_LUT_RES (config.cuh:64)
constexpr float kLamMin = 360.0f, kLamMax = 780.0f;
constexpr float kSpecPi = 3.141592654f;  // CUDART_PI_F

// Offsets (floats) of the table block passed to ar_scene_set_spectral.
constexpr int kTabCmf = 0;                                   // 421 x 3
constexpr int kTabD65 = kTabCmf + 421 * 3;                   // 421
constexpr int kTabRgbInW = kTabD65 + 421;                    // 32 x 32
constexpr int kTabRgbInB = kTabRgbInW + 1024;                // 32
constexpr int kTabRgbBlkW = kTabRgbInB + 32;                 // 7 x 32 x 32
constexpr int kTabRgbBlkB = kTabRgbBlkW + 7 * 1024;          // 7 x 32
constexpr int kTabRgbOutW = kTabRgbBlkB + 7 * 32;            // 4 x 32
constexpr int kTabLamBlkW = kTabRgbOutW + 128;               // 7 x 32 x 32
constexpr int kTabLamBlkB = kTabLamBlkW + 7 * 1024;          // 7 x 32
constexpr int kTabLamOutW = kTabLamBlkB + 7 * 32;            // 4 x 32
constexpr int kTabFloats = kTabLamOutW + 128;                // 17780

struct SpectralView {
    const float* tables;     // kTabFloats values (device)
    const float4* lut_rgb;   // res^3 entries, x fastest
    const float4* lut_lam;   // kLambdaLutRes entries
    int32_t res;
    int32_t pad;
};

// ---------------------------------------------------------------- tables
// D65Norm (ciexyz.cuh:67-82)
AR_HD float d65_norm(const float* tab, float lambda)
{
    const float* d65 = tab + kTabD65;
    const float k = 1.0f / 10567.065f;
    if (lambda <= 360.0f) return d65[0] * k;
    if (lambda >= 780.0f) return d65[420] * k;
    const float x = lambda - 360.0f;
    const int i = static_cast<int>(floorf(x));
    const float t = x - static_cast<float>(i);
    const float v0 = d65[i], v1 = d65[i + 1];
    return (v0 + (v1 - v0) * t) * k;
}

// LambdaToCIE1931_XYZ (ciexyz.cuh:522-541)
AR_HD f3 cmf_xyz(const float* tab, float lambda)
{
    const float* c = tab + kTabCmf;
    if (lambda <= 360.0f) return mk(c[0], c[1], c[2]);
    if (lambda >= 780.0f) return mk(c[1260], c[1261], c[1262]);
    const float u = (lambda - 360.0f) * (1.0f / 1.0f);
    const int i = static_cast<int>(u);
    const float t = u - static_cast<float>(i);
    const float* a = c + 3 * i;
    const float* b = a + 3;
    return mk(a[0] + (b[0] - a[0]) * t, a[1] + (b[1] - a[1]) * t, a[2] + (b[2] - a[2]) * t);
}

// ---------------------------------------------------------------- sampling
AR_HD float erfc_nr(float x)
{
    const float z = fabsf(x);
    const float t = 1.0f / (1.0f + 0.5f * z);
    const float p = -z * z - 1.26551223f +
                    t * (1.00002368f + t * (0.37409196f + t * (0.09678418f + t * (-0.18628806f +
                    t * (0.27886807f + t * (-1.13520398f + t * (1.48851587f + t * (-0.82215223f + t * 0.17087277f))))))));
    const float r = t * exp_det(p);
    return x >= 0.0f ? r : 2.0f - r;
}

// ndtrif (sample_ciexyz.cuh:28-156): Acklam's rational inverse normal CDF with
// one Newton step.
AR_HD float ndtri_newton(float u)
{
    const float uu = fminf(fmaxf(u, 0.0f), 1.0f);
    const float pLow = 0.02425f, pHigh = 1.0f - 0.02425f;
    float x;
    if (uu < pLow || uu > pHigh) {
        const float q = uu < pLow ? sqrtf(-2.0f * log_det(uu)) : sqrtf(-2.0f * log_det(1.0f - uu));
        float num = fmaf(-7.784894002430293e-03f, q, -3.223964580411365e-01f);
        num = fmaf(num, q, -2.400758277161838e+00f);
        num = fmaf(num, q, -2.549732539343734e+00f);
        num = fmaf(num, q, 4.374664141464968e+00f);
        num = fmaf(num, q, 2.938163982698783e+00f);
        float den = fmaf(7.784695709041462e-03f, q, 3.224671290700398e-01f);
        den = fmaf(den, q, 2.445134137142996e+00f);
        den = fmaf(den, q, 3.754408661907416e+00f);
        den = fmaf(den, q, 1.0f);
        x = uu < pLow ? num / den : -num / den;
    } else {
        const float q = uu - 0.5f;
        const float r = q * q;
        float num = fmaf(-3.969683028665376e+01f, r, 2.209460984245205e+02f);
        num = fmaf(num, r, -2.759285104469687e+02f);
        num = fmaf(num, r, 1.383577518672690e+02f);
        num = fmaf(num, r, -3.066479806614716e+01f);
        num = fmaf(num, r, 2.506628277459239e+00f);
        num *= q;
        float den = fmaf(-5.447609879822406e+01f, r, 1.615858368580409e+02f);
        den = fmaf(den, r, -1.556989798598866e+02f);
        den = fmaf(den, r, 6.680131188771972e+01f);
        den = fmaf(den, r, -1.328068155288572e+01f);
        den = fmaf(den, r, 1.0f);
        x = num / den;
    }
    const float pdf = exp_det(fmaf(-0.5f, x * x, 0.0f)) * 0.3989422804014327f;
    const float cdf = 0.5f * erfc_nr(-x * 0.7071067811865476f);
    x -= (cdf - uu) / pdf;
    return x;
}

AR_HD float clamp_lambda(float h) { return h < kLamMin ? kLamMin : (h > kLamMax ? kLamMax : h); }

// Single-lobe analytic CMF fits (Wyman, Sloan and Shirley, JCGT 2(2) 2013) as
// the reference uses them for sampling (sample_ciexyz.cuh:160-279).
AR_HD float cmf_x_fit(float l)
{
    const float k1 = (l - 595.8f) / 33.33f, k2 = (l - 446.8f) / 19.44f;
    return 1.065f * exp_det(-0.5f * k1 * k1) + 0.366f * exp_det(-0.5f * k2 * k2);
}
AR_HD float cmf_y_fit(float l)
{
    const float k = (log_det(l) - 6.3213077f) / 0.075f;
    return 1.014f * exp_det(-0.5f * k * k);
}
AR_HD float cmf_z_fit(float l)
{
    const float k = (log_det(l) - 6.1088030f) / 0.051f;
    return 1.839f * exp_det(-0.5f * k * k);
}

struct LambdaSample { float lambda, pdf; };

// Density of sample_cie1931's wavelength: the mixture of a uniform share and
// the three fitted colour-matching lobes.
AR_HD float pdf_cie1931(float lambda)
{
    const float total = 0.1f + 1.0f + 1.0f + 1.0f;
    const float uniformRatio = 0.1f / total, xRatio = 1.0f / total, yRatio = 1.0f / total, zRatio = 1.0f / total;
    const float pMix = uniformRatio * 1.0f / (780.0f - 360.0f) + xRatio * (cmf_x_fit(lambda) / 106.81109281f) +
                       yRatio * (cmf_y_fit(lambda) / 106.34513640f) + zRatio * (cmf_z_fit(lambda) / 105.88243587f);
    return fmaxf(pMix, 1e-16f);
}

// SampleCIE1931 (sample_ciexyz.cuh:288-325): a 0.1 : 1 : 1 : 1 mixture of the
// uniform density and the three CMF lobes.
AR_HD LambdaSample sample_cie1931(float r0, float r1, float r2)
{
    const float total = 0.1f + 1.0f + 1.0f + 1.0f;
    const float uniformRatio = 0.1f / total, xRatio = 1.0f / total, yRatio = 1.0f / total;
    float lambda;
    if (r0 < uniformRatio) {
        lambda = r1 * (780.0f - 360.0f) + 360.0f;
    } else if (r0 < uniformRatio + xRatio) {
        float h;
        if (r1 < 0.8330258723493694f) {
            const float t0 = 7.4884543e-13f + r2 * (0.9999999836707862f - 7.4884543e-13f);
            h = 595.7999999999999545f + 33.3299999999999983f * ndtri_newton(t0);
        } else {
            const float t1 = 0.0000040030528583f + r2 * (1.0f - 0.0000040030528583f);
            h = 446.8000000000000114f + 19.4400000000000013f * ndtri_newton(t1);
        }
        lambda = clamp_lambda(h);
    } else if (r0 < uniformRatio + xRatio + yRatio) {
        const float t = 0.0000000020798312f + r1 * (0.9999953206338883f - 0.0000000020798312f);
        lambda = clamp_lambda(exp_det(6.3269327170812479f + 0.0750000000000000f * ndtri_newton(t)));
    } else {
        const float t = 0.0000049890553249f + r1 * (1.0f - 0.0000049890553249f);
        lambda = clamp_lambda(exp_det(6.1114040395252154f + 0.0510000000000000f * ndtri_newton(t)));
    }
    LambdaSample s;
    s.lambda = lambda;
    s.pdf = pdf_cie1931(lambda);
    return s;
}

// Four wavelengths per path (extension; the reference traces one): the hero
// and its rotations by a quarter of [360, 780] nm (Wilkie et al., "Hero
// wavelength spectral sampling", 2014).  Wavelength i of a hero h.
AR_HD float rotate_lambda(float h, int i)
{
    float x = h - 360.0f + 105.0f * static_cast<float>(i);
    if (x >= 420.0f) x -= 420.0f;
    return 360.0f + x;
}

// ---------------------------------------------------------------- dispersion
// IORFromAbbeNM / SigmaAFromTiltNM (spectrum.cuh:8-54)
AR_HD float ior_abbe(float lambda, float nd, float vd)
{
    if (!(lambda > 0.0f)) return nd;
    const float invF = 1.0f / 486.1327f, invC = 1.0f / 656.2725f, invD = 1.0f / 587.5618f;
    const float K = (vd > 0.0f) ? (nd - 1.0f) / (vd * (invF - invC)) : 0.0f;
    const float invL = 1.0f / lambda;
    return nd + K * (invL - invD);
}
AR_HD float sigma_tilt(float sigmaA, float lambda, float tilt)
{
    const float invF = 1.0f / 486.1327f, invC = 1.0f / 656.2725f, invD = 1.0f / 587.5618f;
    const float u = 1.0f / fmaxf(lambda, 1.0e-6f);
    const float du = (u - invD) / (invF - invC);
    const float sA = sigmaA * (1.0f + 1.0f * tilt * du);
    return fmaxf(0.0f, sA);
}

// ---------------------------------------------------------------- basis network
// One residual block: h += relu(W h + b), W row-major [out][in], accumulated in
// input order with fmaf (tensor::LinearRowMajor, tensor.cuh:103-176).
AR_HD void spec_block(float* h, const float* W, const float* B)
{
    float t[kSpecWidth];
    for (int i = 0; i < kSpecWidth; ++i) {
        float acc = B[i];
        for (int j = 0; j < kSpecWidth; ++j) acc = fmaf(h[j], W[i * kSpecWidth + j], acc);
        t[i] = fmaxf(acc, 0.0f);
    }
    for (int i = 0; i < kSpecWidth; ++i) h[i] = h[i] + t[i];
}

AR_HD void spec_out(const float* h, const float* W, float* out)
{
    for (int i = 0; i < kSpecKernel; ++i) {
        float acc = 0.0f;
        for (int j = 0; j < kSpecWidth; ++j) acc = fmaf(h[j], W[i * kSpecWidth + j], acc);
        out[i] = acc;
    }
}

// RGBEncode (spectrum_basis.cuh:2273-2378)
AR_HD void rgb_encode(const float* tab, float r, float g, float b, float* outK)
{
    const float scale = fmaxf(fmaxf(r, g), b);
    const float inv = 1.0f / (scale + 0.001f);
    float s[kSpecWidth];
    const float in[3] = {r, g, b};
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 4; ++k)
            sincos_det(in[c] * inv * kSpecPi * static_cast<float>(k + 1), &s[8 * c + k], &s[8 * c + k + 4]);
    for (int k = 0; k < 4; ++k) sincos_det(scale * kSpecPi * static_cast<float>(k + 1), &s[24 + k], &s[28 + k]);
    float h[kSpecWidth];
    const float* W = tab + kTabRgbInW;
    const float* B = tab + kTabRgbInB;
    for (int i = 0; i < kSpecWidth; ++i) {
        float acc = B[i];
        for (int j = 0; j < kSpecWidth; ++j) acc = fmaf(s[j], W[i * kSpecWidth + j], acc);
        h[i] = fmaxf(acc, 0.0f);
    }
    for (int blk = 0; blk < kSpecBlocks; ++blk)
        spec_block(h, tab + kTabRgbBlkW + blk * 1024, tab + kTabRgbBlkB + blk * 32);
    spec_out(h, tab + kTabRgbOutW, outK);
    for (int i = 0; i < kSpecKernel; ++i) outK[i] *= scale;
}

// LambdaEncode (spectrum_basis.cuh:2380-2459)
AR_HD void lambda_encode(const float* tab, float lambda, float* outK)
{
    const float x = fminf(fmaxf((lambda - 360.0f) / (780.0f - 360.0f), 0.0f), 1.0f);
    float h[kSpecWidth];
    for (int k = 0; k < kSpecWidth / 2; ++k) sincos_det(x * kSpecPi * static_cast<float>(k + 1), &h[k], &h[k + 16]);
    for (int blk = 0; blk < kSpecBlocks; ++blk)
        spec_block(h, tab + kTabLamBlkW + blk * 1024, tab + kTabLamBlkB + blk * 32);
    spec_out(h, tab + kTabLamOutW, outK);
}

// SpectralInteract (spectrum_basis.cuh:2461-2470)
AR_HD float spectral_interact(const float* rk, const float* lk)
{
    float acc = 0.0f;
    for (int i = 0; i < kSpecKernel; ++i) acc = fmaf(rk[i], lk[i], acc);
    return fminf(fmaxf(acc, 0.0f), 1.0f);
}

// ---------------------------------------------------------------- LUT queries
// __linear_coord (spectrum_lut.cuh:92-106)
AR_HD void linear_coord(float g, int res, int& i0, int& i1, float& t)
{
    const float fi0 = floorf(g);
    i0 = static_cast<int>(fi0);
    i1 = i0 + 1;
    if (i1 >= res) i1 = res - 1;
    t = g - fi0;
    if (i0 == i1) t = 0.0f;
}

// QueryLambda (spectrum_lut.cuh:181-220)
AR_HD float4 query_lambda(const float4* lut, float lambda)
{
    float u = (lambda - 360.0f) / (780.0f - 360.0f);
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    float g = u * static_cast<float>(kLambdaLutRes) - 0.5f;
    g = fminf(fmaxf(g, 0.0f), static_cast<float>(kLambdaLutRes) - 1.0f);
    int i0, i1;
    float t;
    linear_coord(g, kLambdaLutRes, i0, i1, t);
    const float w0 = 1.0f - t, w1 = t;
    const float4 a = lut[i0], b = lut[i1];
    return make_float4(a.x * w0 + b.x * w1, a.y * w0 + b.y * w1, a.z * w0 + b.z * w1, a.w * w0 + b.w * w1);
}

AR_HD void accum4(float4 v, float w, float* o)
{
    o[0] = fmaf(w, v.x, o[0]);
    o[1] = fmaf(w, v.y, o[1]);
    o[2] = fmaf(w, v.z, o[2]);
    o[3] = fmaf(w, v.w, o[3]);
}

// QueryRGBBasis (spectrum_lut.cuh:124-179): trilinear over the res^3 table.
AR_HD void query_rgb(const float4* lut, int res, f3 rgb, float* k)
{
    const float maxC = static_cast<float>(res) - 1.0f;
    const float gx = fminf(fmaxf(rgb.x * static_cast<float>(res) - 0.5f, 0.0f), maxC);
    const float gy = fminf(fmaxf(rgb.y * static_cast<float>(res) - 0.5f, 0.0f), maxC);
    const float gz = fminf(fmaxf(rgb.z * static_cast<float>(res) - 0.5f, 0.0f), maxC);
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    linear_coord(gx, res, x0, x1, tx);
    linear_coord(gy, res, y0, y1, ty);
    linear_coord(gz, res, z0, z1, tz);
    const float wx0 = 1.0f - tx, wx1 = tx, wy0 = 1.0f - ty, wy1 = ty, wz0 = 1.0f - tz, wz1 = tz;
    const int sy = res, sz = res * res;
    k[0] = k[1] = k[2] = k[3] = 0.0f;
    accum4(lut[x0 + y0 * sy + z0 * sz], wx0 * wy0 * wz0, k);
    accum4(lut[x1 + y0 * sy + z0 * sz], wx1 * wy0 * wz0, k);
    accum4(lut[x0 + y1 * sy + z0 * sz], wx0 * wy1 * wz0, k);
    accum4(lut[x1 + y1 * sy + z0 * sz], wx1 * wy1 * wz0, k);
    accum4(lut[x0 + y0 * sy + z1 * sz], wx0 * wy0 * wz1, k);
    accum4(lut[x1 + y0 * sy + z1 * sz], wx1 * wy0 * wz1, k);
    accum4(lut[x0 + y1 * sy + z1 * sz], wx0 * wy1 * wz1, k);
    accum4(lut[x1 + y1 * sy + z1 * sz], wx1 * wy1 * wz1, k);
}

// spectrum::lut::Interact (spectrum_lut.cuh:222-236): reflectance or emission
// of an RGB colour at the wavelength whose basis is lk; colours above 1 are
// normalised by their maximum and scaled back.
AR_HD float interact(const float4* lut, int res, float4 lk, f3 rgb)
{
    const float lum = fmaxf(rgb.x, fmaxf(rgb.y, rgb.z));
    float k[4];
    const float l4[4] = {lk.x, lk.y, lk.z, lk.w};
    if (lum > 1.0f) {
        query_rgb(lut, res, mk(rgb.x / lum, rgb.y / lum, rgb.z / lum), k);
        return spectral_interact(k, l4) * lum;
    }
    query_rgb(lut, res, rgb, k);
    return spectral_interact(k, l4);
}

}  // namespace ar
