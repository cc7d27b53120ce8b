// tonemap.cuh -- tone curves of the output epilogue, the reference's
// core/tonemap.cuh restated on this project's fixed arithmetic (detmath.h):
//   Gamma      pow(c, 1/2.2)                               (tonemap.cuh:6-9)
//   ACES       RRT+ODT fit: sRGB -> AP0 -> AP1, desaturate 0.96, rational
//              curve, dark->dim surround, desaturate 0.93, AP1 -> XYZ ->
//              D60->D65 -> Rec.709, clamp at 0, gamma      (tonemap.cuh:11-117)
//   XYZ2SRGBLinearD65                                      (tonemap.cuh:119-130)
// The matrices and curve constants are the reference's (published ACES
// colour-space conversions and its curve fit); they have to be the same
// numbers for the outputs to agree.
#pragma once

#include "detmath.h"

namespace ar {

AR_HD m3 rows(f3 a, f3 b, f3 c) { m3 m; m.x = a; m.y = b; m.z = c; return m; }

AR_HD f3 tone_gamma(f3 c)
{
    const float e = 1.0f / 2.2f;
    return mk(pow_det(c.x, e), pow_det(c.y, e), pow_det(c.z, e));
}

AR_HD f3 xyz_to_srgb_linear_d65(f3 xyz)
{
    const m3 M = rows(mk(3.2406f, -1.5372f, -0.4986f), mk(-0.9689f, 1.8758f, 0.0415f), mk(0.0557f, -0.204f, 1.057f));
    const f3 r = mul(M, xyz);
    return mk(fmaxf(0.0f, r.x), fmaxf(0.0f, r.y), fmaxf(0.0f, r.z));
}

AR_HD f3 tone_aces(f3 color)
{
    const m3 AP1_2_XYZ = rows(mk(0.6624541811f, 0.1340042065f, 0.1561876870f),
                              mk(0.2722287168f, 0.6740817658f, 0.0536895174f),
                              mk(-0.0055746495f, 0.0040607335f, 1.0103391003f));
    const m3 SRGB_2_AP0 = rows(mk(0.4397010f, 0.3829780f, 0.1773350f), mk(0.0897923f, 0.8134230f, 0.0967616f),
                               mk(0.0175440f, 0.1115440f, 0.8707040f));
    const m3 AP0_2_AP1 = rows(mk(1.4514393161f, -0.2365107469f, -0.2149285693f),
                              mk(-0.0765537734f, 1.1762296998f, -0.0996759264f),
                              mk(0.0083161484f, -0.0060324498f, 0.9977163014f));
    const m3 XYZ_2_AP1 = rows(mk(1.6410233797f, -0.3248032942f, -0.2364246952f),
                              mk(-0.6636628587f, 1.6153315917f, 0.0167563477f),
                              mk(0.0117218943f, -0.0082844420f, 0.9883948585f));
    const m3 D60_2_D65 = rows(mk(0.98722400f, -0.00611327f, 0.0159533f), mk(-0.00759836f, 1.00186000f, 0.0053302f),
                              mk(0.00307257f, -0.00509595f, 1.0816800f));
    const m3 XYZ_2_REC709 = rows(mk(3.2409699419f, -1.5373831776f, -0.4986107603f),
                                 mk(-0.9692436363f, 1.8759675015f, 0.0415550574f),
                                 mk(0.0556300797f, -0.2039769589f, 1.0569715142f));
    const f3 rgb2y = mk(0.272229f, 0.674082f, 0.0536895f);

    f3 acescg = mul(AP0_2_AP1, mul(SRGB_2_AP0, color));
    float y = dot(acescg, rgb2y);
    acescg = lerp3(mk(y, y, y), acescg, 0.96f);
    const float a = 278.5085f, b = 10.7772f, c = 293.6045f, d = 88.7122f, e = 80.6889f;
    const f3 x = acescg;
    const f3 post = (x * (x * a + mk(b, b, b))) / (x * (x * c + mk(d, d, d)) + mk(e, e, e));

    // dark -> dim surround in xyY
    f3 xyz = mul(AP1_2_XYZ, post);
    const float div = fmaxf(dot(xyz, mk(1.0f, 1.0f, 1.0f)), 1.0e-4f);
    f3 xyY = mk(xyz.x / div, xyz.y / div, xyz.y);
    xyY.z = fminf(fmaxf(xyY.z, 0.0f), 65504.0f);
    xyY.z = pow_det(xyY.z, 0.9811f);
    const float m = xyY.z / fmaxf(xyY.y, 1e-4f);
    xyz = mk(xyY.x, xyY.z, (1.0f - xyY.x - xyY.y));
    xyz.x *= m;
    xyz.z *= m;
    f3 cv = mul(XYZ_2_AP1, xyz);

    y = dot(cv, rgb2y);
    cv = lerp3(mk(y, y, y), cv, 0.93f);
    xyz = mul(D60_2_D65, mul(AP1_2_XYZ, cv));
    const f3 rec = mul(XYZ_2_REC709, xyz);
    return tone_gamma(mk(fmaxf(0.0f, rec.x), fmaxf(0.0f, rec.y), fmaxf(0.0f, rec.z)));
}

// One output pixel of the reference's Tonemap kernel (core/scene.cu:180-199):
// linear RGB (or XYZ when xyz_input) times exposure, tone type 0 = none,
// 1 = gamma, 2 = ACES, saturated and packed as 0xAARRGGBB.
AR_HD uint32_t tonemap_pixel(f3 v, int tone, float exposure, int xyz_input)
{
    if (xyz_input) v = xyz_to_srgb_linear_d65(v);
    v = v * exposure;
    if (tone == 1) v = tone_gamma(v);
    else if (tone == 2) v = tone_aces(v);
    const uint32_t r = static_cast<uint32_t>(255.0f * saturate(v.x));
    const uint32_t g = static_cast<uint32_t>(255.0f * saturate(v.y));
    const uint32_t b = static_cast<uint32_t>(255.0f * saturate(v.z));
    return 0xff000000u | (r << 16) | (g << 8) | b;
}

}  // namespace ar
