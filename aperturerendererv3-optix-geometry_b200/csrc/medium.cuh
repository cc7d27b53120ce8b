// medium.cuh -- a heterogeneous participating medium (an extension: the
// reference has no volumetric media; its Henyey-Greenstein helpers,
// core/render/sample.cuh:110-145, have no call site).
//
// One axis-aligned box per scene holding a density grid (float or half, x
// fastest, trilinear, clamped to the edge) scaled by sigma_t_max; constant
// single-scatter albedo and Henyey-Greenstein asymmetry g.
//   delta_track   free-flight sampling by delta (Woodcock) tracking against the
//                 majorant sigma_t_max * max(density) (Woodcock et al. 1965;
//                 Novak et al., "Monte Carlo methods for volumetric light
//                 transport simulation", 2018): the first real collision on
//                 [0, tmax) or -1
//   hg_sample     direction from the Henyey-Greenstein phase function by
//                 inversion of its CDF (exact importance sampling: phase/pdf = 1)
//   ratio_track   transmittance estimate for shadow rays
//   HashRng       counter-based uniforms for shadow-ray transmittance (the
//                 "lowbias32" integer hash of C. Wellons), seeded from the path
// Every function is host+device so the oracle can replay the same steps.
#pragma once

#include <cuda_fp16.h>

#include "detmath.h"

namespace ar {

struct alignas(16) MediumRec {
    float bmin[3];
    float sigma_max;     // sigma_t of density 1
    float bmax[3];
    float g;             // Henyey-Greenstein asymmetry
    float albedo[3];     // single-scatter albedo
    float majorant;      // sigma_max * max(density)
    int32_t dims[3];
    int32_t fp16;
    const void* data;    // density grid (device for the kernels, host for the builder)
    int32_t pad[2];
};
static_assert(sizeof(MediumRec) == 80, "MediumRec must be 80 bytes");

AR_HD float medium_value(const MediumRec& m, size_t i)
{
#ifdef __CUDA_ARCH__
    if (m.fp16) return __half2float(__ldg(static_cast<const __half*>(m.data) + i));
    return __ldg(static_cast<const float*>(m.data) + i);
#else
    if (m.fp16) return __half2float(static_cast<const __half*>(m.data)[i]);
    return static_cast<const float*>(m.data)[i];
#endif
}

AR_HD int clamp_index(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }

// Density at world point p: trilinear between voxel centres, clamped at the edges.
AR_HD float medium_density(const MediumRec& m, f3 p)
{
    const float gx = (p.x - m.bmin[0]) / (m.bmax[0] - m.bmin[0]) * static_cast<float>(m.dims[0]) - 0.5f;
    const float gy = (p.y - m.bmin[1]) / (m.bmax[1] - m.bmin[1]) * static_cast<float>(m.dims[1]) - 0.5f;
    const float gz = (p.z - m.bmin[2]) / (m.bmax[2] - m.bmin[2]) * static_cast<float>(m.dims[2]) - 0.5f;
    const float fx0 = floorf(gx), fy0 = floorf(gy), fz0 = floorf(gz);
    const float tx = gx - fx0, ty = gy - fy0, tz = gz - fz0;
    const int x0 = clamp_index(static_cast<int>(fx0), m.dims[0] - 1), x1 = clamp_index(static_cast<int>(fx0) + 1, m.dims[0] - 1);
    const int y0 = clamp_index(static_cast<int>(fy0), m.dims[1] - 1), y1 = clamp_index(static_cast<int>(fy0) + 1, m.dims[1] - 1);
    const int z0 = clamp_index(static_cast<int>(fz0), m.dims[2] - 1), z1 = clamp_index(static_cast<int>(fz0) + 1, m.dims[2] - 1);
    const size_t sx = 1, sy = static_cast<size_t>(m.dims[0]), sz = static_cast<size_t>(m.dims[0]) * m.dims[1];
    const float c000 = medium_value(m, x0 * sx + y0 * sy + z0 * sz), c100 = medium_value(m, x1 * sx + y0 * sy + z0 * sz);
    const float c010 = medium_value(m, x0 * sx + y1 * sy + z0 * sz), c110 = medium_value(m, x1 * sx + y1 * sy + z0 * sz);
    const float c001 = medium_value(m, x0 * sx + y0 * sy + z1 * sz), c101 = medium_value(m, x1 * sx + y0 * sy + z1 * sz);
    const float c011 = medium_value(m, x0 * sx + y1 * sy + z1 * sz), c111 = medium_value(m, x1 * sx + y1 * sy + z1 * sz);
    const float c00 = c000 * (1.0f - tx) + c100 * tx, c10 = c010 * (1.0f - tx) + c110 * tx;
    const float c01 = c001 * (1.0f - tx) + c101 * tx, c11 = c011 * (1.0f - tx) + c111 * tx;
    const float c0 = c00 * (1.0f - ty) + c10 * ty, c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}

// Entry and exit distances of the ray in the medium box, clipped to [0, tmax].
AR_HD bool medium_span(const MediumRec& m, f3 o, f3 d, float tmax, float* t0, float* t1)
{
    const f3 inv = mk(inv_safe(d.x), inv_safe(d.y), inv_safe(d.z));
    const f3 a = (mk(m.bmin[0], m.bmin[1], m.bmin[2]) - o) * inv;
    const f3 b = (mk(m.bmax[0], m.bmax[1], m.bmax[2]) - o) * inv;
    const f3 lo = vmin(a, b), hi = vmax(a, b);
    const float tn = fmaxf(fmaxf(fmaxf(lo.x, lo.y), lo.z), 0.0f);
    const float tf = fminf(fminf(fminf(hi.x, hi.y), hi.z), tmax);
    *t0 = tn;
    *t1 = tf;
    return tn < tf && m.majorant > 0.0f;
}

constexpr int kMediumMaxSteps = 4096;  // tentative collisions per segment (bounded loop)

// First real collision along the ray before tmax, or -1.  `next` yields
// uniforms in (0, 1].
template <class Next>
AR_HD float delta_track(const MediumRec& m, f3 o, f3 d, float tmax, Next&& next)
{
    float t0, t1;
    if (!medium_span(m, o, d, tmax, &t0, &t1)) return -1.0f;
    float t = t0;
    for (int i = 0; i < kMediumMaxSteps; ++i) {
        t = t - log_det(1.0f - next() * 0.99999994f) / m.majorant;
        if (t >= t1) return -1.0f;
        const float s = medium_density(m, o + d * t) * m.sigma_max;
        if (next() * m.majorant < s) return t;
    }
    return -1.0f;
}

// Transmittance estimate along [0, tmax) by ratio tracking (Cramer 1978;
// Novak, Selle and Jarosz, "Residual ratio tracking", 2014): the product of
// (1 - sigma_t / majorant) over the tentative collisions.
template <class Next>
AR_HD float ratio_track(const MediumRec& m, f3 o, f3 d, float tmax, Next&& next)
{
    float t0, t1;
    if (!medium_span(m, o, d, tmax, &t0, &t1)) return 1.0f;
    float t = t0, tr = 1.0f;
    for (int i = 0; i < kMediumMaxSteps; ++i) {
        t = t - log_det(1.0f - next() * 0.99999994f) / m.majorant;
        if (t >= t1) break;
        tr = tr * (1.0f - medium_density(m, o + d * t) * m.sigma_max / m.majorant);
        if (tr <= 0.0f) return 0.0f;
    }
    return tr;
}

// Henyey-Greenstein phase function value for the cosine between the
// propagation direction and the scattered direction.
AR_HD float hg_phase(float g, float cosT)
{
    const float den = 1.0f + g * g - 2.0f * g * cosT;
    return (1.0f - g * g) / (4.0f * 3.14159265358979f * den * sqrtf(den));
}

// Henyey-Greenstein: direction around the propagation direction d.
AR_HD f3 hg_sample(f3 d, float g, float u1, float u2)
{
    float cosT;
    if (fabsf(g) < 1e-3f) {
        cosT = 1.0f - 2.0f * u1;
    } else {
        const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
        cosT = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    cosT = fminf(fmaxf(cosT, -1.0f), 1.0f);
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    float sp, cp;
    sincos_det(2.0f * 3.14159265358979f * u2, &sp, &cp);
    const f3 a = fabsf(d.z) < 0.999f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    const f3 t = normalize(cross(a, d));
    const f3 b = cross(d, t);
    return normalize(t * (sinT * cp) + b * (sinT * sp) + d * cosT);
}

// Counter-based uniforms in (0, 1): the lowbias32 hash of (seed, counter).
AR_HD uint32_t lowbias32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
struct HashRng {
    uint32_t seed, n;
    AR_HD float operator()()
    {
        const uint32_t h = lowbias32(seed ^ lowbias32(n++ * 0x9E3779B9u + 0x632BE5ABu));
        return (static_cast<float>(h >> 8) + 0.5f) * (1.0f / 16777216.0f);
    }
};

// Seeds of a path's medium uniforms: a key of the render (seed and first frame
// index), then per sample, pixel, depth and use (salt 0 free flight, 1 shadow).
AR_HD uint32_t medium_frame_key(uint64_t seed, uint64_t frame0)
{
    uint32_t h = lowbias32(static_cast<uint32_t>(seed) ^ 0x6D2B79F5u);
    h = lowbias32(h ^ static_cast<uint32_t>(seed >> 32));
    h = lowbias32(h ^ static_cast<uint32_t>(frame0));
    return lowbias32(h ^ static_cast<uint32_t>(frame0 >> 32));
}
AR_HD uint32_t medium_seed(uint32_t key, uint32_t sample, uint32_t pixel, uint32_t depth, uint32_t salt)
{
    uint32_t h = lowbias32(key ^ sample);
    h = lowbias32(h ^ pixel);
    return lowbias32(h ^ (depth * 2u + salt));
}

}  // namespace ar
