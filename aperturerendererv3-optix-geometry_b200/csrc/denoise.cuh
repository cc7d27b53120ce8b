// denoise.cuh -- per-pixel guide buffers of the screen-space denoiser.
//
// record_gbuffer follows denoise::RecordScreenGBuffer / RecordShadingModel
// (core/denoise/denoise.cuh:86-166): running means over frames kept in half
// precision, each update rounded to half exactly where the reference rounds.
// record_stats follows denoise::RecordScreenStatisticBuffer
// (core/denoise/denoise_statistic.cuh:37-69): Welford mean and second/third
// central moments of the Box-Cox(0.5) transformed sample, the moment updates
// in double.  The reference's powf(x, 0.5f) is sqrtf(x) here: the correctly
// rounded value of the same function, identical on host and device.
#pragma once

#include <cuda_fp16.h>

#include "../../include/aperture_b200.h"
#include "detmath.h"

namespace ar {

constexpr int kDnModels = 5;  // MAT_MAX + 1 (core/render/object.cuh:45-52): [4] = no surface

struct DenoiseView {
    ar_screen_gbuffer* gbuf;  // NULL: not recorded
    ar_screen_stats* stat;    // NULL: not recorded
};

__device__ __forceinline__ float h2f(uint16_t h) { return __half2float(__ushort_as_half(h)); }
__device__ __forceinline__ uint16_t f2h(float f) { return __half_as_ushort(__float2half_rn(f)); }

// RecordShadingModel (denoise.cuh:86-104), on the frame counter before its increment
__device__ __forceinline__ void record_model(ar_screen_gbuffer& g, int model)
{
    if (g.frames == 0) {
#pragma unroll
        for (int i = 0; i < kDnModels; ++i) g.shading_model[i] = 0;
    }
    const float affix = 1.0f / static_cast<float>(g.frames + 1u);
    const float pre = static_cast<float>(g.frames) / static_cast<float>(g.frames + 1u);
#pragma unroll
    for (int i = 0; i < kDnModels; ++i) g.shading_model[i] = f2h(h2f(g.shading_model[i]) * pre);
    g.shading_model[model] = f2h(h2f(g.shading_model[model]) + affix);
}

// RecordScreenGBuffer (denoise.cuh:106-166) for one pixel and frame.
__device__ __forceinline__ void record_gbuffer(ar_screen_gbuffer* gp, bool hit, f3 albedo, f3 normal, float metallic,
                                               float roughness, float depth, int model)
{
    ar_screen_gbuffer g = *gp;
    if (hit) {
        if (g.valid_frames == 0) {
            g.albedo[0] = g.albedo[1] = g.albedo[2] = 0;
            g.normal[0] = g.normal[1] = g.normal[2] = 0;
            g.metallic = g.roughness = 0;
            g.depth = 0.0f;
        }
        const float affix = 1.0f / static_cast<float>(g.valid_frames + 1u);
        const float pre = static_cast<float>(g.valid_frames) / static_cast<float>(g.valid_frames + 1u);
        const float a[3] = {albedo.x, albedo.y, albedo.z};
        const float n[3] = {normal.x, normal.y, normal.z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            g.albedo[c] = f2h(h2f(g.albedo[c]) * pre);
            g.normal[c] = f2h(h2f(g.normal[c]) * pre);
        }
        g.metallic = f2h(h2f(g.metallic) * pre);
        g.roughness = f2h(h2f(g.roughness) * pre);
        g.depth = g.depth * pre;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            g.albedo[c] = f2h(h2f(g.albedo[c]) + affix * a[c]);
            g.normal[c] = f2h(h2f(g.normal[c]) + affix * n[c]);
        }
        g.metallic = f2h(h2f(g.metallic) + affix * metallic);
        g.roughness = f2h(h2f(g.roughness) + affix * roughness);
        g.depth = g.depth + affix * depth;
        ++g.valid_frames;
        record_model(g, model);
    } else {
        record_model(g, kDnModels - 1);
    }
    ++g.frames;
    *gp = g;
}

// RecordScreenStatisticBuffer (denoise_statistic.cuh:37-69) for one pixel and sample.
__device__ __forceinline__ void record_stats(ar_screen_stats* sp, f3 x)
{
    ar_screen_stats s = *sp;
    const uint32_t n0 = s.num, n1 = n0 + 1u;
    s.num = n1;
    const float xs[3] = {x.x, x.y, x.z};
    const float invN1 = 1.0f / static_cast<float>(n1);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float bc = (sqrtf(fmaxf(xs[c], 0.0f)) - 1.0f) * 2.0f;  // BoxCox05 (denoise_statistic.cuh:26-34)
        const float delta = bc - s.mean[c];
        const float dn = delta * invN1;
        const double m2 = static_cast<double>(s.m2_div_n[c]) * static_cast<double>(n0) +
                          static_cast<double>(delta * (delta - dn));
        const float d2 = delta * delta, dn2 = dn * dn;
        const double m3 = (static_cast<double>(s.m3_div_n[c]) * static_cast<double>(n0) -
                           3.0 * (static_cast<double>(dn) * m2)) +
                          static_cast<double>(delta * (d2 - dn2));
        s.mean[c] = s.mean[c] + dn;
        s.m2_div_n[c] = static_cast<float>(m2 / static_cast<double>(n1));
        s.m3_div_n[c] = static_cast<float>(m3 / static_cast<double>(n1));
    }
    *sp = s;
}

}  // namespace ar
