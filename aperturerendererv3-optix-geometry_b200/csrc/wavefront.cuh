// wavefront.cuh -- path state and launch parameters of the wavefront pipeline.
//
// The reference runs one 168-register megakernel thread per pixel per frame
// (RenderCamera, core/scene.cu:201-255, calling CalculateRadiance,
// core/render/render.cuh:460-999).  Here a path's loop body is split at its two
// BVH queries into kernels that communicate through HBM:
//   plan/regen -> extend (closest hit) -> shade (BSDF sample, emission + MIS,
//   light sample, Russian roulette) -> shadow (any hit, adds the NEE term)
//   -> retire (FP64 accumulation)
// and the whole sequence repeats until every sample has been traced.
//
// Layout.  A path is one 128-byte record (one L2 line).  Paths live in two
// dense pools used alternately: extend reads the current pool in order, shade
// writes every surviving path into the next pool at a warp-aggregated append
// position, and new samples are appended behind them, so traversal reads are
// sequential and no index queue is needed for extension rays.  Shading is
// ordered by material (one bucket per shading model plus misses); shadow
// segments and finished paths go to dense side arrays.  Every stage draws its
// uniforms from the path's own curand XORWOW state, seeded as the reference
// seeds it (core/random.cuh:31-39), in the reference's order.
#pragma once

#include <cstdint>

#include "../../include/aperture_b200.h"
#include "denoise.cuh"
#include "guiding.cuh"
#include "nrc.cuh"
#include "spectral.cuh"
#include "traverse.cuh"

namespace ar {

enum : int32_t {
    kFlagPrevNEE = 1,      // previousNEEState.previousDidNEE_
    kFlagInside = 2,       // MediaContext::bInsideMedia_
    kFlagHeroOnly = 4,     // four-wavelength mode: the other wavelengths ended at dispersive glass
};

constexpr int kModelMedium = 4;   // shade bucket of collisions in the participating medium
constexpr int kShadeBuckets = 6;  // miss, then shading model + 1 (medium: kModelMedium + 1)
constexpr int32_t kHitMedium = -2; // hit object of a medium collision

struct alignas(16) PathRec {
    float4 o;     // ray origin xyz; w: depth | nonDeltaDepth << 16 (int bits)
    float4 d;     // ray direction xyz; w: flags | media depth << 8 (int bits)
    float4 mask;  // throughput rgb (spectral: x throughput, y wavelength, z its pdf; four wavelengths:
                  // wavelengths 0-2); w: pixel (int bits)
    float4 rad;   // radiance rgb (spectral: x; four wavelengths: 0-2); w: sample index (int bits)
    uint4 rng0;   // xorwow d, v0, v1, v2
    uint4 rng1;   // xorwow v3, v4; z media object; w uniforms consumed (cache mode: spread sum, float bits)
    float4 prev;  // previous NEE vertex xyz; w previous BSDF pdf (cache mode: +inf after a delta event)
    float4 vloc;  // media vertex location xyz; w (cache mode) square root of the primary spread a0
};
static_assert(sizeof(PathRec) == 128, "PathRec must be one 128-byte line");

struct alignas(16) ShadowRec {
    float4 src;   // segment start xyz; w segment eps
    float4 dst;   // segment end xyz; w target: >= 0 next-pool index, < 0 ~retire index
    float4 nee;   // pending radiance rgb (throughput applied); w bit 0: cosX > 0 && cosY > 0,
                  // bits 1-31: seed of the medium transmittance estimate
};

struct alignas(16) RetireRec {
    float4 rad;   // radiance rgb; w pixel (int bits)
    int4 meta;    // x sample index, y uniforms consumed, z/w wavelength and pdf bits (spectral)
};

// Control block of the path pool (device memory).
struct PoolCtl {
    int32_t count[2];                   // paths in pool buffer 0 / 1
    int32_t shade_count[8];             // shade bucket lengths (kShadeBuckets used)
    int32_t shadow_count;               // shadow segments this iteration
    int32_t retire_count;               // paths that ended this iteration
    int32_t fetch_ext, fetch_shadow, fetch_rays;  // persistent-kernel work counters
    int32_t plan_new;                   // samples started this iteration
    int32_t plan_base;                  // pool index of the first of them
    int32_t pad[3];
    int64_t gen_next;                   // next sample index to start (g = s * npix + p)
    int64_t plan_first;                 // sample index of the first path started this iteration
    int64_t retired;                    // paths finished so far
    int64_t total;                      // samples of this render (spp * npix)
};

struct PathBuffers {
    PathRec* pool[2];
    float4* aux[2];      // four-wavelength mode, per pool index: throughput and radiance of
                         // wavelength 3, hero wavelength, unused
    float* shadow3;      // four-wavelength mode: pending radiance of wavelength 3 per shadow segment
    int4* hit;           // per current-pool index: object, prim slot, t bits
    int32_t* qsh;        // shade buckets, kShadeBuckets x capacity
    ShadowRec* shadow;   // capacity entries
    RetireRec* retire;   // capacity entries
    int32_t capacity;    // paths per pool buffer
    int32_t pad;
};

struct FrameParams {
    // camera (RenderCamera, scene.cu:213-230), precomputed on the host
    float cam_o[3];
    float cam_d[3];
    float right[3];
    float up[3];
    float tan_half_x, tan_half_y;
    int32_t width, height;
    int32_t grid_x;          // ceil(width / 8): reference block grid for the pixel index
    int32_t camera_inside;   // intersection::Overlap at the camera
    int32_t max_depth, rr_depth, use_nee, sky;
    int32_t npix;            // width * height
    int32_t pool;            // paths in flight
    uint64_t seed;
    uint64_t frame0;         // TOTAL_FRAME_INDEX of the first sample
    float eps_tab[9];        // INTERSECT_EPS(0..8)
    int32_t spectral;        // 1: one hero wavelength per path, 4: four wavelengths; XYZ output
    int32_t tri_light_nee;   // 1: NEE also samples triangle lights (extension)
    SpectralView spec;       // tables and lookup tables of the spectral mode
    uint32_t medium_key;     // medium_frame_key(seed, frame0)
    NrcFrame nrc;            // learned radiance cache hooks (enabled = 0: plain tracer)
    int32_t guiding;         // 1: path guiding with `guide` (interactive frames, one path per pixel)
    GuideView guide;
    DenoiseView dn;          // denoiser guide buffers (interactive frames, one path per pixel); NULL: off
};

}  // namespace ar
