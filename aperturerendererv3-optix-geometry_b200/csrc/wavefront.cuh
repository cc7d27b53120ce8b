// wavefront.cuh -- path state and launch parameters of the wavefront pipeline.
//
// The reference runs one 168-register megakernel thread per pixel per frame
// (RenderCamera, core/scene.cu:201-255, calling CalculateRadiance,
// core/render/render.cuh:460-999).  Here a path's loop body is split at its two
// BVH queries into stages that communicate through structure-of-arrays state in
// HBM:
//   raygen  -> extend (closest hit) -> shade (BSDF sample, emission + MIS,
//   light sample, Russian roulette) -> shadow (any hit, adds the NEE term)
//   -> extend ... -> finish (FP64 accumulation).
// Queues of live path slots are compacted with warp ballots.  Every stage
// draws its uniforms from the path's own curand XORWOW state, seeded as the
// reference seeds it (core/random.cuh:31-39), in the reference's order, so a
// path consumes exactly the reference's sample sequence.
#pragma once

#include <cstdint>

#include "../../include/aperture_b200.h"
#include "traverse.cuh"

namespace ar {

enum : int32_t {
    kFlagPrevNEE = 1,      // previousNEEState.previousDidNEE_
    kFlagInside = 2,       // MediaContext::bInsideMedia_
    kFlagNeeCosOK = 4,     // pending NEE term has cosX > 0 && cosY > 0
    kFlagMissThin = 8      // last segment was a thin-surface miss inside media
};

// Control block of the path pool (device memory).  Paths live in `pool` slots;
// retired slots go onto a free stack and are refilled with the next samples
// (sample-major order g = s * npix + p) until `total` samples have been traced.
struct PoolCtl {
    int32_t qcount[2];     // extension queue lengths (ping-pong)
    int32_t shadow_count;  // shadow queue length
    int32_t retire_count;  // paths that ended this iteration
    int32_t fetch_ext, fetch_shadow, fetch_rays;  // persistent-kernel work counters
    int32_t free_count;    // free slots on the stack
    int32_t plan_new;      // samples started this iteration
    int32_t plan_src;      // first free-stack entry they use
    int32_t pad[2];
    int64_t gen_next;      // next sample index to start
    int64_t plan_first;    // sample index of the first path started this iteration
    int64_t retired;       // paths finished so far
    int64_t total;         // samples of this render (spp * npix)
};

struct PathSoA {
    float4* o;       // ray origin xyz
    float4* d;       // ray direction xyz
    float4* mask;    // throughput rgb
    float4* rad;     // radiance rgb
    uint4* rng0;     // xorwow d, v0, v1, v2
    uint2* rng1;     // xorwow v3, v4
    int4* info;      // x pixel, y depth | nonDeltaDepth << 16, z sample index, w flags | media depth << 8
    float4* prev;    // previous vertex xyz, w previous BSDF pdf
    float4* media;   // media vertex location xyz, w media object (int bits)
    int4* hit;       // object, prim slot, t bits
    float4* nee;     // pending NEE radiance rgb (mask already applied)
    float4* sseg0;   // shadow segment source xyz, w segment eps
    float4* sseg1;   // shadow segment target xyz
    int32_t* q[2];   // extension queues (ping-pong)
    int32_t* qs;     // shadow queue
    int32_t* qr;     // paths that ended this iteration
    int32_t* freeq;  // free-slot stack
    int32_t* ucount; // uniforms consumed per slot (debug only)
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
    int32_t pool;            // path slots
    uint64_t seed;
    uint64_t frame0;         // TOTAL_FRAME_INDEX of the first sample
    float eps_tab[9];        // INTERSECT_EPS(0..8)
};

}  // namespace ar
