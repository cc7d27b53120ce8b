/*
 * ref_path_prelude.h -- pre-included (nvcc -include) into ref_path_harness.cu,
 * before any of the reference's headers.  TEST INFRASTRUCTURE ONLY.
 *
 * It selects, without edits, the configuration in which the reference's path
 * loop runs on the host:
 *   - RGB build (USE_SPECTRUM_RENDERING off, config.cuh:61), 32-bit BVH node
 *     layout (BVH_USE_16_BITS_NODE / BVH_PACK_NODE off, bvh.cuh:36-42);
 *   - MAX_TRACING_DEPTH (config.cuh:8) read from the harness at run time
 *     (the reference fixes it at 1000; the benchmark configurations set 8-16);
 *   - RENDER_GLOBAL defined, so that render.cuh's block of __constant__ scene
 *     globals (render.cuh:23-56) is skipped; the harness defines the same
 *     names as host variables before it includes render.cuh.
 * With REF_PATH_DETMATH the transcendental functions the path calls (sinf,
 * cosf, tanf, sincosf, expf, logf, powf) and rsqrtf are routed to the fixed
 * definitions the oracle uses (oracle_math.h), which isolates the algorithm
 * from the host math library; without it they are the host's own.
 */
#pragma once
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include "config.cuh"

#undef USE_SPECTRUM_RENDERING
#undef BVH_USE_16_BITS_NODE
#undef BVH_PACK_NODE
#undef MAX_TRACING_DEPTH
#define MAX_TRACING_DEPTH (ref_path_max_depth())
int ref_path_host_max_depth();
__host__ __device__ __forceinline__ int ref_path_max_depth()
{
#ifdef __CUDA_ARCH__
    return 1000;
#else
    return ref_path_host_max_depth();
#endif
}

#define RENDER_GLOBAL

/* Random numbers and observation hooks (ref_path_patch.py edits 2 and 4). */
float ref_host_uniform(curandState* seed);
void ref_host_trace(curandState* seed, int object_or_minus1);
void ref_host_shadow(curandState* seed, int depth);

__host__ __device__ __forceinline__ float ref_uniform(curandState* seed)
{
#ifdef __CUDA_ARCH__
    return curand_uniform(seed);
#else
    return ref_host_uniform(seed);
#endif
}

__host__ __device__ __forceinline__ float4 ref_tex2d_float4(cudaTextureObject_t t, float x, float y)
{
#ifdef __CUDA_ARCH__
    return tex2D<float4>(t, x, y);
#else
    (void)t; (void)x; (void)y;
    return make_float4(1.0f, 1.0f, 1.0f, 1.0f);  /* unreachable: harness materials carry no texture */
#endif
}

#ifdef __CUDA_ARCH__
#define REF_HOOK_TRACE(seed, tr) ((void)0)
#define REF_HOOK_SHADOW(seed, depth) ((void)0)
#else
#define REF_HOOK_TRACE(seed, tr) \
    ref_host_trace((seed), (tr).intersectionContext_.bHit_ ? (tr).intersectionContext_.objectIndex_ : -1)
#define REF_HOOK_SHADOW(seed, depth) ref_host_shadow((seed), (depth))
#endif

#if defined(REF_PATH_DETMATH) && !defined(__CUDA_ARCH__)
#include "oracle_math.h"
#define sinf(x) om_sinf(x)
#define cosf(x) om_cosf(x)
#define tanf(x) om_tanf(x)
#define expf(x) om_expf(x)
#define logf(x) om_logf(x)
#define powf(x, y) om_powf((x), (y))
#define sincosf(x, s, c) om_sincosf((x), (s), (c))
#define rsqrtf(x) om_rsqrtf(x)
#endif
