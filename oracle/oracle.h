/*
 * oracle.h -- CPU restatement of the reference path tracer's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker for the CUDA core: only
 * the test suite, the smoke check and the CPU-baseline leg of bench.py load it.
 * Nothing in the shipped library links against it.
 *
 * It restates, function by function, ApertureRendererV3's CalculateRadiance
 * stack (core/render/render.cuh:460-999) in scalar C with IEEE single
 * precision, no FMA contraction (-ffp-contract=off) and the deterministic
 * transcendental functions of oracle_math.h, so that the GPU kernels -- built
 * with the same rounding rules -- can be compared bit for bit.  The input
 * format is the public ar_object_desc of include/aperture_b200.h.
 *
 * Pinning: the BVH build and the ray queries are checked against the
 * reference's own code compiled on the host (oracle/_ref, see oracle/Makefile),
 * whose outputs are committed as fixtures under tests/golden/.
 */
#ifndef APERTURE_ORACLE_H
#define APERTURE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/aperture_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scene options. */
enum {
    /* BVH proxies of triangles use the SceneObject centre as the reference's
     * UpdateProxy does (object.cuh:309-342); otherwise the centre of the
     * triangle's world bounds. */
    OR_PROXY_OBJECT_CENTER = 1 << 0,
    /* Triangles hit with the reference's default G-buffer (white, no
     * emission; intersection.cuh:17,63) instead of their material. */
    OR_TRIANGLE_DEFAULT_GBUFFER = 1 << 1,
    /* Inside a medium whose object is a triangle, trace only that triangle
     * (the reference's solo trace, render.cuh:91-94) instead of the scene. */
    OR_TRIANGLE_SOLO_MEDIA = 1 << 2,
    /* Path loop queries use the reference's slab test and first-found tie
     * rule (for pinning against the reference's own code). */
    OR_REFERENCE_TRAVERSAL = 1 << 3
};

/* Query options for or_trace_rays. */
enum {
    OR_TIE_FIRST_FOUND = 0,   /* reference: strict t < best (intersection.cuh:160) */
    OR_TIE_LOWEST_INDEX = 1,  /* the GPU core: equal t goes to the lower object index */
    OR_SLAB_REFERENCE = 0,    /* FastAABBHit as written (bvh.cuh:424-470)           */
    OR_SLAB_STANDARD = 2      /* standard slab test (entry <= exit), widened 1 ulp  */
};

typedef struct or_scene or_scene;

or_scene* or_scene_create(const ar_object_desc* objects, size_t count, int flags,
                          int leaf_size, int bin_count);
/* With the SDF volumes that AR_SDF_VOLUME objects refer to. */
or_scene* or_scene_create_ex(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes,
                             size_t volume_count, int flags, int leaf_size, int bin_count);
void or_scene_destroy(or_scene* s);

/* BVH export: per node bmin[3], bmax[3] floats and left, right, first, count. */
int64_t or_scene_node_count(const or_scene* s);
void or_scene_nodes(const or_scene* s, float* bounds6, int32_t* links4);
void or_scene_indices(const or_scene* s, int32_t* indices);
int64_t or_scene_light_count(const or_scene* s);
void or_scene_lights(const or_scene* s, int32_t* object_index, float* select_prob);

/* Rays as 8 floats: origin.xyz, tmin, direction.xyz, tmax.  Counters (may be
 * NULL) receive per-ray node visits and primitive tests. */
void or_trace_rays(const or_scene* s, const float* rays, int64_t n, int any_hit, int mode,
                   int32_t* hit_object, float* hit_t, int32_t* node_visits,
                   int32_t* prim_tests, int threads);
/* Brute force over all objects, lowest-index tie rule. */
void or_trace_rays_brute(const or_scene* s, const float* rays, int64_t n, int any_hit,
                         int32_t* hit_object, float* hit_t, int threads);

/* Camera rays of RenderCamera (scene.cu:213-230) for jitter values taken
 * from a tape: rays[8] per path, as for or_trace_rays. */
void or_camera_ray(const ar_camera* cam, int i, int j, float jx, float jy, float* ray8);

/* Replay spp samples of every pixel with uniforms read from `tape`
 * (ar_rng_tape layout: per path `per_path` floats, sample major).  Writes one
 * ar_path_record per path.  Returns the number of paths that ran out of tape. */
int64_t or_render_paths(const or_scene* s, const ar_camera* cam, const ar_render_params* p,
                        const float* tape, int per_path, ar_path_record* records,
                        int threads);

/* CPU baseline: render pixels pixel_begin, pixel_begin + step, ... < pixel_end
 * with an own per-path random generator (not curand), FP64 sums added into
 * accum (w*h*3).  Counts closest-hit and shadow queries. */
void or_render_image(const or_scene* s, const ar_camera* cam, const ar_render_params* p,
                     int64_t pixel_begin, int64_t pixel_end, int64_t step, double* accum,
                     int64_t* extension_rays, int64_t* shadow_rays, int threads);

/* Run the CPU baseline path loop over pixels [pb, pe) single-threaded and
 * record every closest-hit query (ext) and any-hit segment (sh) as 8-float rays,
 * up to the given capacities.  Returns the number of queries. */
int64_t or_collect_rays(const or_scene* s, const ar_camera* cam, const ar_render_params* p, int64_t pb, int64_t pe,
                        float* ext, int64_t ext_cap, int64_t* n_ext, float* sh, int64_t sh_cap, int64_t* n_sh);

/* Participating medium (extension): attach (NULL removes) a density box; the
 * medium's pieces for their own tests: density at a point, Henyey-Greenstein
 * sampling (n pairs of uniforms around d3) and value, and per ray (8 floats,
 * tmax in [7]) delta tracking (first collision or -1) or, with ratio = 1,
 * ratio-tracking transmittance, from counter-based uniforms of seeds[i]. */
int or_scene_set_medium(or_scene* s, const ar_medium_desc* m);
float or_medium_density(const or_scene* s, const float* p3);
void or_hg_sample(const float* d3, float g, const float* u2, int64_t n, float* out3);
float or_hg_phase(float g, float cosT);
void or_medium_track(const or_scene* s, const float* rays8, int64_t n, const uint32_t* seeds, int ratio, float* out);

/* Deterministic transcendental functions (exported for their own tests). */
/* Closest hit plus the hit's world position, normal and inside flag
 * (IntersectionContext fields), per ray; misses leave zeros. */
void or_trace_detail(const or_scene* s, const float* rays, int64_t n, int mode, int32_t* hit_object,
                     float* hit_t, float* pos, float* nrm, int32_t* inside, int threads);
/* AnyHitSegmentBVH (intersection.cuh:372-397): segments as src.xyz, dst.xyz,
 * eps of the given loop depth; occluded[i] = 1 when something blocks it. */
void or_segments_occluded(const or_scene* s, const float* seg6, const int32_t* depth, int64_t n, int mode,
                          int32_t* occluded, int threads);
/* intersection::Overlap: first object containing each point, or -1. */
void or_overlap(const or_scene* s, const float* p3, int64_t n, int32_t* object_index);
/* BSDF_PDF (RGB) for one material, normal, ray direction and light direction. */
float or_bsdf_pdf(int model, const ar_material* m, const float* N, const float* ray_dir, const float* L);
/* PowerHeuristic (render.cuh:185-196). */
float or_power_heuristic(float a, float b);

/* Tonemap kernel (scene.cu:180-199): n pixels of RGB (or XYZ) -> 0xAARRGGBB. */
void or_tonemap(const float* rgb, int64_t n, int tone, float exposure, int xyz_input, uint32_t* out);

/* Screen-space denoiser (core/denoise/): one frame recorded per pixel from
 * hits (12 floats: albedo.xyz, normal.xyz, metallic, roughness, depth, shading
 * model, hit flag, unused) and samples (3 floats); either output may be NULL. */
void or_dn_record(const float* hits, const float* samples, int64_t n, ar_screen_gbuffer* gbuffer,
                  ar_screen_stats* stats);
/* Bilateral16x16<7> over the whole image (t_quantiles: 1024 floats). */
void or_dn_bilateral(const float* hdr, float* out, const ar_screen_gbuffer* gb, const ar_screen_stats* st, int width,
                     int height, const float* t_quantiles);

/* One object's hit at loop depth `depth` (SDF tolerance INTERSECT_EPS(depth)/2):
 * t = -1 on a miss, with world position and normal. */
void or_object_isect(const or_scene* s, int32_t obj, const float* rays, int64_t n, int32_t depth, float* t,
                     float* pos, float* nrm);
/* The float grid of SDF volume v as an object of the scene uses it. */
void or_volume_grid(const or_scene* s, int32_t v, float* out);

/* Spectral mode: the reference's tables (17780 floats, ar_scene_set_spectral
 * layout) and lookup tables built from them at RGB resolution res.  0 on success. */
int or_scene_set_spectral(or_scene* s, const float* tables, size_t count, int res, int threads);
void or_spectral_luts(const or_scene* s, float* lambda_lut, float* rgb_lut);
/* SampleCIE1931 for n triples of uniforms. */
void or_spectral_sample(const float* u3, int64_t n, float* lambda, float* pdf);
/* RGBEncode of rgb[3n] and LambdaEncode of lambda[n] (either may be NULL). */
void or_spectral_encode(const float* tables, const float* rgb, const float* lambda, int64_t n, float* rgb_k,
                        float* lam_k);
/* Interact, D65Norm and the colour matching functions through a scene's tables. */
void or_spectral_interact(const or_scene* s, const float* lambda, const float* rgb, int64_t n, float* resp,
                          float* d65, float* xyz);

float or_sinf(float x);
float or_cosf(float x);
float or_expf(float x);
float or_logf(float x);
float or_powf(float x, float y);

#ifdef __cplusplus
}
#endif

#endif /* APERTURE_ORACLE_H */
