/*
 * aperture_b200.h -- C ABI of the B200 (sm_100a) path-tracing core.
 *
 * The reference renderer (ApertureRendererV3) exposes its hot path only as the
 * C++ classes SceneRenderer and Camera (core/scene.hpp:19-154,
 * core/camera.hpp:14-100), whose scene state lives in module-global
 * __constant__ symbols (core/render/render.cuh:26-55).  This header is the
 * drop-in boundary that replaces them: plain C types, plain pointers and sizes,
 * one handle per scene, no device globals, status codes instead of printed
 * errors.  Every entry point below names the reference interface it replaces.
 *
 * Threading: a scene handle may be used by one host thread at a time.  Work is
 * issued on the caller's CUDA stream (passed as void*; NULL = legacy default
 * stream) and every call that returns host data synchronises that stream.
 */
#ifndef APERTURE_B200_H
#define APERTURE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AR_ABI_VERSION 1

typedef enum ar_status {
    AR_OK = 0,
    AR_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, enum value or layout      */
    AR_ERR_CUDA = 2,             /* a CUDA runtime call failed                   */
    AR_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed             */
    AR_ERR_UNSUPPORTED = 4,      /* feature not available for this scene/config  */
    AR_ERR_DEVICE_FAULT = 5,     /* a kernel reported an internal error word     */
    AR_ERR_NO_DEVICE = 6,        /* no CUDA device / extension not usable        */
    AR_ERR_INTERNAL = 7          /* a consistency check of the library failed    */
} ar_status;

/* EObjectType (core/render/object.cuh:29-35). */
enum { AR_OBJ_CUBE = 0, AR_OBJ_SPHERE = 1, AR_OBJ_SDF = 2, AR_OBJ_TRIANGLE = 3 };
/* EShadingModel (core/render/object.cuh:45-52). */
enum { AR_MAT_DIFFUSE = 0, AR_MAT_LIGHT = 1, AR_MAT_GLASS = 2, AR_MAT_GGX = 3 };
/* Where a caller-supplied buffer lives. */
enum { AR_MEM_HOST = 0, AR_MEM_DEVICE = 1 };

typedef struct ar_vec3 { float x, y, z; } ar_vec3;

/* Material = shading model + the GBuffer fields of a pure-colour texture
 * (core/render/object.cuh:60-91, 124-217).  Textures are not supported. */
typedef struct ar_material {
    int32_t shading_model; /* AR_MAT_*                                   */
    ar_vec3 albedo;        /* linear                                     */
    ar_vec3 emissive;      /* linear radiance                            */
    float specular;        /* GGX: F0 = 0.08 * specular                  */
    float metallic;
    float roughness;       /* GGX: alpha = roughness^2                   */
    float ior;             /* glass                                      */
    float sigma_a;         /* glass Beer-Lambert density                 */
    float abbe_number;     /* glass dispersion (spectral)                */
    float tilt_number;
} ar_material;             /* 56 bytes */

/* ESDFType (core/render/object.cuh:37-43) of an AR_OBJ_SDF object. */
enum { AR_SDF_TORUS = 0, AR_SDF_VOLUME = 1 };

/* Vertex (core/render/object.cuh:233-238), object space. */
typedef struct ar_vertex { ar_vec3 position; ar_vec3 normal; float u, v; } ar_vertex; /* 32 B */

/* One scene primitive; the fields of the reference SceneObject that its
 * constructor takes (core/render/object.cuh:344-364).  The world transform is
 * objectToWorld = Rz * (Ry * Rx) from the Euler angles in degrees, then
 * + center, exactly as that constructor builds it. */
typedef struct ar_object_desc {
    int32_t type;          /* AR_OBJ_*                                              */
    ar_vec3 center;
    ar_vec3 extent;        /* cube / SDF box half-size; sphere radius = max component */
    ar_vec3 rotation_deg;  /* Euler (x, y, z) in degrees                            */
    ar_material material;
    union {
        ar_vertex tri[3];  /* AR_OBJ_TRIANGLE: object-space vertices                */
        struct {           /* AR_OBJ_SDF (AdditionalObjectInfo, object.cuh:219-229) */
            float info[4]; /* SDFInfo::sdfInfo0_: torus (R, r) in the unit box      */
            int32_t kind;  /* AR_SDF_TORUS or AR_SDF_VOLUME                         */
            int32_t volume;/* AR_SDF_VOLUME: index into the scene's volume list     */
        } sdf;
    };
    int32_t visible;       /* 0 = skipped by intersection (SceneObject::bVisible_)  */
    int32_t reserved[3];
} ar_object_desc;          /* 208 bytes */

/* A sampled signed-distance volume (SDFVolumeInfo, object/sdf/sdf_volume.cuh:14-45),
 * the grid of an AR_SDF_VOLUME object: dims[0]*dims[1]*dims[2] distances in
 * the unit box [0,1]^3 of the object (x fastest, Index3D), in the object's
 * unit-box distance units.  Either `data` (host memory, precision 32 = float,
 * 16 = IEEE half) or, when data is NULL, filled on the device from an analytic
 * function like SDFCacheManager::AddVolume / FillSDFVolume
 * (object/sdf/sdf_cache_manager.cuh:16-104): fill_kind AR_SDF_TORUS with
 * fill_info (R, r).  Samples are nearest or trilinear as SampleSDFAdaptive01.
 * precision 16 stores the grid as half floats (half the bytes per tap). */
typedef struct ar_sdf_volume {
    int32_t dims[3];
    int32_t precision;     /* 32 or 16                                              */
    const void* data;      /* host values, or NULL to fill from fill_kind           */
    int32_t fill_kind;     /* AR_SDF_TORUS                                          */
    float fill_info[4];
    int32_t reserved;
} ar_sdf_volume;           /* 48 bytes */

/* Pinhole camera of RenderCamera (core/scene.cu:201-230) with the field of view
 * as a parameter instead of the hard-coded 60 degrees. */
typedef struct ar_camera {
    ar_vec3 position;
    ar_vec3 direction;     /* need not be normalised */
    float fov_y_deg;       /* reference: 60                                         */
    int32_t width;
    int32_t height;
} ar_camera;

/* Knobs the reference fixes at compile time (core/config.cuh). */
typedef struct ar_render_params {
    int32_t spp;           /* samples per pixel (frames of the offline Render loop)  */
    int32_t max_depth;     /* MAX_TRACING_DEPTH (reference: 1000)                    */
    int32_t rr_depth;      /* MIN_TRACING_DEPTH: RR from this non-delta depth (3)    */
    int32_t use_nee;       /* SceneSetting::bUseNEE_                                 */
    int32_t sky;           /* 1 = SkyLighting, 0 = DISABLE_SKYLIGHT                  */
    int32_t frame_offset;  /* TOTAL_FRAME_INDEX of the first sample                  */
    uint64_t seed;         /* GLOBAL_SEED (reference: 0x9e3779b97f4a7c15)            */
    int32_t sort_rays;     /* must be 0 (other values: AR_ERR_UNSUPPORTED).  Paths are
                              always shaded in material buckets; a direction-octant
                              sort of the extension rays is not built (measured slower) */
    int32_t wave_paths;    /* paths in flight per wave; 0 = automatic                */
    int32_t spectral;      /* 1 = USE_SPECTRUM_RENDERING: one hero wavelength per path
                              (SampleCIE1931), output linear CIE XYZ; needs
                              ar_scene_set_spectral.  4 = four wavelengths per path
                              (extension): the hero and its rotations by 105 nm in
                              [360, 780], one estimate per rotation set (balance
                              heuristic); dispersive glass continues with the hero
                              alone.  0 = RGB                                        */
    int32_t tri_light_nee; /* 1 = NEE also samples emissive triangles (uniform area
                              sampling, two-sided, MIS with BSDF hits).  The
                              reference samples cube and sphere lights only
                              (nee.cuh:362-369), which 0 reproduces.               */
} ar_render_params;

/* Per-path record of ar_render_debug_paths (one per pixel and sample). */
#define AR_DEBUG_MAX_HITS 16
typedef struct ar_path_record {
    float radiance[3];     /* CalculateRadiance output before accumulation           */
    int32_t segments;      /* loop iterations executed (Trace calls)                 */
    int32_t uniforms;      /* curand_uniform values this path consumed               */
    int32_t nee_rays;      /* shadow rays cast                                        */
    int32_t nee_depth_mask;/* bit d set: a shadow ray was cast at loop depth d (< 32) */
    int32_t reserved;
    int32_t hit_object[AR_DEBUG_MAX_HITS]; /* closest-hit object per segment, -1 = miss,
                                              -2 = collision in the participating medium */
} ar_path_record;          /* 96 bytes */

typedef struct ar_scene_info {
    int64_t objects;
    int64_t triangles;
    int64_t lights;
    int64_t wide_nodes;    /* 8-wide quantised BVH nodes                              */
    int64_t prim_refs;     /* leaf primitive records                                  */
    int64_t device_bytes;  /* bytes held on the device by the scene                   */
    int32_t device;
    int32_t camera_inside; /* reserved */
} ar_scene_info;

/* Counters of one ar_render call.  Passing a stats pointer also times every
 * closest-hit and any-hit traversal launch with CUDA events on the caller's
 * stream (a few microseconds of overhead per launch). */
typedef struct ar_render_stats {
    int64_t paths;           /* camera paths traced                                  */
    int64_t extension_rays;  /* closest-hit BVH queries                              */
    int64_t shadow_rays;     /* any-hit BVH queries actually traversed               */
    int64_t kernel_launches; /* kernels this call launched                           */
    int64_t extend_launches; /* closest-hit traversal launches                       */
    int64_t shadow_launches; /* any-hit traversal launches                           */
    int64_t extend_node_visits; /* reserved (0): node visits of closest-hit queries  */
    int64_t extend_prim_tests;  /* reserved (0)                                       */
    int64_t shadow_node_visits; /* reserved (0)                                       */
    int64_t shadow_prim_tests;  /* reserved (0)                                       */
    float   extend_ms;       /* summed device time of the closest-hit launches       */
    float   shadow_ms;       /* summed device time of the any-hit launches           */
    float   total_ms;        /* device time of the whole render call                 */
    int32_t reserved;
} ar_render_stats;

typedef struct ar_scene ar_scene;

/* Library ABI version (AR_ABI_VERSION). */
int32_t ar_version(void);

/* Message of the last error on the calling thread; "" when none.
 * Replaces the printing CHECK_ERROR macro (core/vector.cuh:22-31). */
const char* ar_get_last_error_string(void);

/* Build a scene on `device`: world-space triangle records, SAH BVH collapsed to
 * 8-wide quantised nodes, light table.  Replaces SceneRenderer::SceneRenderer
 * (core/scene.hpp:113, core/scene.cu:1120-1156) together with the upload it
 * defers to the first Render, UpdateSceneToDeviceIfDirty (core/scene.cu:1025-1118). */
ar_status ar_scene_create(const ar_object_desc* objects, size_t count, int32_t device,
                          ar_scene** out_scene);

/* ar_scene_create with the signed-distance volumes its AR_SDF_VOLUME objects
 * refer to (the reference's SDFCacheManager entries, indexed in order). */
ar_status ar_scene_create_ex(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes,
                             size_t volume_count, int32_t device, ar_scene** out_scene);

/* Release every device allocation of the scene (SceneRenderer::~SceneRenderer,
 * core/scene.cu:1158-1163).  NULL is accepted. */
void ar_scene_destroy(ar_scene* scene);

ar_status ar_scene_get_info(const ar_scene* scene, ar_scene_info* info);

/* Shape of the BVH that ar_scene_create_ex builds for these objects, built on
 * the host alone (no device, nothing uploaded): the 8-wide nodes, primitive
 * records, occupied child slots and the exact worst-case traversal stack
 * depth.  The call also checks the structure -- every primitive record in
 * exactly one leaf slot, every child index in range -- and returns
 * AR_ERR_INTERNAL if it does not hold.  Invalid objects give
 * AR_ERR_INVALID_ARGUMENT and coordinates beyond the quantised grid's range
 * AR_ERR_UNSUPPORTED, as in ar_scene_create_ex. */
typedef struct ar_bvh_info {
    int64_t wide_nodes;
    int64_t prim_refs;
    int64_t leaf_slots;      /* child slots holding a leaf (1-4 primitive records) */
    int64_t internal_slots;  /* child slots holding a wide node (= wide_nodes - 1)  */
    int32_t stack_bound;     /* deepest traversal stack any ray can need           */
    int32_t depth;           /* wide levels                                        */
} ar_bvh_info;

ar_status ar_bvh_build_info(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes,
                            size_t volume_count, ar_bvh_info* info);

/* Offline render: spp samples per pixel, FP64 accumulation, mean written as
 * linear RGB float3 rows (index j*width+i).  Replaces
 * std::vector<float3> SceneRenderer::Render(int2, float3, float3, int)
 * (core/scene.hpp:126, core/scene.cu:276-306).
 *   out_rgb   width*height*3 floats (may be NULL if accum is given)
 *   accum     width*height*3 doubles holding running sums, or NULL; when given it
 *             is ADDED to (resume/extend a render), never cleared
 *   mem_kind  AR_MEM_HOST or AR_MEM_DEVICE for both buffers
 *   stats     optional counters (NULL to skip)                                 */
ar_status ar_render(ar_scene* scene, const ar_camera* camera, const ar_render_params* params,
                    float* out_rgb, double* accum, int32_t mem_kind, void* stream,
                    ar_render_stats* stats);

/* Closest-hit (any_hit = 0) or any-hit (any_hit = 1) queries for n rays laid out
 * as 8 floats each: origin.xyz, tmin, direction.xyz, tmax.  A hit is accepted
 * when tmin <= t < tmax (intersection.cuh:160) and ties in t go to the lowest
 * object index.  hit_t may be NULL.  Replaces intersection::TraverseBVH
 * (core/render/intersection.cuh:235-370) as used by Trace and SegmentTrace. */
ar_status ar_trace_rays(ar_scene* scene, const float* rays, size_t n, int32_t any_hit,
                        int32_t* hit_object, float* hit_t, int32_t mem_kind, void* stream);

/* Closest-hit / any-hit ray queries like ar_trace_rays, for callers that
 * cannot allocate device memory when they query: hosts that give the library
 * a fixed memory budget, real-time threads that must not take allocator
 * locks, processes where another thread may be capturing a CUDA graph.  It
 * calls no cudaMalloc/cudaFree: its scratch (a work counter, an error word and
 * the traversal-stack overflow of its persistent threads) is one file-scope
 * __device__ array of 16 MiB that each GPU loading the library holds until the
 * process exits.  rays, hit_object and hit_t (may be NULL) are device
 * pointers; rays 16-byte aligned; batches above 2^30 rays run as several
 * launches of at most 2^30.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress); make it before any stream capture.  All
 * calls share the array: calls whose work overlaps on the GPU race --
 * serialise them (one stream).  Returns after the queries finished
 * (synchronises `stream`).  While another thread captures a CUDA graph in the
 * global capture mode, pass a stream created with cudaStreamNonBlocking: work
 * on the legacy default stream synchronises with every blocking stream, which
 * invalidates that capture.  No counterpart in the reference. */
ar_status ar_trace_rays_static(const ar_scene* scene, const float* rays, size_t n, int32_t any_hit,
                               int32_t* hit_object, float* hit_t, void* stream);

/* Render spp samples and record every path (width*height*spp records, sample
 * major: record[(s*height + j)*width + i]).  Debug/parity entry; same kernels
 * as ar_render. */
ar_status ar_render_debug_paths(ar_scene* scene, const ar_camera* camera,
                                const ar_render_params* params, ar_path_record* records,
                                int32_t mem_kind, void* stream);

/* The first `per_path` uniforms of the random stream of every path of
 * ar_render (curand XORWOW, seed params->seed, subsequence = the reference's
 * block-linear pixel index of 8x4 blocks, offset = frame * 2^32;
 * core/random.cuh:31-39).  out has spp*height*width*per_path floats, sample
 * major.  Lets a CPU replay consume exactly the GPU's sample sequence. */
ar_status ar_rng_tape(const ar_camera* camera, const ar_render_params* params, int32_t per_path,
                      float* out, int32_t mem_kind, void* stream);

/* Spectral mode set-up for a scene (SceneRenderer::SetupSpectrumLUT,
 * core/scene.cu; spectrum_lut.cuh:12-79): `tables` holds, as float32, the
 * reference's CIE 1931 colour matching functions (421 x 3, 360..780 nm), its
 * D65 spectrum (421) and the weights of its two spectrum-basis networks
 * (spectrum_basis.cuh: RGB_IN_W/B, RGB_BLK0..6_W/B, RGB_OUT_W, LAM_BLK0..6_W/B,
 * LAM_OUT_W), 17780 values in that order.  The wavelength lookup table (840
 * entries) and the RGB lookup table (lut_res^3 entries; the reference's
 * SPECTRUM_RGB_LUT_RES is 512) are then built on the scene's device. */
ar_status ar_scene_set_spectral(ar_scene* scene, const float* tables, size_t count, int32_t lut_res);

/* Builders of the RGB lookup table: AR_LUT_SIMT evaluates the network one
 * thread per entry in fp32 (fmaf in the reference's input order; the table
 * the oracle reproduces bit for bit, used by ar_scene_set_spectral);
 * AR_LUT_TENSOR runs every layer as a 128 x 32 x 32 product on the tcgen05
 * tensor cores with three-term bf16 splits of both operands (fp32 accuracy,
 * other summation order: entries within a few fp32 ulps of the SIMT table). */
enum { AR_LUT_SIMT = 0, AR_LUT_TENSOR = 1 };
ar_status ar_scene_set_spectral_ex(ar_scene* scene, const float* tables, size_t count, int32_t lut_res,
                                   int32_t method);
/* The RGB lookup table alone (res^3 x 4 floats, x fastest) into a 16-byte
 * aligned device buffer of the current device, built by `method`; *ms (may be
 * NULL) gets the device time of the build.  res in [2, 1024].  No counterpart
 * in the reference beyond PrecomputeRGBLUTKernel (spectrum_lut.cuh:12-38). */
ar_status ar_spectral_rgb_lut(const float* tables, size_t count, int32_t res, int32_t method, float* out_device,
                              float* ms);

/* Copies of the spectral lookup tables (840 x 4 and lut_res^3 x 4 floats, x
 * fastest); either pointer may be NULL. */
ar_status ar_scene_get_spectral_luts(const ar_scene* scene, float* lambda_lut, float* rgb_lut);

/* A heterogeneous participating medium (extension: the reference has no
 * volumetric media; its Henyey-Greenstein helpers, core/render/sample.cuh:110-145,
 * have no call site).  One axis-aligned box of world space holds a density grid
 * (dims[0] x dims[1] x dims[2] values, x fastest, trilinear between voxel
 * centres, clamped at the faces); extinction = sigma_t_max * density.  Free
 * flights are sampled by delta tracking, scattering by the Henyey-Greenstein
 * phase function with asymmetry g; every collision scatters with throughput
 * weight `albedo`.  Shadow rays are attenuated by ratio-tracking estimates of
 * the transmittance.  The interior of a dielectric object (a path inside
 * glass) is not part of the medium. */
typedef struct ar_medium_desc {
    float bounds_min[3];
    float bounds_max[3];
    float sigma_t_max;     /* extinction of density 1, world units^-1               */
    float albedo[3];       /* single-scatter albedo, each in [0, 1]                 */
    float g;               /* Henyey-Greenstein asymmetry, (-1, 1)                  */
    int32_t dims[3];
    int32_t precision;     /* 32 = float, 16 = half                                 */
    const void* density;   /* host memory, non-negative finite values               */
} ar_medium_desc;

/* Attach (or with NULL remove) the scene's medium; copies the grid to the
 * scene's device. */
ar_status ar_scene_set_medium(ar_scene* scene, const ar_medium_desc* medium);

/* ------------------------------------------------------------------------ */
/* Learned radiance cache (extension; the reference has none).               */
/* A multiresolution hash-grid encoding of position (half-float tables),     */
/* degree-4 spherical harmonics of the outgoing direction, roughness,        */
/* diffuse albedo and normal feed a 64-wide MLP (5 hidden ReLU layers, exp   */
/* output, bf16 weights and activations, fp32 accumulation) trained online    */
/* with a relative L2 loss and Adam on radiance estimates of a subset of      */
/* full-length "training" paths; the other paths end at the first vertex      */
/* whose path spread exceeds spread_c times the primary footprint and take    */
/* the cache's prediction there (Mueller et al. 2021).                        */
/* ------------------------------------------------------------------------ */
typedef struct ar_nrc ar_nrc;

typedef struct ar_nrc_config {
    int32_t levels;             /* hash-grid levels, <= 16 (16)                      */
    int32_t log2_entries;       /* table entries per level = 2^log2_entries (19)    */
    int32_t base_resolution;    /* coarsest grid resolution (16)                     */
    int32_t max_resolution;     /* finest grid resolution (2048)                     */
    float bounds_min[3];        /* box of the position encoding; bounds_max <=      */
    float bounds_max[3];        /* bounds_min takes the scene's bounding box         */
    int32_t train_paths;        /* training paths per frame (65536)                  */
    int32_t train_batch;        /* samples per optimiser step (16384)                */
    int32_t train_steps;        /* optimiser steps per frame (4)                     */
    int32_t max_train_vertices; /* vertices recorded per training path (8)           */
    float learning_rate;        /* Adam (1e-2; beta1 0.9, beta2 0.99)                */
    float spread_c;             /* termination threshold c (0.01)                    */
    uint64_t seed;              /* initial weights and tables                        */
} ar_nrc_config;

typedef struct ar_nrc_frame_stats {
    float total_ms;             /* device time of the frame                          */
    float render_ms;            /* path tracing (extension + shade + shadow)         */
    float infer_ms;             /* cache queries                                     */
    float train_ms;             /* optimiser steps                                   */
    int64_t queries;            /* paths terminated into the cache                   */
    int64_t train_samples;      /* training samples produced                         */
    int64_t extension_rays;
    int64_t shadow_rays;
    float loss;                 /* mean relative L2 loss of the frame's steps         */
    int32_t reserved;
} ar_nrc_frame_stats;

/* Cache of one scene (the scene must outlive it). */
ar_status ar_nrc_create(ar_scene* scene, const ar_nrc_config* config, ar_nrc** out);
ar_status ar_nrc_destroy(ar_nrc* nrc);
/* One frame of params->spp samples per pixel (1 to 64, RGB): paths that end
 * in the cache add throughput x prediction; sample 0 of every training pixel
 * runs to its end and records training vertices; with train != 0 the frame's
 * training samples then take train_steps optimiser steps.  out_rgb (this
 * frame's mean image) and accum (FP64 sums of all spp samples added) are
 * device buffers; either may be NULL, not both.  stats may be NULL (then no
 * host synchronisation). */
ar_status ar_nrc_render_frame(ar_nrc* nrc, const ar_camera* camera, const ar_render_params* params,
                              float* out_rgb, double* accum, int32_t train, ar_nrc_frame_stats* stats,
                              void* stream);
/* Options: AR_NRC_OPT_TENSOR_PATH selects the inference kernel, 1 (default)
 * tcgen05.mma with tensor-memory accumulators (128 rows per CTA), 0 the
 * warp-level mma.sync kernel (32 rows per warp).  AR_NRC_OPT_SPECTRAL sets
 * the cache's mode before its first frame: 0 (default) RGB, 4 for frames of
 * four wavelengths per path (params->spectral = 4; needs the scene's spectral
 * tables): the 16 outputs are then the outgoing spectral radiance at 16
 * wavelength bins of 26.25 nm over [360, 780] nm, interpolated linearly at
 * each of the path's wavelengths, and the cache adds the path's XYZ estimate. */
enum { AR_NRC_OPT_TENSOR_PATH = 1, AR_NRC_OPT_SPECTRAL = 2 };
ar_status ar_nrc_set_option(ar_nrc* nrc, int32_t option, int32_t value);
/* Parameters as fp32: tables (levels x 2^log2_entries x 2) and MLP weights
 * (21504: layers 0-4 [64][64], layer 5 [16][64], [out][in]); NULL skips. */
ar_status ar_nrc_get_params(const ar_nrc* nrc, float* table, float* weights);
ar_status ar_nrc_set_params(ar_nrc* nrc, const float* table, const float* weights);
/* Direct use of the network: n vertices of 16 floats (position, pad;
 * direction, roughness; normal, pad; albedo, pad) -> n x 3 predictions (RGB
 * cache) or n x 16 spectral bins (four-wavelength cache); and `steps`
 * optimiser steps over n training samples of 20 floats (the vertex layout
 * with the target radiance in the three pad floats: r at 3, g at 11, b at
 * 15; then 4 floats, unused by the RGB cache; the four-wavelength cache reads
 * the targets of wavelengths 0-2 from the pads, that of wavelength 3 from
 * float 16 and the hero wavelength from float 17, a negative target being
 * left out), batches taken in order, the mean loss of each step to
 * losses[steps].  Host buffers. */
ar_status ar_nrc_infer(ar_nrc* nrc, const float* vertices, size_t n, float* out_rgb);
ar_status ar_nrc_train(ar_nrc* nrc, const float* samples, size_t n, int32_t steps, float* losses);
/* Gradients of the mean relative L2 loss over n <= train_batch samples with
 * respect to the table entries and the weights (layouts of
 * ar_nrc_get_params), without an update; loss may be NULL. */
ar_status ar_nrc_gradients(ar_nrc* nrc, const float* samples, size_t n, float* table_grad, float* weight_grad,
                           float* loss);

/* ------------------------------------------------------------------------ */
/* Path guiding (SceneRenderer's interactive mode with bUsePathGuiding:       */
/* core/render/render.cuh:545-640, core/guiding, scene.cu:583-744).           */
/* Probes of incident RGB radiance (8x8 equal-area octahedral maps with mips) */
/* per (0.05-unit voxel, icosahedron face of the reflected direction), filled */
/* from the radiance the frame's paths bring back and sampled with           */
/* probability alpha = 0.5 * min(1, frame / 64)^0.5 (mixture pdf, also in    */
/* MIS).  Interactive frames: one path per pixel per call, RGB.              */
/* ------------------------------------------------------------------------ */
typedef struct ar_guide ar_guide;

typedef struct ar_guide_config {
    int32_t probe_capacity;     /* probes in the pool (131072)                        */
    int32_t log2_table;         /* hash-table slots = 2^log2_table (20)               */
} ar_guide_config;

typedef struct ar_guide_stats {
    int64_t frames;             /* guided frames rendered                             */
    int64_t probes;             /* probes allocated (keys seen, capped by capacity)   */
    int64_t samples;            /* samples of the last frame                          */
    int64_t dropped;            /* samples of the last frame without a probe          */
    float alpha;                /* guiding probability of the last frame              */
    int32_t reserved;
} ar_guide_stats;

ar_status ar_guide_create(ar_scene* scene, const ar_guide_config* config, ar_guide** out);
ar_status ar_guide_destroy(ar_guide* guide);
/* One interactive frame (params->spp must be 1, RGB): render with the current
 * probes, then add the frame's samples to them.  out_rgb / accum as in
 * ar_render with AR_MEM_DEVICE (either may be NULL, not both). */
ar_status ar_guide_render_frame(ar_guide* guide, const ar_camera* camera, const ar_render_params* params,
                                float* out_rgb, double* accum, void* stream);
ar_status ar_guide_get_stats(const ar_guide* guide, ar_guide_stats* stats);
/* Copy of probe `index` (88 float4 texels: 8x8 leaves, 4x4, 2x2, 1x1 mips,
 * padding), or AR_ERR_INVALID_ARGUMENT when it is not allocated. */
ar_status ar_guide_get_probe(const ar_guide* guide, int32_t index, float* texels);

/* The probe math of the guided frames evaluated on the current device, for
 * checks against the reference's Octahedron (core/guiding/octahedron.cuh) and
 * grid (core/guiding/guiding_bin.cuh).  texels: nprobes x 85 x 4 floats (8x8
 * leaves, then the 4x4, 2x2 and 1x1 mips; rgb and one unused float).  Per
 * query i (host arrays): probe probe_of[i], normal normal3, texel weights
 * query3, five uniforms u5 (three for the mip descent, two for the point in
 * the leaf texel).  Out: the hemisphere sample's direction and pdf
 * (SampleOctahedronHemisphere, octahedron.cuh:343-364), the hemisphere pdf of
 * direction eval3 (OctahedronHemispherePDF, octahedron.cuh:366-380) and the
 * (voxel, face) key of point pos3 and direction eval3 (19-bit two's-
 * complement voxel x, y, z in bits 0-56, face index from bit 57; GetVoxelGrid,
 * guiding_bin.cuh:102-114). */
ar_status ar_guide_probe_eval(const float* texels, int32_t nprobes, const int32_t* probe_of, const float* normal3,
                              const float* query3, const float* u5, const float* eval3, const float* pos3, int64_t n,
                              float* out_dir3, float* out_pdf, float* out_eval_pdf, uint64_t* out_key);

/* One job of a batch: a scene (shared between jobs if wanted), a camera, the
 * render parameters and device outputs (mean image and/or FP64 sums added). */
typedef struct ar_job {
    ar_scene* scene;
    ar_camera camera;
    ar_render_params params;
    float* out_rgb;        /* device, width*height*3 floats, or NULL          */
    double* accum;         /* device, width*height*3 doubles (sums added), or NULL */
} ar_job;

typedef struct ar_batch_stats {
    float total_ms;        /* device time of the whole batch                   */
    int32_t iterations_per_graph;
    int64_t paths;
    int64_t extension_rays;
    int64_t shadow_rays;
    int64_t graph_launches;/* launches of the batch graph (1)                  */
    int64_t graph_nodes;   /* nodes of the loop body                           */
    int64_t kernel_launches;/* kernels run (body kernels x loop passes)         */
    int64_t loop_passes;   /* passes of the device-side loop                   */
} ar_batch_stats;

/* Many render jobs of uneven resolution, scene and spp at once (config 5 of
 * the benchmark; the reference renders one camera at a time, scene.cu:276-306).
 * Every job keeps its own wavefront pool; the batch is ONE launch of a CUDA
 * graph whose WHILE conditional node repeats a body of iterations_per_graph
 * (0 = 16; rounded up to even) wavefront iterations of every job -- each job
 * on its own branch so small jobs run side by side -- followed by a drain test
 * that sets the node's condition on the device until every job has retired
 * all of its paths (no host round trip between passes).  path_budget (0 =
 * 2^22) paths in flight are shared among the jobs by their share of the work
 * (a job's own params.wave_paths overrides).  All scenes on one device.
 * Outputs are written on `stream`; the call returns when they are complete. */
ar_status ar_render_batch(const ar_job* jobs, int32_t njobs, int32_t iterations_per_graph, int64_t path_budget,
                          ar_batch_stats* stats, void* stream);

/* Result of ar_batch_autotune. */
typedef struct ar_batch_tuning {
    int32_t iterations_per_graph;  /* chosen graph length                          */
    int32_t candidates;            /* configurations timed                         */
    int64_t path_budget;           /* chosen in-flight path budget                 */
    float best_ms;                 /* probe time of the chosen configuration       */
    float default_ms;              /* probe time of the defaults (16, 2^22)        */
    int32_t trace_blocks_per_sm;   /* chosen traversal grid per job (0: occupancy) */
    int32_t shade_blocks_per_sm;   /* chosen shading/generation/retirement grid    */
} ar_batch_tuning;

/* Autotuner of ar_render_batch: times the batch's probe (every job at
 * min(spp, probe_spp) samples into scratch outputs; the jobs' own buffers are
 * not touched) for graph lengths {4, 8, 16, 32} x path budgets {2^20 .. 2^23},
 * then, at the fastest of those, for each job's kernel grids: traversal
 * blocks per SM {occupancy, 4, 2} x shading / path generation / retirement
 * blocks per SM {4, 2, 1} (jobs run as parallel graph branches, so smaller
 * grids let several jobs' kernels share the GPU); 24 candidates, the fastest
 * in paths per second wins.  The choice is remembered for batches of the same
 * shape (job count, pixels, samples, spectral jobs) and used by
 * ar_render_batch when it is called with iterations_per_graph = 0 and
 * path_budget = 0.  probe_spp <= 0 takes 4. */
ar_status ar_batch_autotune(const ar_job* jobs, int32_t njobs, int32_t probe_spp, ar_batch_tuning* out,
                            void* stream);

/* Running-mean resolve for progressive rendering: out[i] = (float)(accum[i] *
 * scale) for n values (scale = 1 / samples so far).  With ar_render's FP64
 * accum this replaces the reference's per-frame FP32 running mean of the
 * interactive SceneRenderer::Render (target = lerp(target, result,
 * 1/(1+frameIndex)), core/scene.cu:241-242).  mem_kind: where both live. */
ar_status ar_accum_resolve(const double* accum, size_t n, double scale, float* out, int32_t mem_kind,
                           void* stream);

/* Output epilogue of the reference's Tonemap kernel (core/scene.cu:180-199,
 * curves of core/tonemap.cuh): for each of n pixels, linear RGB (or CIE XYZ
 * when xyz_input != 0, converted by XYZ2SRGBLinearD65) times exposure, then
 * tone_type 0 = none, 1 = gamma 1/2.2, 2 = ACES; saturated and packed as
 * 0xAARRGGBB (alpha 0xff) -- the reference's ldrTarget format.  rgb holds 3*n
 * floats; mem_kind says where both buffers live.  The offline path
 * (Camera::RenderToFile, core/camera.cu:64-89) applies the same curves on the
 * host before SaveBMP. */
ar_status ar_tonemap(const float* rgb, size_t n, int32_t tone_type, float exposure, int32_t xyz_input,
                     uint32_t* bgra, int32_t mem_kind, void* stream);

/* The tone curve of ar_tonemap for one pixel, on the host, before
 * quantisation: out3 = Gamma(rgb3) (tone_type 1), ACES(rgb3) (2) or rgb3 (0)
 * (core/tonemap.cuh:6-117).  No device is needed.  Used by the C++ shim's
 * Gamma / ACES functions (include/aperture_b200_renderer.hpp). */
ar_status ar_tone_curve(const float* rgb3, int32_t tone_type, float* out3);

/* ---------------------------------------------------------------- denoiser
 * Per-pixel guide buffers of the reference's screen-space denoiser and its
 * bilateral filter (core/denoise/).  Half-precision fields hold IEEE binary16
 * bit patterns.  Both buffers live on the device, one record per pixel in
 * row-major order (j*width+i), owned by the caller; zero them (cudaMemset 0)
 * before the first frame, as the reference's ResetScreenGBuffer does
 * (core/GUI.hpp:202-230). */

/* Running means over frames of the primary hit: replaces
 * denoise::ScreenGBuffer (core/denoise/denoise.cuh:35-84).  The reference's
 * 64-bit frame counters are 32-bit here. */
typedef struct ar_screen_gbuffer {
    uint16_t albedo[3];         /* half: material albedo at the primary hit   */
    uint16_t normal[3];         /* half: shading normal facing the ray         */
    uint16_t metallic;          /* half                                        */
    uint16_t roughness;         /* half                                        */
    float depth;                /* hit distance                                */
    uint32_t valid_frames;      /* frames whose primary ray hit a surface      */
    uint32_t frames;            /* frames recorded                             */
    uint16_t shading_model[6];  /* half: share of frames per shading model
                                   (AR_MAT_*), [4] = no surface, [5] unused    */
    uint32_t reserved[2];
} ar_screen_gbuffer;            /* 48 bytes */

/* Box-Cox (lambda 0.5) moments of the per-frame samples: replaces
 * denoise::ScreenStatisticsBuffer (core/denoise/denoise_statistic.cuh:11-24). */
typedef struct ar_screen_stats {
    uint32_t num;               /* samples recorded                            */
    float mean[3];              /* mean of BoxCox(sample)                      */
    float m2_div_n[3];          /* second central moment / num                 */
    float m3_div_n[3];          /* third central moment / num                  */
    uint32_t reserved[2];
} ar_screen_stats;              /* 48 bytes */

/* One interactive frame (params->spp must be 1, RGB or single-wavelength
 * spectral) that also records, per pixel, the primary hit into `gbuffer`
 * (denoise::RecordScreenGBuffer at depth 0, core/render/render.cuh:640-643)
 * and the frame's clamped sample into `stats` (RecordScreenStatisticBuffer,
 * render.cuh:988-991, core/denoise/denoise_statistic.cuh:37-69).  Either
 * buffer may be NULL.  out_rgb / accum as in ar_render with AR_MEM_DEVICE
 * (either may be NULL, not both).  Replaces the recording part of the
 * interactive SceneRenderer::Render (core/scene.hpp:128-133). */
ar_status ar_render_frame_denoise(ar_scene* scene, const ar_camera* camera, const ar_render_params* params,
                                  float* out_rgb, double* accum, ar_screen_gbuffer* gbuffer,
                                  ar_screen_stats* stats, void* stream);

/* Records one frame from caller-supplied primary-hit attributes and samples
 * (for a caller with its own primary visibility, and the parity tests):
 * hits holds 12 floats per pixel -- albedo.xyz, normal.xyz, metallic,
 * roughness, depth, shading model (AR_MAT_* as a float), hit flag (nonzero =
 * surface), unused -- and samples 3 floats per pixel (the clamped sample).
 * Either output may be NULL.  Device pointers; n pixels. */
ar_status ar_denoise_record(const float* hits, const float* samples, size_t n, ar_screen_gbuffer* gbuffer,
                            ar_screen_stats* stats, void* stream);

/* Bilateral filter of the reference (denoise::Bilateral16x16<7>,
 * core/denoise/denoise.cuh:359-443): a 15 x 15 window in log(1 + c) space,
 * each neighbour weighted by the guide-buffer similarity (ComputeSVGFWeight,
 * denoise.cuh:185-245), a Gaussian of the pixel offset (sigma 2) and a
 * skewness-corrected Welch t-test at 0.005 between the two pixels' Box-Cox
 * moments (ComputeTStatisticFinal, denoise.cuh:341-356); borders clamp.  A
 * neighbour whose guide weight is not a number (a pixel whose primary ray
 * never hit has a zero normal) contributes nothing.  hdr_in and hdr_out:
 * width*height*3 floats; all pointers on the device; hdr_out must not alias
 * hdr_in.  The call takes 32 bytes per pixel of stream-ordered scratch
 * (cudaMallocAsync / cudaFreeAsync on `stream`) for the tap mask between its
 * two passes. */
ar_status ar_denoise_bilateral(const float* hdr_in, float* hdr_out, const ar_screen_gbuffer* gbuffer,
                               const ar_screen_stats* stats, int32_t width, int32_t height, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* APERTURE_B200_H */
