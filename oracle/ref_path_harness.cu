// ref_path_harness.cu -- runs the reference's own path loop on the host.
// TEST INFRASTRUCTURE ONLY: built by `make -C oracle ref-path` from the
// build-time copy that ref_path_patch.py makes of the reference's core/ (git-
// ignored, oracle/_ref/src/core) into oracle/_ref/libref_path.so (host math)
// and oracle/_ref/libref_path_detmath.so (the oracle's fixed transcendental
// functions, REF_PATH_DETMATH).  Loaded by the fixture generator under
// tests/golden/, by pinning tests and by the CPU legs of bench.py.
//
// Called unchanged (apart from the edits ref_path_patch.py lists):
//   CalculateRadiance<bUseBVH = true, bUseNEE, bUsePathGuiding = false>
//       core/render/render.cuh:460-999, with everything under it: Trace,
//       NEE, SegmentTrace, TraverseBVH, AnyHitSegmentBVH, the intersectors,
//       EvaluateMaterial / SampleBSDF / EvaluateBSDFWithCos / BSDF_PDF,
//       NEESampleLight and the NEE pdfs, Overlap, PowerHeuristic, SkyLighting;
//   the scene through ref_scene_common.h (SceneObject, BuildBVH, light table).
// Restated here because its file (core/scene.cu) needs OptiX and the GUI: the
// per-pixel part of RenderCamera (core/scene.cu:201-240) -- two Rand1 jitters,
// the pinhole ray with the reference's arithmetic (field of view as a
// parameter instead of the fixed 60 degrees) and max(0, result).
//
// Per-path records (ar_path_record) are filled by the observation hooks:
// segments and closest-hit objects after each Trace, shadow rays and their
// loop depth after each NEE segment query, and the uniforms drawn.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "nee/nee.cuh"
#include "guiding/octahedron.cuh"
#include "vector.cuh"
#include "render/sample.cuh"
#include "render/object.cuh"
#include "render/material.cuh"
#include "render/intersection.cuh"
#include "denoise/denoise.cuh"
#include "denoise/denoise_statistic.cuh"
#include "guiding/guiding.cuh"
#include "guiding/guiding_debug.cuh"
#include "spectrum/sample_ciexyz.cuh"

// The scene globals of render.cuh:23-56 (skipped there through RENDER_GLOBAL),
// as host variables for the host pass.
#ifdef __CUDA_ARCH__
#define REF_GLOBAL __device__
#else
#define REF_GLOBAL
#endif
REF_GLOBAL int RESOLUTION = 0;
REF_GLOBAL int FRAME_INDEX = 0;
REF_GLOBAL SceneObject* SCENE_OBJECTS = nullptr;
REF_GLOBAL int SCENE_OBJECT_COUNTS = 0;
REF_GLOBAL AdditionalLightInfo* SCENE_LIGHTS_INFO = nullptr;
REF_GLOBAL int SCENE_LIGHTS_COUNTS = 0;
REF_GLOBAL BVHNode* BVH_NODES = nullptr;
REF_GLOBAL int BVH_NODES_COUNTS = 0;
REF_GLOBAL int* BVH_OBJECT_INDICES = nullptr;
REF_GLOBAL SceneSetting SETTING = {};
REF_GLOBAL Octahedron* SCENE_PROBES = nullptr;
REF_GLOBAL size_t SCENE_PROBES_COUNTS = 0;
REF_GLOBAL int3 INDIRECT_VOLUME_START = {0, 0, 0};
REF_GLOBAL int3 INDIRECT_VOLUME_END = {0, 0, 0};
REF_GLOBAL int3 INDIRECT_VOLUME_SIZE = {0, 0, 0};
REF_GLOBAL size_t* INDIRECT_INDEX_VOLUME = nullptr;
REF_GLOBAL float* SPECTRUM_LUT_RGB = nullptr;
REF_GLOBAL float* SPECTRUM_LUT_LAMBDA = nullptr;

#include "render/render.cuh"

#include "ref_scene_common.h"

// The SDF cache pointers the reference declares extern (object/sdf/sdf_master.cuh:12-13);
// scene.cu defines them in the reference build.  The path scenes have no SDF object.
namespace sdf {
__device__ SDFVolumeInfo* cachedSDFInfoPtrs = nullptr;
__device__ uint32_t cachedSDFInfoPtrsCount = 0;
}  // namespace sdf

namespace {

int g_max_depth = 1000;
std::mutex g_render_mutex;  // the scene globals serve one render at a time

// Per-path state.  The reference passes a curandState* down the whole loop;
// the harness gives it the address of `rng`, the first member, and recovers
// the rest of the state from it in the hooks.
struct PathState {
    curandState rng;
    const float* tape;
    int limit;
    int pos;
    int overflow;
    uint64_t gen;  // host generator (splitmix64) when tape is NULL
    int segments;
    int hits[AR_DEBUG_MAX_HITS];
    int nee_rays;
    int nee_mask;
};
static_assert(offsetof(PathState, rng) == 0, "curandState must be the first member");

PathState* state_of(curandState* s) { return reinterpret_cast<PathState*>(s); }

void begin_path(PathState& st, const float* tape, int limit, uint64_t gen)
{
    std::memset(&st, 0, sizeof(st));
    st.tape = tape;
    st.limit = limit;
    st.gen = gen;
    for (int& h : st.hits) h = -1;
}

void bind_scene(const ref_scene_data& s)
{
    SCENE_OBJECTS = const_cast<SceneObject*>(s.objects.data());
    SCENE_OBJECT_COUNTS = static_cast<int>(s.objects.size());
    SCENE_LIGHTS_INFO = const_cast<AdditionalLightInfo*>(s.lights.data());
    SCENE_LIGHTS_COUNTS = static_cast<int>(s.lights.size());
    BVH_NODES = const_cast<BVHNode*>(s.bvh.nodes_.data());
    BVH_NODES_COUNTS = static_cast<int>(s.bvh.nodes_.size());
    BVH_OBJECT_INDICES = const_cast<int*>(s.bvh.objectIndices_.data());
    FRAME_INDEX = 0;
    SCENE_PROBES = nullptr;
    SCENE_PROBES_COUNTS = 0;
}

// RenderCamera's per-pixel part (core/scene.cu:213-240), field of view from
// the camera instead of the fixed 60 degrees.
float3 camera_sample(const ar_camera& cam, int i, int j, curandState* seed, bool nee)
{
    const int2 size = make_int2(cam.width, cam.height);
    const float3 cameraOrigin = make_float3(cam.position.x, cam.position.y, cam.position.z);
    const float3 cameraDirection = make_float3(cam.direction.x, cam.direction.y, cam.direction.z);
    float u = (i + Rand1(seed)) / static_cast<float>(size.x);
    float v = (j + Rand1(seed)) / static_cast<float>(size.y);
    float2 ndc = make_float2(u * 2.f - 1.f, (1.0 - v) * 2.f - 1.f);
    const float FOV = cam.fov_y_deg * 3.1415926f / 180.0f;
    const float aspect = static_cast<float>(size.x) / max(1.0f, static_cast<float>(size.y));
    const float tanHalfY = tanf(0.5f * FOV);
    const float tanHalfX = tanHalfY * aspect;
    const float sx = ndc.x * tanHalfX;
    const float sy = ndc.y * tanHalfY;
    const float3 right = normalize(cross(cameraDirection, float3{0.0, 1.0, 0.0}));
    const float3 up = normalize(cross(cameraDirection, right));
    const float3 rayDirection = normalize(cameraDirection + right * sx + up * sy);
    const float4 r = nee ? CalculateRadiance<true, true, false>(seed, cameraOrigin, rayDirection, nullptr, nullptr, nullptr)
                         : CalculateRadiance<true, false, false>(seed, cameraOrigin, rayDirection, nullptr, nullptr, nullptr);
    float3 result = make_f3(r);
    result = max(float3{0}, result);
    return result;
}

int check_params(const ar_render_params* p)
{
    // MIN_TRACING_DEPTH (config.cuh:6) is compiled in; the sky is on (DISABLE_SKYLIGHT
    // undefined, config.cuh:55); one hero wavelength needs the spectral build.
    if (p->rr_depth != MIN_TRACING_DEPTH || p->sky != 1 || p->spectral != 0 || p->tri_light_nee != 0) return -1;
    if (p->max_depth < 1) return -1;
    return 0;
}

int thread_count_of(int threads)
{
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

}  // namespace

int ref_path_host_max_depth() { return g_max_depth; }

float ref_host_uniform(curandState* seed)
{
    PathState* st = state_of(seed);
    if (st->tape) {
        if (st->pos >= st->limit) { st->overflow = 1; st->pos++; return 0.5f; }
        return st->tape[st->pos++];
    }
    // splitmix64 -> uniform in (0, 1], for the CPU baseline (not curand's stream)
    uint64_t z = (st->gen += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z = z ^ (z >> 31);
    st->pos++;
    return static_cast<float>((z >> 40) + 1) * 0x1p-24f;
}

void ref_host_trace(curandState* seed, int object)
{
    PathState* st = state_of(seed);
    if (st->segments < AR_DEBUG_MAX_HITS) st->hits[st->segments] = object;
    st->segments++;
}

void ref_host_shadow(curandState* seed, int depth)
{
    PathState* st = state_of(seed);
    st->nee_rays++;
    if (depth < 32) st->nee_mask |= static_cast<int>(1u << depth);
}

struct ref_path_scene : ref_scene_data {};

extern "C" {

ref_path_scene* refp_scene_create(const ar_object_desc* objects, size_t count, int leaf_size, int bin_count)
{
    ref_path_scene* s = new ref_path_scene;
    ref_build_scene(objects, count, leaf_size, bin_count, s);
    return s;
}

void refp_scene_destroy(ref_path_scene* s) { delete s; }

#ifdef REF_PATH_DETMATH
int refp_detmath() { return 1; }
#else
int refp_detmath() { return 0; }
#endif

// Replay spp samples of every pixel with uniforms read from `tape` (the
// ar_rng_tape layout: per path `per_path` floats, sample major) and write one
// ar_path_record per path.  Returns the number of paths that ran out of tape,
// or -1 for parameters this build cannot express.
int64_t refp_render_paths(const ref_path_scene* s, const ar_camera* cam, const ar_render_params* p, const float* tape,
                          int per_path, ar_path_record* rec, int threads)
{
    if (check_params(p)) return -1;
    std::lock_guard<std::mutex> lock(g_render_mutex);
    bind_scene(*s);
    g_max_depth = p->max_depth;
    const int64_t W = cam->width, H = cam->height, S = p->spp;
    int64_t overflow = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : overflow) num_threads(thread_count_of(threads))
    for (int64_t k = 0; k < W * H * S; ++k) {
        const int i = static_cast<int>(k % W), j = static_cast<int>((k / W) % H);
        PathState st;
        begin_path(st, tape + k * per_path, per_path, 0);
        const float3 r = camera_sample(*cam, i, j, &st.rng, p->use_nee != 0);
        ar_path_record* o = &rec[k];
        std::memset(o, 0, sizeof(*o));
        o->radiance[0] = r.x; o->radiance[1] = r.y; o->radiance[2] = r.z;
        o->segments = st.segments;
        o->uniforms = st.pos;
        o->nee_rays = st.nee_rays;
        o->nee_depth_mask = st.nee_mask;
        for (int h = 0; h < AR_DEBUG_MAX_HITS; ++h) o->hit_object[h] = st.hits[h];
        if (st.overflow) overflow++;
    }
    return overflow;
}

// CPU baseline: pixels pb, pb + step, ... < pe, spp samples each from the host
// generator, FP64 sums added into accum (w*h*3); closest-hit and shadow query
// counts.  Returns 0, or -1 for parameters this build cannot express.
int refp_render_image(const ref_path_scene* s, const ar_camera* cam, const ar_render_params* p, int64_t pb, int64_t pe,
                      int64_t step, double* accum, int64_t* ext, int64_t* shadow, int threads)
{
    if (check_params(p)) return -1;
    std::lock_guard<std::mutex> lock(g_render_mutex);
    bind_scene(*s);
    g_max_depth = p->max_depth;
    const int64_t W = cam->width;
    if (step < 1) step = 1;
    const int64_t count = (pe - pb + step - 1) / step;
    int64_t e = 0, sh = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : e, sh) num_threads(thread_count_of(threads))
    for (int64_t k = 0; k < count; ++k) {
        const int64_t pix = pb + k * step;
        const int i = static_cast<int>(pix % W), j = static_cast<int>(pix / W);
        double acc[3] = {0.0, 0.0, 0.0};
        for (int smp = 0; smp < p->spp; ++smp) {
            PathState st;
            begin_path(st, nullptr, 0,
                       p->seed ^ (static_cast<uint64_t>(pix) * 0x9e3779b97f4a7c15ull) ^
                           (static_cast<uint64_t>(smp + p->frame_offset) << 40));
            const float3 r = camera_sample(*cam, i, j, &st.rng, p->use_nee != 0);
            acc[0] += r.x; acc[1] += r.y; acc[2] += r.z;
            e += st.segments;
            sh += st.nee_rays;
        }
        accum[3 * pix + 0] += acc[0]; accum[3 * pix + 1] += acc[1]; accum[3 * pix + 2] += acc[2];
    }
    if (ext) *ext = e;
    if (shadow) *shadow = sh;
    return 0;
}

}  // extern "C"

// ---- path guiding probes (core/guiding/octahedron.cuh, guiding_bin.cuh), for
// pinning the CUDA core's probe math: the reference's 20 face normals
// (FaceNormal20FromIndex, guiding_bin.cuh:40-66), its (voxel, face) grid of a
// point and direction (GetVoxelGrid, guiding_bin.cuh:102-114), and per query
// SampleOctahedronHemisphere (octahedron.cuh:343-364; three mip-descent
// uniforms and two for the point in the leaf texel, read from u5) and
// OctahedronHemispherePDF (octahedron.cuh:366-380) of given probes.
extern "C" {

void refp_guiding_faces(float* out60)
{
    for (int f = 0; f < PATH_GUIDING_FACE_COUNT; ++f) {
        const float3 n = pg::FaceNormal20FromIndex(f);
        out60[3 * f] = n.x; out60[3 * f + 1] = n.y; out60[3 * f + 2] = n.z;
    }
}

void refp_guiding_voxel(const float* pos3, const float* dir3, int64_t n, int32_t* out4)
{
    for (int64_t i = 0; i < n; ++i) {
        const int4 g = pg::GetVoxelGrid(make_float3(pos3[3 * i], pos3[3 * i + 1], pos3[3 * i + 2]),
                                        make_float3(dir3[3 * i], dir3[3 * i + 1], dir3[3 * i + 2]));
        out4[4 * i] = g.x; out4[4 * i + 1] = g.y; out4[4 * i + 2] = g.z; out4[4 * i + 3] = g.w;
    }
}

// texels: nprobes x 85 x 4 floats (leaves 8x8, then the 4x4, 2x2, 1x1 mips; rgb + unused)
void refp_guiding_sample(const float* texels, int32_t nprobes, const int32_t* probe_of, const float* normal3,
                         const float* query3, const float* u5, const float* eval3, int64_t n, float* out_dir3,
                         float* out_pdf, float* out_eval_pdf)
{
    std::vector<Octahedron> probes(static_cast<size_t>(nprobes));
    for (int32_t p = 0; p < nprobes; ++p) {
        std::memset(&probes[p], 0, sizeof(Octahedron));
        for (int t = 0; t < Octahedron::totalPixelCount_; ++t) {
            const float* s = texels + (static_cast<size_t>(p) * Octahedron::totalPixelCount_ + t) * 4;
            probes[p].data_[t] = make_float4(s[0], s[1], s[2], s[3]);
        }
    }
    for (int64_t i = 0; i < n; ++i) {
        const Octahedron& o = probes[static_cast<size_t>(probe_of[i])];
        const float3 nrm = make_float3(normal3[3 * i], normal3[3 * i + 1], normal3[3 * i + 2]);
        const float3 q = make_float3(query3[3 * i], query3[3 * i + 1], query3[3 * i + 2]);
        PathState st;
        begin_path(st, u5 + 5 * i, 5, 0);
        const Sample smp = o.SampleOctahedronHemisphere(&st.rng, nrm, q);
        out_dir3[3 * i] = smp.direction_.x; out_dir3[3 * i + 1] = smp.direction_.y; out_dir3[3 * i + 2] = smp.direction_.z;
        out_pdf[i] = smp.pdf_;
        out_eval_pdf[i] = o.OctahedronHemispherePDF(make_float3(eval3[3 * i], eval3[3 * i + 1], eval3[3 * i + 2]), nrm, q);
    }
}

}  // extern "C"
