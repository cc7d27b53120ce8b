// capi.cu -- implementation of the C ABI declared in include/aperture_b200.h.
//
// Host orchestration only: scene upload, workspace management and the order of
// kernel launches.  All arithmetic on scene data happens in scene_build.cpp
// (host, once per scene) and render.cu (device).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/aperture_b200.h"
#include "render_kernels.h"
#include "scene_build.h"
#include "sdf.cuh"
#include "xorwow_jump.h"

namespace {

thread_local std::string g_last_error;

ar_status fail(ar_status s, const std::string& msg)
{
    g_last_error = msg;
    return s;
}

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t c, const std::string& where)
        : std::runtime_error(where + ": " + cudaGetErrorString(c)), code(c) {}
};

void ck(cudaError_t e, const char* where)
{
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(e, where);
    }
}

template <class T>
T* dalloc(size_t count, const char* what)
{
    if (count == 0) count = 1;
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw CudaError(e, std::string("cudaMalloc ") + what);
    }
    return static_cast<T*>(p);
}

template <class T>
T* upload(const std::vector<T>& v, const char* what)
{
    T* p = dalloc<T>(v.size(), what);
    if (!v.empty()) ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
    return p;
}

class DeviceGuard {
public:
    explicit DeviceGuard(int dev)
    {
        ck(cudaGetDevice(&prev_), "cudaGetDevice");
        if (prev_ != dev) ck(cudaSetDevice(dev), "cudaSetDevice");
        changed_ = prev_ != dev;
    }
    ~DeviceGuard() { if (changed_) cudaSetDevice(prev_); }
private:
    int prev_ = 0;
    bool changed_ = false;
};

// The same for destructors: never throws (the runtime may already be shutting
// down when a handle is released at process exit).
class QuietDeviceGuard {
public:
    explicit QuietDeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev_) == cudaSuccess && prev_ != dev) changed_ = cudaSetDevice(dev) == cudaSuccess;
        cudaGetLastError();
    }
    ~QuietDeviceGuard() { if (changed_) cudaSetDevice(prev_); }
private:
    int prev_ = 0;
    bool changed_ = false;
};

constexpr int64_t kMaxPool = int64_t(1) << 21;  // paths in flight

}  // namespace

struct ar_scene {
    int device = 0;
    int sm_count = 148;
    ar::SceneView view{};
    int grid_trace = 0;
    const uint32_t* jump_table = nullptr;  // A^(2^32) lookup table of the XORWOW register
    const uint32_t* jump_table67 = nullptr;  // A^(2^67): one curand subsequence
    int64_t objects = 0, triangles = 0, lights = 0, nodes = 0, prims = 0;
    int64_t device_bytes = 0;
    std::vector<void*> owned;
    // host copy for the camera overlap test (intersection::Overlap)
    std::vector<ar::ObjInfo> h_objects;
    std::vector<ar::Analytic> h_analytic;
    // spectral mode (ar_scene_set_spectral): reference tables and lookup tables
    float* spec_tables = nullptr;
    float4* spec_lut_lam = nullptr;
    float4* spec_lut_rgb = nullptr;
    int spec_res = 0;
    void* medium_grid = nullptr;                // density grid of the participating medium
    float bounds[6] = {0, 0, 0, 0, 0, 0};       // box of the BVH root (min xyz, max xyz)
    std::vector<ar::SdfRec> h_sdf;              // data pointers into h_volumes
    std::vector<ar::HostVolume> h_volumes;
    // render workspace
    char* ws = nullptr;
    size_t ws_bytes = 0;
    int64_t ws_wave = 0;
    int64_t ws_pix = 0;
    ar::PathBuffers bufs{};
    uint4* base0 = nullptr;
    uint2* base1 = nullptr;
    // the per-pixel generator states in base0/base1 are those of frame
    // rng_next_frame for (rng_seed, rng_width, rng_height) when rng_valid
    bool rng_valid = false;
    uint64_t rng_seed = 0, rng_next_frame = 0;
    int rng_width = 0, rng_height = 0;
    double* accum = nullptr;
    float* fout = nullptr;
    ar::PoolCtl* ctl = nullptr;
    unsigned long long* stats = nullptr;
    int* err = nullptr;
    uint32_t* ovf = nullptr;  // traversal stack overflow slabs, one per persistent thread
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> timer_ext, timer_sh;  // event pairs around traversal launches

    ~ar_scene()
    {
        QuietDeviceGuard g(device);
        for (void* p : owned) cudaFree(p);
        if (ws) cudaFree(ws);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        for (cudaEvent_t e : timer_ext) cudaEventDestroy(e);
        for (cudaEvent_t e : timer_sh) cudaEventDestroy(e);
    }
};

namespace {

// Carve the two path pools, side arrays, queues and per-pixel buffers from one
// allocation (re-used across calls; grown when a larger pool or image comes).
void ensure_workspace(ar_scene* s, int64_t pool, int64_t npix)
{
    if (s->ws && s->ws_wave >= pool && s->ws_pix >= npix) return;
    if (s->ws) { cudaFree(s->ws); s->ws = nullptr; }
    pool = std::max(pool, s->ws_wave);
    npix = std::max(npix, s->ws_pix);
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t W = static_cast<size_t>(pool), N = static_cast<size_t>(npix);
    const size_t o_p0 = take(sizeof(ar::PathRec) * W), o_p1 = take(sizeof(ar::PathRec) * W);
    const size_t o_hit = take(16 * W), o_qsh = take(4 * W * ar::kShadeBuckets);
    const size_t o_sh = take(sizeof(ar::ShadowRec) * W), o_rt = take(sizeof(ar::RetireRec) * W);
    const size_t o_ax0 = take(16 * W), o_ax1 = take(16 * W), o_sh3 = take(4 * W);
    const size_t o_b0 = take(16 * N), o_b1 = take(8 * N), o_acc = take(24 * N), o_fout = take(12 * N);
    const size_t o_cnt = take(sizeof(ar::PoolCtl)), o_stats = take(64), o_err = take(64);
    const size_t o_ovf = take(static_cast<size_t>(s->grid_trace) * ar::kTraceBlock * ar::kStackOverflow * 4);
    s->ws = dalloc<char>(off, "render workspace");
    s->ws_bytes = off;
    s->ws_wave = pool;
    s->ws_pix = npix;
    s->rng_valid = false;
    char* b = s->ws;
    ar::PathBuffers& B = s->bufs;
    B.pool[0] = reinterpret_cast<ar::PathRec*>(b + o_p0);
    B.pool[1] = reinterpret_cast<ar::PathRec*>(b + o_p1);
    B.hit = reinterpret_cast<int4*>(b + o_hit);
    B.qsh = reinterpret_cast<int32_t*>(b + o_qsh);
    B.shadow = reinterpret_cast<ar::ShadowRec*>(b + o_sh);
    B.retire = reinterpret_cast<ar::RetireRec*>(b + o_rt);
    B.aux[0] = reinterpret_cast<float4*>(b + o_ax0);
    B.aux[1] = reinterpret_cast<float4*>(b + o_ax1);
    B.shadow3 = reinterpret_cast<float*>(b + o_sh3);
    B.capacity = static_cast<int32_t>(pool);
    s->base0 = reinterpret_cast<uint4*>(b + o_b0);
    s->base1 = reinterpret_cast<uint2*>(b + o_b1);
    s->accum = reinterpret_cast<double*>(b + o_acc);
    s->fout = reinterpret_cast<float*>(b + o_fout);
    s->ctl = reinterpret_cast<ar::PoolCtl*>(b + o_cnt);
    s->stats = reinterpret_cast<unsigned long long*>(b + o_stats);
    s->err = reinterpret_cast<int*>(b + o_err);
    s->ovf = reinterpret_cast<uint32_t*>(b + o_ovf);
}

// intersection::Overlap (intersection.cuh:399-414) at the camera position; the
// reference scans every object per path, here it is done once per render.
bool camera_inside(const ar_scene* s, ar::f3 p)
{
    using namespace ar;
    for (size_t i = 0; i < s->h_objects.size(); ++i) {
        const ObjInfo& oi = s->h_objects[i];
        if (oi.type == AR_OBJ_SDF) {
            const SdfRec& g = s->h_sdf[oi.aux];
            if (sdf_contains(g, s->h_analytic[g.analytic], p)) return true;
            continue;
        }
        if (oi.type != AR_OBJ_CUBE && oi.type != AR_OBJ_SPHERE) continue;
        const Analytic& an = s->h_analytic[oi.aux];
        m3 w2o;
        w2o.x = mk(an.w2o[0], an.w2o[1], an.w2o[2]);
        w2o.y = mk(an.w2o[3], an.w2o[4], an.w2o[5]);
        w2o.z = mk(an.w2o[6], an.w2o[7], an.w2o[8]);
        const f3 l = mul(w2o, p - mk(an.center[0], an.center[1], an.center[2]));
        if (oi.type == AR_OBJ_CUBE) {
            const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
            if (-e.x < l.x && -e.y < l.y && -e.z < l.z && e.x > l.x && e.y > l.y && e.z > l.z) return true;
        } else {
            if (dot(l, l) < an.radius * an.radius) return true;
        }
    }
    return false;
}

ar_status check_camera(const ar_camera* c)
{
    if (!c) return fail(AR_ERR_INVALID_ARGUMENT, "camera is NULL");
    if (c->width <= 0 || c->height <= 0) return fail(AR_ERR_INVALID_ARGUMENT, "camera width/height must be positive");
    if (static_cast<int64_t>(c->width) * c->height > (int64_t(1) << 28))
        return fail(AR_ERR_INVALID_ARGUMENT, "image larger than 2^28 pixels");
    if (!(c->fov_y_deg > 0.0f && c->fov_y_deg < 180.0f)) return fail(AR_ERR_INVALID_ARGUMENT, "fov_y_deg must be in (0, 180)");
    return AR_OK;
}

ar_status check_params(const ar_render_params* p)
{
    if (!p) return fail(AR_ERR_INVALID_ARGUMENT, "params is NULL");
    if (p->spp <= 0) return fail(AR_ERR_INVALID_ARGUMENT, "spp must be positive");
    if (p->max_depth <= 0 || p->max_depth > 4096) return fail(AR_ERR_INVALID_ARGUMENT, "max_depth must be in [1, 4096]");
    if (p->rr_depth < 0) return fail(AR_ERR_INVALID_ARGUMENT, "rr_depth must be >= 0");
    if (p->frame_offset < 0) return fail(AR_ERR_INVALID_ARGUMENT, "frame_offset must be >= 0");
    if (p->spectral != 0 && p->spectral != 1 && p->spectral != 4)
        return fail(AR_ERR_INVALID_ARGUMENT, "spectral must be 0, 1 or 4");
    if (p->tri_light_nee != 0 && p->tri_light_nee != 1)
        return fail(AR_ERR_INVALID_ARGUMENT, "tri_light_nee must be 0 or 1");
    if (p->sort_rays != 0)
        return fail(AR_ERR_UNSUPPORTED,
                    "sort_rays: only 0 is supported (paths are always shaded in material buckets; a direction-octant "
                    "sort of the extension rays is not built)");
    return AR_OK;
}

ar::FrameParams make_frame(const ar_scene* s, const ar_camera* c, const ar_render_params* p)
{
    using namespace ar;
    FrameParams fp;
    std::memset(&fp, 0, sizeof(fp));
    const f3 cd = mk(c->direction.x, c->direction.y, c->direction.z);
    // RenderCamera (scene.cu:218-230) with the field of view as a parameter
    const float fov = c->fov_y_deg * 3.1415926f / 180.0f;
    const float aspect = static_cast<float>(c->width) / std::max(1.0f, static_cast<float>(c->height));
    const float tanHalfY = tan_det(0.5f * fov);
    fp.tan_half_y = tanHalfY;
    fp.tan_half_x = tanHalfY * aspect;
    const f3 right = normalize(cross(cd, mk(0.0f, 1.0f, 0.0f)));
    const f3 up = normalize(cross(cd, right));
    fp.cam_o[0] = c->position.x; fp.cam_o[1] = c->position.y; fp.cam_o[2] = c->position.z;
    fp.cam_d[0] = cd.x; fp.cam_d[1] = cd.y; fp.cam_d[2] = cd.z;
    fp.right[0] = right.x; fp.right[1] = right.y; fp.right[2] = right.z;
    fp.up[0] = up.x; fp.up[1] = up.y; fp.up[2] = up.z;
    fp.width = c->width;
    fp.height = c->height;
    fp.grid_x = (c->width + 7) / 8;
    fp.npix = c->width * c->height;
    fp.camera_inside = camera_inside(s, mk(c->position.x, c->position.y, c->position.z)) ? 1 : 0;
    if (p) {
        fp.max_depth = p->max_depth;
        fp.rr_depth = p->rr_depth;
        fp.use_nee = p->use_nee;
        fp.sky = p->sky;
        fp.seed = p->seed;
        fp.frame0 = static_cast<uint64_t>(p->frame_offset);
        fp.tri_light_nee = p->tri_light_nee;
        fp.medium_key = medium_frame_key(fp.seed, fp.frame0);
        if (p->spectral) {
            fp.spectral = p->spectral;
            fp.spec.tables = s->spec_tables;
            fp.spec.lut_lam = s->spec_lut_lam;
            fp.spec.lut_rgb = s->spec_lut_rgb;
            fp.spec.res = s->spec_res;
        }
    }
    for (int d = 0; d <= 8; ++d) fp.eps_tab[d] = 1.0e-3f * exp_det(fminf(static_cast<float>(d) * 0.5f, 4.0f));
    return fp;
}

ar_status run_render(ar_scene* s, const ar_camera* cam, const ar_render_params* p, ar_path_record* rec_dev,
                     cudaStream_t st, ar_render_stats* stats, const ar::NrcFrame* nrc = nullptr,
                     const ar::GuideView* guide = nullptr, const ar::DenoiseView* dn = nullptr)
{
    using namespace ar;
    if (p->spectral && !s->spec_tables)
        return fail(AR_ERR_UNSUPPORTED, "spectral rendering needs ar_scene_set_spectral first");
    ar::FrameParams fp = make_frame(s, cam, p);
    const int64_t npix = fp.npix;
    const int64_t total = npix * p->spp;
    int64_t pool = p->wave_paths > 0 ? std::min<int64_t>(p->wave_paths, kMaxPool) : kMaxPool;
    pool = std::max<int64_t>(1, std::min<int64_t>(pool, total));
    fp.pool = static_cast<int32_t>(pool);
    if (nrc) fp.nrc = *nrc;
    if (guide) {
        fp.guiding = 1;
        fp.guide = *guide;
    }
    if (dn) fp.dn = *dn;
    ensure_workspace(s, pool, npix);
    PathBuffers B = s->bufs;
    B.capacity = static_cast<int32_t>(pool);
    ck(cudaMemsetAsync(s->accum, 0, sizeof(double) * 3 * npix, st), "memset accum");
    ck(cudaMemsetAsync(s->stats, 0, 64, st), "memset stats");
    ck(cudaMemsetAsync(s->err, 0, 64, st), "memset err");
    if (!s->ev0) { ck(cudaEventCreate(&s->ev0), "event"); ck(cudaEventCreate(&s->ev1), "event"); }
    ck(cudaEventRecord(s->ev0, st), "event record");
    // curand_init of every pixel (a skip-ahead per pixel) only when the stored
    // states are not already those of this render's first frame: a render that
    // continues the previous one (frame_offset = previous offset + spp, same
    // seed and image) starts from the states the previous one left.
    if (!(s->rng_valid && s->rng_seed == fp.seed && s->rng_width == fp.width && s->rng_height == fp.height &&
          s->rng_next_frame == fp.frame0))
        ck(launch_rng_init(fp, s->base0, s->base1, s->jump_table67, st), "rng init");
    s->rng_valid = false;
    ck(launch_pool_init(s->ctl, total, st), "pool init");
    int64_t launches = 2;
    const int grid_trace = s->grid_trace;
    const int grid_other = s->sm_count * 4;
    LaunchTimers tm;
    LaunchTimers* tmp = stats ? &tm : nullptr;
    constexpr int kBatch = 16;
    // every iteration retires or advances each path by one segment and admits up
    // to min(pool, npix) new samples (k_plan): a hard bound
    const int64_t admit = std::max<int64_t>(1, std::min<int64_t>(pool, npix));
    const int64_t max_iter = (total / admit + 2) * (static_cast<int64_t>(p->max_depth) + 2) + kBatch;
    int cur = 0;
    int64_t iters = 0;
    int64_t retired = 0;
    for (;;) {
        if (tmp) {
            const size_t need = static_cast<size_t>(2 * (iters + kBatch));
            for (auto* v : {&s->timer_ext, &s->timer_sh}) {
                while (v->size() < need) {
                    cudaEvent_t e;
                    ck(cudaEventCreate(&e), "event create");
                    v->push_back(e);
                }
            }
            // the vectors may have grown: re-point; recorded pairs keep their handles
            tm.extend_ev = s->timer_ext.data();
            tm.shadow_ev = s->timer_sh.data();
            tm.cap = static_cast<int>(need / 2);
        }
        ck(launch_iterations(s->view, fp, B, s->ctl, s->base0, s->base1, s->jump_table, s->stats, s->ovf, s->err,
                             s->accum, rec_dev,
                             kBatch, &cur, grid_trace, grid_other, st, &launches, tmp),
           "render launch");
        iters += kBatch;
        ck(cudaMemcpyAsync(&retired, &s->ctl->retired, sizeof(int64_t), cudaMemcpyDeviceToHost, st), "poll");
        ck(cudaStreamSynchronize(st), "sync");
        if (retired >= total) break;
        if (iters > max_iter) return fail(AR_ERR_DEVICE_FAULT, "path pool did not drain");
    }
    // every pixel's state advanced by one frame per sample (k_regen)
    s->rng_valid = true;
    s->rng_seed = fp.seed;
    s->rng_width = fp.width;
    s->rng_height = fp.height;
    s->rng_next_frame = fp.frame0 + static_cast<uint64_t>(p->spp);
    ck(cudaEventRecord(s->ev1, st), "event record");
    if (stats) {
        unsigned long long h[6];
        ck(cudaMemcpyAsync(h, s->stats, sizeof(h), cudaMemcpyDeviceToHost, st), "stats copy");
        ck(cudaStreamSynchronize(st), "sync");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, s->ev0, s->ev1);
        std::memset(stats, 0, sizeof(*stats));
        stats->paths = total;
        stats->extension_rays = static_cast<int64_t>(h[0]);
        stats->shadow_rays = static_cast<int64_t>(h[1]);
        stats->kernel_launches = launches;
        stats->total_ms = ms;
        stats->extend_launches = iters;
        stats->shadow_launches = iters;
        stats->extend_node_visits = static_cast<int64_t>(h[2]);
        stats->extend_prim_tests = static_cast<int64_t>(h[3]);
        stats->shadow_node_visits = static_cast<int64_t>(h[4]);
        stats->shadow_prim_tests = static_cast<int64_t>(h[5]);
        float e_ms = 0.0f, s_ms = 0.0f;
        for (int k = 0; k < tm.n_extend; ++k) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, tm.extend_ev[2 * k], tm.extend_ev[2 * k + 1]);
            e_ms += t;
        }
        for (int k = 0; k < tm.n_shadow; ++k) {
            float t = 0.0f;
            cudaEventElapsedTime(&t, tm.shadow_ev[2 * k], tm.shadow_ev[2 * k + 1]);
            s_ms += t;
        }
        stats->extend_ms = e_ms;
        stats->shadow_ms = s_ms;
    }
    return AR_OK;
}

ar_status check_err(ar_scene* s, cudaStream_t st)
{
    int e = 0;
    ck(cudaMemcpyAsync(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost, st), "error word copy");
    ck(cudaStreamSynchronize(st), "sync");
    if (e != 0) return fail(AR_ERR_DEVICE_FAULT, "traversal stack overflow reported by a kernel");
    return AR_OK;
}

#define AR_GUARD_BEGIN try {
#define AR_GUARD_END                                                              \
    }                                                                             \
    catch (const CudaError& e) {                                                  \
        return fail(e.code == cudaErrorMemoryAllocation ? AR_ERR_OUT_OF_MEMORY    \
                                                        : AR_ERR_CUDA, e.what()); \
    }                                                                             \
    catch (const std::bad_alloc&) { return fail(AR_ERR_OUT_OF_MEMORY, "host allocation failed"); } \
    catch (const std::domain_error& e) { return fail(AR_ERR_UNSUPPORTED, e.what()); } \
    catch (const std::invalid_argument& e) { return fail(AR_ERR_INVALID_ARGUMENT, e.what()); } \
    catch (const std::exception& e) { return fail(AR_ERR_CUDA, e.what()); }

}  // namespace

namespace ar {
// Internal accessors for entry points defined in other translation units.
bool scene_view_of(const ar_scene* s, SceneView* v, int* device, int* sm_count)
{
    if (!s) return false;
    *v = s->view;
    *device = s->device;
    *sm_count = s->sm_count;
    return true;
}
ar_status set_error(ar_status st, const std::string& msg) { return fail(st, msg); }
}  // namespace ar

extern "C" {

int32_t ar_version(void) { return AR_ABI_VERSION; }

const char* ar_get_last_error_string(void) { return g_last_error.c_str(); }

ar_status ar_scene_create(const ar_object_desc* objects, size_t count, int32_t device, ar_scene** out_scene)
{
    return ar_scene_create_ex(objects, count, nullptr, 0, device, out_scene);
}

ar_status ar_scene_create_ex(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes,
                             size_t volume_count, int32_t device, ar_scene** out_scene)
{
    g_last_error.clear();
    if (!out_scene) return fail(AR_ERR_INVALID_ARGUMENT, "out_scene is NULL");
    *out_scene = nullptr;
    if (count > 0 && !objects) return fail(AR_ERR_INVALID_ARGUMENT, "objects is NULL");
    AR_GUARD_BEGIN
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(AR_ERR_INVALID_ARGUMENT, "device index out of range");
    if (volume_count > 0 && !volumes) return fail(AR_ERR_INVALID_ARGUMENT, "volumes is NULL");
    ar::HostScene hs = ar::build_scene(objects, count, volumes, volume_count);
    DeviceGuard g(device);
    ar_scene* s = new ar_scene();
    s->device = device;
    if (!hs.nodes.empty()) {   // root box: origin + the largest quantised child upper bound
        const ar::WideNode& r = hs.nodes[0];
        const float o[3] = {r.ox, r.oy, r.oz};
        const uint8_t* qhi[3] = {r.qhi_x, r.qhi_y, r.qhi_z};
        const uint8_t* qlo[3] = {r.qlo_x, r.qlo_y, r.qlo_z};
        for (int a = 0; a < 3; ++a) {
            const int e = static_cast<int>((r.exps >> (8 * a)) & 0xFFu) - 127;
            const float sc = std::ldexp(1.0f, e);
            float hi = o[a];
            for (int k = 0; k < 8; ++k)
                if (qlo[a][k] <= qhi[a][k]) hi = std::max(hi, o[a] + static_cast<float>(qhi[a][k]) * sc);
            s->bounds[a] = o[a];
            s->bounds[3 + a] = hi;
        }
    }
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, device);
    try {
        auto own = [&](void* p, size_t bytes) { s->owned.push_back(p); s->device_bytes += static_cast<int64_t>(bytes); return p; };
        ar::SceneView& v = s->view;
        v.nodes = static_cast<const ar::WideNode*>(own(upload(hs.nodes, "nodes"), hs.nodes.size() * sizeof(ar::WideNode)));
        v.prims = static_cast<const ar::PrimRec*>(own(upload(hs.prims, "prims"), hs.prims.size() * sizeof(ar::PrimRec)));
        v.objects = static_cast<const ar::ObjInfo*>(own(upload(hs.objects, "objects"), hs.objects.size() * sizeof(ar::ObjInfo)));
        v.trishade = static_cast<const ar::TriShade*>(own(upload(hs.trishade, "trishade"), hs.trishade.size() * sizeof(ar::TriShade)));
        v.analytic = static_cast<const ar::Analytic*>(own(upload(hs.analytic, "analytic"), hs.analytic.size() * sizeof(ar::Analytic)));
        v.materials = static_cast<const ar::MaterialRec*>(own(upload(hs.materials, "materials"), hs.materials.size() * sizeof(ar::MaterialRec)));
        v.light_object = static_cast<const int32_t*>(own(upload(hs.light_object, "lights"), hs.light_object.size() * 4));
        v.light_prob = static_cast<const float*>(own(upload(hs.light_prob, "lights"), hs.light_prob.size() * 4));
        v.light_tri = static_cast<const float4*>(own(upload(hs.light_tri, "light triangles"), hs.light_tri.size() * 16));
        {
            static const std::vector<uint32_t> jt = ar::xorwow_jump_table_2p32();
            s->jump_table = static_cast<const uint32_t*>(own(upload(jt, "rng jump table"), jt.size() * 4));
            static const std::vector<uint32_t> js = ar::xorwow_jump_table_pow2(67);
            s->jump_table67 = static_cast<const uint32_t*>(own(upload(js, "rng subsequence table"), js.size() * 4));
        }
        {
            // SDF volumes, then the SDF records pointing at them (device and host copies)
            std::vector<const void*> vdev(hs.volumes.size());
            for (size_t k = 0; k < hs.volumes.size(); ++k) {
                const std::vector<unsigned char>& b = hs.volumes[k].bytes;
                vdev[k] = own(upload(b, "sdf volume"), b.size());
            }
            std::vector<ar::SdfRec> dsdf = hs.sdf;
            s->h_volumes = std::move(hs.volumes);
            s->h_sdf = hs.sdf;
            for (size_t k = 0; k < dsdf.size(); ++k) {
                if (dsdf[k].kind != ar::kSdfVolume) continue;
                const size_t vi = static_cast<size_t>(dsdf[k].pad[0]);
                dsdf[k].data = vdev[vi];
                s->h_sdf[k].data = s->h_volumes[vi].bytes.data();
            }
            v.sdf = static_cast<const ar::SdfRec*>(own(upload(dsdf, "sdf"), dsdf.size() * sizeof(ar::SdfRec)));
            v.num_sdf = static_cast<int32_t>(dsdf.size());
        }
        v.num_nodes = static_cast<int32_t>(hs.prims.empty() ? 0 : hs.nodes.size());
        v.num_objects = static_cast<int32_t>(hs.objects.size());
        v.num_lights = static_cast<int32_t>(hs.light_object.size());
        if (hs.stack_bound > ar::kStackMax) throw std::domain_error("BVH too deep for the traversal stack");
        s->grid_trace = ar::trace_grid(s->sm_count);
        {
            ar_camera c0{};
            c0.width = c0.height = 1;
            c0.fov_y_deg = 60.0f;
            const ar::FrameParams f0 = make_frame(s, &c0, nullptr);
            ck(ar::set_intersect_eps(f0.eps_tab), "upload INTERSECT_EPS");
        }
        s->objects = static_cast<int64_t>(count);
        s->triangles = hs.triangles;
        s->lights = static_cast<int64_t>(hs.light_object.size());
        s->nodes = static_cast<int64_t>(hs.nodes.size());
        s->prims = static_cast<int64_t>(hs.prims.size());
        s->h_objects = std::move(hs.objects);
        s->h_analytic = std::move(hs.analytic);
    } catch (...) {
        delete s;
        throw;
    }
    *out_scene = s;
    return AR_OK;
    AR_GUARD_END
}

void ar_scene_destroy(ar_scene* scene)
{
    try { delete scene; } catch (...) {}
}

ar_status ar_scene_get_info(const ar_scene* s, ar_scene_info* info)
{
    if (!s || !info) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    std::memset(info, 0, sizeof(*info));
    info->objects = s->objects;
    info->triangles = s->triangles;
    info->lights = s->lights;
    info->wide_nodes = s->nodes;
    info->prim_refs = s->prims;
    info->device_bytes = s->device_bytes;
    info->device = s->device;
    return AR_OK;
}

ar_status ar_bvh_build_info(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes,
                            size_t volume_count, ar_bvh_info* info)
{
    g_last_error.clear();
    if (!info) return fail(AR_ERR_INVALID_ARGUMENT, "info is NULL");
    std::memset(info, 0, sizeof(*info));
    if (count > 0 && !objects) return fail(AR_ERR_INVALID_ARGUMENT, "objects is NULL");
    if (volume_count > 0 && !volumes) return fail(AR_ERR_INVALID_ARGUMENT, "volumes is NULL");
    try {
        const ar::HostScene hs = ar::build_scene(objects, count, volumes, volume_count);
        // every primitive record in exactly one leaf slot, every child index in range
        std::vector<uint8_t> seen(hs.prims.size(), 0);
        for (size_t w = 0; w < hs.nodes.size(); ++w) {
            const ar::WideNode& nd = hs.nodes[w];
            for (int k = 0; k < ar::kWide; ++k) {
                const uint32_t m = ((k < 4 ? nd.meta_lo : nd.meta_hi) >> (8 * (k & 3))) & 0xFFu;
                if (m == ar::kMetaEmpty) continue;
                if (m & ar::kMetaInternal) {
                    const uint64_t c = static_cast<uint64_t>(nd.child_base) + (m & 7u);
                    if (c == 0 || c >= hs.nodes.size())
                        return fail(AR_ERR_INTERNAL, "BVH: child index out of range");
                    ++info->internal_slots;
                } else {
                    const uint32_t cnt = ((m >> 5) & 3u) + 1u;
                    for (uint32_t q = 0; q < cnt; ++q) {
                        const uint64_t pi = static_cast<uint64_t>(nd.prim_base) + (m & 31u) + q;
                        if (pi >= hs.prims.size() || seen[pi]++)
                            return fail(AR_ERR_INTERNAL, "BVH: primitive record out of range or shared");
                    }
                    ++info->leaf_slots;
                }
            }
        }
        for (uint8_t v : seen)
            if (v != 1) return fail(AR_ERR_INTERNAL, "BVH: primitive record in no leaf");
        info->wide_nodes = static_cast<int64_t>(hs.nodes.size());
        info->prim_refs = static_cast<int64_t>(hs.prims.size());
        info->stack_bound = hs.stack_bound;
        info->depth = hs.wide_depth;
        return AR_OK;
    } catch (const std::bad_alloc&) {
        return fail(AR_ERR_OUT_OF_MEMORY, "host allocation failed");
    } catch (const std::domain_error& e) {
        return fail(AR_ERR_UNSUPPORTED, e.what());
    } catch (const std::runtime_error& e) {   // the builder's own consistency checks
        return fail(AR_ERR_INTERNAL, e.what());
    } catch (const std::exception& e) {
        return fail(AR_ERR_INVALID_ARGUMENT, e.what());
    }
}

ar_status ar_render(ar_scene* s, const ar_camera* cam, const ar_render_params* p, float* out_rgb, double* accum,
                    int32_t mem_kind, void* stream, ar_render_stats* stats)
{
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (!out_rgb && !accum) return fail(AR_ERR_INVALID_ARGUMENT, "out_rgb and accum are both NULL");
    if (mem_kind != AR_MEM_HOST && mem_kind != AR_MEM_DEVICE) return fail(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (ar_status e = run_render(s, cam, p, nullptr, st, stats)) return e;
    if (stats) stats->kernel_launches += (out_rgb ? 1 : 0) + (accum ? 1 : 0);
    const int64_t n = static_cast<int64_t>(cam->width) * cam->height * 3;
    const double inv = 1.0 / static_cast<double>(p->spp);
    if (mem_kind == AR_MEM_DEVICE) {
        if (out_rgb) ck(ar::launch_mean(s->accum, n, inv, out_rgb, st), "mean");
        if (accum) ck(ar::launch_add(s->accum, n, accum, st), "accumulate");
    } else {
        if (out_rgb) {
            ck(ar::launch_mean(s->accum, n, inv, s->fout, st), "mean");
            ck(cudaMemcpyAsync(out_rgb, s->fout, n * sizeof(float), cudaMemcpyDeviceToHost, st), "copy image");
        }
        if (accum) {
            std::vector<double> tmp(static_cast<size_t>(n));
            ck(cudaMemcpyAsync(tmp.data(), s->accum, n * sizeof(double), cudaMemcpyDeviceToHost, st), "copy accum");
            ck(cudaStreamSynchronize(st), "sync");
            for (int64_t i = 0; i < n; ++i) accum[i] += tmp[static_cast<size_t>(i)];
        }
    }
    return check_err(s, st);
    AR_GUARD_END
}

ar_status ar_scene_set_spectral(ar_scene* s, const float* tables, size_t count, int32_t lut_res)
{
    return ar_scene_set_spectral_ex(s, tables, count, lut_res, AR_LUT_SIMT);
}

ar_status ar_scene_set_spectral_ex(ar_scene* s, const float* tables, size_t count, int32_t lut_res, int32_t method)
{
    if (method != AR_LUT_SIMT && method != AR_LUT_TENSOR)
        return fail(AR_ERR_INVALID_ARGUMENT, "method must be AR_LUT_SIMT or AR_LUT_TENSOR");
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (!tables) return fail(AR_ERR_INVALID_ARGUMENT, "tables is NULL");
    if (count != static_cast<size_t>(ar::kTabFloats))
        return fail(AR_ERR_INVALID_ARGUMENT, "tables must hold " + std::to_string(ar::kTabFloats) + " floats");
    if (lut_res < 2 || lut_res > 512) return fail(AR_ERR_INVALID_ARGUMENT, "lut_res must be in [2, 512]");
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    auto drop = [&](void* p) {
        if (!p) return;
        for (auto it = s->owned.begin(); it != s->owned.end(); ++it)
            if (*it == p) { s->owned.erase(it); break; }
        cudaFree(p);
    };
    drop(s->spec_tables); drop(s->spec_lut_lam); drop(s->spec_lut_rgb);
    s->spec_tables = nullptr; s->spec_lut_lam = nullptr; s->spec_lut_rgb = nullptr; s->spec_res = 0;
    const size_t nrgb = static_cast<size_t>(lut_res) * lut_res * lut_res;
    float* tab = dalloc<float>(count, "spectral tables");
    s->owned.push_back(tab);
    float4* lam = dalloc<float4>(ar::kLambdaLutRes, "spectral lambda table");
    s->owned.push_back(lam);
    float4* rgb = dalloc<float4>(nrgb, "spectral rgb table");
    s->owned.push_back(rgb);
    ck(cudaMemcpy(tab, tables, count * sizeof(float), cudaMemcpyHostToDevice), "copy spectral tables");
    ck(ar::launch_spectral_luts(tab, lut_res, lam, rgb, s->sm_count, nullptr), "spectral tables");
    if (method == AR_LUT_TENSOR) {   // the RGB table again, on the tensor cores
        int* err = dalloc<int>(1, "error word");
        ck(cudaMemset(err, 0, sizeof(int)), "memset");
        cudaError_t e = ar::launch_spectral_rgb_lut_tc(tab, lut_res, rgb, err, s->sm_count, nullptr);
        int h = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(err);
        ck(e, "spectral rgb table on the tensor cores");
        if (h) return fail(AR_ERR_DEVICE_FAULT, "tensor-core table build: an MMA did not complete within its wait limit");
    }
    ck(cudaDeviceSynchronize(), "spectral tables");
    s->spec_tables = tab;
    s->spec_lut_lam = lam;
    s->spec_lut_rgb = rgb;
    s->spec_res = lut_res;
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_scene_set_medium(ar_scene* s, const ar_medium_desc* m)
{
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    size_t count = 0;
    if (m) {
        for (int a = 0; a < 3; ++a) {
            if (!(m->bounds_max[a] > m->bounds_min[a]) || !std::isfinite(m->bounds_min[a]) || !std::isfinite(m->bounds_max[a]))
                return fail(AR_ERR_INVALID_ARGUMENT, "medium bounds must be finite with max > min");
            if (m->dims[a] < 1 || m->dims[a] > 4096) return fail(AR_ERR_INVALID_ARGUMENT, "medium dims must be in [1, 4096]");
            if (!(m->albedo[a] >= 0.0f && m->albedo[a] <= 1.0f)) return fail(AR_ERR_INVALID_ARGUMENT, "medium albedo must be in [0, 1]");
        }
        if (!(m->sigma_t_max >= 0.0f) || !std::isfinite(m->sigma_t_max))
            return fail(AR_ERR_INVALID_ARGUMENT, "sigma_t_max must be finite and non-negative");
        if (!(m->g > -1.0f && m->g < 1.0f)) return fail(AR_ERR_INVALID_ARGUMENT, "g must be in (-1, 1)");
        if (m->precision != 16 && m->precision != 32) return fail(AR_ERR_INVALID_ARGUMENT, "precision must be 16 or 32");
        if (!m->density) return fail(AR_ERR_INVALID_ARGUMENT, "density is NULL");
        count = static_cast<size_t>(m->dims[0]) * m->dims[1] * m->dims[2];
        if (count > (size_t(1) << 31)) return fail(AR_ERR_INVALID_ARGUMENT, "medium grid above 2^31 values");
    }
    AR_GUARD_BEGIN
    float dmax = 0.0f;
    for (size_t i = 0; i < count; ++i) {
        const float v = m->precision == 16 ? __half2float(static_cast<const __half*>(m->density)[i])
                                           : static_cast<const float*>(m->density)[i];
        if (!(v >= 0.0f) || !std::isfinite(v)) return fail(AR_ERR_INVALID_ARGUMENT, "density values must be finite and non-negative");
        dmax = std::max(dmax, v);
    }
    DeviceGuard g(s->device);
    if (s->medium_grid) {
        for (auto it = s->owned.begin(); it != s->owned.end(); ++it)
            if (*it == s->medium_grid) { s->owned.erase(it); break; }
        cudaFree(s->medium_grid);
        s->medium_grid = nullptr;
    }
    s->view.has_medium = 0;
    std::memset(&s->view.medium, 0, sizeof(s->view.medium));
    if (!m) return AR_OK;
    const size_t bytes = count * (m->precision == 16 ? 2 : 4);
    unsigned char* grid = dalloc<unsigned char>(bytes, "medium grid");
    s->owned.push_back(grid);
    s->medium_grid = grid;
    ck(cudaMemcpy(grid, m->density, bytes, cudaMemcpyHostToDevice), "copy medium grid");
    ar::MediumRec& r = s->view.medium;
    for (int a = 0; a < 3; ++a) {
        r.bmin[a] = m->bounds_min[a];
        r.bmax[a] = m->bounds_max[a];
        r.albedo[a] = m->albedo[a];
        r.dims[a] = m->dims[a];
    }
    r.sigma_max = m->sigma_t_max;
    r.g = m->g;
    r.majorant = m->sigma_t_max * dmax;
    r.fp16 = m->precision == 16 ? 1 : 0;
    r.data = grid;
    s->view.has_medium = 1;
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_scene_get_spectral_luts(const ar_scene* s, float* lambda_lut, float* rgb_lut)
{
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (!s->spec_tables) return fail(AR_ERR_UNSUPPORTED, "no spectral tables set");
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    if (lambda_lut)
        ck(cudaMemcpy(lambda_lut, s->spec_lut_lam, sizeof(float4) * ar::kLambdaLutRes, cudaMemcpyDeviceToHost),
           "copy lambda table");
    if (rgb_lut)
        ck(cudaMemcpy(rgb_lut, s->spec_lut_rgb, sizeof(float4) * static_cast<size_t>(s->spec_res) * s->spec_res * s->spec_res,
                      cudaMemcpyDeviceToHost), "copy rgb table");
    return AR_OK;
    AR_GUARD_END
}

// ------------------------------------------------------------------ batches
namespace {

// Workspace of one job of a batch (the same layout as a scene's own).
struct JobWs {
    char* mem = nullptr;
    ar::PathBuffers B{};
    uint4* base0 = nullptr;
    uint2* base1 = nullptr;
    double* accum = nullptr;
    ar::PoolCtl* ctl = nullptr;
    unsigned long long* stats = nullptr;
    int* err = nullptr;
    uint32_t* ovf = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    ar::FrameParams fp{};
    int64_t total = 0, pool = 0, npix = 0;
    int cur = 0;
};

void job_alloc(JobWs& w, int64_t pool, int64_t npix, int grid_trace)
{
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t W = static_cast<size_t>(pool), N = static_cast<size_t>(npix);
    const size_t o_p0 = take(sizeof(ar::PathRec) * W), o_p1 = take(sizeof(ar::PathRec) * W);
    const size_t o_hit = take(16 * W), o_qsh = take(4 * W * ar::kShadeBuckets);
    const size_t o_sh = take(sizeof(ar::ShadowRec) * W), o_rt = take(sizeof(ar::RetireRec) * W);
    const size_t o_ax0 = take(16 * W), o_ax1 = take(16 * W), o_sh3 = take(4 * W);
    const size_t o_b0 = take(16 * N), o_b1 = take(8 * N), o_acc = take(24 * N);
    const size_t o_cnt = take(sizeof(ar::PoolCtl)), o_stats = take(64), o_err = take(64);
    const size_t o_ovf = take(static_cast<size_t>(grid_trace) * ar::kTraceBlock * ar::kStackOverflow * 4);
    w.mem = dalloc<char>(off, "batch job workspace");
    char* b = w.mem;
    w.B.pool[0] = reinterpret_cast<ar::PathRec*>(b + o_p0);
    w.B.pool[1] = reinterpret_cast<ar::PathRec*>(b + o_p1);
    w.B.hit = reinterpret_cast<int4*>(b + o_hit);
    w.B.qsh = reinterpret_cast<int32_t*>(b + o_qsh);
    w.B.shadow = reinterpret_cast<ar::ShadowRec*>(b + o_sh);
    w.B.retire = reinterpret_cast<ar::RetireRec*>(b + o_rt);
    w.B.aux[0] = reinterpret_cast<float4*>(b + o_ax0);
    w.B.aux[1] = reinterpret_cast<float4*>(b + o_ax1);
    w.B.shadow3 = reinterpret_cast<float*>(b + o_sh3);
    w.B.capacity = static_cast<int32_t>(pool);
    w.base0 = reinterpret_cast<uint4*>(b + o_b0);
    w.base1 = reinterpret_cast<uint2*>(b + o_b1);
    w.accum = reinterpret_cast<double*>(b + o_acc);
    w.ctl = reinterpret_cast<ar::PoolCtl*>(b + o_cnt);
    w.stats = reinterpret_cast<unsigned long long*>(b + o_stats);
    w.err = reinterpret_cast<int*>(b + o_err);
    w.ovf = reinterpret_cast<uint32_t*>(b + o_ovf);
}

// Device-side end test of the batch loop: after each pass of the loop body
// every job's retired-path count is compared with its total; the conditional
// handle keeps the WHILE node looping while a job has paths left and the pass
// count is below its bound (then the error word gets bit 0 and the loop ends).
struct BatchDrain {
    const ar::PoolCtl* const* ctl;  // per job
    const int64_t* total;           // per job
    int32_t jobs;
    int32_t max_passes;
    int32_t* passes;                // [0] passes run, [1] error word
};

__global__ void k_batch_drain(BatchDrain d, cudaGraphConditionalHandle h)
{
    __shared__ int open;
    if (threadIdx.x == 0) open = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < d.jobs; j += blockDim.x)
        if (d.ctl[j]->retired < d.total[j]) atomicOr(&open, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int n = d.passes[0] + 1;
        d.passes[0] = n;
        const bool again = open != 0 && n < d.max_passes;
        if (open != 0 && !again) d.passes[1] |= 1;
        cudaGraphSetConditional(h, again ? 1u : 0u);
    }
}

struct BatchResources {
    std::vector<JobWs> jobs;
    void* drain_mem = nullptr;      // BatchDrain tables and counters
    cudaEvent_t fork = nullptr;
    cudaStream_t orch = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~BatchResources()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (fork) cudaEventDestroy(fork);
        if (drain_mem) cudaFree(drain_mem);
        if (orch) cudaStreamDestroy(orch);
        for (JobWs& w : jobs) {
            if (w.done) cudaEventDestroy(w.done);
            if (w.st) cudaStreamDestroy(w.st);
            if (w.mem) cudaFree(w.mem);
        }
    }
};

}  // namespace

}  // extern "C"

namespace {
// Batch shape of the autotuner's memory: job count, pixels, samples, spectral jobs.
struct BatchKey {
    int32_t jobs;
    int32_t spectral;
    int64_t pixels, samples;
    bool operator<(const BatchKey& o) const
    {
        return std::tie(jobs, spectral, pixels, samples) < std::tie(o.jobs, o.spectral, o.pixels, o.samples);
    }
};
BatchKey batch_key(const ar_job* jobs, int32_t njobs)
{
    BatchKey k{njobs, 0, 0, 0};
    for (int j = 0; j < njobs; ++j) {
        const int64_t px = static_cast<int64_t>(jobs[j].camera.width) * jobs[j].camera.height;
        k.pixels += px;
        k.samples += px * jobs[j].params.spp;
        k.spectral += jobs[j].params.spectral ? 1 : 0;
    }
    return k;
}
// Launch knobs of a batch: graph length, in-flight path budget, resident
// blocks per SM of each job's traversal kernels and of its shading, path
// generation and retirement kernels (0: the defaults -- the traversal
// kernels' occupancy and 4).  Jobs run as parallel graph branches, so smaller
// grids let kernels of several jobs share the GPU.
struct BatchKnobs {
    int32_t iterations = 0;
    int64_t budget = 0;
    int32_t trace_bps = 0;
    int32_t shade_bps = 0;
};
std::mutex g_tune_mutex;
std::map<BatchKey, BatchKnobs> g_tuned;

ar_status render_batch(const ar_job* jobs, int32_t njobs, BatchKnobs kn, ar_batch_stats* stats, void* stream);
}  // namespace

extern "C" {

ar_status ar_render_batch(const ar_job* jobs, int32_t njobs, int32_t iterations_per_graph, int64_t path_budget,
                          ar_batch_stats* stats, void* stream)
{
    g_last_error.clear();
    if (njobs <= 0 || !jobs) return fail(AR_ERR_INVALID_ARGUMENT, "jobs is NULL or empty");
    BatchKnobs kn;
    kn.iterations = iterations_per_graph;
    kn.budget = path_budget;
    if (iterations_per_graph == 0 && path_budget == 0) {   // autotuned knobs for this batch shape
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(batch_key(jobs, njobs));
        if (it != g_tuned.end()) kn = it->second;
    }
    return render_batch(jobs, njobs, kn, stats, stream);
}

}  // extern "C"

namespace {
ar_status render_batch(const ar_job* jobs, int32_t njobs, BatchKnobs kn, ar_batch_stats* stats, void* stream)
{
    const int32_t iterations_per_graph = kn.iterations;
    const int64_t path_budget = kn.budget;
    if (njobs <= 0 || !jobs) return fail(AR_ERR_INVALID_ARGUMENT, "jobs is NULL or empty");
    if (iterations_per_graph < 0 || iterations_per_graph > 256)
        return fail(AR_ERR_INVALID_ARGUMENT, "iterations_per_graph must be in [0, 256]");
    const ar_scene* s0 = jobs[0].scene;
    for (int j = 0; j < njobs; ++j) {
        const ar_job& jb = jobs[j];
        if (!jb.scene) return fail(AR_ERR_INVALID_ARGUMENT, "job " + std::to_string(j) + ": scene is NULL");
        if (jb.scene->device != s0->device) return fail(AR_ERR_INVALID_ARGUMENT, "jobs span several devices");
        if (ar_status e = check_camera(&jb.camera)) return e;
        if (ar_status e = check_params(&jb.params)) return e;
        if (!jb.out_rgb && !jb.accum) return fail(AR_ERR_INVALID_ARGUMENT, "job " + std::to_string(j) + ": no output");
        if (jb.params.spectral && !jb.scene->spec_tables)
            return fail(AR_ERR_UNSUPPORTED, "job " + std::to_string(j) + ": spectral tables not set");
    }
    if (kn.trace_bps < 0 || kn.trace_bps > 64 || kn.shade_bps < 0 || kn.shade_bps > 64)
        return fail(AR_ERR_INVALID_ARGUMENT, "blocks per SM must be in [0, 64]");
    AR_GUARD_BEGIN
    DeviceGuard g(s0->device);
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    int K = iterations_per_graph > 0 ? iterations_per_graph : 16;
    K += K & 1;  // even: both pool buffers back in place after a replay
    // In-flight paths: a shared budget split by each job's share of the work
    // (a job never gets more than it has paths, nor fewer than 2^14).
    int64_t totalAll = 0;
    for (int j = 0; j < njobs; ++j)
        totalAll += static_cast<int64_t>(jobs[j].camera.width) * jobs[j].camera.height * jobs[j].params.spp;
    const int64_t budget = path_budget > 0 ? path_budget : (int64_t(1) << 22);
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    ck(cudaEventCreate(&t0), "event");
    ck(cudaEventCreate(&t1), "event");
    struct Ev { cudaEvent_t a, b; ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); } } evs{t0, t1};
    BatchResources R;
    R.jobs.resize(static_cast<size_t>(njobs));
    ck(cudaEventCreateWithFlags(&R.fork, cudaEventDisableTiming), "event");
    // the batch runs on a stream of its own (the legacy default stream cannot
    // be captured), ordered after the caller's stream
    ck(cudaStreamCreateWithFlags(&R.orch, cudaStreamNonBlocking), "stream");
    cudaStream_t st = R.orch;
    ck(cudaEventRecord(R.fork, user), "event record");
    ck(cudaStreamWaitEvent(st, R.fork, 0), "order after caller");
    ck(cudaEventRecord(t0, st), "event record");
    ck(cudaEventRecord(R.fork, st), "event record");
    for (int j = 0; j < njobs; ++j) {
        JobWs& w = R.jobs[j];
        const ar_job& jb = jobs[j];
        w.npix = static_cast<int64_t>(jb.camera.width) * jb.camera.height;
        w.total = w.npix * jb.params.spp;
        int64_t pool = static_cast<int64_t>(static_cast<double>(budget) * static_cast<double>(w.total) /
                                            static_cast<double>(totalAll));
        if (jb.params.wave_paths > 0) pool = jb.params.wave_paths;
        pool = std::max<int64_t>(std::min<int64_t>(pool, kMaxPool), int64_t(1) << 14);
        w.pool = std::max<int64_t>(1, std::min<int64_t>(pool, w.total));
        w.fp = make_frame(jb.scene, &jb.camera, &jb.params);
        w.fp.pool = static_cast<int32_t>(w.pool);
        job_alloc(w, w.pool, w.npix, jb.scene->grid_trace);
        ck(cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming), "event");
        ck(cudaStreamWaitEvent(w.st, R.fork, 0), "fork");
        ck(cudaMemsetAsync(w.accum, 0, sizeof(double) * 3 * w.npix, w.st), "memset");
        ck(cudaMemsetAsync(w.stats, 0, 64, w.st), "memset");
        ck(cudaMemsetAsync(w.err, 0, 64, w.st), "memset");
        ck(ar::launch_rng_init(w.fp, w.base0, w.base1, jb.scene->jump_table67, w.st), "rng init");
        ck(ar::launch_pool_init(w.ctl, w.total, w.st), "pool init");
        ck(cudaEventRecord(w.done, w.st), "event record");
        ck(cudaStreamWaitEvent(st, w.done, 0), "join");
    }
    int64_t maxDepth = 0, maxRatio = 0;
    for (int j = 0; j < njobs; ++j) {
        maxDepth = std::max<int64_t>(maxDepth, jobs[j].params.max_depth);
        const int64_t admit = std::max<int64_t>(1, std::min<int64_t>(R.jobs[j].pool, R.jobs[j].npix));
        maxRatio = std::max<int64_t>(maxRatio, R.jobs[j].total / admit + 2);
    }
    const int64_t maxPasses = (maxRatio * (maxDepth + 2)) / K + 2;
    // The drain test's tables: per job its pool control block and path total.
    {
        const size_t nj = static_cast<size_t>(njobs);
        R.drain_mem = dalloc<unsigned char>(nj * 16 + 64, "batch drain tables");
        std::vector<const ar::PoolCtl*> ctls(nj);
        std::vector<int64_t> totals(nj);
        for (size_t j = 0; j < nj; ++j) {
            ctls[j] = R.jobs[j].ctl;
            totals[j] = R.jobs[j].total;
        }
        unsigned char* m = static_cast<unsigned char*>(R.drain_mem);
        ck(cudaMemcpyAsync(m, ctls.data(), nj * 8, cudaMemcpyHostToDevice, st), "drain tables");
        ck(cudaMemcpyAsync(m + nj * 8, totals.data(), nj * 8, cudaMemcpyHostToDevice, st), "drain tables");
        ck(cudaMemsetAsync(m + nj * 16, 0, 64, st), "drain counters");
    }
    BatchDrain dr;
    dr.ctl = reinterpret_cast<const ar::PoolCtl* const*>(R.drain_mem);
    dr.total = reinterpret_cast<const int64_t*>(static_cast<unsigned char*>(R.drain_mem) + njobs * 8);
    dr.jobs = njobs;
    dr.max_passes = static_cast<int32_t>(std::min<int64_t>(maxPasses, INT32_MAX));
    dr.passes = reinterpret_cast<int32_t*>(static_cast<unsigned char*>(R.drain_mem) + njobs * 16);
    // One graph, launched once: a WHILE conditional node whose body runs K
    // wavefront iterations of every job (each job on its own branch) and then
    // the drain test, which sets the node's condition on the device -- no host
    // round trip between passes.
    ck(cudaGraphCreate(&R.graph, 0), "graph create");
    cudaGraphConditionalHandle cond;
    ck(cudaGraphConditionalHandleCreate(&cond, R.graph, 1, cudaGraphCondAssignDefault), "conditional handle");
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop;
    ck(cudaGraphAddNode(&loop, R.graph, nullptr, 0, &cp), "conditional node");
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    ck(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
       "begin capture");
    ck(cudaEventRecord(R.fork, st), "fork");
    int64_t launches = 0;
    for (int j = 0; j < njobs; ++j) {
        JobWs& w = R.jobs[j];
        const ar_job& jb = jobs[j];
        ck(cudaStreamWaitEvent(w.st, R.fork, 0), "fork");
        // persistent traversal kernels fetch work dynamically: any grid up to
        // the one the overflow slabs were sized for is complete
        const int gt = kn.trace_bps > 0 ? std::min(jb.scene->grid_trace, jb.scene->sm_count * kn.trace_bps)
                                        : jb.scene->grid_trace;
        const int go = jb.scene->sm_count * (kn.shade_bps > 0 ? kn.shade_bps : 4);
        ck(ar::launch_iterations(jb.scene->view, w.fp, w.B, w.ctl, w.base0, w.base1, jb.scene->jump_table, w.stats,
                                 w.ovf, w.err, w.accum, nullptr, K, &w.cur, gt, go, w.st, &launches, nullptr),
           "capture iterations");
        ck(cudaEventRecord(w.done, w.st), "join");
        ck(cudaStreamWaitEvent(st, w.done, 0), "join");
    }
    k_batch_drain<<<1, 256, 0, st>>>(dr, cond);
    ck(cudaGetLastError(), "drain test");
    cudaGraph_t captured = nullptr;
    ck(cudaStreamEndCapture(st, &captured), "end capture");
    ck(cudaGraphInstantiate(&R.exec, R.graph, 0), "graph instantiate");
    size_t nodes = 0;
    cudaGraphGetNodes(body, nullptr, &nodes);
    ck(cudaGraphLaunch(R.exec, st), "graph launch");
    int32_t dres[2] = {0, 0};
    ck(cudaMemcpyAsync(dres, dr.passes, sizeof(dres), cudaMemcpyDeviceToHost, st), "pass count");
    ck(cudaStreamSynchronize(st), "sync");
    if (dres[1] != 0) return fail(AR_ERR_DEVICE_FAULT, "batch path pools did not drain");
    const int64_t replays = dres[0];
    // outputs, counters, error words
    unsigned long long ext = 0, sh = 0;
    for (int j = 0; j < njobs; ++j) {
        JobWs& w = R.jobs[j];
        const ar_job& jb = jobs[j];
        const int64_t n = w.npix * 3;
        if (jb.out_rgb) ck(ar::launch_mean(w.accum, n, 1.0 / static_cast<double>(jb.params.spp), jb.out_rgb, st), "mean");
        if (jb.accum) ck(ar::launch_add(w.accum, n, jb.accum, st), "accumulate");
        unsigned long long h[2];
        int e = 0;
        ck(cudaMemcpyAsync(h, w.stats, sizeof(h), cudaMemcpyDeviceToHost, st), "stats");
        ck(cudaMemcpyAsync(&e, w.err, sizeof(int), cudaMemcpyDeviceToHost, st), "error word");
        ck(cudaStreamSynchronize(st), "sync");
        if (e != 0) return fail(AR_ERR_DEVICE_FAULT, "job " + std::to_string(j) + ": traversal stack overflow");
        ext += h[0];
        sh += h[1];
    }
    ck(cudaEventRecord(t1, st), "event record");
    ck(cudaEventSynchronize(t1), "sync");
    ck(cudaStreamWaitEvent(user, t1, 0), "order caller after batch");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        stats->total_ms = ms;
        stats->paths = totalAll;
        stats->extension_rays = static_cast<int64_t>(ext);
        stats->shadow_rays = static_cast<int64_t>(sh);
        stats->graph_launches = 1;
        stats->loop_passes = replays;
        stats->graph_nodes = static_cast<int64_t>(nodes);
        stats->kernel_launches = launches * replays;
        stats->iterations_per_graph = K;
    }
    return AR_OK;
    AR_GUARD_END
}
}  // namespace

extern "C" {

ar_status ar_accum_resolve(const double* accum, size_t n, double scale, float* out, int32_t mem_kind, void* stream)
{
    g_last_error.clear();
    if (n == 0) return AR_OK;
    if (!accum || !out) return fail(AR_ERR_INVALID_ARGUMENT, "accum/out is NULL");
    if (mem_kind == AR_MEM_HOST) {
        for (size_t i = 0; i < n; ++i) out[i] = static_cast<float>(accum[i] * scale);
        return AR_OK;
    }
    if (mem_kind != AR_MEM_DEVICE) return fail(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    AR_GUARD_BEGIN
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    ck(ar::launch_mean(accum, static_cast<int64_t>(n), scale, out, static_cast<cudaStream_t>(stream)), "resolve");
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_trace_rays(ar_scene* s, const float* rays, size_t n, int32_t any_hit, int32_t* hit_object, float* hit_t,
                        int32_t mem_kind, void* stream)
{
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (n == 0) return AR_OK;
    if (!rays || !hit_object) return fail(AR_ERR_INVALID_ARGUMENT, "rays/hit_object is NULL");
    if (mem_kind != AR_MEM_HOST && mem_kind != AR_MEM_DEVICE) return fail(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    if (mem_kind == AR_MEM_DEVICE && (reinterpret_cast<uintptr_t>(rays) & 15u))
        return fail(AR_ERR_INVALID_ARGUMENT, "device ray buffer must be 16-byte aligned");
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!s->err) ensure_workspace(s, 1, 1);
    ck(cudaMemsetAsync(s->err, 0, 64, st), "memset err");
    const float4* drays;
    int32_t* dobj;
    float* dt;
    std::vector<void*> tmp;
    if (mem_kind == AR_MEM_HOST) {
        float4* rr = dalloc<float4>(2 * n, "rays");
        tmp.push_back(rr);
        ck(cudaMemcpyAsync(rr, rays, n * 32, cudaMemcpyHostToDevice, st), "copy rays");
        drays = rr;
        dobj = dalloc<int32_t>(n, "hits"); tmp.push_back(dobj);
        dt = hit_t ? dalloc<float>(n, "t") : nullptr;
        if (dt) tmp.push_back(dt);
    } else {
        drays = reinterpret_cast<const float4*>(rays);
        dobj = hit_object;
        dt = hit_t;
    }
    cudaError_t e = cudaSuccess;
    const size_t chunk = size_t(1) << 30;
    for (size_t first = 0; first < n && e == cudaSuccess; first += chunk) {
        const int cnt = static_cast<int>(std::min(chunk, n - first));
        e = cudaMemsetAsync(&s->ctl->fetch_rays, 0, sizeof(int32_t), st);
        if (e == cudaSuccess)
            e = ar::launch_trace_rays(s->view, drays + 2 * first, cnt, any_hit ? 1 : 0, dobj + first,
                                      dt ? dt + first : nullptr, s->ctl, s->ovf, s->err, s->grid_trace, st);
    }
    if (e == cudaSuccess && mem_kind == AR_MEM_HOST) {
        e = cudaMemcpyAsync(hit_object, dobj, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && hit_t) e = cudaMemcpyAsync(hit_t, dt, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    for (void* p : tmp) cudaFree(p);
    ck(e, "trace rays");
    return check_err(s, st);
    AR_GUARD_END
}

ar_status ar_render_debug_paths(ar_scene* s, const ar_camera* cam, const ar_render_params* p, ar_path_record* records,
                                int32_t mem_kind, void* stream)
{
    g_last_error.clear();
    if (!s || !records) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (mem_kind != AR_MEM_HOST && mem_kind != AR_MEM_DEVICE) return fail(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t nrec = static_cast<size_t>(cam->width) * cam->height * p->spp;
    ar_path_record* drec = records;
    if (mem_kind == AR_MEM_HOST) drec = dalloc<ar_path_record>(nrec, "path records");
    cudaError_t e = cudaMemsetAsync(drec, 0, nrec * sizeof(ar_path_record), st);
    ar_status rs = AR_OK;
    if (e == cudaSuccess) {
        try { rs = run_render(s, cam, p, drec, st, nullptr); } catch (...) { if (mem_kind == AR_MEM_HOST) cudaFree(drec); throw; }
    }
    if (e == cudaSuccess && rs == AR_OK && mem_kind == AR_MEM_HOST) {
        e = cudaMemcpyAsync(records, drec, nrec * sizeof(ar_path_record), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (mem_kind == AR_MEM_HOST) cudaFree(drec);
    ck(e, "debug render");
    if (rs != AR_OK) return rs;
    return check_err(s, st);
    AR_GUARD_END
}

ar_status ar_rng_tape(const ar_camera* cam, const ar_render_params* p, int32_t per_path, float* out, int32_t mem_kind,
                      void* stream)
{
    g_last_error.clear();
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (per_path <= 0 || !out) return fail(AR_ERR_INVALID_ARGUMENT, "per_path must be positive and out non-NULL");
    if (mem_kind != AR_MEM_HOST && mem_kind != AR_MEM_DEVICE) return fail(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    AR_GUARD_BEGIN
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ar::FrameParams fp;
    std::memset(&fp, 0, sizeof(fp));
    fp.width = cam->width;
    fp.height = cam->height;
    fp.grid_x = (cam->width + 7) / 8;
    fp.npix = cam->width * cam->height;
    fp.seed = p->seed;
    fp.frame0 = static_cast<uint64_t>(p->frame_offset);
    const size_t n = static_cast<size_t>(fp.npix) * p->spp * per_path;
    float* dout = out;
    if (mem_kind == AR_MEM_HOST) dout = dalloc<float>(n, "tape");
    cudaError_t e = ar::launch_rng_tape(fp, p->spp, per_path, dout, st);
    if (e == cudaSuccess && mem_kind == AR_MEM_HOST) {
        e = cudaMemcpyAsync(out, dout, n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (mem_kind == AR_MEM_HOST) cudaFree(dout);
    ck(e, "rng tape");
    return AR_OK;
    AR_GUARD_END
}

}  // extern "C"

// ------------------------------------------------------------------ learned radiance cache
struct ar_nrc {
    ar_scene* scene = nullptr;
    ar_nrc_config cfg{};
    ar::NrcGrid grid{};
    ar::NrcParams P{};
    ar::NrcTrainBuffers T{};
    int step = 0;
    ar::NrcQuery* queries = nullptr;
    int64_t query_cap = 0;
    ar::NrcTrainVertex* tverts = nullptr;
    ar::NrcSample* samples = nullptr;
    int32_t* counters = nullptr;   // [0] queries, [1] samples, [2..] slot vertex counts
    int slots = 0, sample_cap = 0;
    int* tc_err = nullptr;         // error word of the tcgen05 inference kernel
    int tensor_path = 1;           // inference: 1 tcgen05 (default), 0 mma.sync
    int spectral = 0;              // 0 RGB cache, 4 four-wavelength cache (16 spectral bins)
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<void*> owned;

    ar::NrcNet net() const
    {
        ar::NrcNet n;
        n.grid = grid;
        n.table = P.table_h;
        n.w = P.w_bf;
        n.wt = P.wt_bf;
        n.spectral = spectral;
        n.tables = scene->spec_tables;
        return n;
    }
    ~ar_nrc()
    {
        QuietDeviceGuard g(scene->device);
        for (void* p : owned) cudaFree(p);
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace {

template <class T>
T* nrc_alloc(ar_nrc* c, size_t count, const char* what)
{
    T* p = dalloc<T>(count, what);
    c->owned.push_back(p);
    return p;
}

void nrc_ensure_queries(ar_nrc* c, int64_t n)
{
    if (n <= c->query_cap) return;
    for (auto it = c->owned.begin(); it != c->owned.end(); ++it)
        if (*it == c->queries) { c->owned.erase(it); break; }
    if (c->queries) cudaFree(c->queries);
    c->queries = nrc_alloc<ar::NrcQuery>(c, static_cast<size_t>(n), "cache queries");
    c->query_cap = n;
}

cudaError_t nrc_run_infer(ar_nrc* c, const ar::NrcQuery* q, const int32_t* count, int cap, double* accum,
                          float* out_rgb, cudaStream_t st)
{
    if (c->tensor_path == 1)
        return ar::nrc_infer_tc(c->net(), q, count, cap, accum, out_rgb, c->tc_err, c->scene->sm_count, st);
    return ar::nrc_infer(c->net(), q, count, cap, accum, out_rgb, c->scene->sm_count, st);
}

ar_status nrc_check(ar_nrc* c, cudaStream_t st)
{
    int e = 0;
    ck(cudaMemcpyAsync(&e, c->tc_err, sizeof(int), cudaMemcpyDeviceToHost, st), "copy error word");
    ck(cudaStreamSynchronize(st), "sync");
    if (e != 0) {
        ck(cudaMemsetAsync(c->tc_err, 0, sizeof(int), st), "memset");
        return fail(AR_ERR_DEVICE_FAULT, "cache tensor-core kernels: an MMA did not complete within its wait limit");
    }
    return AR_OK;
}

ar_status nrc_train_steps(ar_nrc* c, const ar::NrcSample* samples, const int32_t* count, int steps, cudaStream_t st)
{
    for (int k = 0; k < steps; ++k)
        ck(ar::nrc_train_step(c->net(), c->P, samples, count, k * c->cfg.train_batch, c->cfg.train_batch, c->T,
                              c->cfg.learning_rate, ++c->step, c->scene->sm_count, st, true,
                              c->tensor_path ? c->tc_err : nullptr), "cache training");
    return AR_OK;
}

}  // namespace

extern "C" {

ar_status ar_nrc_create(ar_scene* s, const ar_nrc_config* cfg, ar_nrc** out)
{
    g_last_error.clear();
    if (!s || !cfg || !out) return fail(AR_ERR_INVALID_ARGUMENT, "scene, config or out is NULL");
    *out = nullptr;
    if (cfg->levels < 1 || cfg->levels > ar::kNrcMaxLevels) return fail(AR_ERR_INVALID_ARGUMENT, "levels must be in [1, 16]");
    if (cfg->log2_entries < 8 || cfg->log2_entries > 24) return fail(AR_ERR_INVALID_ARGUMENT, "log2_entries must be in [8, 24]");
    if (cfg->base_resolution < 2 || cfg->max_resolution < cfg->base_resolution || cfg->max_resolution > (1 << 16))
        return fail(AR_ERR_INVALID_ARGUMENT, "need 2 <= base_resolution <= max_resolution <= 65536");
    if (cfg->train_paths < 1 || cfg->train_batch < 32 || cfg->train_steps < 0 || cfg->max_train_vertices < 1 ||
        cfg->max_train_vertices > 64)
        return fail(AR_ERR_INVALID_ARGUMENT, "bad training sizes");
    if (!(cfg->learning_rate > 0.0f) || !(cfg->spread_c > 0.0f)) return fail(AR_ERR_INVALID_ARGUMENT, "learning_rate and spread_c must be positive");
    float bmin[3], bmax[3];
    bool given = true;
    for (int a = 0; a < 3; ++a) given = given && cfg->bounds_max[a] > cfg->bounds_min[a];
    for (int a = 0; a < 3; ++a) {
        bmin[a] = given ? cfg->bounds_min[a] : s->bounds[a];
        bmax[a] = given ? cfg->bounds_max[a] : s->bounds[3 + a];
        if (!(bmax[a] > bmin[a])) return fail(AR_ERR_INVALID_ARGUMENT, "scene has no extent: give bounds");
    }
    AR_GUARD_BEGIN
    DeviceGuard g(s->device);
    std::unique_ptr<ar_nrc> c(new ar_nrc());
    c->scene = s;
    c->cfg = *cfg;
    ar::NrcGrid& gr = c->grid;
    gr.levels = cfg->levels;
    const uint32_t entries = 1u << cfg->log2_entries;
    gr.mask = entries - 1u;
    const double b = cfg->levels > 1 ? std::exp((std::log(static_cast<double>(cfg->max_resolution)) -
                                                 std::log(static_cast<double>(cfg->base_resolution))) / (cfg->levels - 1))
                                     : 1.0;
    for (int l = 0; l < ar::kNrcMaxLevels; ++l) {
        const int r = l < cfg->levels ? static_cast<int>(std::floor(cfg->base_resolution * std::pow(b, l) + 1e-6)) : 1;
        gr.res[l] = r;
        const double cells = std::pow(static_cast<double>(r + 1), 3.0);
        gr.dense[l] = cells <= static_cast<double>(entries) ? 1 : 0;
    }
    for (int a = 0; a < 3; ++a) {
        gr.bmin[a] = bmin[a];
        gr.inv_ext[a] = 1.0f / (bmax[a] - bmin[a]);
    }
    ar::NrcParams& P = c->P;
    P.table_floats = static_cast<int64_t>(cfg->levels) * entries * 2;
    const size_t tf = static_cast<size_t>(P.table_floats);
    P.table_f32 = nrc_alloc<float>(c.get(), tf, "cache table");
    P.table_m = nrc_alloc<float>(c.get(), tf, "cache table moments");
    P.table_v = nrc_alloc<float>(c.get(), tf, "cache table moments");
    P.table_g = nrc_alloc<float>(c.get(), tf, "cache table gradients");
    P.table_h = nrc_alloc<__half2>(c.get(), tf / 2, "cache table half");
    P.w_f32 = nrc_alloc<float>(c.get(), ar::kNrcParams, "cache weights");
    P.w_m = nrc_alloc<float>(c.get(), ar::kNrcParams, "cache weights");
    P.w_v = nrc_alloc<float>(c.get(), ar::kNrcParams, "cache weights");
    P.w_g = nrc_alloc<float>(c.get(), ar::kNrcParams, "cache weights");
    P.w_bf = nrc_alloc<__nv_bfloat16>(c.get(), ar::kNrcParams, "cache weights bf16");
    P.wt_bf = nrc_alloc<__nv_bfloat16>(c.get(), ar::kNrcParams, "cache weights bf16");
    ck(cudaMemset(P.table_m, 0, tf * 4), "memset");
    ck(cudaMemset(P.table_v, 0, tf * 4), "memset");
    ck(cudaMemset(P.table_g, 0, tf * 4), "memset");
    ck(cudaMemset(P.w_m, 0, ar::kNrcParams * 4), "memset");
    ck(cudaMemset(P.w_v, 0, ar::kNrcParams * 4), "memset");
    ck(cudaMemset(P.w_g, 0, ar::kNrcParams * 4), "memset");
    const size_t B = static_cast<size_t>(cfg->train_batch);
    ar::NrcTrainBuffers& T = c->T;
    T.acts = nrc_alloc<__nv_bfloat16>(c.get(), B * ar::kNrcIn * ar::kNrcLayers, "cache activations");
    T.dz = nrc_alloc<__nv_bfloat16>(c.get(), B * ar::kNrcIn * ar::kNrcLayers, "cache gradients");
    T.raw = nrc_alloc<float>(c.get(), B * 16, "cache outputs");
    T.dx = nrc_alloc<float>(c.get(), B * 32, "cache input gradients");
    T.loss = nrc_alloc<float>(c.get(), 1, "cache loss");
    c->slots = cfg->train_paths + 1;
    c->sample_cap = std::max(cfg->train_paths * cfg->max_train_vertices, cfg->train_batch * std::max(cfg->train_steps, 1));
    c->tverts = nrc_alloc<ar::NrcTrainVertex>(c.get(), static_cast<size_t>(c->slots) * cfg->max_train_vertices, "cache training vertices");
    c->samples = nrc_alloc<ar::NrcSample>(c.get(), static_cast<size_t>(c->sample_cap), "cache samples");
    c->counters = nrc_alloc<int32_t>(c.get(), static_cast<size_t>(c->slots) + 2, "cache counters");
    c->tc_err = nrc_alloc<int>(c.get(), 1, "cache error word");
    ck(cudaMemset(c->tc_err, 0, sizeof(int)), "memset");
    ck(ar::nrc_init_params(P, cfg->seed, nullptr), "cache init");
    for (cudaEvent_t& e : c->ev) ck(cudaEventCreate(&e), "event");
    ck(cudaDeviceSynchronize(), "cache init");
    *out = c.release();
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_nrc_destroy(ar_nrc* c)
{
    g_last_error.clear();
    delete c;
    return AR_OK;
}

ar_status ar_nrc_render_frame(ar_nrc* c, const ar_camera* cam, const ar_render_params* p, float* out_rgb,
                              double* accum, int32_t train, ar_nrc_frame_stats* stats, void* stream)
{
    g_last_error.clear();
    if (!c) return fail(AR_ERR_INVALID_ARGUMENT, "cache is NULL");
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (p->spp > 64) return fail(AR_ERR_INVALID_ARGUMENT, "cache frames take 1 to 64 samples per pixel");
    if (p->spectral != c->spectral)
        return fail(p->spectral == 1 ? AR_ERR_UNSUPPORTED : AR_ERR_INVALID_ARGUMENT,
                    "params->spectral must match the cache's mode (AR_NRC_OPT_SPECTRAL: 0 RGB, 4 four wavelengths; "
                    "one wavelength per path has no cache)");
    if (c->spectral && !c->scene->spec_tables) return fail(AR_ERR_UNSUPPORTED, "no spectral tables set");
    if (!out_rgb && !accum) return fail(AR_ERR_INVALID_ARGUMENT, "out_rgb and accum are both NULL");
    AR_GUARD_BEGIN
    ar_scene* s = c->scene;
    DeviceGuard g(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t npix = static_cast<int64_t>(cam->width) * cam->height;
    nrc_ensure_queries(c, npix * p->spp);   // at most one cache query per path
    ck(cudaMemsetAsync(c->counters, 0, sizeof(int32_t) * (static_cast<size_t>(c->slots) + 2), st), "memset");
    if (stats) ck(cudaMemsetAsync(c->T.loss, 0, sizeof(float), st), "memset");
    ar::NrcFrame f{};
    f.enabled = 1;
    f.spectral = c->spectral;
    f.stride = static_cast<int32_t>(std::max<int64_t>(1, (npix + c->cfg.train_paths - 1) / c->cfg.train_paths));
    f.offset = static_cast<int32_t>(ar::lowbias32(static_cast<uint32_t>(p->frame_offset) * 0x9E3779B9u ^
                                                  static_cast<uint32_t>(p->seed)) % static_cast<uint32_t>(f.stride));
    f.max_train_vertices = c->cfg.max_train_vertices;
    f.spread_c = c->cfg.spread_c;
    f.query_cap = static_cast<int32_t>(c->query_cap);
    f.sample_cap = c->sample_cap;
    f.slots = c->slots;
    f.queries = c->queries;
    f.query_count = c->counters;
    f.train_vertices = c->tverts;
    f.slot_count = c->counters + 2;
    f.samples = c->samples;
    f.sample_count = c->counters + 1;
    ar_render_stats rs;
    ck(cudaEventRecord(c->ev[0], st), "event");
    if (ar_status e = run_render(s, cam, p, nullptr, st, stats ? &rs : nullptr, &f)) return e;
    ck(cudaEventRecord(c->ev[1], st), "event");
    ck(nrc_run_infer(c, c->queries, c->counters, static_cast<int>(c->query_cap), s->accum, nullptr, st),
       "cache inference");
    ck(cudaEventRecord(c->ev[2], st), "event");
    if (train) nrc_train_steps(c, c->samples, c->counters + 1, c->cfg.train_steps, st);
    ck(cudaEventRecord(c->ev[3], st), "event");
    const int64_t n = npix * 3;
    if (out_rgb) ck(ar::launch_mean(s->accum, n, 1.0 / static_cast<double>(p->spp), out_rgb, st), "mean");
    if (accum) ck(ar::launch_add(s->accum, n, accum, st), "accumulate");
    if (stats) {
        int32_t cnt[2];
        float loss = 0.0f;
        ck(cudaMemcpyAsync(cnt, c->counters, sizeof(cnt), cudaMemcpyDeviceToHost, st), "copy counters");
        ck(cudaMemcpyAsync(&loss, c->T.loss, sizeof(float), cudaMemcpyDeviceToHost, st), "copy loss");
        ck(cudaStreamSynchronize(st), "sync");
        std::memset(stats, 0, sizeof(*stats));
        cudaEventElapsedTime(&stats->total_ms, c->ev[0], c->ev[3]);
        cudaEventElapsedTime(&stats->render_ms, c->ev[0], c->ev[1]);
        cudaEventElapsedTime(&stats->infer_ms, c->ev[1], c->ev[2]);
        cudaEventElapsedTime(&stats->train_ms, c->ev[2], c->ev[3]);
        stats->queries = cnt[0];
        stats->train_samples = cnt[1];
        stats->extension_rays = rs.extension_rays;
        stats->shadow_rays = rs.shadow_rays;
        stats->loss = train && c->cfg.train_steps > 0 ? loss / static_cast<float>(c->cfg.train_steps) : 0.0f;
    }
    if (ar_status e = nrc_check(c, st)) return e;
    return check_err(s, st);
    AR_GUARD_END
}

ar_status ar_nrc_set_option(ar_nrc* c, int32_t option, int32_t value)
{
    g_last_error.clear();
    if (!c) return fail(AR_ERR_INVALID_ARGUMENT, "cache is NULL");
    if (option == AR_NRC_OPT_TENSOR_PATH && (value == 0 || value == 1)) {
        c->tensor_path = value;
        return AR_OK;
    }
    if (option == AR_NRC_OPT_SPECTRAL && (value == 0 || value == 4)) {
        if (value == 4 && !c->scene->spec_tables) return fail(AR_ERR_UNSUPPORTED, "no spectral tables set");
        c->spectral = value;
        return AR_OK;
    }
    return fail(AR_ERR_INVALID_ARGUMENT, "unknown option or value");
}

ar_status ar_nrc_get_params(const ar_nrc* c, float* table, float* weights)
{
    g_last_error.clear();
    if (!c) return fail(AR_ERR_INVALID_ARGUMENT, "cache is NULL");
    AR_GUARD_BEGIN
    DeviceGuard g(c->scene->device);
    if (table) ck(cudaMemcpy(table, c->P.table_f32, static_cast<size_t>(c->P.table_floats) * 4, cudaMemcpyDeviceToHost), "copy table");
    if (weights) ck(cudaMemcpy(weights, c->P.w_f32, ar::kNrcParams * 4, cudaMemcpyDeviceToHost), "copy weights");
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_nrc_set_params(ar_nrc* c, const float* table, const float* weights)
{
    g_last_error.clear();
    if (!c) return fail(AR_ERR_INVALID_ARGUMENT, "cache is NULL");
    AR_GUARD_BEGIN
    DeviceGuard g(c->scene->device);
    if (table) ck(cudaMemcpy(c->P.table_f32, table, static_cast<size_t>(c->P.table_floats) * 4, cudaMemcpyHostToDevice), "copy table");
    if (weights) ck(cudaMemcpy(c->P.w_f32, weights, ar::kNrcParams * 4, cudaMemcpyHostToDevice), "copy weights");
    ck(ar::nrc_publish(c->P, nullptr), "publish");
    ck(cudaDeviceSynchronize(), "sync");
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_nrc_infer(ar_nrc* c, const float* vertices, size_t n, float* out_rgb)
{
    g_last_error.clear();
    if (!c || (n && (!vertices || !out_rgb))) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n > static_cast<size_t>(INT32_MAX)) return fail(AR_ERR_INVALID_ARGUMENT, "too many vertices");
    if (n == 0) return AR_OK;
    AR_GUARD_BEGIN
    DeviceGuard g(c->scene->device);
    ar::NrcQuery* q = dalloc<ar::NrcQuery>(n, "queries");
    float* out = nullptr;
    int32_t* cnt = nullptr;
    cudaError_t e = cudaSuccess;
    try {
        out = dalloc<float>(n * (c->spectral ? ar::kNrcBins : 3), "predictions");
        cnt = dalloc<int32_t>(1, "count");
        std::vector<ar::NrcQuery> h(n);
        for (size_t i = 0; i < n; ++i) {
            std::memcpy(&h[i].v, vertices + 16 * i, sizeof(ar::NrcVertex));
            h[i].t = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        }
        const int32_t ni = static_cast<int32_t>(n);
        ck(cudaMemcpy(q, h.data(), n * sizeof(ar::NrcQuery), cudaMemcpyHostToDevice), "copy vertices");
        ck(cudaMemcpy(cnt, &ni, 4, cudaMemcpyHostToDevice), "copy count");
        e = nrc_run_infer(c, q, cnt, ni, nullptr, out, nullptr);
        if (e == cudaSuccess)
            e = cudaMemcpy(out_rgb, out, n * 4 * (c->spectral ? ar::kNrcBins : 3), cudaMemcpyDeviceToHost);
    } catch (...) {
        cudaFree(q); cudaFree(out); cudaFree(cnt);
        throw;
    }
    cudaFree(q); cudaFree(out); cudaFree(cnt);
    ck(e, "cache inference");
    return nrc_check(c, nullptr);
    AR_GUARD_END
}

ar_status ar_nrc_gradients(ar_nrc* c, const float* samples, size_t n, float* table_grad, float* weight_grad,
                           float* loss)
{
    g_last_error.clear();
    if (!c || !samples || n == 0) return fail(AR_ERR_INVALID_ARGUMENT, "bad argument");
    if (n > static_cast<size_t>(c->cfg.train_batch)) return fail(AR_ERR_INVALID_ARGUMENT, "n exceeds train_batch");
    AR_GUARD_BEGIN
    DeviceGuard g(c->scene->device);
    ar::NrcSample* d = dalloc<ar::NrcSample>(n, "samples");
    int32_t* cnt = nullptr;
    try {
        cnt = dalloc<int32_t>(1, "count");
        const int32_t ni = static_cast<int32_t>(n);
        ck(cudaMemcpy(d, samples, n * sizeof(ar::NrcSample), cudaMemcpyHostToDevice), "copy samples");
        ck(cudaMemcpy(cnt, &ni, 4, cudaMemcpyHostToDevice), "copy count");
        ck(cudaMemset(c->T.loss, 0, 4), "memset");
        ck(ar::nrc_train_step(c->net(), c->P, d, cnt, 0, c->cfg.train_batch, c->T, c->cfg.learning_rate, c->step + 1,
                              c->scene->sm_count, nullptr, false, c->tensor_path ? c->tc_err : nullptr),
           "cache gradients");
        const size_t tf = static_cast<size_t>(c->P.table_floats);
        std::vector<float> tg(tf), wg(ar::kNrcParams);
        ck(cudaMemcpy(tg.data(), c->P.table_g, tf * 4, cudaMemcpyDeviceToHost), "copy gradients");
        ck(cudaMemcpy(wg.data(), c->P.w_g, ar::kNrcParams * 4, cudaMemcpyDeviceToHost), "copy gradients");
        if (loss) ck(cudaMemcpy(loss, c->T.loss, 4, cudaMemcpyDeviceToHost), "copy loss");
        ck(cudaMemset(c->P.table_g, 0, tf * 4), "memset");
        ck(cudaMemset(c->P.w_g, 0, ar::kNrcParams * 4), "memset");
        const float inv = 1.0f / ar::kNrcLossScale;
        if (table_grad) for (size_t i = 0; i < tf; ++i) table_grad[i] = tg[i] * inv;
        if (weight_grad) for (int i = 0; i < ar::kNrcParams; ++i) weight_grad[i] = wg[static_cast<size_t>(i)] * inv;
    } catch (...) {
        cudaFree(d); cudaFree(cnt);
        throw;
    }
    cudaFree(d); cudaFree(cnt);
    return nrc_check(c, nullptr);
    AR_GUARD_END
}

ar_status ar_nrc_train(ar_nrc* c, const float* samples, size_t n, int32_t steps, float* losses)
{
    g_last_error.clear();
    if (!c || (n && !samples) || steps < 0) return fail(AR_ERR_INVALID_ARGUMENT, "bad argument");
    if (n > static_cast<size_t>(INT32_MAX)) return fail(AR_ERR_INVALID_ARGUMENT, "too many samples");
    AR_GUARD_BEGIN
    DeviceGuard g(c->scene->device);
    ar::NrcSample* d = dalloc<ar::NrcSample>(std::max<size_t>(n, 1), "samples");
    int32_t* cnt = nullptr;
    try {
        cnt = dalloc<int32_t>(1, "count");
        const int32_t ni = static_cast<int32_t>(n);
        if (n) ck(cudaMemcpy(d, samples, n * sizeof(ar::NrcSample), cudaMemcpyHostToDevice), "copy samples");
        ck(cudaMemcpy(cnt, &ni, 4, cudaMemcpyHostToDevice), "copy count");
        for (int k = 0; k < steps; ++k) {
            ck(cudaMemset(c->T.loss, 0, 4), "memset");
            ck(ar::nrc_train_step(c->net(), c->P, d, cnt, k * c->cfg.train_batch, c->cfg.train_batch, c->T,
                                  c->cfg.learning_rate, ++c->step, c->scene->sm_count, nullptr, true,
                                  c->tensor_path ? c->tc_err : nullptr), "cache training");
            float l = 0.0f;
            ck(cudaMemcpy(&l, c->T.loss, 4, cudaMemcpyDeviceToHost), "copy loss");
            if (losses) losses[k] = l;
        }
    } catch (...) {
        cudaFree(d); cudaFree(cnt);
        throw;
    }
    cudaFree(d); cudaFree(cnt);
    return nrc_check(c, nullptr);
    AR_GUARD_END
}

ar_status ar_batch_autotune(const ar_job* jobs, int32_t njobs, int32_t probe_spp, ar_batch_tuning* out, void* stream)
{
    g_last_error.clear();
    if (!jobs || njobs <= 0 || !out) return fail(AR_ERR_INVALID_ARGUMENT, "jobs or out is NULL");
    for (int j = 0; j < njobs; ++j)
        if (!jobs[j].scene) return fail(AR_ERR_INVALID_ARGUMENT, "job " + std::to_string(j) + ": scene is NULL");
    if (probe_spp <= 0) probe_spp = 4;
    AR_GUARD_BEGIN
    DeviceGuard g(jobs[0].scene->device);
    std::vector<ar_job> probe(jobs, jobs + njobs);
    std::vector<float*> scratch;
    struct Free {
        std::vector<float*>& v;
        ~Free() { for (float* p : v) cudaFree(p); }
    } release{scratch};
    for (ar_job& jb : probe) {
        const size_t n = static_cast<size_t>(jb.camera.width) * static_cast<size_t>(jb.camera.height) * 3;
        float* p = dalloc<float>(std::max<size_t>(n, 1), "autotune scratch");
        scratch.push_back(p);
        jb.out_rgb = p;
        jb.accum = nullptr;
        jb.params.spp = std::min(jb.params.spp, probe_spp);
        jb.params.wave_paths = 0;
    }
    const int32_t ks[4] = {4, 8, 16, 32};
    const int64_t bs[4] = {int64_t(1) << 20, int64_t(1) << 21, int64_t(1) << 22, int64_t(1) << 23};
    const int32_t tbs[3] = {0, 4, 2};   // traversal blocks per SM (0: the kernels' occupancy)
    const int32_t sbs[3] = {4, 2, 1};   // shading / generation / retirement blocks per SM
    ar_batch_stats st;
    // first use of every workspace (allocations, graph set-up) outside the timing
    BatchKnobs cur;
    cur.iterations = 16;
    cur.budget = bs[2];
    if (ar_status e = render_batch(probe.data(), njobs, cur, &st, stream)) return e;
    ar_batch_tuning best{16, 0, bs[2], 0.0f, 0.0f, 0, 4};
    BatchKnobs bestk = cur;
    double best_rate = -1.0;
    auto run = [&](const BatchKnobs& k) -> ar_status {
        if (ar_status e = render_batch(probe.data(), njobs, k, &st, stream)) return e;
        const double rate = static_cast<double>(st.paths) / std::max(1e-6, static_cast<double>(st.total_ms));
        if (k.iterations == 16 && k.budget == bs[2] && k.trace_bps == 0 && k.shade_bps == 0) best.default_ms = st.total_ms;
        ++best.candidates;
        if (rate > best_rate) {
            best_rate = rate;
            bestk = k;
            best.best_ms = st.total_ms;
        }
        return AR_OK;
    };
    // graph length x path budget at the default grids, then the grids at the best of those
    for (int32_t k : ks)
        for (int64_t b : bs) {
            BatchKnobs c;
            c.iterations = k;
            c.budget = b;
            if (ar_status e = run(c)) return e;
        }
    const BatchKnobs base = bestk;
    for (int32_t t : tbs)
        for (int32_t sb : sbs) {
            if (t == 0 && sb == 4) continue;   // measured above
            BatchKnobs c = base;
            c.trace_bps = t;
            c.shade_bps = sb;
            if (ar_status e = run(c)) return e;
        }
    best.iterations_per_graph = bestk.iterations;
    best.path_budget = bestk.budget;
    best.trace_blocks_per_sm = bestk.trace_bps;
    best.shade_blocks_per_sm = bestk.shade_bps > 0 ? bestk.shade_bps : 4;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[batch_key(jobs, njobs)] = bestk;
    }
    *out = best;
    return AR_OK;
    AR_GUARD_END
}

}  // extern "C"

// ------------------------------------------------------------------ path guiding
struct ar_guide {
    ar_scene* scene = nullptr;
    ar::GuideView view{};
    size_t table_size = 0;
    int64_t frames = 0;
    int64_t npix = 0;
    float* faces = nullptr;
    std::vector<void*> owned;
    std::vector<void*> frame_bufs;
    ~ar_guide()
    {
        QuietDeviceGuard g(scene->device);
        for (void* p : owned) cudaFree(p);
        for (void* p : frame_bufs) cudaFree(p);
    }
};

namespace {
template <class T>
T* guide_alloc(std::vector<void*>& v, size_t count, const char* what)
{
    T* p = dalloc<T>(count, what);
    v.push_back(p);
    return p;
}
void guide_ensure_frame(ar_guide* g, int64_t npix)
{
    if (npix <= g->npix) return;
    for (void* p : g->frame_bufs) cudaFree(p);
    g->frame_bufs.clear();
    const size_t n = static_cast<size_t>(npix);
    g->view.events = guide_alloc<float4>(g->frame_bufs, n * ar::kPgEvents * 3, "guiding events");
    g->view.event_lb = guide_alloc<float4>(g->frame_bufs, n * ar::kPgEvents, "guiding events");
    g->view.event_count = guide_alloc<int32_t>(g->frame_bufs, n, "guiding events");
    g->view.sample_cap = static_cast<int32_t>(std::min<int64_t>(npix * ar::kPgCollect, int64_t(1) << 22));
    g->view.samples = guide_alloc<float4>(g->frame_bufs, static_cast<size_t>(g->view.sample_cap) * 3, "guiding samples");
    ck(cudaMemset(g->view.event_count, 0, n * sizeof(int32_t)), "memset");
    g->npix = npix;
}
}  // namespace

extern "C" {

ar_status ar_guide_create(ar_scene* s, const ar_guide_config* cfg, ar_guide** out)
{
    g_last_error.clear();
    if (!s || !out) return fail(AR_ERR_INVALID_ARGUMENT, "scene or out is NULL");
    *out = nullptr;
    const int cap = cfg && cfg->probe_capacity > 0 ? cfg->probe_capacity : 131072;
    const int lt = cfg && cfg->log2_table > 0 ? cfg->log2_table : 20;
    if (cap > (1 << 24)) return fail(AR_ERR_INVALID_ARGUMENT, "probe_capacity above 2^24");
    if (lt < 10 || lt > 28) return fail(AR_ERR_INVALID_ARGUMENT, "log2_table must be in [10, 28]");
    AR_GUARD_BEGIN
    DeviceGuard dg(s->device);
    std::unique_ptr<ar_guide> g(new ar_guide());
    g->scene = s;
    g->table_size = size_t(1) << lt;
    ar::GuideView& v = g->view;
    v.capacity = cap;
    v.table_mask = static_cast<uint32_t>(g->table_size - 1);
    v.keys = guide_alloc<uint64_t>(g->owned, g->table_size, "guiding table");
    v.slots = guide_alloc<int32_t>(g->owned, g->table_size, "guiding table");
    v.probes = guide_alloc<float4>(g->owned, static_cast<size_t>(cap) * ar::kPgStride, "guiding probes");
    v.accum = guide_alloc<float4>(g->owned, static_cast<size_t>(cap) * ar::kPgRes * ar::kPgRes, "guiding sums");
    v.counts = guide_alloc<unsigned long long>(g->owned, static_cast<size_t>(cap), "guiding counts");
    v.frame_counts = guide_alloc<unsigned int>(g->owned, static_cast<size_t>(cap), "guiding counts");
    v.touched = guide_alloc<int32_t>(g->owned, static_cast<size_t>(cap), "guiding list");
    v.counters = guide_alloc<int32_t>(g->owned, 6, "guiding counters");
    float faces[60];
    ar::pg_face_normals(faces);
    float* df = guide_alloc<float>(g->owned, 60, "guiding faces");
    ck(cudaMemcpy(df, faces, sizeof(faces), cudaMemcpyHostToDevice), "copy faces");
    v.faces = df;
    ck(ar::pg_clear(v, g->table_size, nullptr), "guiding clear");
    ck(cudaDeviceSynchronize(), "guiding init");
    *out = g.release();
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_guide_destroy(ar_guide* g)
{
    g_last_error.clear();
    delete g;
    return AR_OK;
}

ar_status ar_guide_render_frame(ar_guide* g, const ar_camera* cam, const ar_render_params* p, float* out_rgb,
                                double* accum, void* stream)
{
    g_last_error.clear();
    if (!g) return fail(AR_ERR_INVALID_ARGUMENT, "guide is NULL");
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (p->spp != 1) return fail(AR_ERR_INVALID_ARGUMENT, "guided frames take spp = 1");
    if (p->spectral) return fail(AR_ERR_UNSUPPORTED, "path guiding is RGB only");
    if (!out_rgb && !accum) return fail(AR_ERR_INVALID_ARGUMENT, "out_rgb and accum are both NULL");
    AR_GUARD_BEGIN
    ar_scene* s = g->scene;
    DeviceGuard dg(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t npix = static_cast<int64_t>(cam->width) * cam->height;
    guide_ensure_frame(g, npix);
    // events of a frame that did not complete must not leak into this one
    ck(cudaMemsetAsync(g->view.event_count, 0, static_cast<size_t>(npix) * sizeof(int32_t), st), "memset");
    g->view.alpha = ar::pg_alpha(g->frames);
    if (ar_status e = run_render(s, cam, p, nullptr, st, nullptr, nullptr, &g->view)) return e;
    ck(ar::pg_update(g->view, s->sm_count, st), "guiding update");
    ++g->frames;
    const int64_t n = npix * 3;
    if (out_rgb) ck(ar::launch_mean(s->accum, n, 1.0 / static_cast<double>(p->spp), out_rgb, st), "mean");
    if (accum) ck(ar::launch_add(s->accum, n, accum, st), "accumulate");
    return check_err(s, st);
    AR_GUARD_END
}

// ------------------------------------------------------------------ denoiser recording
ar_status ar_render_frame_denoise(ar_scene* s, const ar_camera* cam, const ar_render_params* p, float* out_rgb,
                                  double* accum, ar_screen_gbuffer* gbuffer, ar_screen_stats* stats, void* stream)
{
    g_last_error.clear();
    if (!s) return fail(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (ar_status e = check_camera(cam)) return e;
    if (ar_status e = check_params(p)) return e;
    if (p->spp != 1) return fail(AR_ERR_INVALID_ARGUMENT, "denoiser frames take spp = 1");
    if (!out_rgb && !accum) return fail(AR_ERR_INVALID_ARGUMENT, "out_rgb and accum are both NULL");
    AR_GUARD_BEGIN
    DeviceGuard dg(s->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ar::DenoiseView dn;
    dn.gbuf = gbuffer;
    dn.stat = stats;
    if (ar_status e = run_render(s, cam, p, nullptr, st, nullptr, nullptr, nullptr, &dn)) return e;
    const int64_t n = static_cast<int64_t>(cam->width) * cam->height * 3;
    if (out_rgb) ck(ar::launch_mean(s->accum, n, 1.0, out_rgb, st), "mean");
    if (accum) ck(ar::launch_add(s->accum, n, accum, st), "accumulate");
    return check_err(s, st);
    AR_GUARD_END
}

ar_status ar_guide_get_stats(const ar_guide* g, ar_guide_stats* out)
{
    g_last_error.clear();
    if (!g || !out) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    AR_GUARD_BEGIN
    DeviceGuard dg(g->scene->device);
    int32_t c[6];
    ck(cudaMemcpy(c, g->view.counters, sizeof(c), cudaMemcpyDeviceToHost), "copy counters");
    std::memset(out, 0, sizeof(*out));
    out->frames = g->frames;
    out->probes = std::min<int64_t>(c[0], g->view.capacity);
    out->samples = c[4];
    out->dropped = c[5];
    out->alpha = ar::pg_alpha(std::max<int64_t>(0, g->frames - 1));
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_guide_get_probe(const ar_guide* g, int32_t index, float* texels)
{
    g_last_error.clear();
    if (!g || !texels) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    AR_GUARD_BEGIN
    DeviceGuard dg(g->scene->device);
    int32_t c[4];
    ck(cudaMemcpy(c, g->view.counters, sizeof(c), cudaMemcpyDeviceToHost), "copy counters");
    if (index < 0 || index >= std::min(c[0], g->view.capacity)) return fail(AR_ERR_INVALID_ARGUMENT, "probe not allocated");
    ck(cudaMemcpy(texels, g->view.probes + static_cast<size_t>(index) * ar::kPgStride, sizeof(float4) * ar::kPgStride,
                  cudaMemcpyDeviceToHost), "copy probe");
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_spectral_rgb_lut(const float* tables, size_t count, int32_t res, int32_t method, float* out_device,
                              float* ms)
{
    g_last_error.clear();
    if (!tables || !out_device) return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    if (count != static_cast<size_t>(ar::kTabFloats))
        return fail(AR_ERR_INVALID_ARGUMENT, "tables must hold " + std::to_string(ar::kTabFloats) + " floats");
    if (res < 2 || res > 1024) return fail(AR_ERR_INVALID_ARGUMENT, "res must be in [2, 1024]");
    if (method != AR_LUT_SIMT && method != AR_LUT_TENSOR)
        return fail(AR_ERR_INVALID_ARGUMENT, "method must be AR_LUT_SIMT or AR_LUT_TENSOR");
    if (reinterpret_cast<uintptr_t>(out_device) & 15u) return fail(AR_ERR_INVALID_ARGUMENT, "out must be 16-byte aligned");
    AR_GUARD_BEGIN
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return fail(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    float* tab = dalloc<float>(count, "spectral tables");
    float4* lam = dalloc<float4>(ar::kLambdaLutRes, "spectral lambda table");
    int* err = dalloc<int>(1, "error word");
    struct Free { void* a; void* b; void* c; ~Free() { cudaFree(a); cudaFree(b); cudaFree(c); } } fr{tab, lam, err};
    ck(cudaMemcpy(tab, tables, count * sizeof(float), cudaMemcpyHostToDevice), "copy spectral tables");
    ck(cudaMemset(err, 0, sizeof(int)), "memset");
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    struct Ev { cudaEvent_t a, b; ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); } } ev{e0, e1};
    float4* out = reinterpret_cast<float4*>(out_device);
    ck(cudaEventRecord(e0, nullptr), "event");
    if (method == AR_LUT_TENSOR) ck(ar::launch_spectral_rgb_lut_tc(tab, res, out, err, sms, nullptr), "table build");
    else ck(ar::launch_spectral_luts(tab, res, lam, out, sms, nullptr), "table build");
    ck(cudaEventRecord(e1, nullptr), "event");
    ck(cudaEventSynchronize(e1), "sync");
    int h = 0;
    ck(cudaMemcpy(&h, err, sizeof(int), cudaMemcpyDeviceToHost), "error word");
    if (h) return fail(AR_ERR_DEVICE_FAULT, "tensor-core table build: an MMA did not complete within its wait limit");
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    return AR_OK;
    AR_GUARD_END
}

ar_status ar_guide_probe_eval(const float* texels, int32_t nprobes, const int32_t* probe_of, const float* normal3,
                              const float* query3, const float* u5, const float* eval3, const float* pos3, int64_t n,
                              float* out_dir3, float* out_pdf, float* out_eval_pdf, uint64_t* out_key)
{
    g_last_error.clear();
    if (n < 0 || nprobes <= 0) return fail(AR_ERR_INVALID_ARGUMENT, "n must be >= 0 and nprobes > 0");
    if (n == 0) return AR_OK;
    if (!texels || !probe_of || !normal3 || !query3 || !u5 || !eval3 || !pos3 || !out_dir3 || !out_pdf ||
        !out_eval_pdf || !out_key)
        return fail(AR_ERR_INVALID_ARGUMENT, "NULL argument");
    for (int64_t i = 0; i < n; ++i)
        if (probe_of[i] < 0 || probe_of[i] >= nprobes) return fail(AR_ERR_INVALID_ARGUMENT, "probe index out of range");
    AR_GUARD_BEGIN
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    const size_t m = static_cast<size_t>(n);
    std::vector<float4> padded(static_cast<size_t>(nprobes) * ar::kPgStride, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    for (int32_t p = 0; p < nprobes; ++p)
        for (int t = 0; t < ar::kPgTexels; ++t) {
            const float* src = texels + (static_cast<size_t>(p) * ar::kPgTexels + t) * 4;
            padded[static_cast<size_t>(p) * ar::kPgStride + t] = make_float4(src[0], src[1], src[2], src[3]);
        }
    float faces[60];
    ar::pg_face_normals(faces);
    std::vector<void*> tmp;
    struct Free {
        std::vector<void*>& v;
        ~Free() { for (void* p : v) cudaFree(p); }
    } fr{tmp};
    auto up = [&](const void* src, size_t bytes) {
        void* d = dalloc<unsigned char>(bytes, "probe eval input");
        tmp.push_back(d);
        ck(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice), "copy probe eval input");
        return d;
    };
    auto dn = [&](size_t bytes) {
        void* d = dalloc<unsigned char>(bytes, "probe eval output");
        tmp.push_back(d);
        return d;
    };
    const float4* dp = static_cast<const float4*>(up(padded.data(), padded.size() * sizeof(float4)));
    const int32_t* dpo = static_cast<const int32_t*>(up(probe_of, m * 4));
    const float* dn3 = static_cast<const float*>(up(normal3, m * 12));
    const float* dq3 = static_cast<const float*>(up(query3, m * 12));
    const float* du5 = static_cast<const float*>(up(u5, m * 20));
    const float* de3 = static_cast<const float*>(up(eval3, m * 12));
    const float* dp3 = static_cast<const float*>(up(pos3, m * 12));
    const float* dfc = static_cast<const float*>(up(faces, sizeof(faces)));
    float* odir = static_cast<float*>(dn(m * 12));
    float* opdf = static_cast<float*>(dn(m * 4));
    float* oepdf = static_cast<float*>(dn(m * 4));
    unsigned long long* okey = static_cast<unsigned long long*>(dn(m * 8));
    ck(ar::pg_eval(dp, dpo, dn3, dq3, du5, de3, dp3, n, dfc, odir, opdf, oepdf, okey, nullptr), "probe eval");
    ck(cudaMemcpy(out_dir3, odir, m * 12, cudaMemcpyDeviceToHost), "copy directions");
    ck(cudaMemcpy(out_pdf, opdf, m * 4, cudaMemcpyDeviceToHost), "copy pdfs");
    ck(cudaMemcpy(out_eval_pdf, oepdf, m * 4, cudaMemcpyDeviceToHost), "copy pdfs");
    ck(cudaMemcpy(out_key, okey, m * 8, cudaMemcpyDeviceToHost), "copy keys");
    return AR_OK;
    AR_GUARD_END
}

}  // extern "C"

