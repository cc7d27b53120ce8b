// aperture_b200_renderer.hpp -- the reference renderer's host API (SceneObject,
// Material, SceneRenderer, Camera) over the C ABI of aperture_b200.h.
//
// ApertureRendererV3 is driven through C++ classes: a caller fills a
// std::vector<SceneObject> (core/render/object.cuh:250-365), builds a
// SceneRenderer from it (core/scene.hpp:113) and calls
// SceneRenderer::Render(size, origin, direction, spp) (core/scene.cu:276-306) or
// Camera::RenderToFile(path, spp, tonemap, exposure) (core/camera.cu:64-89).
// This header keeps those names, signatures and argument meanings so such a
// caller recompiles against it unchanged; every call forwards to the sm_100a
// library (libaperture_b200.so).  Header-only; needs CUDA's vector_types.h for
// float3 / int2, like the reference.
//
// Conventions kept from the reference: errors are printed, not thrown (the
// reference's CHECK_ERROR prints and continues; here a failed call prints the
// library's message and leaves the output zeroed); the camera's field of view is
// 60 degrees and MAX_TRACING_DEPTH 1000; the scene is uploaded lazily on the
// first Render after construction or MarkAsDirty().
//
// Differences a caller may notice:
//   * samples are accumulated in FP64 (the reference keeps an FP32 running mean);
//   * triangles are shaded with their own material (the reference's software
//     tracer shades triangles white);
//   * Camera::RenderToFile indexes rows by the image width and writes a correct
//     top-down 32-bit BMP for any aspect ratio (the reference indexes by height
//     and swaps channels over width x height, right only for square images);
//   * the interactive Render's odd/even variance targets, path-guiding sample
//     buffer and denoiser buffers are not supported (a message is printed when
//     one is passed); path guiding is inert in the reference's offline render.
#pragma once

#include <cuda_runtime.h>
#include <vector_types.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <string>
#include <vector>

#include "aperture_b200.h"

namespace pg { struct PathGuidingSample; }
namespace denoise { struct ScreenGBuffer; struct ScreenStatisticsBuffer; }

// EObjectType / EShadingModel (core/render/object.cuh:29-52)
enum class EObjectType { OBJ_CUBE = 0, OBJ_SPHERE = 1, OBJ_SDF = 2, OBJ_TRIANGLE = 3 };
enum class EShadingModel { MAT_DIFFUSE = 0, MAT_LIGHT = 1, MAT_GLASS = 2, MAT_GGX = 3, MAT_MAX = 4 };
enum class ETextureType { TEX_PURE_COLOR = 0 };

// GBuffer fields of a pure-colour texture (core/render/object.cuh:60-91), defaults as there.
struct GBuffer {
    float3 albedo_ = {1.0f, 1.0f, 1.0f};
    float3 emissive_ = {0.0f, 0.0f, 0.0f};
    float specular_ = 0.0f;
    float metallic_ = 0.0f;
    float roughness_ = 0.0f;
    float IOR_ = 1.5f;
    float sigmaA_ = 100.0f;
    float3 normal_ = {0.0f, 0.0f, 1.0f};
    float abbeNumber_ = 20.0f;
    float tiltNumber_ = 0.0f;
};

struct Texture {
    ETextureType textureType_ = ETextureType::TEX_PURE_COLOR;
    GBuffer baseTexture_ = {};
};

namespace aperture_b200_detail {
inline float clampf(float v, float a, float b) { return v < a ? a : (v > b ? b : v); }
}  // namespace aperture_b200_detail

// Material and its factories (core/render/object.cuh:124-217).
struct Material {
    EShadingModel shadingModel_ = EShadingModel::MAT_DIFFUSE;
    Texture texture_ = {};

    static Material CreateDiffusePureColor(const float3 color, const float3 emissive = float3{0.0f, 0.0f, 0.0f})
    {
        Material m;
        m.texture_.baseTexture_.albedo_ = color;
        m.texture_.baseTexture_.emissive_ = emissive;
        return m;
    }
    static Material CreateLight(const float3 emissive)
    {
        Material m;
        m.shadingModel_ = EShadingModel::MAT_LIGHT;
        m.texture_.baseTexture_.albedo_ = float3{0.0f, 0.0f, 0.0f};
        m.texture_.baseTexture_.emissive_ = emissive;
        return m;
    }
    static Material CreateGlassPureColor(const float3 color, const float IOR, const float sigmaA,
                                         const float abbeNumber = 20.0f, const float tiltNumber = 0.0f)
    {
        Material m;
        m.shadingModel_ = EShadingModel::MAT_GLASS;
        GBuffer& g = m.texture_.baseTexture_;
        g.albedo_ = color;
        g.IOR_ = IOR;
        g.sigmaA_ = sigmaA;
        g.abbeNumber_ = abbeNumber;
        g.tiltNumber_ = tiltNumber;
        return m;
    }
    static Material CreateGGXGlassPureColor(const float3 color, const float IOR, const float sigmaA, const float roughness)
    {
        Material m;
        m.shadingModel_ = EShadingModel::MAT_GLASS;
        GBuffer& g = m.texture_.baseTexture_;
        g.albedo_ = color;
        g.IOR_ = IOR;
        g.sigmaA_ = sigmaA;
        g.roughness_ = roughness;
        return m;
    }
    static Material CreateGGXPureColor(const float3 baseColor, const float roughness, const float metallic,
                                       const float specular, const float3 emissive = float3{0.0f, 0.0f, 0.0f})
    {
        using aperture_b200_detail::clampf;
        Material m;
        m.shadingModel_ = EShadingModel::MAT_GGX;
        GBuffer& g = m.texture_.baseTexture_;
        g.albedo_ = baseColor;
        g.roughness_ = clampf(roughness, 0.01f, 1.0f);
        g.metallic_ = clampf(metallic, 0.0f, 1.0f);
        g.specular_ = clampf(specular, 0.0f, 1.0f);
        g.emissive_ = emissive;
        return m;
    }
};

// Triangle vertex data (core/render/object.cuh:232-248), object space.
struct Vertex { float3 position_; float3 normal_; float2 uv_; };
struct TriangleInfo { Vertex v0_; Vertex v1_; Vertex v2_; };
struct AdditionalObjectInfo { TriangleInfo triangleInfo_ = {}; };

// SceneObject (core/render/object.cuh:250-365): the constructor's arguments are
// kept; the world transform is built by the library from rotation_ exactly as
// the reference's constructor builds it (Rz * (Ry * Rx), degrees).
struct SceneObject {
    float3 center_ = {0.0f, 0.0f, 0.0f};
    float3 extent_ = {0.0f, 0.0f, 0.0f};
    Material material_ = {};
    float3 rotation_ = {0.0f, 0.0f, 0.0f};
    EObjectType type_ = EObjectType::OBJ_CUBE;
    AdditionalObjectInfo additionalObjectInfo_ = {};
    bool bVisible_ = true;

    SceneObject() = default;
    SceneObject(const float3 center, const float3 extent, const Material& material, const float3 rotation,
                const EObjectType type = EObjectType::OBJ_CUBE, const AdditionalObjectInfo& additionalObjectInfo = {})
        : center_(center), extent_{std::fabs(extent.x), std::fabs(extent.y), std::fabs(extent.z)},
          material_(material), rotation_(rotation), type_(type), additionalObjectInfo_(additionalObjectInfo)
    {
    }

    ar_object_desc ToDesc() const
    {
        ar_object_desc d;
        std::memset(&d, 0, sizeof(d));
        d.type = static_cast<int32_t>(type_);
        d.center = {center_.x, center_.y, center_.z};
        d.extent = {extent_.x, extent_.y, extent_.z};
        d.rotation_deg = {rotation_.x, rotation_.y, rotation_.z};
        const GBuffer& g = material_.texture_.baseTexture_;
        d.material.shading_model = static_cast<int32_t>(material_.shadingModel_);
        d.material.albedo = {g.albedo_.x, g.albedo_.y, g.albedo_.z};
        d.material.emissive = {g.emissive_.x, g.emissive_.y, g.emissive_.z};
        d.material.specular = g.specular_;
        d.material.metallic = g.metallic_;
        d.material.roughness = g.roughness_;
        d.material.ior = g.IOR_;
        d.material.sigma_a = g.sigmaA_;
        d.material.abbe_number = g.abbeNumber_;
        d.material.tilt_number = g.tiltNumber_;
        const Vertex* v[3] = {&additionalObjectInfo_.triangleInfo_.v0_, &additionalObjectInfo_.triangleInfo_.v1_,
                              &additionalObjectInfo_.triangleInfo_.v2_};
        for (int k = 0; k < 3; ++k) {
            d.tri[k].position = {v[k]->position_.x, v[k]->position_.y, v[k]->position_.z};
            d.tri[k].normal = {v[k]->normal_.x, v[k]->normal_.y, v[k]->normal_.z};
            d.tri[k].u = v[k]->uv_.x;
            d.tri[k].v = v[k]->uv_.y;
        }
        d.visible = bVisible_ ? 1 : 0;
        return d;
    }
};

// SceneSetting (core/render/object.cuh:10-27); only bUseNEE_ changes the image
// here (BVH traversal is always on, path guiding is inert offline).
struct SceneSetting {
    bool bUseBVH_ = true;
    bool bUseNEE_ = true;
    bool bUsePathGuiding_ = true;
    bool bDenoise_ = false;
};

class SceneRenderer {
public:
    std::vector<SceneObject> sceneObjects_;
    SceneSetting sceneSetting_;

    explicit SceneRenderer(const std::vector<SceneObject>& sceneObjects) : sceneObjects_(sceneObjects) {}
    SceneRenderer(const SceneRenderer&) = delete;
    ~SceneRenderer()
    {
        MarkNeedResetGuiding();
        if (scene_) ar_scene_destroy(scene_);
        FreeAccum();
    }

    void SetExposure(float exp) { exposure_ = exp; }
    float GetExposure() const { return exposure_; }
    void MarkAsDirty() { dirty_ = true; }
    // Path guiding of the interactive render (the reference's
    // CalculateRadiance<..., bUsePathGuiding>): off by default here.
    void SetPathGuiding(bool on) { useGuiding_ = on; }
    void MarkNeedResetGuiding()
    {
        if (guide_) ar_guide_destroy(guide_);
        guide_ = nullptr;
    }

    // Offline render: linear RGB, row j*size.x + i, mean of sampleNum samples
    // (frames 0 .. sampleNum-1).
    std::vector<float3> Render(const int2 size, const float3 cameraOrigin, const float3 cameraDirection,
                               int sampleNum = 1024)
    {
        std::vector<float3> out(static_cast<size_t>(size.x > 0 ? size.x : 0) * (size.y > 0 ? size.y : 0),
                                float3{0.0f, 0.0f, 0.0f});
        if (out.empty() || !Upload()) return out;
        const ar_camera cam = MakeCamera(size, cameraOrigin, cameraDirection);
        const ar_render_params p = MakeParams(sampleNum, 0);
        Check(ar_render(scene_, &cam, &p, reinterpret_cast<float*>(out.data()), nullptr, AR_MEM_HOST, nullptr,
                        nullptr));
        return out;
    }

    // Interactive render of frame `frameIndex` into caller-owned device buffers:
    // hdrTarget (float3, W*H) receives the running mean of frames 0..frameIndex,
    // ldrTarget (0xAARRGGBB, W*H, may be null) its tone-mapped image
    // (toneType 0 none, 1 gamma, 2 ACES; exposure from SetExposure).
    void Render(float3* hdrTarget, unsigned int* ldrTarget, const int2 size, const float3 cameraOrigin,
                const float3 cameraDirection, int frameIndex, int toneType, float3* oddTarget = nullptr,
                float3* evenTarget = nullptr, pg::PathGuidingSample* radianceSampleBuffer = nullptr,
                denoise::ScreenGBuffer* screenGBuffer = nullptr,
                denoise::ScreenStatisticsBuffer* screenStatisticsBuffer = nullptr)
    {
        if (oddTarget || evenTarget || radianceSampleBuffer || screenGBuffer || screenStatisticsBuffer)
            std::cout << "aperture_b200: odd/even, path-guiding sample and denoiser buffers are not supported; ignored\n";
        if (!hdrTarget || size.x <= 0 || size.y <= 0 || !Upload()) return;
        const size_t n = static_cast<size_t>(size.x) * size.y * 3;
        if (!EnsureAccum(n)) return;
        if (frameIndex <= 0 && !ZeroAccum()) return;
        const ar_camera cam = MakeCamera(size, cameraOrigin, cameraDirection);
        const ar_render_params p = MakeParams(1, frameIndex > 0 ? frameIndex : 0);
        if (useGuiding_) {
            if (!guide_ && !Check(ar_guide_create(scene_, nullptr, &guide_))) return;
            if (!Check(ar_guide_render_frame(guide_, &cam, &p, nullptr, accum_, nullptr))) return;
        } else if (!Check(ar_render(scene_, &cam, &p, nullptr, accum_, AR_MEM_DEVICE, nullptr, nullptr))) {
            return;
        }
        const double scale = 1.0 / static_cast<double>((frameIndex > 0 ? frameIndex : 0) + 1);
        if (!Check(ar_accum_resolve(accum_, n, scale, reinterpret_cast<float*>(hdrTarget), AR_MEM_DEVICE, nullptr)))
            return;
        if (ldrTarget)
            Check(ar_tonemap(reinterpret_cast<const float*>(hdrTarget), n / 3, toneType, exposure_, 0, ldrTarget,
                             AR_MEM_DEVICE, nullptr));
    }

    // The library's scene handle (uploads the scene if needed); null on failure.
    ar_scene* Handle() { return Upload() ? scene_ : nullptr; }

private:
    ar_scene* scene_ = nullptr;
    ar_guide* guide_ = nullptr;
    bool useGuiding_ = false;
    bool dirty_ = true;
    float exposure_ = 1.0f;
    double* accum_ = nullptr;
    size_t accum_n_ = 0;

    static bool Check(ar_status st)
    {
        if (st == AR_OK) return true;
        std::cout << "aperture_b200 ERROR: " << ar_get_last_error_string() << "\n";
        return false;
    }

    bool Upload()
    {
        if (!dirty_ && scene_) return true;
        MarkNeedResetGuiding();
        if (scene_) {
            ar_scene_destroy(scene_);
            scene_ = nullptr;
        }
        std::vector<ar_object_desc> desc;
        desc.reserve(sceneObjects_.size());
        for (const SceneObject& o : sceneObjects_) desc.push_back(o.ToDesc());
        if (!Check(ar_scene_create(desc.data(), desc.size(), 0, &scene_))) return false;
        dirty_ = false;
        return true;
    }

    bool EnsureAccum(size_t n);
    void FreeAccum();
    bool ZeroAccum();

    static ar_camera MakeCamera(int2 size, float3 origin, float3 direction)
    {
        ar_camera c;
        c.position = {origin.x, origin.y, origin.z};
        c.direction = {direction.x, direction.y, direction.z};
        c.fov_y_deg = 60.0f;  // RenderCamera's FOV (core/scene.cu:220)
        c.width = size.x;
        c.height = size.y;
        return c;
    }

    ar_render_params MakeParams(int spp, int frame) const
    {
        ar_render_params p;
        std::memset(&p, 0, sizeof(p));
        p.spp = spp;
        p.max_depth = 1000;  // MAX_TRACING_DEPTH (core/config.cuh:8)
        p.rr_depth = 3;      // MIN_TRACING_DEPTH (core/config.cuh:7)
        p.use_nee = sceneSetting_.bUseNEE_ ? 1 : 0;
        p.sky = 1;
        p.frame_offset = frame;
        p.seed = 0x9e3779b97f4a7c15ull;  // GLOBAL_SEED (core/random.cuh:13)
        return p;
    }
};

// The interactive accumulator (FP64, 3 values per pixel) is device memory that
// the shim allocates with the CUDA runtime, like the caller's own hdr/ldr
// targets, and frees in the destructor.
inline bool SceneRenderer::EnsureAccum(size_t n)
{
    if (accum_ && accum_n_ == n) return true;
    FreeAccum();
    if (cudaMalloc(reinterpret_cast<void**>(&accum_), n * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        accum_ = nullptr;
        std::cout << "aperture_b200 ERROR: cannot allocate the accumulation buffer\n";
        return false;
    }
    accum_n_ = n;
    return ZeroAccum();
}

inline void SceneRenderer::FreeAccum()
{
    if (accum_) cudaFree(accum_);
    accum_ = nullptr;
    accum_n_ = 0;
}

inline bool SceneRenderer::ZeroAccum()
{
    if (cudaMemset(accum_, 0, accum_n_ * sizeof(double)) == cudaSuccess) return true;
    cudaGetLastError();
    std::cout << "aperture_b200 ERROR: cannot clear the accumulation buffer\n";
    return false;
}

// Tone curves as host functions with the reference's names and signature
// (core/tonemap.cuh: Gamma, ACES), usable as its ToneMapFunction; they call the
// library's own curves (ar_tone_curve) so host and GPU results agree.
typedef std::function<float3(const float3 radiance)> ToneMapFunction;

inline float3 Gamma(float3 color)
{
    const float in[3] = {color.x, color.y, color.z};
    float out[3] = {0.0f, 0.0f, 0.0f};
    ar_tone_curve(in, 1, out);
    return float3{out[0], out[1], out[2]};
}

inline float3 ACES(float3 color)
{
    const float in[3] = {color.x, color.y, color.z};
    float out[3] = {0.0f, 0.0f, 0.0f};
    ar_tone_curve(in, 2, out);
    return float3{out[0], out[1], out[2]};
}

namespace aperture_b200_detail {
inline int tone_of(const ToneMapFunction& f)
{
    if (!f) return 0;
    auto t = f.target<float3 (*)(float3)>();
    if (t && *t == &::ACES) return 2;
    if (t && *t == &::Gamma) return 1;
    return -1;
}
}  // namespace aperture_b200_detail

// SaveBMP (core/camera.cu:10-62): writes `filename`.bmp, 32-bit, top-down;
// image holds R, G, B, A bytes per pixel, row j at offset 4*j*imageWidth.
inline int SaveBMP(unsigned char* image, int imageWidth, int imageHeight, const char* filename)
{
    unsigned char header[54] = {0x42, 0x4d};
    const uint32_t data = static_cast<uint32_t>(imageWidth) * static_cast<uint32_t>(imageHeight) * 4u;
    const uint32_t file_size = data + 54u;
    auto put32 = [&](int at, uint32_t v) {
        for (int k = 0; k < 4; ++k) header[at + k] = static_cast<unsigned char>((v >> (8 * k)) & 0xffu);
    };
    put32(2, file_size);
    put32(10, 54u);
    put32(14, 40u);
    put32(18, static_cast<uint32_t>(imageWidth));
    put32(22, static_cast<uint32_t>(-imageHeight));  // negative: top-down rows
    header[26] = 1;
    header[28] = 32;
    put32(34, data);
    std::string name = std::string(filename) + ".bmp";
    FILE* f = std::fopen(name.c_str(), "wb");
    if (!f) return -1;
    std::vector<unsigned char> bgra(image, image + data);
    for (size_t i = 0; i + 3 < bgra.size(); i += 4) std::swap(bgra[i], bgra[i + 2]);
    std::fwrite(header, 1, 54, f);
    std::fwrite(bgra.data(), 1, bgra.size(), f);
    std::fclose(f);
    return 0;
}

// Camera (core/camera.hpp:14-100).
class Camera {
protected:
    float3 position_;
    float3 direction_;

public:
    SceneRenderer* sceneRenderer_;
    int resolutionX_;
    int resolutionY_;
    std::string name_;
    mutable double variance_ = 0.0;

    Camera(SceneRenderer& sceneRenderer, const std::string& name = "test camera", const int resolutionX = 1080,
           int resolutionY = 720, const float3 position = {0.0f, 0.75f, 0.75f},
           const float3 direction = {0.0f, 0.0f, -0.75f})
    {
        SetPositionAndDirection(position, direction);
        name_ = name;
        sceneRenderer_ = &sceneRenderer;
        resolutionX_ = resolutionX;
        resolutionY_ = resolutionY;
    }

    void SetPosition(const float3 position) { position_ = position; }
    float3 GetPosition() const { return position_; }
    void SetDirection(const float3 d)
    {
        const float l2 = d.x * d.x + d.y * d.y + d.z * d.z;
        const float inv = l2 > 1e-20f ? 1.0f / std::sqrt(l2) : 0.0f;
        direction_ = float3{d.x * inv, d.y * inv, d.z * inv};
    }
    float3 GetDirection() const { return direction_; }
    void SetPositionAndDirection(const float3 position, const float3 direction)
    {
        SetPosition(position);
        SetDirection(direction);
    }
    void SetVolume(SceneRenderer& sceneRenderer) { sceneRenderer_ = &sceneRenderer; }

    // Render sampleNum samples, apply exposure and the tone curve, write
    // `path`.bmp.  ACES and Gamma run on the GPU (ar_tonemap); any other
    // function is applied per pixel on the host, as the reference does.
    void RenderToFile(const std::string& path, const int sampleNum = 1, const ToneMapFunction tonemapFunction = ACES,
                      const float exp = 1.0) const
    {
        const int w = resolutionX_, h = resolutionY_;
        const std::vector<float3> img = sceneRenderer_->Render(int2{w, h}, GetPosition(), GetDirection(), sampleNum);
        std::vector<unsigned char> data(static_cast<size_t>(w) * h * 4, 0);
        const int tone = aperture_b200_detail::tone_of(tonemapFunction);
        if (tone >= 0) {
            std::vector<uint32_t> packed(static_cast<size_t>(w) * h);
            if (ar_tonemap(reinterpret_cast<const float*>(img.data()), packed.size(), tone, exp, 0, packed.data(),
                           AR_MEM_HOST, nullptr) != AR_OK) {
                std::cout << "aperture_b200 ERROR: " << ar_get_last_error_string() << "\n";
            }
            for (size_t i = 0; i < packed.size(); ++i) {
                data[4 * i + 0] = static_cast<unsigned char>((packed[i] >> 16) & 0xffu);
                data[4 * i + 1] = static_cast<unsigned char>((packed[i] >> 8) & 0xffu);
                data[4 * i + 2] = static_cast<unsigned char>(packed[i] & 0xffu);
                data[4 * i + 3] = 255;
            }
        } else {
            for (size_t i = 0; i < img.size(); ++i) {
                const float3 v = tonemapFunction(float3{img[i].x * exp, img[i].y * exp, img[i].z * exp});
                auto q = [](float x) {
                    x = (x != x) ? 0.0f : (x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x));
                    return static_cast<unsigned char>(x * 255);
                };
                data[4 * i + 0] = q(v.x);
                data[4 * i + 1] = q(v.y);
                data[4 * i + 2] = q(v.z);
                data[4 * i + 3] = 255;
            }
        }
        SaveBMP(data.data(), w, h, path.c_str());
    }

    // Interactive frame into device buffers (the reference's Camera::Render).
    void Render(float3* target, float3* oddTarget, float3* evenTarget, pg::PathGuidingSample* sampleTarget,
                denoise::ScreenGBuffer* screenGBuffer, denoise::ScreenStatisticsBuffer* screenStatisticsBuffer,
                unsigned int* target2, const int2 size, const int frame, const int tone = 2) const
    {
        sceneRenderer_->Render(target, target2, size, GetPosition(), GetDirection(), frame, tone, oddTarget,
                               evenTarget, sampleTarget, screenGBuffer, screenStatisticsBuffer);
    }
};

