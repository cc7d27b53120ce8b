// A caller of the reference's C++ API, compiled against the shim header
// (include/aperture_b200_renderer.hpp); run by tests/test_cpu_shim.py and
// tests/test_gpu_shim.py.
//
//   shim_render OUTDIR WIDTH HEIGHT SPP
//
// Builds a Cornell-style scene with the reference's factories (triangle walls,
// a rotated GGX cube, a glass sphere, a thin cube light), then
//   OUTDIR/objects.bin  the ar_object_desc array the shim hands to the library
//   OUTDIR/image.f32    SceneRenderer::Render(size, origin, direction, SPP)
//   OUTDIR/shot.bmp     Camera::RenderToFile(OUTDIR/shot, SPP, ACES, 1.3)
//   OUTDIR/custom.bmp   Camera::RenderToFile with a host tone function
//   OUTDIR/frames.f32   interactive Render, 3 frames into device buffers
//                       (hdr after frame 2, then the ldr words as floats' bits)
// and prints "shim done".
#include <cstdio>
#include <string>
#include <vector>

#include "aperture_b200_renderer.hpp"

namespace {

void quad(std::vector<SceneObject>& out, float3 a, float3 b, float3 c, float3 d, float3 n, const Material& m)
{
    AdditionalObjectInfo t1, t2;
    t1.triangleInfo_ = {{a, n, {0, 0}}, {b, n, {1, 0}}, {c, n, {1, 1}}};
    t2.triangleInfo_ = {{a, n, {0, 0}}, {c, n, {1, 1}}, {d, n, {0, 1}}};
    out.emplace_back(float3{0, 0, 0}, float3{0, 0, 0}, m, float3{0, 0, 0}, EObjectType::OBJ_TRIANGLE, t1);
    out.emplace_back(float3{0, 0, 0}, float3{0, 0, 0}, m, float3{0, 0, 0}, EObjectType::OBJ_TRIANGLE, t2);
}

std::vector<SceneObject> make_scene()
{
    std::vector<SceneObject> s;
    const float h = 0.5f;
    const Material grey = Material::CreateDiffusePureColor({0.73f, 0.73f, 0.73f});
    quad(s, {-h, -h, -h}, {-h, -h, h}, {h, -h, h}, {h, -h, -h}, {0, 1, 0}, grey);
    quad(s, {-h, h, -h}, {h, h, -h}, {h, h, h}, {-h, h, h}, {0, -1, 0}, grey);
    quad(s, {-h, -h, -h}, {h, -h, -h}, {h, h, -h}, {-h, h, -h}, {0, 0, 1}, grey);
    quad(s, {-h, -h, -h}, {-h, h, -h}, {-h, h, h}, {-h, -h, h}, {1, 0, 0},
         Material::CreateDiffusePureColor({0.65f, 0.05f, 0.05f}));
    quad(s, {h, -h, -h}, {h, -h, h}, {h, h, h}, {h, h, -h}, {-1, 0, 0},
         Material::CreateDiffusePureColor({0.12f, 0.45f, 0.15f}));
    s.emplace_back(float3{0.17f, -0.35f, -0.1f}, float3{0.15f, 0.15f, 0.15f},
                   Material::CreateGGXPureColor({0.9f, 0.6f, 0.3f}, 0.3f, 1.0f, 0.5f), float3{0, 25.0f, 0});
    s.emplace_back(float3{-0.18f, -0.3f, 0.05f}, float3{0.2f, 0.2f, 0.2f},
                   Material::CreateGlassPureColor({0.95f, 0.95f, 0.95f}, 1.5f, 0.5f), float3{0, 0, 0},
                   EObjectType::OBJ_SPHERE);
    s.emplace_back(float3{0.0f, h - 0.01f, 0.0f}, float3{0.125f, 0.01f, 0.125f},
                   Material::CreateLight({17.0f, 12.0f, 4.0f}), float3{0, 0, 0});
    return s;
}

float3 custom_tone(const float3 c) { return float3{c.x / (1.0f + c.x), c.y / (1.0f + c.y), c.z / (1.0f + c.z)}; }

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 5) {
        std::fprintf(stderr, "usage: shim_render OUTDIR WIDTH HEIGHT SPP\n");
        return 2;
    }
    const std::string dir = argv[1];
    const int w = std::atoi(argv[2]), hgt = std::atoi(argv[3]), spp = std::atoi(argv[4]);
    const std::vector<SceneObject> scene = make_scene();
    {
        FILE* f = std::fopen((dir + "/objects.bin").c_str(), "wb");
        for (const SceneObject& o : scene) {
            const ar_object_desc d = o.ToDesc();
            std::fwrite(&d, sizeof(d), 1, f);
        }
        std::fclose(f);
    }
    SceneRenderer renderer(scene);
    const float3 origin{0.0f, 0.0f, 1.9f}, direction{0.0f, 0.0f, -1.0f};
    const std::vector<float3> img = renderer.Render(int2{w, hgt}, origin, direction, spp);
    {
        FILE* f = std::fopen((dir + "/image.f32").c_str(), "wb");
        std::fwrite(img.data(), sizeof(float3), img.size(), f);
        std::fclose(f);
    }
    Camera camera(renderer, "shim camera", w, hgt, origin, direction);
    camera.RenderToFile(dir + "/shot", spp, ACES, 1.3f);
    camera.RenderToFile(dir + "/custom", spp, custom_tone, 1.0f);

    // interactive: three frames into device buffers
    const size_t n = static_cast<size_t>(w) * hgt;
    float3* hdr = nullptr;
    unsigned int* ldr = nullptr;
    std::vector<float> frames(n * 4, 0.0f);
    if (cudaMalloc(reinterpret_cast<void**>(&hdr), n * sizeof(float3)) == cudaSuccess &&
        cudaMalloc(reinterpret_cast<void**>(&ldr), n * sizeof(unsigned int)) == cudaSuccess) {
        for (int frame = 0; frame < 3; ++frame)
            camera.Render(hdr, nullptr, nullptr, nullptr, nullptr, nullptr, ldr, int2{w, hgt}, frame, 2);
        cudaMemcpy(frames.data(), hdr, n * sizeof(float3), cudaMemcpyDeviceToHost);
        cudaMemcpy(frames.data() + 3 * n, ldr, n * sizeof(unsigned int), cudaMemcpyDeviceToHost);
        cudaFree(hdr);
        cudaFree(ldr);
    } else {
        cudaGetLastError();
        std::printf("no device buffers for the interactive render\n");
    }
    {
        FILE* f = std::fopen((dir + "/frames.f32").c_str(), "wb");
        std::fwrite(frames.data(), sizeof(float), frames.size(), f);
        std::fclose(f);
    }
    std::printf("shim done\n");
    return 0;
}
