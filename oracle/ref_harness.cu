// ref_harness.cu -- drives the reference renderer's own host-callable code, to
// pin the C restatement (oracle.c).  TEST INFRASTRUCTURE ONLY: built by
// `make -C oracle ref` into oracle/_ref/libref.so from the reference's headers
// where they lie (include path REF_CORE), never shipped, loaded only by the
// fixture generator under tests/golden/ and by pinning tests.
//
// Everything called here is the reference's code, unchanged:
//   SceneObject(center, extent, material, rotation, type, info)
//       core/render/object.cuh:344-364 (world transform, BVH proxy)
//   SceneObject::GetArea / GetEmissivePower   core/render/object.cuh:270-306
//   BuildBVH                                  core/bvh/bvh.cuh:142-422
//   intersection::TraverseBVH<bAnyHit>        core/render/intersection.cuh:235-370
//   intersection::AnyHitSegmentBVH            core/render/intersection.cuh:372-397
//   intersection::Intersect (linear scan)     core/render/intersection.cuh:175-205
//   IntersectBase, sdf::IntersectSDFObject    core/render/intersection.cuh:93-113,
//       core/object/sdf/sdf_base.cuh:54-163 (torus and volume functors)
//   intersection::Overlap                     core/render/intersection.cuh:399-414
//   BSDF_PDF (RGB)                            core/render/material.cuh:332-387
//   Gamma, ACES, XYZ2SRGBLinearD65            core/tonemap.cuh (the per-pixel steps of
//       the Tonemap kernel around them, core/scene.cu:180-199, are repeated below:
//       scene.cu itself needs OptiX and the GUI)
// The light table follows UpdateSceneToDeviceIfDirty (core/scene.cu:1046-1080):
// this file repeats its loop because scene.cu itself needs OptiX and the GUI.
#include <cstdint>
#include <vector>

#include "bvh/bvh.cuh"
#include "render/intersection.cuh"
#include "render/material.cuh"
#include "tonemap.cuh"
#include "spectrum/ciexyz.cuh"
#include "spectrum/sample_ciexyz.cuh"

#include "ref_scene_common.h"

// The SDF cache pointers the reference declares extern (object/sdf/sdf_master.cuh:12-13);
// scene.cu defines them in the reference build.  No SDF object is used here.
namespace sdf {
__device__ SDFVolumeInfo* cachedSDFInfoPtrs = nullptr;
__device__ uint32_t cachedSDFInfoPtrsCount = 0;
}  // namespace sdf

struct ref_scene : ref_scene_data {};

extern "C" {

ref_scene* ref_scene_create(const ar_object_desc* objects, size_t count, int leaf_size, int bin_count)
{
    ref_scene* s = new ref_scene;
    ref_build_scene(objects, count, leaf_size, bin_count, s);
    return s;
}

void ref_scene_destroy(ref_scene* s) { delete s; }

int64_t ref_scene_node_count(const ref_scene* s) { return static_cast<int64_t>(s->bvh.nodes_.size()); }

void ref_scene_nodes(const ref_scene* s, float* b6, int32_t* l4)
{
    for (size_t i = 0; i < s->bvh.nodes_.size(); ++i) {
        const BVHNode& n = s->bvh.nodes_[i];
        b6[6 * i + 0] = n.boundMin_.x; b6[6 * i + 1] = n.boundMin_.y; b6[6 * i + 2] = n.boundMin_.z;
        b6[6 * i + 3] = n.boundMax_.x; b6[6 * i + 4] = n.boundMax_.y; b6[6 * i + 5] = n.boundMax_.z;
        l4[4 * i + 0] = n.left_; l4[4 * i + 1] = n.right_; l4[4 * i + 2] = n.first_; l4[4 * i + 3] = n.count_;
    }
}

void ref_scene_indices(const ref_scene* s, int32_t* idx)
{
    for (size_t i = 0; i < s->bvh.objectIndices_.size(); ++i) idx[i] = s->bvh.objectIndices_[i];
}

int64_t ref_scene_light_count(const ref_scene* s) { return static_cast<int64_t>(s->lights.size()); }

void ref_scene_lights(const ref_scene* s, int32_t* object_index, float* select_prob)
{
    for (size_t i = 0; i < s->lights.size(); ++i) {
        object_index[i] = s->lights[i].objectIndex_;
        select_prob[i] = s->lights[i].selectProb_;
    }
}

// Rays as 8 floats (origin, tmin, direction, tmax).  mode 0: TraverseBVH over
// the reference BVH; mode 1: the linear Intersect scan.  Closest hits also
// return the hit position, normal and inside flag.
void ref_trace_rays(const ref_scene* s, const float* rays, int64_t n, int any_hit, int mode, int32_t* hit_object,
                    float* hit_t, float* pos, float* nrm, int32_t* inside, int threads)
{
    const intersection::SceneObjectsIntersector isect{s->objects.data(), static_cast<int>(s->objects.size())};
    const BVHNode* nodes = s->bvh.nodes_.data();
    const int node_count = static_cast<int>(s->bvh.nodes_.size());
    const int* indices = s->bvh.objectIndices_.data();
#pragma omp parallel for schedule(dynamic, 256) num_threads(thread_count(threads))
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        const float3 o = make_float3(q[0], q[1], q[2]);
        const float3 d = make_float3(q[4], q[5], q[6]);
        IntersectionContext c;
        if (mode == 1)
            c = intersection::Intersect(0, o, d, isect, -1, q[3], q[7]);
        else if (any_hit)
            c = intersection::TraverseBVH<true>(0, o, d, isect, nodes, node_count, indices, q[3], q[7]);
        else
            c = intersection::TraverseBVH<false>(0, o, d, isect, nodes, node_count, indices, q[3], q[7]);
        hit_object[i] = c.bHit_ ? c.objectIndex_ : -1;
        if (hit_t) hit_t[i] = c.bHit_ ? c.distance_ : q[7];
        if (pos) { pos[3 * i] = c.bHit_ ? c.hitPosition_.x : 0.0f; pos[3 * i + 1] = c.bHit_ ? c.hitPosition_.y : 0.0f; pos[3 * i + 2] = c.bHit_ ? c.hitPosition_.z : 0.0f; }
        if (nrm) { nrm[3 * i] = c.bHit_ ? c.hitNormal_.x : 0.0f; nrm[3 * i + 1] = c.bHit_ ? c.hitNormal_.y : 0.0f; nrm[3 * i + 2] = c.bHit_ ? c.hitNormal_.z : 0.0f; }
        if (inside) inside[i] = c.bHit_ ? static_cast<int32_t>(c.isInside_) : 0;
    }
}

// AnyHitSegmentBVH for segments src.xyz, dst.xyz at the given loop depth.
void ref_segments_occluded(const ref_scene* s, const float* seg6, const int32_t* depth, int64_t n,
                           int32_t* occluded, int threads)
{
    const intersection::SceneObjectsIntersector isect{s->objects.data(), static_cast<int>(s->objects.size())};
    const BVHNode* nodes = s->bvh.nodes_.data();
    const int node_count = static_cast<int>(s->bvh.nodes_.size());
    const int* indices = s->bvh.objectIndices_.data();
#pragma omp parallel for schedule(dynamic, 256) num_threads(thread_count(threads))
    for (int64_t i = 0; i < n; ++i) {
        const float* q = seg6 + 6 * i;
        const IntersectionContext c = intersection::AnyHitSegmentBVH(
            depth[i], make_float3(q[0], q[1], q[2]), make_float3(q[3], q[4], q[5]), isect, nodes, node_count, indices);
        occluded[i] = c.bHit_ ? 1 : 0;
    }
}

void ref_overlap(const ref_scene* s, const float* p3, int64_t n, int32_t* object_index)
{
    for (int64_t i = 0; i < n; ++i) {
        const OverlapContext c = intersection::Overlap(make_float3(p3[3 * i], p3[3 * i + 1], p3[3 * i + 2]),
                                                       s->objects.data(), static_cast<int>(s->objects.size()));
        object_index[i] = c.bOverlap_ ? c.objectIndex_ : -1;
    }
}

float ref_bsdf_pdf(int model, const ar_material* m, const float* N, const float* ray_dir, const float* L)
{
    const GBuffer g = material_of(*m).texture_.baseTexture_;
    return BSDF_PDF(static_cast<EShadingModel>(model), g, make_float3(0.0f, 0.0f, 0.0f), make_float3(N[0], N[1], N[2]),
                    make_float3(ray_dir[0], ray_dir[1], ray_dir[2]), make_float3(L[0], L[1], L[2]));
}

// The default branch of the Tonemap kernel (core/scene.cu:180-199) per pixel;
// exposure is the kernel's __device__ `exposure` (SetExposure).
void ref_tonemap(const float* rgb, int64_t n, int tone, float exposure, int xyz_input, uint32_t* out)
{
    for (int64_t i = 0; i < n; ++i) {
        const float3 in = make_float3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        const float3 result = xyz_input ? XYZ2SRGBLinearD65(in) : in;
        float3 value = result * exposure;
        if (tone == 1) value = Gamma(value);
        else if (tone == 2) value = ACES(value);
        const unsigned int red = static_cast<unsigned int>(255.0f * saturate_(value.x));
        const unsigned int green = static_cast<unsigned int>(255.0f * saturate_(value.y));
        const unsigned int blue = static_cast<unsigned int>(255.0f * saturate_(value.z));
        out[i] = 0xff000000u | (red << 16) | (green << 8) | blue;
    }
}

// One object's intersection at loop depth `depth` (IntersectBase, with the
// volume functor of sdf_volume.cuh built on a host grid for SDF volumes: the
// reference reads its volumes through a device-only pointer table).  Rays as
// for ref_trace_rays (tmin/tmax ignored); t = -1 on a miss.
void ref_object_isect(const ref_scene* s, int32_t obj, const float* grid, const int32_t* dims, const float* rays,
                      int64_t n, int32_t depth, float* t, float* pos, float* nrm)
{
    const SceneObject& o = s->objects[static_cast<size_t>(obj)];
    sdf::SDFVolumeInfo vi{};
    const bool volume = o.type_ == EObjectType::OBJ_SDF && o.additionalObjectInfo_.sdfType_ == ESDFType::SDF_VOLUME;
    if (volume) {
        vi.volumePtr_ = const_cast<float*>(grid);
        vi.dim_ = make_int3(dims[0], dims[1], dims[2]);
        vi.ComputeVoxelSize();
    }
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        const float3 ro = make_float3(q[0], q[1], q[2]), rd = make_float3(q[4], q[5], q[6]);
        const IntersectionContext c =
            volume ? sdf::IntersectSDFObject<sdf::SDFVolumeFunctor, true>(depth, ro, rd, o, sdf::SDFVolumeFunctor(vi))
                   : intersection::IntersectBase(depth, ro, rd, o);
        t[i] = c.bHit_ ? c.distance_ : -1.0f;
        pos[3 * i] = c.hitPosition_.x; pos[3 * i + 1] = c.hitPosition_.y; pos[3 * i + 2] = c.hitPosition_.z;
        nrm[3 * i] = c.hitNormal_.x; nrm[3 * i + 1] = c.hitNormal_.y; nrm[3 * i + 2] = c.hitNormal_.z;
        if (!c.bHit_) for (int k = 0; k < 3; ++k) pos[3 * i + k] = nrm[3 * i + k] = 0.0f;
    }
}

// The grid FillSDFVolume (object/sdf/sdf_cache_manager.cuh:16-38) writes for
// the torus functor, evaluated on the host with the reference's functor.
void ref_fill_torus(const int32_t* dims, float R, float r, float* out)
{
    const SDFInfo info{make_float4(R, r, 0.0f, 0.0f)};
    const sdf::SDFTorusFunctor f{};
    size_t i = 0;
    for (int z = 0; z < dims[2]; ++z)
        for (int y = 0; y < dims[1]; ++y)
            for (int x = 0; x < dims[0]; ++x, ++i) {
                const float nx = (dims[0] > 1) ? static_cast<float>(x) / static_cast<float>(dims[0] - 1) : 0.0f;
                const float ny = (dims[1] > 1) ? static_cast<float>(y) / static_cast<float>(dims[1] - 1) : 0.0f;
                const float nz = (dims[2] > 1) ? static_cast<float>(z) / static_cast<float>(dims[2] - 1) : 0.0f;
                out[i] = f(make_float3(nx, ny, nz) - 0.5f, info);
            }
}

// Spectral pieces, on the host: RGBEncode / LambdaEncode (spectrum_basis.cuh),
// SampleCIE1931 (sample_ciexyz.cuh), D65Norm and LambdaToCIE1931_XYZ
// (ciexyz.cuh), and the network weights as compiled (to check their extraction).
void ref_spectral_encode(const float* rgb, const float* lambda, int64_t n, float* rgb_k, float* lam_k)
{
    for (int64_t i = 0; i < n; ++i) {
        if (rgb) spectrum::query::RGBEncode(rgb + 3 * i, rgb_k + 4 * i);
        if (lambda) spectrum::query::LambdaEncode(lambda + i, lam_k + 4 * i);
    }
}

void ref_spectral_sample(const float* u3, int64_t n, float* lambda, float* pdf)
{
    for (int64_t i = 0; i < n; ++i) {
        const spectrum::sample::SpectrumSample smp =
            spectrum::sample::SampleCIE1931(make_float3(u3[3 * i], u3[3 * i + 1], u3[3 * i + 2]));
        lambda[i] = smp.lambda_;
        pdf[i] = smp.pdf_;
    }
}

void ref_spectral_weights(const float* lambda, int64_t n, float* d65, float* xyz)
{
    for (int64_t i = 0; i < n; ++i) {
        d65[i] = spectrum::D65Norm(lambda[i]);
        const float3 c = spectrum::LambdaToCIE1931_XYZ(lambda[i]);
        xyz[3 * i] = c.x; xyz[3 * i + 1] = c.y; xyz[3 * i + 2] = c.z;
    }
}

// The table block in ar_scene_set_spectral order (17780 floats).
void ref_spectral_tables(float* out)
{
    using namespace spectrum::query;
    size_t o = 0;
    auto put = [&](const float* a, size_t n) { for (size_t i = 0; i < n; ++i) out[o++] = a[i]; };
    for (int i = 0; i < spectrum::CIEXYZ_COUNT; ++i) {
        out[o++] = spectrum::CIEXYZ_CMF[i].x; out[o++] = spectrum::CIEXYZ_CMF[i].y; out[o++] = spectrum::CIEXYZ_CMF[i].z;
    }
    put(spectrum::D65_SPD, spectrum::D65_COUNT);
    put(RGB_IN_W, 1024); put(RGB_IN_B, 32);
    const float* rw[7] = {RGB_BLK0_W, RGB_BLK1_W, RGB_BLK2_W, RGB_BLK3_W, RGB_BLK4_W, RGB_BLK5_W, RGB_BLK6_W};
    const float* rb[7] = {RGB_BLK0_B, RGB_BLK1_B, RGB_BLK2_B, RGB_BLK3_B, RGB_BLK4_B, RGB_BLK5_B, RGB_BLK6_B};
    const float* lw[7] = {LAM_BLK0_W, LAM_BLK1_W, LAM_BLK2_W, LAM_BLK3_W, LAM_BLK4_W, LAM_BLK5_W, LAM_BLK6_W};
    const float* lb[7] = {LAM_BLK0_B, LAM_BLK1_B, LAM_BLK2_B, LAM_BLK3_B, LAM_BLK4_B, LAM_BLK5_B, LAM_BLK6_B};
    for (int k = 0; k < 7; ++k) put(rw[k], 1024);
    for (int k = 0; k < 7; ++k) put(rb[k], 32);
    put(RGB_OUT_W, 128);
    for (int k = 0; k < 7; ++k) put(lw[k], 1024);
    for (int k = 0; k < 7; ++k) put(lb[k], 32);
    put(LAM_OUT_W, 128);
}

// INTERSECT_EPS (config.cuh:3) as the reference's host pass evaluates it.
float ref_intersect_eps(int depth) { return INTERSECT_EPS(depth); }

}  // extern "C"
