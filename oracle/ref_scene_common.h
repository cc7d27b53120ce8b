// ref_scene_common.h -- scene conversion shared by the two reference harnesses
// (ref_harness.cu: queries from the pristine sources; ref_path_harness.cu: the
// path loop from the build-time copy).  TEST INFRASTRUCTURE ONLY.
//
// An ar_object_desc becomes the reference's SceneObject through its own
// constructor (core/render/object.cuh:344-364); the BVH is the reference's
// BuildBVH (core/bvh/bvh.cuh:142-422) over the objects' proxies; the light
// table repeats the loop of UpdateSceneToDeviceIfDirty (core/scene.cu:1046-1080)
// over the reference's GetArea * GetEmissivePower, because scene.cu itself
// needs OptiX and the GUI.
#pragma once
#include <vector>

#include "../include/aperture_b200.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

float3 f3(const ar_vec3& v) { return make_float3(v.x, v.y, v.z); }

Material material_of(const ar_material& m)
{
    Material r = {};
    r.shadingModel_ = static_cast<EShadingModel>(m.shading_model);
    r.texture_.textureType_ = ETextureType::TEX_PURE_COLOR;
    GBuffer& g = r.texture_.baseTexture_;
    g.albedo_ = f3(m.albedo);
    g.emissive_ = f3(m.emissive);
    g.specular_ = m.specular;
    g.metallic_ = m.metallic;
    g.roughness_ = m.roughness;
    g.IOR_ = m.ior;
    g.sigmaA_ = m.sigma_a;
    g.abbeNumber_ = m.abbe_number;
    g.tiltNumber_ = m.tilt_number;
    return r;
}

SceneObject object_of(const ar_object_desc& d)
{
    AdditionalObjectInfo info = {};
    if (d.type == AR_OBJ_SDF) {
        info.sdfType_ = d.sdf.kind == AR_SDF_TORUS ? ESDFType::SDF_TORUS : ESDFType::SDF_VOLUME;
        info.sdfInfo_.sdfInfo0_ = make_float4(d.sdf.info[0], d.sdf.info[1], d.sdf.info[2], d.sdf.info[3]);
        info.sdfInfo_.cachedVolumeIndex_ = d.sdf.volume;
    }
    if (d.type == AR_OBJ_TRIANGLE) {
        Vertex* v[3] = {&info.triangleInfo_.v0_, &info.triangleInfo_.v1_, &info.triangleInfo_.v2_};
        for (int k = 0; k < 3; ++k) {
            v[k]->position_ = f3(d.tri[k].position);
            v[k]->normal_ = f3(d.tri[k].normal);
            v[k]->uv_ = make_float2(d.tri[k].u, d.tri[k].v);
        }
    }
    SceneObject o(f3(d.center), f3(d.extent), material_of(d.material), f3(d.rotation_deg),
                  static_cast<EObjectType>(d.type), info);
    o.bVisible_ = d.visible != 0;
    return o;
}

int thread_count(int threads)
{
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

}  // namespace

struct ref_scene_data {
    std::vector<SceneObject> objects;
    BVHHost bvh;
    std::vector<AdditionalLightInfo> lights;
};


inline void ref_build_scene(const ar_object_desc* objects, size_t count, int leaf_size, int bin_count,
                            ref_scene_data* s)
{
    s->objects.reserve(count);
    for (size_t i = 0; i < count; ++i) s->objects.push_back(object_of(objects[i]));
    std::vector<PrimitiveProxy> proxies;
    proxies.reserve(count);
    for (const SceneObject& o : s->objects) proxies.push_back(o.proxy_);
    s->bvh = BuildBVH(proxies, leaf_size, bin_count);
    float total = 0.0f;
    for (size_t i = 0; i < s->objects.size(); ++i) {
        SceneObject& o = s->objects[i];
        o.objectIndex_ = static_cast<int>(i);
        if (o.material_.shadingModel_ == EShadingModel::MAT_LIGHT) {
            o.lightIndex_ = static_cast<int>(s->lights.size());
            AdditionalLightInfo li;
            li.objectIndex_ = static_cast<int>(i);
            li.importanceWeight_ = fmaxf(o.GetArea() * o.GetEmissivePower(), 1.0e-20f);
            total += li.importanceWeight_;
            s->lights.push_back(li);
        } else {
            o.lightIndex_ = -1;
        }
    }
    for (AdditionalLightInfo& li : s->lights) li.selectProb_ = li.importanceWeight_ / total;
}
