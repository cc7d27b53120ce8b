// scene_build.h -- host-side scene ingest and BVH construction.
#pragma once

#include <cstddef>
#include <string>
#include <vector>

#include "../../include/aperture_b200.h"
#include "detmath.h"
#include "scene_types.h"

namespace ar {

// A signed-distance volume as uploaded: float or half values, x fastest.
struct float4_ { float x, y, z, w; };

struct HostVolume {
    int dims[3] = {0, 0, 0};
    bool fp16 = false;
    std::vector<unsigned char> bytes;
    float voxel_size_max = 0.0f;
};

struct HostScene {
    std::vector<ObjInfo> objects;
    std::vector<TriShade> trishade;
    std::vector<Analytic> analytic;
    std::vector<MaterialRec> materials;
    std::vector<PrimRec> prims;
    std::vector<WideNode> nodes;
    std::vector<SdfRec> sdf;           // data pointers index `volumes` until upload
    std::vector<HostVolume> volumes;
    std::vector<float4_> light_tri;        // per light: v0 + area, e1, e2 (world; triangles only)
    std::vector<int32_t> light_object;
    std::vector<float> light_prob;
    int64_t triangles = 0;
    int stack_bound = 0;      // exact worst-case traversal stack depth
    int wide_depth = 0;
    bool root_leaf_only = false;
};

// Ingest the reference SceneObject fields (object.cuh:254-364) and build the
// scene: world-space triangles, light table (scene.cu:1056-1080), SAH BVH
// collapsed to 8-wide quantised nodes.  Throws std::runtime_error on invalid
// input.
HostScene build_scene(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes = nullptr,
                      size_t volume_count = 0);

// objectToWorld = Rz * (Ry * Rx) from Euler degrees with host libm, exactly as
// the SceneObject constructor (object.cuh:344-364, vector.cuh:378-416).
void euler_matrices(f3 deg, m3* o2w, m3* w2o);

}  // namespace ar
