// scene_types.h -- device-resident scene layout (shared by host builder and kernels).
//
// HBM layout of one scene (all arrays 16-byte aligned, read with 128-bit loads):
//   WideNode  nodes[]     80 B  8-wide BVH node, child boxes quantised to 8 bits
//   PrimRec   prims[]     48 B  leaf-ordered primitive: world-space v0, e1, e2 of a
//                               triangle (the exact operands of the reference's
//                               Moller-Trumbore test) or a reference to an
//                               analytic object
//   ObjInfo   objects[]   16 B  per reference SceneObject: type, material, light, aux
//   TriShade  trishade[]  48 B  world vertex normals of triangle objects (shading)
//   Analytic  analytic[] 112 B  cube / sphere / SDF transform records
//   SdfRec    sdf[]       64 B  SDF objects (tested after the BVH), volume grids
//   MaterialRec materials[] 64 B  de-duplicated materials
//   lights: object index + selection probability, in object order
#pragma once

#include <cstdint>

namespace ar {

constexpr int kWide = 8;
constexpr uint8_t kMetaEmpty = 0xFF;
constexpr uint8_t kMetaInternal = 0x80;  // | rank of the internal child (0..7)
// leaf meta: ((count - 1) << 5) | offset, count 1..4, offset 0..28

struct alignas(16) WideNode {
    float ox, oy, oz;        // quantisation origin
    uint32_t exps;           // ex | ey << 8 | ez << 16 (biased exponents, scale = 2^(e-127))
    uint32_t child_base;     // first internal child (wide node index)
    uint32_t prim_base;      // first primitive of the leaf children
    uint32_t meta_lo;        // meta bytes of slots 0..3
    uint32_t meta_hi;        // meta bytes of slots 4..7
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "WideNode must be 80 bytes");

enum : int32_t { kPrimTriangle = 0, kPrimAnalytic = 1 };

struct alignas(16) PrimRec {
    float v0[3]; int32_t object;
    float e1[3]; int32_t kind;
    float e2[3]; int32_t pad;
};
static_assert(sizeof(PrimRec) == 48, "PrimRec must be 48 bytes");

struct alignas(16) ObjInfo {
    int32_t type;      // AR_OBJ_*
    int32_t material;  // index into materials
    int32_t light;     // light index or -1
    int32_t aux;       // triangle: index into trishade; analytic: index into analytic
};

struct alignas(16) TriShade {
    float n0[3], n1[3], n2[3];
    float pad[3];
};

struct alignas(16) Analytic {
    float center[3]; float radius;
    float extent[3]; float pad0;
    float o2w[9];
    float w2o[9];
    float pad1[2];
};
static_assert(sizeof(Analytic) == 112, "Analytic must be 112 bytes");

// Signed-distance object (SDF torus or sampled volume).  SDF objects are not
// BVH primitives: every query tests them after its BVH traversal (there are a
// few per scene, each behind its own box test).
enum : int32_t { kSdfTorus = 0, kSdfVolume = 1 };

struct alignas(16) SdfRec {
    int32_t object;         // scene object index
    int32_t analytic;       // centre, extent and matrices in analytic[]
    int32_t kind;           // kSdfTorus / kSdfVolume
    int32_t fp16;           // volume values stored as half floats
    float info[4];          // SDFInfo::sdfInfo0_
    int32_t dims[3];        // volume grid
    float voxel_size_max;   // SDFVolumeInfo::voxelSizeMax_
    const void* data;       // volume values (device), x fastest
    int32_t pad[2];
};
static_assert(sizeof(SdfRec) == 64, "SdfRec must be 64 bytes");

struct alignas(16) MaterialRec {
    int32_t model;
    float albedo[3];
    float emissive[3];
    float specular;
    float metallic, roughness, ior, sigma_a;
    float abbe, tilt;        // glass dispersion / absorption tilt (spectral mode)
    float pad[2];
};
static_assert(sizeof(MaterialRec) == 64, "MaterialRec must be 64 bytes");

}  // namespace ar
