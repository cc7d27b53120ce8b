// sdf.cuh -- signed-distance objects: the analytic torus and sampled volumes,
// sphere-traced inside the object's box (the reference's object/sdf/*.cuh).
//
// Functions are host+device so that the scene builder (camera-inside test)
// and the kernels evaluate the same arithmetic.  Rounding contract as
// everywhere: no FMA contraction, 1/sqrtf for normalisation.
//   sdf_torus          SdfTorus (sdf_torus.cuh:14-18)
//   grid_*             SampleSDFNearest01 / SampleSDFTrilinear01 /
//                      SampleSDFAdaptive01 (sdf_volume.cuh:69-162)
//   sdf_eval           SDFTorusFunctor / SDFVolumeFunctor (u + 0.5 into [0,1]^3)
//   sdf_march          IntersectSDFObject + RaymarchLocal (sdf_base.cuh:54-163):
//                      box entry, sphere tracing up to 512 steps with step
//                      max(|d|, eps/2) (volumes: max(0.9|d|, eps/2)), hit when
//                      the distance changes sign to within SDF_EPS(depth)
//   sdf_surface        hit position and central-difference normal
//                      (sdfNormalUnit, UnitNormalToLocal, sdf_base.cuh:29-52)
#pragma once

#include <cuda_fp16.h>

#include "detmath.h"
#include "scene_types.h"

namespace ar {

constexpr int kSdfSteps = 512;               // SDF_STEPS (config.cuh:75)
constexpr float kSdfVolumeStepScale = 0.9f;  // SDF_VOLUME_STEP_SCALE (config.cuh:76)
constexpr float kSdfNearestScale = 2.5f;     // SDF_VOLUME_USE_NEAREST_SCALE (config.cuh:77)

AR_HD float sdf_torus(f3 u, float R, float r)
{
    const float qx = sqrtf(u.x * u.x + u.z * u.z) - R;
    return sqrtf(qx * qx + u.y * u.y) - r;
}

// One value of a volume grid (host or device memory, float or half).
AR_HD float grid_value(const SdfRec& g, size_t i)
{
#ifdef __CUDA_ARCH__
    if (g.fp16) return __half2float(__ldg(static_cast<const __half*>(g.data) + i));
    return __ldg(static_cast<const float*>(g.data) + i);
#else
    if (g.fp16) return __half2float(static_cast<const __half*>(g.data)[i]);
    return static_cast<const float*>(g.data)[i];
#endif
}

AR_HD size_t grid_index(int x, int y, int z, const SdfRec& g)
{
    return static_cast<size_t>(z) * g.dims[0] * g.dims[1] + static_cast<size_t>(y) * g.dims[0] + x;
}

AR_HD int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

AR_HD float grid_nearest(f3 p, const SdfRec& g)
{
    const f3 q = mk(p.x * static_cast<float>(g.dims[0] - 1), p.y * static_cast<float>(g.dims[1] - 1),
                    p.z * static_cast<float>(g.dims[2] - 1));
    const int x = clampi(static_cast<int>(floorf(q.x + 0.5f)), 0, g.dims[0] - 1);
    const int y = clampi(static_cast<int>(floorf(q.y + 0.5f)), 0, g.dims[1] - 1);
    const int z = clampi(static_cast<int>(floorf(q.z + 0.5f)), 0, g.dims[2] - 1);
    return grid_value(g, grid_index(x, y, z, g));
}

AR_HD float grid_trilinear(f3 p, const SdfRec& g)
{
    const f3 q = mk(p.x * static_cast<float>(g.dims[0] - 1), p.y * static_cast<float>(g.dims[1] - 1),
                    p.z * static_cast<float>(g.dims[2] - 1));
    int x0 = static_cast<int>(floorf(q.x)), y0 = static_cast<int>(floorf(q.y)), z0 = static_cast<int>(floorf(q.z));
    const int x1 = clampi(x0 + 1, 0, g.dims[0] - 1);
    const int y1 = clampi(y0 + 1, 0, g.dims[1] - 1);
    const int z1 = clampi(z0 + 1, 0, g.dims[2] - 1);
    x0 = clampi(x0, 0, g.dims[0] - 1);
    y0 = clampi(y0, 0, g.dims[1] - 1);
    z0 = clampi(z0, 0, g.dims[2] - 1);
    const float fx = fminf(fmaxf(q.x - static_cast<float>(x0), 0.0f), 1.0f);
    const float fy = fminf(fmaxf(q.y - static_cast<float>(y0), 0.0f), 1.0f);
    const float fz = fminf(fmaxf(q.z - static_cast<float>(z0), 0.0f), 1.0f);
    const float c000 = grid_value(g, grid_index(x0, y0, z0, g)), c100 = grid_value(g, grid_index(x1, y0, z0, g));
    const float c010 = grid_value(g, grid_index(x0, y1, z0, g)), c110 = grid_value(g, grid_index(x1, y1, z0, g));
    const float c001 = grid_value(g, grid_index(x0, y0, z1, g)), c101 = grid_value(g, grid_index(x1, y0, z1, g));
    const float c011 = grid_value(g, grid_index(x0, y1, z1, g)), c111 = grid_value(g, grid_index(x1, y1, z1, g));
    const float c00 = c000 * (1.0f - fx) + c100 * fx;
    const float c10 = c010 * (1.0f - fx) + c110 * fx;
    const float c01 = c001 * (1.0f - fx) + c101 * fx;
    const float c11 = c011 * (1.0f - fx) + c111 * fx;
    const float c0 = c00 * (1.0f - fy) + c10 * fy;
    const float c1 = c01 * (1.0f - fy) + c11 * fy;
    return c0 * (1.0f - fz) + c1 * fz;
}

// Distance at u in the object's unit box [-0.5, 0.5]^3.
AR_HD float sdf_eval(const SdfRec& g, f3 u)
{
    if (g.kind == kSdfTorus) return sdf_torus(u, g.info[0], g.info[1]);
    if (!g.data || g.dims[0] * g.dims[1] * g.dims[2] == 0) return 1.0e20f;
    const f3 p = mk(u.x + 0.5f, u.y + 0.5f, u.z + 0.5f);
    const float dn = grid_nearest(p, g);
    return fabsf(dn) > g.voxel_size_max ? dn : grid_trilinear(p, g);
}

AR_HD f3 to_unit(f3 pl, f3 e)
{
    const float ex = fmaxf(e.x, 1e-8f), ey = fmaxf(e.y, 1e-8f), ez = fmaxf(e.z, 1e-8f);
    return mk(pl.x / (2.0f * ex), pl.y / (2.0f * ey), pl.z / (2.0f * ez));
}

AR_HD m3 m3_of(const float* m)
{
    m3 r;
    r.x = mk(m[0], m[1], m[2]);
    r.y = mk(m[3], m[4], m[5]);
    r.z = mk(m[6], m[7], m[8]);
    return r;
}

// Sphere-traced hit distance along the normalised local ray, or -1.  eps_isect
// is INTERSECT_EPS(depth) of the query; SDF_EPS = eps_isect / 2 (config.cuh:73).
AR_HD float sdf_march(const SdfRec& g, const Analytic& an, f3 ro, f3 rd, float eps_isect)
{
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    const m3 w2o = m3_of(an.w2o);
    const f3 lo = mul(w2o, ro - c);
    const f3 ld = normalize(mul(w2o, rd));
    const f3 dv = mk(inv_safe(ld.x), inv_safe(ld.y), inv_safe(ld.z));
    const f3 t1 = (-e - lo) * dv;
    const f3 t2 = (e - lo) * dv;
    const f3 tmn = vmin(t1, t2), tmx = vmax(t1, t2);
    const float tEnter = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
    const float tExit = fminf(fminf(tmx.x, tmx.y), tmx.z);
    if (tEnter > tExit || tExit <= 0.0f) return -1.0f;
    const float eps = eps_isect * 0.5f;
    const float minStep = eps * 0.5f;
    const float scale = g.kind == kSdfVolume ? kSdfVolumeStepScale : 1.0f;
    const bool startInside = sdf_eval(g, to_unit(lo, e)) <= 0.0f;
    const float sMin = 2.0f * fminf(e.x, fminf(e.y, e.z));
    float t = fmaxf(0.0f, tEnter);
    for (int i = 0; i < kSdfSteps; ++i) {
        const float tLast = t;
        const f3 pl = lo + ld * t;
        const float dLocal = sdf_eval(g, to_unit(pl, e)) * sMin;
        if (startInside ? (dLocal > 0.0f && dLocal < eps) : (dLocal < 0.0f && -dLocal < eps)) return tLast;
        const float adv = g.kind == kSdfVolume ? fmaxf(fabsf(dLocal) * scale, minStep) : fmaxf(fabsf(dLocal), minStep);
        t += adv;
        if (t > tExit) break;
    }
    return -1.0f;
}

// World position and normal of a hit at distance t (from sdf_march).
AR_HD void sdf_surface(const SdfRec& g, const Analytic& an, f3 ro, f3 rd, float t, float eps_isect, f3* pos, f3* nrm)
{
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    const m3 w2o = m3_of(an.w2o), o2w = m3_of(an.o2w);
    const f3 lo = mul(w2o, ro - c);
    const f3 ld = normalize(mul(w2o, rd));
    const f3 pl = lo + ld * t;
    const float sMin = 2.0f * fminf(e.x, fminf(e.y, e.z));
    const float h = (eps_isect * 0.5f) / fmaxf(sMin, 1e-8f);
    const f3 u = to_unit(pl, e);
    const float dx = sdf_eval(g, u + mk(h, 0.0f, 0.0f)) - sdf_eval(g, u - mk(h, 0.0f, 0.0f));
    const float dy = sdf_eval(g, u + mk(0.0f, h, 0.0f)) - sdf_eval(g, u - mk(0.0f, h, 0.0f));
    const float dz = sdf_eval(g, u + mk(0.0f, 0.0f, h)) - sdf_eval(g, u - mk(0.0f, 0.0f, h));
    const f3 nu = normalize(mk(dx, dy, dz));
    const float ex = fmaxf(e.x, 1e-8f), ey = fmaxf(e.y, 1e-8f), ez = fmaxf(e.z, 1e-8f);
    const f3 nl = normalize(mk(nu.x / (2.0f * ex), nu.y / (2.0f * ey), nu.z / (2.0f * ez)));
    *pos = mul(o2w, pl) + c;
    *nrm = normalize(mul(o2w, nl));
}

// OverlapSDFObject (sdf_base.cuh:166-177): p inside the surface.
AR_HD bool sdf_contains(const SdfRec& g, const Analytic& an, f3 p)
{
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    return sdf_eval(g, to_unit(mul(m3_of(an.w2o), p - c), e)) <= 0.0f;
}

// The values FillSDFVolume (object/sdf/sdf_cache_manager.cuh:16-38) writes for
// the torus functor: grid point (x, y, z) at pos01 = index / (dims - 1), minus 0.5.
AR_HD float torus_fill_value(int x, int y, int z, const int dims[3], float R, float r)
{
    const float nx = dims[0] > 1 ? static_cast<float>(x) / static_cast<float>(dims[0] - 1) : 0.0f;
    const float ny = dims[1] > 1 ? static_cast<float>(y) / static_cast<float>(dims[1] - 1) : 0.0f;
    const float nz = dims[2] > 1 ? static_cast<float>(z) / static_cast<float>(dims[2] - 1) : 0.0f;
    return sdf_torus(mk(nx - 0.5f, ny - 0.5f, nz - 0.5f), R, r);
}

// SDFVolumeInfo::ComputeVoxelSize (sdf_volume.cuh:24-44)
AR_HD float voxel_size_max(const int dims[3])
{
    const f3 inv = mk(1.0f / fmaxf(static_cast<float>(dims[0]), 1.0f), 1.0f / fmaxf(static_cast<float>(dims[1]), 1.0f),
                      1.0f / fmaxf(static_cast<float>(dims[2]), 1.0f));
    return length(inv) * kSdfNearestScale;
}

}  // namespace ar
