// traverse.cuh -- sm_100a BVH traversal and primitive intersection.
//
// Replaces intersection::TraverseBVH (core/render/intersection.cuh:235-370) and
// the per-shape intersectors it calls.  One thread per ray; the traversal stack
// of each warp lives in shared memory, interleaved by lane (entry k of lane l at
// [k * 32 + l]) so pushes and pops are bank-conflict free.  Nodes are 80-byte
// 8-wide records read with five 128-bit read-only loads; the child boxes are
// decoded from 8-bit grid coordinates with one byte permute per plane and one
// packed two-lane FMA per axis (near and far plane together):
//     t(q) = fma(2^15 + q, a, b),  a = scale * inv_dir,
//     b = (origin - ray_origin) * inv_dir - 2^15 * a   (once per node).
// The box test is conservative (every child box is padded by a grid step on
// all sides, far distance widened by 2^-20 relative), so the set of primitives
// tested is a superset of the exact one and the closest hit equals a
// brute-force search.  Ties in t go to the lowest object index; the
// reference keeps the first primitive its traversal happens to find.
#pragma once

#include <cstdint>

#include "detmath.h"
#include "../../include/aperture_b200.h"
#include "scene_types.h"
#include "medium.cuh"
#include "sdf.cuh"

namespace ar {

struct SceneView {
    const WideNode* nodes;
    const PrimRec* prims;
    const ObjInfo* objects;
    const TriShade* trishade;
    const Analytic* analytic;
    const MaterialRec* materials;
    const int32_t* light_object;
    const float* light_prob;
    const SdfRec* sdf;       // SDF objects, tested after the BVH
    const float4* light_tri; // per light: v0 + area, e1, e2 (triangle lights)
    int32_t num_nodes;
    int32_t num_objects;
    int32_t num_lights;
    int32_t num_sdf;
    int32_t has_medium;      // 1: `medium` holds the participating medium
    MediumRec medium;
};

constexpr float kSlabWiden = 1.000001f;
constexpr float kMinDir = 0x1p-64f;

__device__ __forceinline__ float4 ldg4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ uint4 ldgu4(const void* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// Moller-Trumbore exactly as IntersectTriangleObject (intersection.cuh:31-57),
// operands precomputed with the same expressions.  Returns t or -1.
__device__ __forceinline__ float mt_triangle(f3 o, f3 d, f3 v0, f3 e1, f3 e2)
{
    const f3 h = cross(d, e2);
    const float a = dot(e1, h);
    if (a > -1e-6f && a < 1e-6f) return -1.0f;
    const float f = __frcp_rn(a);  // == 1.0f / a, IEEE
    const f3 s = o - v0;
    const float u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const f3 q = cross(s, e1);
    const float v = f * dot(d, q);
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = f * dot(e2, q);
    return (t > 1e-5f) ? t : -1.0f;
}

__device__ __forceinline__ m3 load_m3(const float* m)
{
    m3 r;
    r.x = mk(m[0], m[1], m[2]); r.y = mk(m[3], m[4], m[5]); r.z = mk(m[6], m[7], m[8]);
    return r;
}

// IntersectAABBObject (object/aabb.cuh:28-89).  Fills pos/nrm when wanted.
template <bool kDetail>
__device__ __forceinline__ float isect_cube(const Analytic& an, f3 ro, f3 rd, f3* pos, f3* nrm)
{
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    const m3 w2o = load_m3(an.w2o);
    const f3 lo = mul(w2o, ro - c);
    const f3 ld = normalize(mul(w2o, rd));
    const f3 dv = mk(inv_safe(ld.x), inv_safe(ld.y), inv_safe(ld.z));
    const f3 t1 = (-e - lo) * dv;
    const f3 t2 = (e - lo) * dv;
    const f3 tmn = vmin(t1, t2), tmx = vmax(t1, t2);
    const float tEnter = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
    const float tExit = fminf(fminf(tmx.x, tmx.y), tmx.z);
    if (tEnter > tExit) return -1.0f;
    if (tExit <= 0.0f) return -1.0f;
    const bool inside = (tEnter < 0.0f);
    const float tHit = inside ? tExit : tEnter;
    if (kDetail) {
        const m3 o2w = load_m3(an.o2w);
        const f3 lp = lo + ld * tHit;
        *pos = mul(o2w, lp) + c;
        const float rx = fabsf(lp.x) / e.x;
        const float ry = fabsf(lp.y) / e.y;
        const float rz = fabsf(lp.z) / e.z;
        f3 ln;
        if (rx >= ry && rx >= rz) ln = mk((lp.x > 0.0f) ? 1.0f : -1.0f, 0.0f, 0.0f);
        else if (ry >= rz) ln = mk(0.0f, (lp.y > 0.0f) ? 1.0f : -1.0f, 0.0f);
        else ln = mk(0.0f, 0.0f, (lp.z > 0.0f) ? 1.0f : -1.0f);
        if (inside) ln = -ln;
        *nrm = normalize(mul(o2w, ln));
    }
    return tHit;
}

// IntersectSphereObject (object/sphere.cuh:9-70)
template <bool kDetail>
__device__ __forceinline__ float isect_sphere(const Analytic& an, f3 ro, f3 rd, f3* pos, f3* nrm)
{
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const m3 w2o = load_m3(an.w2o);
    const f3 lo = mul(w2o, ro - c);
    const f3 ld = normalize(mul(w2o, rd));
    const float r = an.radius;
    const float b = dot(lo, ld);
    const float cc = dot(lo, lo) - r * r;
    const float disc = b * b - 1.0f * cc;
    if (disc < 0.0f) return -1.0f;
    const float sq = sqrtf(disc);
    float t = -b - sq;
    bool inside = false;
    if (t <= 0.0f) { t = -b + sq; inside = true; }
    if (t <= 0.0f) return -1.0f;
    if (kDetail) {
        const m3 o2w = load_m3(an.o2w);
        const f3 lp = lo + ld * t;
        const f3 ln = normalize(lp) * (inside ? -1.0f : 1.0f);
        *pos = mul(o2w, lp) + c;
        *nrm = normalize(mul(o2w, ln));
    }
    return t;
}

__device__ __forceinline__ float isect_analytic_t(const SceneView& s, int obj, f3 ro, f3 rd)
{
    const ObjInfo oi = s.objects[obj];
    const Analytic& an = s.analytic[oi.aux];
    f3 p, n;
    if (oi.type == 0) return isect_cube<false>(an, ro, rd, &p, &n);
    if (oi.type == 1) return isect_sphere<false>(an, ro, rd, &p, &n);
    return -1.0f;
}

// The same test out of line, for the traversal loop: analytic primitives are
// rare leaf entries, and one copy of their code keeps the unrolled leaf loop
// small.
static __device__ __noinline__ float isect_analytic_leaf(const ObjInfo* objects, const Analytic* analytic, int obj,
                                                         f3 ro, f3 rd)
{
    const ObjInfo oi = objects[obj];
    const Analytic& an = analytic[oi.aux];
    f3 p, n;
    if (oi.type == 0) return isect_cube<false>(an, ro, rd, &p, &n);
    if (oi.type == 1) return isect_sphere<false>(an, ro, rd, &p, &n);
    return -1.0f;
}

// INTERSECT_EPS(0) = 1e-3 * exp(0) (config.cuh:3): the tolerance of standalone ray queries.
constexpr float kEpsDepth0 = 1.0e-3f;

// SDF objects are not in the BVH: each query tests them after its traversal
// with the same acceptance rule as a leaf (tmin <= t < best; an equal
// distance goes to the lower object index).  eps is INTERSECT_EPS(depth) of
// the query, which sets the sphere-tracing tolerance.  Out of line: the
// marching loop stays out of the traversal kernels' register budget.
static __device__ __noinline__ void sdf_closest(const SceneView& s, f3 o, f3 d, float tmin, float eps, float* best_t,
                                         int32_t* best_obj)
{
    for (int k = 0; k < s.num_sdf; ++k) {
        const SdfRec g = s.sdf[k];
        const float t = sdf_march(g, s.analytic[g.analytic], o, d, eps);
        if (t < 0.0f || t < tmin) continue;
        if (t < *best_t || (t == *best_t && *best_obj >= 0 && g.object < *best_obj)) {
            *best_t = t;
            *best_obj = g.object;
        }
    }
}

// Any SDF object hit in [tmin, tmax): its object index, else -1.
static __device__ __noinline__ int32_t sdf_any(const SceneView& s, f3 o, f3 d, float tmin, float tmax, float eps)
{
    for (int k = 0; k < s.num_sdf; ++k) {
        const SdfRec g = s.sdf[k];
        const float t = sdf_march(g, s.analytic[g.analytic], o, d, eps);
        if (t >= 0.0f && !(t < tmin) && t < tmax) return g.object;
    }
    return -1;
}

// Hit position and normal on an SDF object (out of line, for the shading kernels).
static __device__ __noinline__ void sdf_surface_of(const SceneView& s, int aux, f3 ro, f3 rd, float t, float eps,
                                                   f3* pos, f3* nrm)
{
    const SdfRec g = s.sdf[aux];
    sdf_surface(g, s.analytic[g.analytic], ro, rd, t, eps, pos, nrm);
}

// Solo trace of an SDF object (the medium a path is inside).
static __device__ __noinline__ float sdf_solo_t(const SceneView& s, int obj, f3 ro, f3 rd, float eps)
{
    const SdfRec g = s.sdf[s.objects[obj].aux];
    return sdf_march(g, s.analytic[g.analytic], ro, rd, eps);
}

struct Hit {
    float t;
    int32_t obj;   // object index, -1 = miss
    int32_t prim;  // leaf-order primitive slot, -1 = none
};

// Traversal stack: kStackShared entries per lane in shared memory, the rest in
// a per-thread slab of global memory (only deep BVH paths reach it).
constexpr int kStackShared = 32;
constexpr int kStackOverflow = 96;
constexpr int kStackMax = kStackShared + kStackOverflow;

struct RayState {
    f3 o, d;
    float ix, iy, iz;  // reciprocal direction, |d| clamped to 2^-64
    float tmin;
    Hit best;
    uint32_t node;
    int sp;
    uint32_t visits;  // nodes visited
    uint32_t tests;   // primitives tested
};

__device__ __forceinline__ void ray_begin(RayState& r, f3 o, f3 d, float tmin, float tmax)
{
    r.o = o;
    r.d = d;
    const float dx = fabsf(d.x) < kMinDir ? copysignf(kMinDir, d.x) : d.x;
    const float dy = fabsf(d.y) < kMinDir ? copysignf(kMinDir, d.y) : d.y;
    const float dz = fabsf(d.z) < kMinDir ? copysignf(kMinDir, d.z) : d.z;
    r.ix = __frcp_rn(dx);
    r.iy = __frcp_rn(dy);
    r.iz = __frcp_rn(dz);
    r.tmin = tmin;
    r.best.t = tmax;
    r.best.obj = -1;
    r.best.prim = -1;
    r.node = 0;
    r.sp = 0;
    r.visits = 0;
    r.tests = 0;
}

// byte q = byte k of w placed in bits 8-15 of the float 2^15: the value
// 2^15 + q, exact, with one byte permute and no conversion instruction.
__device__ __forceinline__ float byte_biased(uint32_t w, int k)
{
    return __uint_as_float(__byte_perm(w, 0x47000000u, 0x7404u + (static_cast<uint32_t>(k) << 4)));
}
constexpr float kByteBias = 32768.0f;  // 2^15, the offset byte_biased adds

__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// (d0, d1) = (q0 * a + b, q1 * a + b): the near and far plane of one axis in
// one packed fma.rn.f32x2 (sm_100; each lane rounds exactly like fmaf).  On
// the 1M-triangle sphere field this cut the closest-hit stage 2 % and the
// any-hit stage 4 %.
__device__ __forceinline__ void ffma2(float& d0, float& d1, float q0, float q1, float a, float b)
{
    asm("{\n\t.reg .b64 rq, ra, rb, rd;\n\t"
        "mov.b64 rq, {%2, %3};\n\t"
        "mov.b64 ra, {%4, %4};\n\t"
        "mov.b64 rb, {%5, %5};\n\t"
        "fma.rn.f32x2 rd, rq, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d0), "=f"(d1) : "f"(q0), "f"(q1), "f"(a), "f"(b));
}

// a[k] for a run-time k without indexing the register array
__device__ __forceinline__ uint32_t pick8(const uint32_t (&a)[8], int k)
{
    const bool k1 = k & 1, k2 = k & 2, k4 = k & 4;
    const uint32_t b0 = k1 ? a[1] : a[0], b1 = k1 ? a[3] : a[2], b2 = k1 ? a[5] : a[4], b3 = k1 ? a[7] : a[6];
    const uint32_t c0 = k2 ? b1 : b0, c1 = k2 ? b3 : b2;
    return k4 ? c1 : c0;
}

__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b)
{
    const uint32_t lo = min(a, b), hi = max(a, b);
    a = lo; b = hi;
}

// Sort key of a hit child in one byte permute (prmt with sign replication):
// byte 0 = meta byte b of `meta`, bytes 1-2 = the top 16 bits of tnear, byte 3
// = the meta byte's bit 7 replicated (0xFF for internal and empty slots, 0 for
// leaves).  tnear >= 0, so its top 16 bits order like its value.
__device__ __forceinline__ uint32_t child_key(float tnear, uint32_t meta, int b)
{
    uint32_t r;
    const uint32_t sel = 0x0324u + static_cast<uint32_t>(b) + (static_cast<uint32_t>(0xC + b) << 12);
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(__float_as_uint(tnear)), "r"(meta), "r"(sel));
    return r;
}

// The entry distance a key carries, rounded down to 16 bits (bytes 1-2 of
// the key moved to bytes 2-3 of a float, zeros below).
__device__ __forceinline__ float key_distance(uint32_t key)
{
    return __uint_as_float(__byte_perm(key, 0u, 0x2144u));
}

// Closest-hit stack entries carry the child's entry distance with the node
// index: (bits(tnear) & ~mask) | node, mask = all ones up to the highest bit
// of (num_nodes | 255).  Clearing low bits of a non-negative float rounds it
// down, so the stored distance never exceeds the true one, and a node popped
// after a nearer hit was found is dropped without being fetched, by the same
// test that culls children at push time.  Any-hit queries never lower their
// limit below what their entries passed and push bare node indices.
__device__ __forceinline__ uint32_t stack_node_mask(int num_nodes)
{
    return 0xFFFFFFFFu >> __clz(static_cast<uint32_t>(num_nodes) | 255u);
}

// Visit node r.node: test its 8 child boxes, intersect the primitives of hit
// leaf children nearest first, push hit internal children far to near (a
// closest-hit query keeps the nearest as its next node), else pop the next
// node that can still hold a nearer hit.  Returns true when the ray is
// finished (stack empty, any-hit found, or stack overflow reported through
// *err).
template <bool kAny, bool kCount>
__device__ __forceinline__ bool ray_step(const SceneView& s, RayState& r, uint32_t* stack, uint32_t* ovf, int* err)
{
    const uint32_t nmask = kAny ? 0u : stack_node_mask(s.num_nodes);
    const WideNode* np = s.nodes + r.node;
    if (kCount) ++r.visits;
    const float4 w0 = ldg4(reinterpret_cast<const char*>(np));
    const uint4 w1 = ldgu4(reinterpret_cast<const char*>(np) + 16);
    const uint4 w2 = ldgu4(reinterpret_cast<const char*>(np) + 32);
    const uint4 w3 = ldgu4(reinterpret_cast<const char*>(np) + 48);
    const uint4 w4 = ldgu4(reinterpret_cast<const char*>(np) + 64);
    const uint32_t exps = __float_as_uint(w0.w);
    const float sx = __uint_as_float((exps & 0xFFu) << 23);
    const float sy = __uint_as_float(((exps >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((exps >> 16) & 0xFFu) << 23);
    const float ax = sx * r.ix, ay = sy * r.iy, az = sz * r.iz;
    // plane q at t = q * a + (origin - o) * inv_dir = fma(2^15 + q, a, b) with
    // b = (origin - o) * inv_dir - 2^15 * a; the extra rounding of b is at most
    // 2^-24 (|b| + 2^15 |a|), far below the one-grid-step padding of the boxes
    const float bx = fmaf(-kByteBias, ax, (w0.x - r.o.x) * r.ix);
    const float by = fmaf(-kByteBias, ay, (w0.y - r.o.y) * r.iy);
    const float bz = fmaf(-kByteBias, az, (w0.z - r.o.z) * r.iz);
    // w2 = qlo_x | qlo_y, w3 = qlo_z | qhi_x, w4 = qhi_y | qhi_z (8 bytes each)
    const bool nx = r.ix < 0.0f, ny = r.iy < 0.0f, nz = r.iz < 0.0f;
    const uint32_t nx0 = nx ? w3.z : w2.x, nx1 = nx ? w3.w : w2.y, fx0 = nx ? w2.x : w3.z, fx1 = nx ? w2.y : w3.w;
    const uint32_t ny0 = ny ? w4.x : w2.z, ny1 = ny ? w4.y : w2.w, fy0 = ny ? w2.z : w4.x, fy1 = ny ? w2.w : w4.y;
    const uint32_t nz0 = nz ? w4.z : w3.x, nz1 = nz ? w4.w : w3.y, fz0 = nz ? w3.x : w4.z, fz1 = nz ? w3.y : w4.w;
    const uint32_t meta0 = w1.z, meta1 = w1.w;
    const float limit = fminf(r.best.t, FLT_MAX);
    // every accepted hit has t > 0, so the box test may start at max(tmin, 0),
    // which also makes every tnear non-negative (its bits order like its value)
    const float tlow = fmaxf(r.tmin, 0.0f);
    uint32_t key[8];
    uint32_t hm = 0;  // bit k: slot k's box is hit
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int b = k & 3;
        float tnx, tfx, tny, tfy, tnz, tfz;
        ffma2(tnx, tfx, byte_biased(k < 4 ? nx0 : nx1, b), byte_biased(k < 4 ? fx0 : fx1, b), ax, bx);
        ffma2(tny, tfy, byte_biased(k < 4 ? ny0 : ny1, b), byte_biased(k < 4 ? fy0 : fy1, b), ay, by);
        ffma2(tnz, tfz, byte_biased(k < 4 ? nz0 : nz1, b), byte_biased(k < 4 ? fz0 : fz1, b), az, bz);
        const float tnear = max3f(tnx, tny, fmaxf(tnz, tlow));
        const float tfar = min3f(tfx, tfy, fminf(tfz, limit)) * kSlabWiden;
        // key (child_key): the top 16 bits of tnear with the child's meta byte
        // below and the meta byte's sign above, so that the sort puts every
        // hit leaf (nearest first) before every hit internal child (nearest
        // first) and the misses last.  Empty slots have inverted
        // boxes (lo 255, hi 0) and fail this test unless the ray starts some
        // 2^28 grid steps away; they then sort as internal children, and their
        // meta byte kMetaEmpty keeps them off the stack.
        const bool hit = tnear <= tfar;
        key[k] = hit ? child_key(tnear, k < 4 ? meta0 : meta1, b) : 0xFFFFFFFFu;
        hm |= static_cast<uint32_t>(hit) << k;
    }
    // visit children nearest first -- sort the 8 keys (Batcher odd-even merge
    // network, 19 comparators).  Any-hit queries profit too: the occluder of a
    // shadow segment is usually close to its start.
    cswap(key[0], key[1]); cswap(key[2], key[3]); cswap(key[4], key[5]); cswap(key[6], key[7]);
    cswap(key[0], key[2]); cswap(key[1], key[3]); cswap(key[4], key[6]); cswap(key[5], key[7]);
    cswap(key[1], key[2]); cswap(key[5], key[6]);
    cswap(key[0], key[4]); cswap(key[1], key[5]); cswap(key[2], key[6]); cswap(key[3], key[7]);
    cswap(key[2], key[4]); cswap(key[3], key[5]);
    cswap(key[1], key[2]); cswap(key[3], key[4]); cswap(key[5], key[6]);
    // hit leaves occupy sorted positions [0, nl), hit internal children
    // [nl, nh).  Leaf slots: meta bytes with bit 7 clear, gathered from the two
    // meta words (bits 7, 15, 23, 31 to bits 0-3 by one multiply-high).
    const uint32_t ls = ((__umulhi(~meta0 & 0x80808080u, 0x10204080u) >> 3) & 0xFu) |
                        (((__umulhi(~meta1 & 0x80808080u, 0x10204080u) >> 3) & 0xFu) << 4);
    const int nh = __popc(hm), nl = __popc(hm & ls);
    // leaves, nearest first, in one flat loop over (leaf, primitive) pairs: a
    // single copy of the primitive tests, and a warp runs as many iterations
    // as its busiest lane has primitives instead of the sum over leaf ranks of
    // the per-rank maximum.  A leaf is entered only while its entry distance
    // does not exceed the current hit (later leaves are farther).
    const uint32_t prim_base = w1.y;
    int lk = 0, left = 0;
    uint32_t pidx = 0;
    if (nl > 0) {
        const uint32_t kk = key[0];
        if (key_distance(kk) <= fminf(r.best.t, FLT_MAX) * kSlabWiden) {
            left = static_cast<int>((kk & 0xFFu) >> 5) + 1;
            pidx = prim_base + (kk & 31u);
        }
    }
#pragma unroll 1
    while (left > 0) {
        const PrimRec* pr = s.prims + pidx;
        if (kCount) ++r.tests;
        // all three words at once: one memory round trip per primitive
        const float4 a = ldg4(&pr->v0[0]);
        const float4 e1 = ldg4(&pr->e1[0]);
        const float4 e2 = ldg4(&pr->e2[0]);
        const int obj = __float_as_int(a.w);
        float t;
        if (__float_as_int(e1.w) == kPrimTriangle) {
            t = mt_triangle(r.o, r.d, mk(a.x, a.y, a.z), mk(e1.x, e1.y, e1.z), mk(e2.x, e2.y, e2.z));
        } else {
            t = isect_analytic_t(s, obj, r.o, r.d);
        }
        if (!(t < 0.0f || t < r.tmin) &&
            (t < r.best.t || (r.best.obj >= 0 && t == r.best.t && obj < r.best.obj))) {
            r.best.t = t;
            r.best.obj = obj;
            r.best.prim = static_cast<int>(pidx);
            if (kAny) return true;
        }
        ++pidx;
        if (--left == 0 && ++lk < nl) {
            const uint32_t kk = pick8(key, lk);
            if (key_distance(kk) <= fminf(r.best.t, FLT_MAX) * kSlabWiden) {
                left = static_cast<int>((kk & 0xFFu) >> 5) + 1;
                pidx = prim_base + (kk & 31u);
            }
        }
    }
    // internal children far to near.  Any-hit queries push them all and pop
    // the nearest; closest-hit queries push all but the nearest, which they
    // visit next without a trip through the stack (the same order: -2 % time
    // for closest-hit queries; any-hit queries, whose nodes hold fewer hit
    // children, measured no gain).
    const uint32_t child_base = w1.x;
    const float lim_push = fminf(r.best.t, FLT_MAX) * kSlabWiden;
    uint32_t held = 0xFFFFFFFFu;   // closest hit: the nearest child so far (distance bits | node)
#pragma unroll 1
    for (int k = nh - 1; k >= nl; --k) {
        const uint32_t kk = pick8(key, k);
        if ((kk & 0xFFu) == kMetaEmpty) continue;
        const float tn = key_distance(kk);
        if (!(tn <= lim_push)) continue;
        const uint32_t child = child_base + (kk & 7u);
        const uint32_t entry = kAny ? child : ((__float_as_uint(tn) & ~nmask) | child);
        uint32_t push = entry;
        if (!kAny) {
            push = held;
            held = entry;
            if (push == 0xFFFFFFFFu) continue;
        }
        if (r.sp < kStackShared) stack[r.sp * 32] = push;
        else if (r.sp < kStackMax) ovf[r.sp - kStackShared] = push;
        else { atomicOr(err, 1); return true; }
        ++r.sp;
    }
    if (!kAny && held != 0xFFFFFFFFu) {
        r.node = held & nmask;
        return false;
    }
    if (kAny) {
        if (r.sp == 0) return true;
        --r.sp;
        r.node = (r.sp < kStackShared) ? stack[r.sp * 32] : ovf[r.sp - kStackShared];
        return false;
    }
    const float lim = fminf(r.best.t, FLT_MAX) * kSlabWiden;
    for (;;) {
        if (r.sp == 0) return true;
        --r.sp;
        const uint32_t e = (r.sp < kStackShared) ? stack[r.sp * 32] : ovf[r.sp - kStackShared];
        if (__uint_as_float(e & ~nmask) <= lim) {
            r.node = e & nmask;
            return false;
        }
    }
}

// Persistent traversal loop shared by every ray-query kernel.  Each warp keeps
// 32 rays in flight.  Lanes whose rays finish are refilled in batches of at
// least refill_min(kAny) (or when the whole warp is idle): the refill stores
// their results and loads new queue entries (one atomic per warp per refill),
// so the lane-divergent store/load code runs once for several lanes instead of
// once per finishing lane, while no lane idles for long.  Measured on the
// 1M-triangle sphere field: 8 for closest-hit queries; 16 for any-hit queries,
// whose short lives make refills frequent (2 and 4 were 6-14 % slower for
// both).  IO supplies load() -> item id or -1 when the entry finished without
// traversal, and store().
constexpr int refill_min(bool any) { return any ? 16 : 8; }

template <bool kAny, class IO, bool kCount = false>
__device__ __forceinline__ void traverse_queue(const SceneView& s, IO& io, int n, int* fetch, uint32_t* stack,
                                               uint32_t* ovf, int* err, unsigned long long* work)
{
    const unsigned lane = threadIdx.x & 31u;
    RayState r;
    int item = -1;   // ray in flight
    int pend = -1;   // finished ray whose result waits in r for the next refill
    unsigned long long visits = 0, tests = 0;
    bool exhausted = false;
    for (;;) {
        const unsigned idle = __ballot_sync(0xFFFFFFFFu, item < 0);
        const bool refill = !exhausted && idle != 0u && (__popc(idle) >= refill_min(kAny) || idle == 0xFFFFFFFFu);
        if ((refill || exhausted) && pend >= 0) {
            io.store(s, pend, r);
            if (kCount) {
                visits += r.visits;
                tests += r.tests;
            }
            pend = -1;
        }
        if (refill) {
            const int leader = __ffs(idle) - 1;
            int base = 0;
            if (static_cast<int>(lane) == leader) base = atomicAdd(fetch, __popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (base + __popc(idle) >= n) exhausted = true;
            if (item < 0) {
                const int k = base + __popc(idle & ((1u << lane) - 1u));
                if (k < n) item = io.load(s, k, r);
            }
        }
        const unsigned busy = __ballot_sync(0xFFFFFFFFu, item >= 0);
        if (busy == 0) {
            if (exhausted) break;
            continue;
        }
        if (item >= 0) {
            const bool done = (s.num_nodes == 0) || ray_step<kAny, kCount>(s, r, stack, ovf, err);
            if (done) {
                pend = item;
                item = -1;
            }
        }
    }
    if (kCount && work) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            visits += __shfl_xor_sync(0xFFFFFFFFu, visits, o);
            tests += __shfl_xor_sync(0xFFFFFFFFu, tests, o);
        }
        if (lane == 0) {
            atomicAdd(&work[0], visits);
            atomicAdd(&work[1], tests);
        }
    }
}

}  // namespace ar
