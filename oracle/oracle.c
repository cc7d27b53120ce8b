/*
 * oracle.c -- CPU restatement of ApertureRendererV3's path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Scalar C, IEEE single precision,
 * compiled with -ffp-contract=off so that every a*b+c rounds twice, exactly
 * like the reference's source expressions read and like the CUDA core built
 * with --fmad=false.  Expression order follows the reference token by token;
 * each function cites the reference lines it restates (paths relative to the
 * reference's core/ directory).
 *
 * Deliberate, documented choices where the reference's exact arithmetic cannot
 * be reproduced on two machines:
 *   - sinf/cosf/sincosf/expf/logf/powf -> oracle_math.h (fixed definitions);
 *   - rsqrtf(x) -> 1/sqrtf(x) (IEEE);
 *   - INTERSECT_EPS(d) = 1e-3f * expf(min(d/2, 4)) -> 9-entry table of the same.
 */
#define _GNU_SOURCE
#include "oracle.h"
#include "oracle_math.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* float3 helpers (vector.cuh:127-262)                                       */
/* ------------------------------------------------------------------------ */
typedef struct { float x, y, z; } V3;
typedef struct { V3 x, y, z; } M3; /* rows, float3x3 (vector.cuh:320-420) */

static inline V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vmul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3 vscale(V3 a, float b) { return v3(a.x * b, a.y * b, a.z * b); }
static inline V3 vdivs(V3 a, float b) { return v3(a.x / b, a.y / b, a.z / b); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 vadds(V3 a, float b) { return v3(a.x + b, a.y + b, a.z + b); }
static inline float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross3(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len3(V3 a) { return sqrtf(dot3(a, a)); }
static inline V3 vmin3(V3 a, V3 b) { return v3(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
static inline V3 vmax3(V3 a, V3 b) { return v3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
static inline V3 vmaxs(V3 a, float b) { return v3(fmaxf(a.x, b), fmaxf(a.y, b), fmaxf(a.z, b)); }
static inline float max3f(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
static inline V3 vabs(V3 a) { return v3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static inline int all_zero(V3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }

/* vector.cuh:222-231 with rsqrtf -> 1/sqrtf */
static inline V3 vnormalize(V3 v)
{
    const float l2 = dot3(v, v);
    if (l2 <= 1e-20f) return v3(0.0f, 0.0f, 0.0f);
    const float inv = om_rsqrtf(l2);
    return vscale(v, inv);
}
static inline float clampf_(float v, float a, float b) { return isnan(v) ? 0.0f : fminf(fmaxf(v, a), b); }
static inline float saturatef_(float v) { return isnan(v) ? 0.0f : fminf(fmaxf(v, 0.0f), 1.0f); }
static inline float signf_(float a) { return a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f); }
static inline float lerpf_(float a, float b, float v) { return a * (1.0f - v) + b * v; }
static inline V3 vlerp(V3 a, V3 b, float v) { return v3(lerpf_(a.x, b.x, v), lerpf_(a.y, b.y, v), lerpf_(a.z, b.z, v)); }
static inline float luminance3(V3 c) { return dot3(c, v3(0.2126f, 0.7152f, 0.0722f)); }
/* v - 2*dot(v,n)*n (vector.cuh:296-299) */
static inline V3 vreflect(V3 v, V3 n) { return vsub(v, vscale(n, 2.0f * dot3(v, n))); }
/* vector.cuh:254-262 */
static inline V3 vrefract(V3 in, V3 normal, float eta)
{
    const V3 n = (dot3(normal, in) > 0.0f) ? vneg(normal) : normal;
    const float cosI = -dot3(n, in);
    const float k = 1.0f - (eta * eta) * fmaxf(0.0f, 1.0f - cosI * cosI);
    const float cosT = sqrtf(fmaxf(0.0f, k));
    return vadd(vscale(in, eta), vscale(n, eta * cosI - cosT));
}
static inline float inv_safe(float x) { return (x == 0.0f) ? (x >= 0 ? FLT_MAX : -FLT_MAX) : 1.0f / x; }
static inline V3 mmul(const M3* m, V3 v) { return v3(dot3(m->x, v), dot3(m->y, v), dot3(m->z, v)); }
static inline float fix_nan_inf(float x)
{
    if (isnan(x)) return 0.0f;
    if (isinf(x)) return x > 0.0f ? 0.0f : -0.0f;
    return x;
}

/* BuildTangentBasis (vector.cuh:264-269) */
static inline void tangent_basis(V3 n, V3* t, V3* b)
{
    const V3 a = (fabsf(n.z) < 0.999f) ? v3(0.0f, 0.0f, 1.0f) : v3(1.0f, 0.0f, 0.0f);
    *t = vnormalize(cross3(a, n));
    *b = cross3(n, *t);
}
/* BuildTangentBasisRandom (vector.cuh:271-283) */
static inline void tangent_basis_random(V3 n, V3* t, V3* b, float e)
{
    const V3 a = (fabsf(n.z) < 0.999f) ? v3(0.0f, 0.0f, 1.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t0 = vnormalize(cross3(a, n));
    const V3 b0 = cross3(n, t0);
    float s, c;
    om_sincosf(e * 3.14159265358979f * 2.0f, &s, &c);
    *t = vadd(vscale(t0, c), vscale(b0, s));
    *b = vadd(vscale(t0, -s), vscale(b0, c));
}

#define OR_PI 3.14159265358979f /* CUDART_PI_F rounds to the same float */

/* ------------------------------------------------------------------------ */
/* Scene                                                                      */
/* ------------------------------------------------------------------------ */
typedef struct {
    int type, visible, light_index;
    V3 center, extent;
    M3 o2w, w2o;
    ar_material mat;
    V3 p0, p1, p2;        /* world-space triangle vertices */
    V3 n0, n1, n2;        /* objectToWorld * vertex normal */
    V3 bmin, bmax, pc;    /* PrimitiveProxy */
    int sdf_kind;         /* AR_SDF_* of AR_OBJ_SDF objects */
    float sdf_info[4];    /* SDFInfo::sdfInfo0_ */
    const float* vol;     /* AR_SDF_VOLUME: grid values (x fastest) */
    int dims[3];
    float vmax;           /* SDFVolumeInfo::voxelSizeMax_ */
} OObj;

typedef struct { V3 bmin, bmax; int left, right, first, count; } ONode;

struct or_scene {
    int n;
    OObj* o;
    float** vols;          /* SDF volume grids (float copies) */
    int nvol;
    float* spec_tab;       /* spectral tables (or_scene_set_spectral) */
    float* lut_lam;        /* 840 x 4 */
    float* lut_rgb;        /* res^3 x 4 */
    int spec_res;
    ONode* nodes;
    int nn, cap;
    int* idx;
    int nl;
    int* lobj;
    float* lprob;
    int flags;
    int fallbacks;
    float eps_tab[9];
    /* participating medium (or_scene_set_medium; extension, no reference counterpart) */
    int has_medium;
    float m_bmin[3], m_bmax[3], m_sigma, m_g, m_albedo[3], m_major;
    int m_dims[3];
    float* m_grid;         /* density values as float (half grids converted exactly) */
};

/* float3x3::rotX/Y/Z and mul (vector.cuh:378-416), host libm as in the
 * reference's SceneObject constructor (object.cuh:344-364). */
static M3 mat_mul(const M3* a, const M3* m)
{
    const V3 c0 = v3(m->x.x, m->y.x, m->z.x);
    const V3 c1 = v3(m->x.y, m->y.y, m->z.y);
    const V3 c2 = v3(m->x.z, m->y.z, m->z.z);
    M3 r;
    r.x = v3(dot3(a->x, c0), dot3(a->x, c1), dot3(a->x, c2));
    r.y = v3(dot3(a->y, c0), dot3(a->y, c1), dot3(a->y, c2));
    r.z = v3(dot3(a->z, c0), dot3(a->z, c1), dot3(a->z, c2));
    return r;
}
static void euler_to_matrix(V3 deg, M3* o2w, M3* w2o)
{
    const float k = 3.14159265358979f / 180.0f; /* deg2rad (vector.cuh:76-80) */
    const float ax = deg.x * k, ay = deg.y * k, az = deg.z * k;
    M3 rx, ry, rz;
    float c = cosf(ax), s = sinf(ax);
    rx.x = v3(1, 0, 0); rx.y = v3(0, c, -s); rx.z = v3(0, s, c);
    c = cosf(ay); s = sinf(ay);
    ry.x = v3(c, 0, s); ry.y = v3(0, 1, 0); ry.z = v3(-s, 0, c);
    c = cosf(az); s = sinf(az);
    rz.x = v3(c, -s, 0); rz.y = v3(s, c, 0); rz.z = v3(0, 0, 1);
    const M3 yx = mat_mul(&ry, &rx);
    *o2w = mat_mul(&rz, &yx);
    w2o->x = v3(o2w->x.x, o2w->y.x, o2w->z.x);
    w2o->y = v3(o2w->x.y, o2w->y.y, o2w->z.y);
    w2o->z = v3(o2w->x.z, o2w->y.z, o2w->z.z);
}

static V3 from_ar(ar_vec3 a) { return v3(a.x, a.y, a.z); }

/* SceneObject::GetArea (object.cuh:278-302) */
static float object_area(const OObj* o, const ar_object_desc* d)
{
    if (o->type == AR_OBJ_CUBE || o->type == AR_OBJ_SDF) {
        const float ex = fabsf(o->extent.x), ey = fabsf(o->extent.y), ez = fabsf(o->extent.z);
        return 8.0f * (ex * ey + ex * ez + ey * ez);
    } else if (o->type == AR_OBJ_SPHERE) {
        const float r = fabsf(o->extent.x);
        return 4.0f * OR_PI * r * r;
    } else if (o->type == AR_OBJ_TRIANGLE) {
        const V3 e1 = vsub(from_ar(d->tri[1].position), from_ar(d->tri[0].position));
        const V3 e2 = vsub(from_ar(d->tri[2].position), from_ar(d->tri[0].position));
        return 0.5f * len3(cross3(e1, e2));
    }
    return 0.0f;
}

/* SceneObject::UpdateProxy (object.cuh:309-342) */
static void update_proxy(OObj* o, int object_center)
{
    o->pc = o->center;
    if (o->type == AR_OBJ_CUBE || o->type == AR_OBJ_SDF) {
        const V3 ax = mmul(&o->o2w, v3(1.0f, 0.0f, 0.0f));
        const V3 ay = mmul(&o->o2w, v3(0.0f, 1.0f, 0.0f));
        const V3 az = mmul(&o->o2w, v3(0.0f, 0.0f, 1.0f));
        V3 h;
        h.x = fabsf(ax.x) * o->extent.x + fabsf(ay.x) * o->extent.y + fabsf(az.x) * o->extent.z;
        h.y = fabsf(ax.y) * o->extent.x + fabsf(ay.y) * o->extent.y + fabsf(az.y) * o->extent.z;
        h.z = fabsf(ax.z) * o->extent.x + fabsf(ay.z) * o->extent.y + fabsf(az.z) * o->extent.z;
        o->bmin = v3(o->center.x - h.x, o->center.y - h.y, o->center.z - h.z);
        o->bmax = v3(o->center.x + h.x, o->center.y + h.y, o->center.z + h.z);
    } else if (o->type == AR_OBJ_SPHERE) {
        const float r = max3f(o->extent);
        const V3 h = v3(r, r, r);
        o->bmin = vsub(o->center, h);
        o->bmax = vadd(o->center, h);
    } else if (o->type == AR_OBJ_TRIANGLE) {
        const V3 p0 = o->p0, p1 = o->p1, p2 = o->p2;
        o->bmin = v3(fminf(fminf(p0.x, p1.x), p2.x), fminf(fminf(p0.y, p1.y), p2.y), fminf(fminf(p0.z, p1.z), p2.z));
        o->bmax = v3(fmaxf(fmaxf(p0.x, p1.x), p2.x), fmaxf(fmaxf(p0.y, p1.y), p2.y), fmaxf(fmaxf(p0.z, p1.z), p2.z));
        if (!object_center)
            o->pc = v3(0.5f * (o->bmin.x + o->bmax.x), 0.5f * (o->bmin.y + o->bmax.y), 0.5f * (o->bmin.z + o->bmax.z));
    } else {
        o->bmin = o->center;
        o->bmax = o->center;
    }
}

/* ------------------------------------------------------------------------ */
/* BuildBVH (bvh/bvh.cuh:142-422), 32-bit node layout                        */
/* ------------------------------------------------------------------------ */
static float aabb_area(V3 mn, V3 mx)
{
    const V3 d = v3(fmaxf(0.0f, mx.x - mn.x), fmaxf(0.0f, mx.y - mn.y), fmaxf(0.0f, mx.z - mn.z));
    return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}
static float axis_of(V3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

typedef struct { or_scene* s; int leaf, bins; } BuildCtx;

static int bin_of(const OObj* p, int axis, float cmin, float invW, int bins)
{
    const float key = axis_of(p->pc, axis);
    int b = invW > 0.0f ? (int)((key - cmin) * invW) : 0;
    b = (b < 0) ? 0 : (b >= bins ? bins - 1 : b);
    return b;
}

static int cmp_key_axis;
static const OObj* cmp_objs;
static int cmp_idx_key(const void* a, const void* b)
{
    const int ia = *(const int*)a, ib = *(const int*)b;
    const float ka = axis_of(cmp_objs[ia].pc, cmp_key_axis), kb = axis_of(cmp_objs[ib].pc, cmp_key_axis);
    if (ka < kb) return -1;
    if (ka > kb) return 1;
    return (ia < ib) ? -1 : (ia > ib);
}

static int new_node(or_scene* s)
{
    if (s->nn == s->cap) {
        s->cap = s->cap ? 2 * s->cap : 1024;
        s->nodes = (ONode*)realloc(s->nodes, (size_t)s->cap * sizeof(ONode));
    }
    memset(&s->nodes[s->nn], 0, sizeof(ONode));
    return s->nn++;
}

static void make_leaf(ONode* node, int start, int count)
{
    node->left = -1; node->right = -1; node->first = start; node->count = count;
}

static int build_rec(BuildCtx* c, int start, int end)
{
    or_scene* s = c->s;
    const int count = end - start;
    const int ni = new_node(s);
    V3 bmin = v3(FLT_MAX, FLT_MAX, FLT_MAX), bmax = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    V3 cmin = bmin, cmax = bmax;
    for (int i = start; i < end; ++i) {
        const OObj* p = &s->o[s->idx[i]];
        bmin = vmin3(bmin, p->bmin); bmax = vmax3(bmax, p->bmax);
        cmin = vmin3(cmin, p->pc); cmax = vmax3(cmax, p->pc);
    }
    s->nodes[ni].bmin = bmin; s->nodes[ni].bmax = bmax;
    if (count <= c->leaf) { make_leaf(&s->nodes[ni], start, count); return ni; }
    const V3 ce = v3(cmax.x - cmin.x, cmax.y - cmin.y, cmax.z - cmin.z);
    int axis = 0;
    if (ce.y > ce.x && ce.y >= ce.z) axis = 1;
    else if (ce.z > ce.x && ce.z >= ce.y) axis = 2;
    if (ce.x <= 1e-6f && ce.y <= 1e-6f && ce.z <= 1e-6f) { make_leaf(&s->nodes[ni], start, count); return ni; }
    const float cminA = axis_of(cmin, axis), cmaxA = axis_of(cmax, axis);
    const int B = c->bins;
    const float invW = (cmaxA > cminA) ? (float)B / (cmaxA - cminA) : 0.0f;
    V3 binMin[64], binMax[64];
    int binCount[64];
    float leftArea[64], rightArea[64];
    int leftCount[64], rightCount[64];
    for (int b = 0; b < B; ++b) {
        binMin[b] = v3(FLT_MAX, FLT_MAX, FLT_MAX); binMax[b] = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX); binCount[b] = 0;
    }
    for (int i = start; i < end; ++i) {
        const OObj* p = &s->o[s->idx[i]];
        const int b = bin_of(p, axis, cminA, invW, B);
        binMin[b] = vmin3(binMin[b], p->bmin); binMax[b] = vmax3(binMax[b], p->bmax); binCount[b]++;
    }
    V3 rmin = v3(FLT_MAX, FLT_MAX, FLT_MAX), rmax = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    int run = 0;
    for (int b = 0; b < B; ++b) {
        if (binCount[b] > 0) { rmin = vmin3(rmin, binMin[b]); rmax = vmax3(rmax, binMax[b]); }
        run += binCount[b];
        leftArea[b] = (run > 0) ? aabb_area(rmin, rmax) : 0.0f;
        leftCount[b] = run;
    }
    rmin = v3(FLT_MAX, FLT_MAX, FLT_MAX); rmax = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX); run = 0;
    for (int b = B - 1; b >= 0; --b) {
        if (binCount[b] > 0) { rmin = vmin3(rmin, binMin[b]); rmax = vmax3(rmax, binMax[b]); }
        run += binCount[b];
        rightArea[b] = (run > 0) ? aabb_area(rmin, rmax) : 0.0f;
        rightCount[b] = run;
    }
    const float parentArea = aabb_area(bmin, bmax);
    float bestCost = FLT_MAX;
    int bestSplit = -1;
    for (int b = 0; b < B - 1; ++b) {
        const int nl = leftCount[b], nr = rightCount[b + 1];
        if (nl == 0 || nr == 0) continue;
        const float sah = 1.0f + (leftArea[b] * (float)nl + rightArea[b + 1] * (float)nr) / fmaxf(parentArea, 1e-20f) * 1.0f;
        if (sah < bestCost) { bestCost = sah; bestSplit = b; }
    }
    int mid = -1;
    if (bestSplit >= 0) {
        /* std::partition on a random-access range: the classic two-pointer
         * (Hoare) scheme -- advance from the front past elements that satisfy
         * the predicate, retreat from the back past those that do not, swap. */
        int* first = s->idx + start;
        int* last = s->idx + end;
        for (;;) {
            for (;;) {
                if (first == last) goto done;
                if (bin_of(&s->o[*first], axis, cminA, invW, B) <= bestSplit) ++first; else break;
            }
            --last;
            for (;;) {
                if (first == last) goto done;
                if (!(bin_of(&s->o[*last], axis, cminA, invW, B) <= bestSplit)) --last; else break;
            }
            { const int t = *first; *first = *last; *last = t; }
            ++first;
        }
    done:
        mid = (int)(first - s->idx);
        if (mid == start || mid == end) bestSplit = -1;
    }
    if (bestSplit < 0) {
        /* Median fallback (bvh.cuh:357-392).  The reference uses
         * std::nth_element, whose placement of the other elements is
         * implementation defined; this restatement sorts instead and counts the
         * event so that pinned scenes can assert it never happens. */
        s->fallbacks++;
        const int m = start + count / 2;
        cmp_key_axis = axis; cmp_objs = s->o;
        qsort(s->idx + start, (size_t)count, sizeof(int), cmp_idx_key);
        mid = m;
        if (mid == start || mid == end) { make_leaf(&s->nodes[ni], start, count); return ni; }
    }
    const int l = build_rec(c, start, mid);
    const int r = build_rec(c, mid, end);
    s->nodes[ni].left = l; s->nodes[ni].right = r; s->nodes[ni].first = -1; s->nodes[ni].count = 0;
    return ni;
}

static float sdf_torus(V3 u, float R, float r);

/* float -> IEEE half, round to nearest even */
static uint16_t float_to_half_rn(float f)
{
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
    const uint32_t ax = x & 0x7FFFFFFFu;
    if (ax >= 0x7F800000u) return (uint16_t)(sign | (ax > 0x7F800000u ? 0x7E00u : 0x7C00u));
    if (ax >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);          /* rounds to infinity */
    if (ax < 0x38800000u) {                                            /* half subnormal or zero */
        if (ax < 0x33000000u) return sign;
        const uint32_t e = ax >> 23;
        const uint32_t m = (ax & 0x7FFFFFu) | 0x800000u;
        const uint32_t shift = 126u - e;
        uint32_t r = m >> shift;
        const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1u);
        if (rem > half || (rem == half && (r & 1u))) ++r;
        return (uint16_t)(sign | r);
    }
    uint32_t h = (ax >> 13) - (112u << 10);
    const uint32_t rem = ax & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
    return (uint16_t)(sign | h);
}

/* IEEE half -> float (exact) */
static float half_to_float(uint16_t h)
{
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t ex = (h >> 10) & 0x1Fu, man = h & 0x3FFu;
    uint32_t bits;
    if (ex == 0) {
        if (man == 0) bits = sign;
        else {                       /* subnormal: renormalise */
            int e = -1;
            uint32_t m = man;
            do { m <<= 1; ++e; } while (!(m & 0x400u));
            bits = sign | ((uint32_t)(112 - e) << 23) | ((m & 0x3FFu) << 13);
        }
    } else if (ex == 31) {
        bits = sign | 0x7F800000u | (man << 13);
    } else {
        bits = sign | ((ex + 112u) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

/* SDF volumes as float grids: the caller's values, or the torus fill of
 * FillSDFVolume (object/sdf/sdf_cache_manager.cuh:16-38).  Half-precision
 * volumes keep their half values (rounded once, as the device stores them). */
static float* make_volume(const ar_sdf_volume* v)
{
    const size_t n = (size_t)v->dims[0] * v->dims[1] * v->dims[2];
    float* g = (float*)malloc((n ? n : 1) * sizeof(float));
    if (v->data) {
        for (size_t i = 0; i < n; ++i)
            g[i] = v->precision == 16 ? half_to_float(((const uint16_t*)v->data)[i]) : ((const float*)v->data)[i];
        return g;
    }
    size_t i = 0;
    for (int z = 0; z < v->dims[2]; ++z)
        for (int y = 0; y < v->dims[1]; ++y)
            for (int x = 0; x < v->dims[0]; ++x, ++i) {
                const float nx = v->dims[0] > 1 ? (float)x / (float)(v->dims[0] - 1) : 0.0f;
                const float ny = v->dims[1] > 1 ? (float)y / (float)(v->dims[1] - 1) : 0.0f;
                const float nz = v->dims[2] > 1 ? (float)z / (float)(v->dims[2] - 1) : 0.0f;
                const float d = sdf_torus(v3(nx - 0.5f, ny - 0.5f, nz - 0.5f), v->fill_info[0], v->fill_info[1]);
                g[i] = v->precision == 16 ? half_to_float(float_to_half_rn(d)) : d;
            }
    return g;
}

or_scene* or_scene_create(const ar_object_desc* objects, size_t count, int flags, int leaf_size, int bin_count)
{
    return or_scene_create_ex(objects, count, NULL, 0, flags, leaf_size, bin_count);
}

or_scene* or_scene_create_ex(const ar_object_desc* objects, size_t count, const ar_sdf_volume* volumes, size_t nvol,
                             int flags, int leaf_size, int bin_count)
{
    or_scene* s = (or_scene*)calloc(1, sizeof(or_scene));
    s->nvol = (int)nvol;
    s->vols = (float**)calloc(nvol ? nvol : 1, sizeof(float*));
    for (size_t v = 0; v < nvol; ++v) s->vols[v] = make_volume(&volumes[v]);
    s->n = (int)count;
    s->flags = flags;
    s->o = (OObj*)calloc(count ? count : 1, sizeof(OObj));
    for (int d = 0; d <= 8; ++d)   /* INTERSECT_EPS (config.cuh:3) */
        s->eps_tab[d] = 1.0e-3f * om_expf(fminf((float)d * 0.5f, 4.0f));
    for (size_t i = 0; i < count; ++i) {
        const ar_object_desc* d = &objects[i];
        OObj* o = &s->o[i];
        o->type = d->type;
        o->visible = d->visible;
        o->center = from_ar(d->center);
        o->extent = vabs(from_ar(d->extent));
        o->mat = d->material;
        euler_to_matrix(from_ar(d->rotation_deg), &o->o2w, &o->w2o);
        if (o->type == AR_OBJ_SDF) {
            o->sdf_kind = d->sdf.kind;
            for (int k = 0; k < 4; ++k) o->sdf_info[k] = d->sdf.info[k];
            if (o->sdf_kind == AR_SDF_VOLUME && d->sdf.volume >= 0 && d->sdf.volume < s->nvol) {
                const ar_sdf_volume* v = &volumes[d->sdf.volume];
                o->vol = s->vols[d->sdf.volume];
                for (int k = 0; k < 3; ++k) o->dims[k] = v->dims[k];
                /* SDFVolumeInfo::ComputeVoxelSize (sdf_volume.cuh:24-44) */
                const V3 inv = v3(1.0f / fmaxf((float)v->dims[0], 1.0f), 1.0f / fmaxf((float)v->dims[1], 1.0f),
                                  1.0f / fmaxf((float)v->dims[2], 1.0f));
                o->vmax = len3(inv) * 2.5f;
            }
        }
        if (o->type == AR_OBJ_TRIANGLE) {
            /* intersection.cuh:27-29 and 75-77 */
            o->p0 = vadd(mmul(&o->o2w, from_ar(d->tri[0].position)), o->center);
            o->p1 = vadd(mmul(&o->o2w, from_ar(d->tri[1].position)), o->center);
            o->p2 = vadd(mmul(&o->o2w, from_ar(d->tri[2].position)), o->center);
            o->n0 = mmul(&o->o2w, from_ar(d->tri[0].normal));
            o->n1 = mmul(&o->o2w, from_ar(d->tri[1].normal));
            o->n2 = mmul(&o->o2w, from_ar(d->tri[2].normal));
        }
        update_proxy(o, (flags & OR_PROXY_OBJECT_CENTER) != 0);
    }
    /* BuildBVH */
    if (leaf_size <= 0) leaf_size = 8;
    if (bin_count <= 0) bin_count = 12;
    BuildCtx c;
    c.s = s;
    c.bins = bin_count < 4 ? 4 : (bin_count > 64 ? 64 : bin_count);
    c.leaf = leaf_size < 1 ? 1 : (leaf_size > 16 ? 16 : leaf_size);
    s->idx = (int*)malloc((count ? count : 1) * sizeof(int));
    for (size_t i = 0; i < count; ++i) s->idx[i] = (int)i;
    if (count > 0) build_rec(&c, 0, (int)count);
    /* Light table (scene.cu:1056-1080) */
    s->lobj = (int*)malloc((count ? count : 1) * sizeof(int));
    s->lprob = (float*)malloc((count ? count : 1) * sizeof(float));
    float total = 0.0f;
    for (size_t i = 0; i < count; ++i) {
        OObj* o = &s->o[i];
        if (o->mat.shading_model == AR_MAT_LIGHT) {
            o->light_index = s->nl;
            const float w = fmaxf(object_area(o, &objects[i]) * luminance3(from_ar(o->mat.emissive)), 1.0e-20f);
            s->lobj[s->nl] = (int)i;
            s->lprob[s->nl] = w;
            total += w;
            s->nl++;
        } else {
            o->light_index = -1;
        }
    }
    for (int l = 0; l < s->nl; ++l) s->lprob[l] = s->lprob[l] / total;
    return s;
}

void or_scene_destroy(or_scene* s)
{
    if (!s) return;
    for (int v = 0; v < s->nvol; ++v) free(s->vols[v]);
    free(s->vols);
    free(s->spec_tab); free(s->lut_lam); free(s->lut_rgb);
    free(s->m_grid);
    free(s->o); free(s->nodes); free(s->idx); free(s->lobj); free(s->lprob); free(s);
}

int64_t or_scene_node_count(const or_scene* s) { return s->nn; }
void or_scene_nodes(const or_scene* s, float* b6, int32_t* l4)
{
    for (int i = 0; i < s->nn; ++i) {
        const ONode* n = &s->nodes[i];
        b6[6 * i + 0] = n->bmin.x; b6[6 * i + 1] = n->bmin.y; b6[6 * i + 2] = n->bmin.z;
        b6[6 * i + 3] = n->bmax.x; b6[6 * i + 4] = n->bmax.y; b6[6 * i + 5] = n->bmax.z;
        l4[4 * i + 0] = n->left; l4[4 * i + 1] = n->right; l4[4 * i + 2] = n->first; l4[4 * i + 3] = n->count;
    }
}
void or_scene_indices(const or_scene* s, int32_t* idx) { memcpy(idx, s->idx, (size_t)s->n * sizeof(int32_t)); }
int64_t or_scene_light_count(const or_scene* s) { return s->nl; }
void or_scene_lights(const or_scene* s, int32_t* obj, float* prob)
{
    for (int l = 0; l < s->nl; ++l) { obj[l] = s->lobj[l]; prob[l] = s->lprob[l]; }
}

/* ------------------------------------------------------------------------ */
/* Intersection (intersection.cuh:15-113, object/aabb.cuh, object/sphere.cuh) */
/* ------------------------------------------------------------------------ */
typedef struct {
    int hit, obj, light;
    float dist;
    V3 pos, nrm;
    int inside;
    /* GBuffer fields used by shading (spectral: responses at the path's
     * wavelength in all three components) */
    V3 albedo, emissive;
    float specular, metallic, roughness, ior, sigma_a;
    int spectral;
} Isect;

static void gbuffer_default(Isect* c)
{
    c->albedo = v3(1.0f, 1.0f, 1.0f); c->emissive = v3(0.0f, 0.0f, 0.0f);
    c->specular = 0.0f; c->metallic = 0.0f; c->roughness = 0.0f; c->ior = 1.5f; c->sigma_a = 100.0f;
}
static void gbuffer_material(Isect* c, const ar_material* m)
{
    c->albedo = from_ar(m->albedo); c->emissive = from_ar(m->emissive);
    c->specular = m->specular; c->metallic = m->metallic; c->roughness = m->roughness;
    c->ior = m->ior; c->sigma_a = m->sigma_a;
}

/* IntersectTriangleObject (intersection.cuh:15-89); world vertices precomputed
 * with the same expression as lines 27-29. */
static int isect_triangle(const or_scene* s, const OObj* o, V3 ro, V3 rd, Isect* out)
{
    if (!o->visible) return 0;
    const V3 e1 = vsub(o->p1, o->p0);
    const V3 e2 = vsub(o->p2, o->p0);
    const V3 h = cross3(rd, e2);
    const float a = dot3(e1, h);
    if (a > -1e-6f && a < 1e-6f) return 0;
    const float f = 1.0f / a;
    const V3 sv = vsub(ro, o->p0);
    const float u = f * dot3(sv, h);
    if (u < 0.0f || u > 1.0f) return 0;
    const V3 q = cross3(sv, e1);
    const float v = f * dot3(rd, q);
    if (v < 0.0f || u + v > 1.0f) return 0;
    const float t = f * dot3(e2, q);
    if (!(t > 1e-5f)) return 0;
    out->hit = 1;
    out->dist = t;
    if (out->obj != -2) { /* -2: caller wants only t */
        out->pos = vadd(ro, vscale(rd, t));
        const float w = 1.0f - u - v;
        const V3 ni = vnormalize(vadd(vadd(vscale(o->n0, w), vscale(o->n1, u)), vscale(o->n2, v)));
        out->inside = dot3(rd, ni) > 0.0f;
        out->nrm = out->inside ? vneg(ni) : ni;
        if (s->flags & OR_TRIANGLE_DEFAULT_GBUFFER) gbuffer_default(out); else gbuffer_material(out, &o->mat);
    }
    return 1;
}

/* IntersectAABBObject (object/aabb.cuh:9-89) */
static int isect_cube(const OObj* o, V3 ro, V3 rd, Isect* out)
{
    const V3 lo = mmul(&o->w2o, vsub(ro, o->center));
    const V3 ld = vnormalize(mmul(&o->w2o, rd));
    const V3 bmin = vneg(o->extent), bmax = o->extent;
    const V3 dv = v3(inv_safe(ld.x), inv_safe(ld.y), inv_safe(ld.z));
    const V3 t1 = vmul(vsub(bmin, lo), dv);
    const V3 t2 = vmul(vsub(bmax, lo), dv);
    const V3 tmn = vmin3(t1, t2), tmx = vmax3(t1, t2);
    const float tEnter = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
    const float tExit = fminf(fminf(tmx.x, tmx.y), tmx.z);
    if (tEnter > tExit) return 0;
    if (tExit <= 0.0f) return 0;
    const int inside = (tEnter < 0.0f);
    const float tHit = inside ? tExit : tEnter;
    out->hit = 1;
    out->dist = tHit;
    if (out->obj != -2) {
        const V3 lp = vadd(lo, vscale(ld, tHit));
        out->pos = vadd(mmul(&o->o2w, lp), o->center);
        const float rx = fabsf(lp.x) / o->extent.x;
        const float ry = fabsf(lp.y) / o->extent.y;
        const float rz = fabsf(lp.z) / o->extent.z;
        V3 ln;
        if (rx >= ry && rx >= rz) ln = v3((lp.x > 0.0f) ? 1.0f : -1.0f, 0.0f, 0.0f);
        else if (ry >= rz) ln = v3(0.0f, (lp.y > 0.0f) ? 1.0f : -1.0f, 0.0f);
        else ln = v3(0.0f, 0.0f, (lp.z > 0.0f) ? 1.0f : -1.0f);
        if (inside) ln = vneg(ln);
        out->nrm = vnormalize(mmul(&o->o2w, ln));
        out->inside = 0;
        gbuffer_material(out, &o->mat);
    }
    return 1;
}

/* IntersectSphereObject (object/sphere.cuh:9-70) */
static int isect_sphere(const OObj* o, V3 ro, V3 rd, Isect* out)
{
    const V3 lo = mmul(&o->w2o, vsub(ro, o->center));
    const V3 ld = vnormalize(mmul(&o->w2o, rd));
    const float r = max3f(o->extent);
    const float b = dot3(lo, ld);
    const float c = dot3(lo, lo) - r * r;
    const float disc = b * b - 1.0f * c;
    if (disc < 0.0f) return 0;
    const float sq = sqrtf(disc);
    float t = -b - sq;
    int inside = 0;
    if (t <= 0.0f) { t = -b + sq; inside = 1; }
    if (t <= 0.0f) return 0;
    out->hit = 1;
    out->dist = t;
    if (out->obj != -2) {
        const V3 lp = vadd(lo, vscale(ld, t));
        const V3 ln = vscale(vnormalize(lp), inside ? -1.0f : 1.0f);
        out->pos = vadd(mmul(&o->o2w, lp), o->center);
        out->nrm = vnormalize(mmul(&o->o2w, ln));
        out->inside = 0;
        gbuffer_material(out, &o->mat);
    }
    return 1;
}

/* ------------------------------------------------------------------------ */
/* SDF objects (object/sdf/ of the reference)                                 */
/* ------------------------------------------------------------------------ */
/* SdfTorus (sdf_torus.cuh:14-18) */
static float sdf_torus(V3 u, float R, float r)
{
    const float qx = sqrtf(u.x * u.x + u.z * u.z) - R;
    return sqrtf(qx * qx + u.y * u.y) - r;
}
static int clampi_(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static size_t grid_index(const OObj* o, int x, int y, int z)
{
    return (size_t)z * o->dims[0] * o->dims[1] + (size_t)y * o->dims[0] + x;
}
/* SampleSDFNearest01 (sdf_volume.cuh:69-83) */
static float grid_nearest(const OObj* o, V3 p)
{
    const V3 q = v3(p.x * (float)(o->dims[0] - 1), p.y * (float)(o->dims[1] - 1), p.z * (float)(o->dims[2] - 1));
    const int x = clampi_((int)floorf(q.x + 0.5f), 0, o->dims[0] - 1);
    const int y = clampi_((int)floorf(q.y + 0.5f), 0, o->dims[1] - 1);
    const int z = clampi_((int)floorf(q.z + 0.5f), 0, o->dims[2] - 1);
    return o->vol[grid_index(o, x, y, z)];
}
/* SampleSDFTrilinear01 (sdf_volume.cuh:85-124) */
static float grid_trilinear(const OObj* o, V3 p)
{
    const V3 q = v3(p.x * (float)(o->dims[0] - 1), p.y * (float)(o->dims[1] - 1), p.z * (float)(o->dims[2] - 1));
    int x0 = (int)floorf(q.x), y0 = (int)floorf(q.y), z0 = (int)floorf(q.z);
    const int x1 = clampi_(x0 + 1, 0, o->dims[0] - 1);
    const int y1 = clampi_(y0 + 1, 0, o->dims[1] - 1);
    const int z1 = clampi_(z0 + 1, 0, o->dims[2] - 1);
    x0 = clampi_(x0, 0, o->dims[0] - 1);
    y0 = clampi_(y0, 0, o->dims[1] - 1);
    z0 = clampi_(z0, 0, o->dims[2] - 1);
    const float fx = fminf(fmaxf(q.x - (float)x0, 0.0f), 1.0f);
    const float fy = fminf(fmaxf(q.y - (float)y0, 0.0f), 1.0f);
    const float fz = fminf(fmaxf(q.z - (float)z0, 0.0f), 1.0f);
    const float* v = o->vol;
    const float c000 = v[grid_index(o, x0, y0, z0)], c100 = v[grid_index(o, x1, y0, z0)];
    const float c010 = v[grid_index(o, x0, y1, z0)], c110 = v[grid_index(o, x1, y1, z0)];
    const float c001 = v[grid_index(o, x0, y0, z1)], c101 = v[grid_index(o, x1, y0, z1)];
    const float c011 = v[grid_index(o, x0, y1, z1)], c111 = v[grid_index(o, x1, y1, z1)];
    const float c00 = c000 * (1.0f - fx) + c100 * fx;
    const float c10 = c010 * (1.0f - fx) + c110 * fx;
    const float c01 = c001 * (1.0f - fx) + c101 * fx;
    const float c11 = c011 * (1.0f - fx) + c111 * fx;
    const float c0 = c00 * (1.0f - fy) + c10 * fy;
    const float c1 = c01 * (1.0f - fy) + c11 * fy;
    return c0 * (1.0f - fz) + c1 * fz;
}
/* SDFTorusFunctor / SDFVolumeFunctor + SampleSDFAdaptive01 (sdf_volume.cuh:143-171) */
static float sdf_eval(const OObj* o, V3 u)
{
    if (o->sdf_kind == AR_SDF_TORUS) return sdf_torus(u, o->sdf_info[0], o->sdf_info[1]);
    if (!o->vol || o->dims[0] * o->dims[1] * o->dims[2] == 0) return 1.0e20f;
    const V3 p = v3(u.x + 0.5f, u.y + 0.5f, u.z + 0.5f);
    const float dn = grid_nearest(o, p);
    return fabsf(dn) > o->vmax ? dn : grid_trilinear(o, p);
}
/* ToUnitSpace (sdf_base.cuh:12-21) */
static V3 to_unit(V3 pl, V3 e)
{
    const float ex = fmaxf(e.x, 1e-8f), ey = fmaxf(e.y, 1e-8f), ez = fmaxf(e.z, 1e-8f);
    return v3(pl.x / (2.0f * ex), pl.y / (2.0f * ey), pl.z / (2.0f * ez));
}
/* IntersectSDFObject + RaymarchLocal + sdfNormalUnit (sdf_base.cuh:40-163);
 * eps_d = INTERSECT_EPS(depth), SDF_EPS = eps_d / 2 (config.cuh:73). */
static int isect_sdf(const OObj* o, V3 ro, V3 rd, float eps_d, Isect* out)
{
    const V3 lo = mmul(&o->w2o, vsub(ro, o->center));
    const V3 ld = vnormalize(mmul(&o->w2o, rd));
    const V3 e = o->extent;
    const V3 dv = v3(inv_safe(ld.x), inv_safe(ld.y), inv_safe(ld.z));
    const V3 t1 = vmul(vsub(vneg(e), lo), dv);
    const V3 t2 = vmul(vsub(e, lo), dv);
    const V3 tmn = vmin3(t1, t2), tmx = vmax3(t1, t2);
    const float tEnter = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
    const float tExit = fminf(fminf(tmx.x, tmx.y), tmx.z);
    if (tEnter > tExit || tExit <= 0.0f) return 0;
    const float eps = eps_d * 0.5f;
    const float minStep = eps * 0.5f;
    const int inside = sdf_eval(o, to_unit(lo, e)) <= 0.0f;
    const float sMin = 2.0f * fminf(e.x, fminf(e.y, e.z));
    float t = fmaxf(0.0f, tEnter);
    float tHit = -1.0f;
    V3 pHit = v3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < 512; ++i) {
        const float tLast = t;
        const V3 pl = vadd(lo, vscale(ld, t));
        const float dLocal = sdf_eval(o, to_unit(pl, e)) * sMin;
        if (inside ? (dLocal > 0.0f && dLocal < eps) : (dLocal < 0.0f && -dLocal < eps)) {
            tHit = tLast;
            pHit = pl;
            break;
        }
        const float adv = o->sdf_kind == AR_SDF_VOLUME ? fmaxf(fabsf(dLocal) * 0.9f, minStep) : fmaxf(fabsf(dLocal), minStep);
        t += adv;
        if (t > tExit) break;
    }
    if (tHit < 0.0f) return 0;
    out->hit = 1;
    out->dist = tHit;
    if (out->obj != -2) {
        const float h = eps / fmaxf(sMin, 1e-8f);
        const V3 u = to_unit(pHit, e);
        const float dx = sdf_eval(o, vadd(u, v3(h, 0.0f, 0.0f))) - sdf_eval(o, vsub(u, v3(h, 0.0f, 0.0f)));
        const float dy = sdf_eval(o, vadd(u, v3(0.0f, h, 0.0f))) - sdf_eval(o, vsub(u, v3(0.0f, h, 0.0f)));
        const float dz = sdf_eval(o, vadd(u, v3(0.0f, 0.0f, h))) - sdf_eval(o, vsub(u, v3(0.0f, 0.0f, h)));
        const V3 nu = vnormalize(v3(dx, dy, dz));
        const float ex = fmaxf(e.x, 1e-8f), ey = fmaxf(e.y, 1e-8f), ez = fmaxf(e.z, 1e-8f);
        const V3 nl = vnormalize(v3(nu.x / (2.0f * ex), nu.y / (2.0f * ey), nu.z / (2.0f * ez)));
        out->pos = vadd(mmul(&o->o2w, pHit), o->center);
        out->nrm = vnormalize(mmul(&o->o2w, nl));
        out->inside = 0;
        gbuffer_material(out, &o->mat);
    }
    return 1;
}

/* IntersectBase (intersection.cuh:93-113).  SDF objects are not part of this
 * restatement; they never hit. */
static int isect_object(const or_scene* s, int i, V3 ro, V3 rd, float eps_d, Isect* out)
{
    const OObj* o = &s->o[i];
    switch (o->type) {
    case AR_OBJ_CUBE: return isect_cube(o, ro, rd, out);
    case AR_OBJ_SPHERE: return isect_sphere(o, ro, rd, out);
    case AR_OBJ_SDF: return isect_sdf(o, ro, rd, eps_d, out);
    case AR_OBJ_TRIANGLE: return isect_triangle(s, o, ro, rd, out);
    default: return 0;
    }
}

/* distance of a hit only (same arithmetic) */
static int isect_t(const or_scene* s, int i, V3 ro, V3 rd, float eps_d, float* t)
{
    Isect c;
    c.hit = 0; c.obj = -2;
    if (!isect_object(s, i, ro, rd, eps_d, &c)) return 0;
    *t = c.dist;
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Traversal (intersection.cuh:235-370, bvh.cuh:424-470)                      */
/* ------------------------------------------------------------------------ */
static inline int slab_ref(V3 ro, V3 inv, V3 mn, V3 mx, float tMin, float tMax, float* tEnterOut)
{
    float t0 = (mn.x - ro.x) * inv.x, t1 = (mx.x - ro.x) * inv.x;
    float te = fminf(t0, t1), tx = fmaxf(t0, t1);
    t0 = (mn.y - ro.y) * inv.y; t1 = (mx.y - ro.y) * inv.y;
    te = fmaxf(te, fminf(t0, t1)); tx = fminf(tx, fmaxf(t0, t1));
    t0 = (mn.z - ro.z) * inv.z; t1 = (mx.z - ro.z) * inv.z;
    te = fmaxf(te, fminf(t0, t1)); tx = fminf(tx, fmaxf(t0, t1));
    if (tx >= fmaxf(0.0f, tMin) && te <= tMax) { *tEnterOut = te; return 1; }
    return 0;
}
static inline int slab_std(V3 ro, V3 inv, V3 mn, V3 mx, float tMin, float tMax, float* tEnterOut)
{
    float t0 = (mn.x - ro.x) * inv.x, t1 = (mx.x - ro.x) * inv.x;
    float te = fminf(t0, t1), tx = fmaxf(t0, t1);
    t0 = (mn.y - ro.y) * inv.y; t1 = (mx.y - ro.y) * inv.y;
    te = fmaxf(te, fminf(t0, t1)); tx = fminf(tx, fmaxf(t0, t1));
    t0 = (mn.z - ro.z) * inv.z; t1 = (mx.z - ro.z) * inv.z;
    te = fmaxf(te, fminf(t0, t1)); tx = fminf(tx, fmaxf(t0, t1));
    te = fmaxf(te, fmaxf(0.0f, tMin));
    tx = fminf(tx * 1.0000004f, tMax);
    if (te <= tx) { *tEnterOut = te; return 1; }
    return 0;
}

typedef struct { int obj; float t; int visits, tests; } TraceResult;

static TraceResult traverse(const or_scene* s, V3 ro, V3 rd, float tMin, float tMax, int any, int mode, float eps_d)
{
    TraceResult r;
    r.obj = -1; r.t = tMax; r.visits = 0; r.tests = 0;
    if (s->nn == 0) return r;
    const int tie_lowest = (mode & OR_TIE_LOWEST_INDEX) != 0;
    const int std_slab = (mode & OR_SLAB_STANDARD) != 0;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    const V3 inv = v3(inv_safe(rd.x), inv_safe(rd.y), inv_safe(rd.z));
    while (sp) {
        const ONode* n = &s->nodes[stack[--sp]];
        r.visits++;
        float te;
        const int ok = std_slab ? slab_std(ro, inv, n->bmin, n->bmax, tMin, r.t, &te)
                                : slab_ref(ro, inv, n->bmin, n->bmax, tMin, r.t, &te);
        if (!ok) continue;
        if (n->count > 0) {
            for (int i = 0; i < n->count; ++i) {
                const int oi = s->idx[n->first + i];
                float t;
                r.tests++;
                if (!isect_t(s, oi, ro, rd, eps_d, &t)) continue;
                if (t < tMin) continue;
                if (t < r.t || (tie_lowest && r.obj >= 0 && t == r.t && oi < r.obj)) {
                    r.t = t; r.obj = oi;
                    if (any) return r;
                }
            }
        } else {
            const ONode* L = &s->nodes[n->left];
            const ONode* R = &s->nodes[n->right];
            float tL = 0.0f, tR = 0.0f;
            const int hL = std_slab ? slab_std(ro, inv, L->bmin, L->bmax, tMin, r.t, &tL)
                                    : slab_ref(ro, inv, L->bmin, L->bmax, tMin, r.t, &tL);
            const int hR = std_slab ? slab_std(ro, inv, R->bmin, R->bmax, tMin, r.t, &tR)
                                    : slab_ref(ro, inv, R->bmin, R->bmax, tMin, r.t, &tR);
            if (hL && hR) {
                if (tL > tR) { if (sp < 128) stack[sp++] = n->left; if (sp < 128) stack[sp++] = n->right; }
                else { if (sp < 128) stack[sp++] = n->right; if (sp < 128) stack[sp++] = n->left; }
            } else if (hL) { if (sp < 128) stack[sp++] = n->left; }
            else if (hR) { if (sp < 128) stack[sp++] = n->right; }
        }
    }
    return r;
}

static TraceResult brute(const or_scene* s, V3 ro, V3 rd, float tMin, float tMax, int any, float eps_d)
{
    TraceResult r;
    r.obj = -1; r.t = tMax; r.visits = 0; r.tests = 0;
    for (int i = 0; i < s->n; ++i) {
        float t;
        if (!isect_t(s, i, ro, rd, eps_d, &t)) continue;
        if (t < tMin || t >= r.t) continue;
        r.t = t; r.obj = i;
        if (any) return r;
    }
    return r;
}

void or_trace_rays(const or_scene* s, const float* rays, int64_t n, int any_hit, int mode,
                   int32_t* hit_object, float* hit_t, int32_t* node_visits, int32_t* prim_tests, int threads)
{
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        const TraceResult r = traverse(s, v3(q[0], q[1], q[2]), v3(q[4], q[5], q[6]), q[3], q[7], any_hit, mode,
                                       s->eps_tab[0]);
        hit_object[i] = r.obj;
        if (hit_t) hit_t[i] = r.obj >= 0 ? r.t : q[7];
        if (node_visits) node_visits[i] = r.visits;
        if (prim_tests) prim_tests[i] = r.tests;
    }
}

void or_trace_rays_brute(const or_scene* s, const float* rays, int64_t n, int any_hit,
                         int32_t* hit_object, float* hit_t, int threads)
{
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        const TraceResult r = brute(s, v3(q[0], q[1], q[2]), v3(q[4], q[5], q[6]), q[3], q[7], any_hit, s->eps_tab[0]);
        hit_object[i] = r.obj;
        if (hit_t) hit_t[i] = r.obj >= 0 ? r.t : q[7];
    }
}

/* Forward declarations of the per-query exports below (defined after the
 * shading helpers they use). */
static int overlap_index(const or_scene* s, V3 p);

/* ------------------------------------------------------------------------ */
/* Random numbers: a tape of curand uniforms, or an own generator             */
/* ------------------------------------------------------------------------ */
typedef struct {
    const float* tape;
    int limit, pos, overflow;
    uint64_t state; /* own generator when tape == NULL */
} Rng;

static inline float rng1(Rng* g)
{
    if (g->tape) {
        if (g->pos >= g->limit) { g->overflow = 1; g->pos++; return 0.5f; }
        return g->tape[g->pos++];
    }
    /* splitmix64 -> uniform in (0, 1] (for the CPU baseline only) */
    uint64_t z = (g->state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z = z ^ (z >> 31);
    g->pos++;
    return (float)((z >> 40) + 1) * 0x1p-24f;
}

/* ------------------------------------------------------------------------ */
/* Sampling and BSDFs (render/sample.cuh, render/brdf.cuh, render/material.cuh) */
/* ------------------------------------------------------------------------ */
typedef struct { V3 dir; float pdf; } Smp;

/* ConcentricSampleDisk (sample.cuh:63-86) */
static void concentric_disk(float ux, float uy, float* dx, float* dy)
{
    const float sx = 2.0f * ux - 1.0f;
    const float sy = 2.0f * uy - 1.0f;
    if (sx == 0.0f && sy == 0.0f) { *dx = 0.0f; *dy = 0.0f; return; }
    float r, phi;
    if (fabsf(sx) > fabsf(sy)) {
        r = sx;
        phi = (OR_PI / 4.0f) * (sy / fmaxf(fabsf(sx), 1e-20f));
    } else {
        r = sy;
        phi = (OR_PI / 2.0f) - (OR_PI / 4.0f) * (sx / fmaxf(fabsf(sy), 1e-20f));
    }
    float sn, cs;
    om_sincosf(phi, &sn, &cs);
    *dx = r * cs; *dy = r * sn;
}

/* SampleCosineWeightedHemisphere (sample.cuh:88-108) */
static Smp sample_cosine(float e0, float e1, float e2, V3 n)
{
    V3 T, Bv;
    tangent_basis_random(n, &T, &Bv, e2);
    float x, y;
    concentric_disk(e0, e1, &x, &y);
    const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
    const V3 dir = vadd(vadd(vscale(T, x), vscale(Bv, y)), vscale(n, z));
    Smp s;
    s.pdf = z / OR_PI;
    s.dir = vnormalize(dir);
    return s;
}

/* FresnelDielectricExact (brdf.cuh:25-32) */
static float fresnel_exact(float cosI, float cosT, float eta)
{
    const float invE = 1.0f / eta;
    const float rPar = (invE * cosI - cosT) / (invE * cosI + cosT);
    const float rPerp = (cosI - invE * cosT) / (cosI + invE * cosT);
    return 0.5f * (rPar * rPar + rPerp * rPerp);
}
static V3 fresnel_schlick3(V3 F0, float cosX)
{
    const float c = clampf_(1.0f - cosX, 0.0f, 1.0f);
    const float c5 = c * c * c * c * c;
    return v3(F0.x + (1.0f - F0.x) * c5, F0.y + (1.0f - F0.y) * c5, F0.z + (1.0f - F0.z) * c5);
}
static float ggx_g_correlated(float alpha, float NoL, float NoV)
{
    const float a2 = alpha * alpha;
    const float gv = NoL * sqrtf(a2 + (1.0f - a2) * NoV * NoV);
    const float gl = NoV * sqrtf(a2 + (1.0f - a2) * NoL * NoL);
    const float denom = gv + gl;
    return (denom > 0.0f) ? (2.0f * NoL * NoV) / denom : 0.0f;
}
static float f0_ue(float spec) { const float s = clampf_(spec, 0.0f, 1.0f); return 0.08f * s; }
static float ggx_d(float alpha, float NoH)
{
    const float a2 = alpha * alpha;
    const float d = NoH * NoH * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxf(OR_PI * d * d, 1e-12f);
}
/* GGXLambert_BRDF (brdf.cuh:96-112) */
static V3 ggx_lambert(V3 V, V3 L, V3 N, V3 F0, float NoV, float kD, float alpha, V3 albedo)
{
    const float NoL = fmaxf(0.0f, dot3(N, L));
    const V3 Hn = vnormalize(vadd(V, L));
    const float NoH = fmaxf(0.0f, dot3(N, Hn));
    const float LoH = fmaxf(0.0f, dot3(L, Hn));
    const V3 F = fresnel_schlick3(F0, LoH);
    const float D = ggx_d(alpha, NoH);
    const float G = ggx_g_correlated(alpha, NoL, NoV);
    V3 spec;
    if (NoL > 0.0f) spec = vdivs(vscale(vscale(F, D), G), fmaxf(4.0f * NoV, 1e-7f));
    else spec = v3(0.0f, 0.0f, 0.0f);
    const V3 omF = v3(1.0f - F.x, 1.0f - F.y, 1.0f - F.z);
    const V3 diff = vscale(vmul(vscale(omF, kD), albedo), NoL / OR_PI);
    return vadd(spec, diff);
}
/* SampleGGXBoundedVNDF (sample.cuh:179-222) */
static Smp sample_ggx_vndf(V3 V, V3 N, float alpha, float r0, float r1, float r2)
{
    V3 X, Y;
    tangent_basis_random(N, &X, &Y, r2);
    const float XoV = dot3(X, V), YoV = dot3(Y, V), NoV = dot3(N, V);
    const V3 localV = v3(XoV, YoV, NoV);
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const V3 lstd = vdivs(v3(XoV * alpha, YoV * alpha, NoV), sqrtf(a2 + (1.0f - a2) * NoV2));
    const float phi = 2.0f * OR_PI * r0;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float b = NoV > 0 ? k * lstd.z : lstd.z;
    const float z = fmaf(1.0f - r1, 1.0f + b, -b);
    const float sinT = sqrtf(saturatef_(1.0f - z * z));
    float sp, cp;
    om_sincosf(phi, &sp, &cp);
    const V3 ostd = v3(sinT * cp, sinT * sp, z);
    const V3 mstd = vadd(lstd, ostd);
    const V3 lh = vnormalize(v3(mstd.x * alpha, mstd.y * alpha, mstd.z));
    const V3 ll = vreflect(vneg(localV), lh);
    const V3 dir = vadd(vadd(vscale(X, ll.x), vscale(Y, ll.y)), vscale(N, ll.z));
    const float ndf = ggx_d(alpha, lh.z);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    Smp s;
    s.dir = dir;
    s.pdf = ndf / (2.0f * (k * NoV + t));
    return s;
}
/* GGXBoundedVNDF_PDF (sample.cuh:224-248) */
static float ggx_vndf_pdf(V3 V, V3 N, V3 L, float alpha)
{
    const float NoV = dot3(N, V), NoL = dot3(N, L);
    if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
    const V3 H = vnormalize(vadd(V, L));
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float NoH = fmaxf(0.0f, dot3(N, H));
    const float ndf = ggx_d(alpha, NoH);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    const float pdf = ndf / (2.0f * (k * NoV + t));
    return fmaxf(pdf, 1e-12f);
}

typedef struct { int inside; V3 vloc; int obj; int depth; } Media; /* MediaContext (material.cuh:12-18) */
typedef struct {
    V3 next; float pdf; V3 emis; V3 brdf;
    int terminate, pure_light, delta, miss_thin;
    Media media;
} SCtx; /* SampleContext (material.cuh:19-37) */

static void sctx_init(SCtx* c)
{
    memset(c, 0, sizeof(*c));
    c->pdf = 1.0f;
    c->media.obj = -1;
}

static V3 bsdf_ggx_params(const Isect* g, float* alpha, float* kD, V3* F0)
{
    *alpha = g->roughness * g->roughness;
    const float f0d = f0_ue(g->specular);
    *F0 = vlerp(v3(f0d, f0d, f0d), g->albedo, g->metallic);
    *kD = 1.0f - g->metallic;
    return *F0;
}

/* EvaluateBSDFWithCos, RGB (material.cuh:48-175) */
static V3 eval_bsdf_cos(int model, V3 rayDir, V3 L, const Isect* ic, const Media* m)
{
    const V3 N = ic->nrm;
    const float NoL = fmaxf(0.0f, dot3(N, L));
    if (model == AR_MAT_DIFFUSE) return vscale(ic->albedo, NoL / OR_PI);
    if (model == AR_MAT_LIGHT) return v3(0.0f, 0.0f, 0.0f);
    if (model == AR_MAT_GGX) {
        const V3 V = vnormalize(vneg(rayDir));
        const float NoV = fmaxf(0.0f, dot3(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
        float alpha, kD; V3 F0;
        bsdf_ggx_params(ic, &alpha, &kD, &F0);
        return ggx_lambert(V, L, N, F0, NoV, kD, alpha, ic->albedo);
    }
    if (model == AR_MAT_GLASS) {
        const float IOR = ic->ior;
        V3 tr = v3(1.0f, 1.0f, 1.0f);
        if (m->inside) {
            /* BeerLambert (brdf.cuh:15-18): exp(d * sigmaA * log(clamp(albedo))) */
            const float d = len3(vsub(m->vloc, ic->pos));
            const V3 al = vmin3(vmaxs(ic->albedo, 1.0e-12f), v3(1.0f, 1.0f, 1.0f));
            const float ds = d * ic->sigma_a;
            tr = v3(om_expf(ds * om_logf(al.x)), om_expf(ds * om_logf(al.y)), om_expf(ds * om_logf(al.z)));
        }
        const V3 nIn = (dot3(N, rayDir) > 0.0f) ? vneg(N) : N;
        const float eta = m->inside ? IOR : 1.0f / IOR;
        const float cosI = -dot3(nIn, rayDir);
        const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
        const float k = 1.0f - sin2I * (eta * eta);
        if (k <= 0.0f) return vscale(tr, 0.99f);
        const float cosT = sqrtf(k);
        const float Fr = fresnel_exact(cosI, cosT, eta);
        const V3 R = vreflect(rayDir, nIn);
        const V3 T = vrefract(rayDir, nIn, eta);
        const float dR = dot3(L, R), dT = dot3(L, T);
        if (dR >= dT) return vscale(tr, Fr);
        const float weight = (eta * eta) * (fabsf(cosT) / fmaxf(1e-6f, cosI));
        return vscale(vscale(tr, 1.0f - Fr), weight);
    }
    return v3(0.0f, 0.0f, 0.0f);
}

/* SampleBSDF, RGB (material.cuh:177-330) */
static SCtx sample_bsdf(Rng* g, int model, V3 rayDir, const Isect* ic, const Media* m)
{
    SCtx r;
    sctx_init(&r);
    const V3 N = ic->nrm;
    const V3 V = vneg(rayDir);
    if (model == AR_MAT_DIFFUSE) {
        const float e0 = rng1(g), e1 = rng1(g), e2 = rng1(g);
        const Smp s = sample_cosine(e0, e1, e2, N);
        r.next = s.dir; r.pdf = s.pdf; r.emis = ic->emissive;
        r.media.inside = m->inside; r.media.vloc = ic->pos;
        return r;
    }
    if (model == AR_MAT_LIGHT) {
        r.pdf = 1.0f; r.emis = ic->emissive; r.terminate = 1; r.pure_light = 1;
        return r;
    }
    if (model == AR_MAT_GLASS) {
        const float IOR = ic->ior;
        r.delta = 1;
        const int inside = m->inside;
        const float eta = inside ? IOR : 1.0f / IOR;
        const V3 nIn = (dot3(N, rayDir) > 0.0f) ? vneg(N) : N;
        const float cosI = -dot3(nIn, rayDir);
        const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
        const float k = 1.0f - sin2I * (eta * eta);
        r.emis = v3(0.0f, 0.0f, 0.0f);
        if (k <= 0.0f) {
            if (m->depth < 1024) {
                r.next = vreflect(rayDir, nIn); r.pdf = 1.0f; r.media.inside = inside; r.media.vloc = ic->pos;
            } else {
                r.next = rayDir; r.pdf = 1.0f; r.media.inside = !inside; r.media.vloc = ic->pos;
            }
            return r;
        }
        const float cosT = sqrtf(k);
        const float Fr = fresnel_exact(cosI, cosT, eta);
        if (rng1(g) < Fr) {
            r.next = vreflect(rayDir, nIn); r.pdf = Fr; r.media.inside = inside; r.media.vloc = ic->pos;
        } else {
            r.next = vrefract(rayDir, nIn, eta); r.pdf = 1.0f - Fr; r.media.inside = !inside; r.media.vloc = ic->pos;
        }
        return r;
    }
    if (model == AR_MAT_GGX) {
        r.emis = ic->emissive;
        const float NoV = fmaxf(0.0f, dot3(N, V));
        if (NoV <= 0.0f) { r.terminate = 1; return r; }
        float alpha, kD; V3 F0;
        bsdf_ggx_params(ic, &alpha, &kD, &F0);
        const float pSpec = clampf_(ic->spectral ? F0.x : luminance3(F0), 0.1f, 0.9f);
        const float u = rng1(g);
        if (u < pSpec) {
            const float e0 = rng1(g), e1 = rng1(g), e2 = rng1(g);
            const Smp s = sample_ggx_vndf(V, N, alpha, e0, e1, e2);
            const V3 L = s.dir;
            const float NoL = fmaxf(0.0f, dot3(N, L));
            if (NoL <= 0.0f) { r.terminate = 1; return r; }
            const float pdfSpec = s.pdf;
            const float pdfDiff = NoL / OR_PI;
            r.next = L; r.pdf = pSpec * pdfSpec + (1.0f - pSpec) * pdfDiff;
        } else {
            const float e0 = rng1(g), e1 = rng1(g), e2 = rng1(g);
            const Smp s = sample_cosine(e0, e1, e2, N);
            const V3 L = s.dir;
            const float pdfDiff = s.pdf;
            const float pdfSpec = ggx_vndf_pdf(V, N, L, alpha);
            r.next = L; r.pdf = pSpec * pdfSpec + (1.0f - pSpec) * pdfDiff;
        }
        r.media.inside = m->inside; r.media.vloc = ic->pos;
        return r;
    }
    return r;
}

/* BSDF_PDF, RGB (material.cuh:332-387) */
static float bsdf_pdf(int model, const Isect* ic, V3 N, V3 rayDir, V3 L)
{
    const V3 V = vneg(rayDir);
    const float NoL = fmaxf(0.0f, dot3(N, L));
    if (model == AR_MAT_DIFFUSE) return NoL > 0.0f ? (NoL * (1.0f / OR_PI)) : 0.0f;
    if (model == AR_MAT_GGX) {
        const float NoV = fmaxf(0.0f, dot3(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
        float alpha, kD; V3 F0;
        bsdf_ggx_params(ic, &alpha, &kD, &F0);
        const float pSpec = clampf_(ic->spectral ? F0.x : luminance3(F0), 0.1f, 0.9f);
        const float pdfSpec = ggx_vndf_pdf(V, N, L, alpha);
        const float pdfDiff = NoL * (1.0f / OR_PI);
        return fmaxf(0.0f, pSpec * pdfSpec + (1.0f - pSpec) * pdfDiff);
    }
    return 0.0f;
}

/* ------------------------------------------------------------------------ */
/* NEE (nee/nee.cuh)                                                          */
/* ------------------------------------------------------------------------ */
typedef struct { int obj; V3 p, n, emis; float pFacet, pA; int valid; } LSmp;

static void obb_axes(const OObj* o, V3* ux, V3* uy, V3* uz)
{
    const M3* M = &o->o2w;
    *ux = vnormalize(v3(M->x.x, M->y.x, M->z.x));
    *uy = vnormalize(v3(M->x.y, M->y.y, M->z.y));
    *uz = vnormalize(v3(M->x.z, M->y.z, M->z.z));
}
static float area_to_solid_angle(V3 sp, V3 lp, V3 ln, float pA)
{
    const V3 s2l = vsub(lp, sp);
    const float d2 = fmaxf(dot3(s2l, s2l), 1e-20f);
    const V3 dir = vscale(s2l, om_rsqrtf(d2));
    const float cosY = fmaxf(0.0f, dot3(ln, vneg(dir)));
    if (cosY <= 0.0f) return 0.0f;
    return pA * (d2 / cosY);
}
static float facing_weight(V3 fn, V3 fc, V3 sp, float area)
{
    const V3 l2s = vnormalize(vsub(sp, fc));
    const float c = fmaxf(0.0f, dot3(fn, l2s));
    return area * c;
}
static void box_facets(const OObj* o, V3 fn[6], V3 fc[6], V3 ft[6], V3 fb[6], float s1[6], float s2[6], float area[6])
{
    V3 ux, uy, uz;
    obb_axes(o, &ux, &uy, &uz);
    const V3 c = o->center, e = o->extent;
    fn[0] = ux; fn[1] = vneg(ux); fn[2] = uy; fn[3] = vneg(uy); fn[4] = uz; fn[5] = vneg(uz);
    fc[0] = vadd(c, vscale(ux, e.x)); fc[1] = vsub(c, vscale(ux, e.x));
    fc[2] = vadd(c, vscale(uy, e.y)); fc[3] = vsub(c, vscale(uy, e.y));
    fc[4] = vadd(c, vscale(uz, e.z)); fc[5] = vsub(c, vscale(uz, e.z));
    ft[0] = uy; ft[1] = uy; ft[2] = ux; ft[3] = ux; ft[4] = ux; ft[5] = ux;
    fb[0] = uz; fb[1] = uz; fb[2] = uz; fb[3] = uz; fb[4] = uy; fb[5] = uy;
    s1[0] = e.y; s1[1] = e.y; s1[2] = e.x; s1[3] = e.x; s1[4] = e.x; s1[5] = e.x;
    s2[0] = e.z; s2[1] = e.z; s2[2] = e.z; s2[3] = e.z; s2[4] = e.y; s2[5] = e.y;
    for (int f = 0; f < 6; ++f) area[f] = 4.0f * s1[f] * s2[f];
}

/* NEEPDFOmegaFromHit_Box (nee.cuh:64-151) */
static float pdf_box(const OObj* o, float selectProb, V3 sp, V3 lp, V3 ln)
{
    V3 fn[6], fc[6], ft[6], fb[6];
    float s1[6], s2[6], area[6];
    box_facets(o, fn, fc, ft, fb, s1, s2, area);
    int hitFacet = -1;
    for (int f = 0; f < 6; ++f) if (dot3(fn[f], ln) > 0.999f) { hitFacet = f; break; }
    if (hitFacet < 0) {
        float best = 1e30f;
        for (int f = 0; f < 6; ++f) {
            const float d = fabsf(dot3(fn[f], vsub(lp, fc[f])));
            if (d < best) { best = d; hitFacet = f; }
        }
    }
    float sum = 0.0f, wHit = 0.0f, aHit = 0.0f;
    for (int f = 0; f < 6; ++f) {
        const float w = facing_weight(fn[f], fc[f], sp, area[f]);
        sum += w;
        if (f == hitFacet) { wHit = w; aHit = area[f]; }
    }
    if (sum <= 0.0f || wHit <= 0.0f) return 0.0f;
    const float pA = selectProb * (1.0f / aHit) * (wHit / sum);
    return area_to_solid_angle(sp, lp, ln, pA);
}

/* NEESampleBoxAreaFacing (nee.cuh:154-251) */
static LSmp sample_box(Rng* g, const OObj* o, V3 cp)
{
    LSmp ls;
    memset(&ls, 0, sizeof(ls));
    V3 fn[6], fc[6], ft[6], fb[6];
    float s1[6], s2[6], area[6];
    box_facets(o, fn, fc, ft, fb, s1, s2, area);
    int vi[6];
    float vw[6];
    int nv = 0;
    float wsum = 0.0f;
    for (int f = 0; f < 6; ++f) {
        const float w = facing_weight(fn[f], fc[f], cp, area[f]);
        if (w > 0.0f) { vi[nv] = f; vw[nv] = w; wsum += w; ++nv; }
    }
    if (nv == 0) return ls;
    int slot = 0, fi = vi[0];
    {
        const float r = rng1(g) * wsum;
        float acc = 0.0f;
        for (int k = 0; k < nv; ++k) {
            acc += vw[k];
            if (r <= acc) { slot = k; fi = vi[k]; break; }
        }
    }
    const float u1 = 2.0f * rng1(g) - 1.0f;
    const float u2 = 2.0f * rng1(g) - 1.0f;
    ls.p = vadd(vadd(fc[fi], vscale(ft[fi], u1 * s1[fi])), vscale(fb[fi], u2 * s2[fi]));
    ls.n = fn[fi];
    ls.emis = from_ar(o->mat.emissive);
    ls.pFacet = 1.0f * (vw[slot] / wsum);
    ls.pA = 1.0f / area[fi];
    ls.valid = 1;
    return ls;
}

/* NEEPDFOmegaFromHit_Sphere (nee.cuh:254-271) */
static float pdf_sphere(const OObj* o, float selectProb, V3 sp, V3 lp, V3 ln)
{
    const float R = max3f(o->extent);
    const float dist = len3(vsub(sp, o->center));
    if (dist <= R) return 0.0f;
    const float cosC = clampf_(R / dist, 0.0f, 1.0f);
    const float areaCap = 2.0f * OR_PI * R * R * (1.0f - cosC);
    if (areaCap <= 1e-20f) return 0.0f;
    const float pA = selectProb / areaCap;
    return area_to_solid_angle(sp, lp, ln, pA);
}

/* NEESampleSphereCapArea (nee.cuh:274-310) */
static LSmp sample_sphere(Rng* g, const OObj* o, V3 cp)
{
    LSmp ls;
    memset(&ls, 0, sizeof(ls));
    const V3 c = o->center;
    const float R = max3f(o->extent);
    const V3 p2c = vsub(cp, c);
    const float dist = len3(p2c);
    if (dist <= R) return ls;
    const V3 axis = vdivs(p2c, dist);
    const float cosC = clampf_(R / dist, 0.0f, 1.0f);
    const float areaCap = 2.0f * OR_PI * R * R * (1.0f - cosC);
    const float u = rng1(g);
    const float vphi = rng1(g);
    const float cosT = lerpf_(cosC, 1.0f, u);
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    const float phi = 2.0f * OR_PI * vphi;
    V3 t, b;
    tangent_basis(axis, &t, &b);
    float sp, cph;
    om_sincosf(phi, &sp, &cph);
    const V3 n = vadd(vadd(vscale(t, cph * sinT), vscale(b, sp * sinT)), vscale(axis, cosT));
    ls.p = vadd(c, vscale(n, R));
    ls.n = n;
    ls.emis = from_ar(o->mat.emissive);
    ls.pFacet = 1.0f;
    ls.pA = 1.0f / areaCap;
    ls.valid = 1;
    return ls;
}

/* NEESampleLight (nee.cuh:330-377) */
/* Extension (not in the reference): emissive triangles as NEE lights, a
 * uniform point by the square-root warp, two-sided (normal turned to p). */
static V3 tri_light_normal(const OObj* o, V3 p, V3 lp)
{
    const V3 n = vnormalize(cross3(vsub(o->p1, o->p0), vsub(o->p2, o->p0)));
    return dot3(n, vsub(p, lp)) < 0.0f ? vneg(n) : n;
}
static float tri_light_area(const OObj* o) { return 0.5f * len3(cross3(vsub(o->p1, o->p0), vsub(o->p2, o->p0))); }
static LSmp sample_triangle(Rng* g, const OObj* o, V3 sp)
{
    LSmp ls;
    memset(&ls, 0, sizeof(ls));
    const float area = tri_light_area(o);
    if (!(area > 0.0f)) return ls;
    const float u1 = rng1(g), u2 = rng1(g);
    const float su = sqrtf(u1);
    const V3 e1 = vsub(o->p1, o->p0), e2 = vsub(o->p2, o->p0);
    ls.p = vadd(vadd(o->p0, vscale(e1, su * (1.0f - u2))), vscale(e2, su * u2));
    ls.n = tri_light_normal(o, sp, ls.p);
    ls.emis = from_ar(o->mat.emissive);
    ls.pFacet = 1.0f;
    ls.pA = 1.0f / area;
    ls.valid = 1;
    return ls;
}

static LSmp sample_light(const or_scene* s, V3 sp, Rng* g, int tri)
{
    LSmp none;
    memset(&none, 0, sizeof(none));
    if (s->nl <= 0) return none;
    int pick = s->nl - 1;
    float pprob = 0.0f;
    {
        const float rr = rng1(g);
        float acc = 0.0f;
        for (int l = 0; l < s->nl; ++l) {
            const float p = s->lprob[l];
            acc += p;
            if (rr < acc) { pick = l; pprob = p; break; }
        }
    }
    const OObj* lo = &s->o[s->lobj[pick]];
    LSmp ls = none;
    if (lo->type == AR_OBJ_CUBE) ls = sample_box(g, lo, sp);
    else if (lo->type == AR_OBJ_SPHERE) ls = sample_sphere(g, lo, sp);
    else if (tri && lo->type == AR_OBJ_TRIANGLE) ls = sample_triangle(g, lo, sp);
    if (!ls.valid) return none;
    ls.obj = s->lobj[pick];
    ls.pFacet = ls.pFacet * pprob;
    return ls;
}

static float area_to_solid_angle(V3 sp, V3 lp, V3 ln, float pA);
static float pdf_light_from_hit(const or_scene* s, int obj, V3 sp, V3 lp, V3 ln, int tri)
{
    const OObj* o = &s->o[obj];
    const float sel = s->lprob[o->light_index];
    if (o->type == AR_OBJ_CUBE) return pdf_box(o, sel, sp, lp, ln);
    if (o->type == AR_OBJ_SPHERE) return pdf_sphere(o, sel, sp, lp, ln);
    if (tri && o->type == AR_OBJ_TRIANGLE) {
        const float area = tri_light_area(o);
        if (!(area > 0.0f)) return 0.0f;
        return area_to_solid_angle(sp, lp, tri_light_normal(o, sp, lp), sel * (1.0f / area));
    }
    return 0.0f;
}

static float power_heuristic(float pA, float pB)
{
    const float a = pA * pA, b = pB * pB;
    return a / fmaxf(1e-24f, a + b);
}

/* SkyLighting (render.cuh:58-73) */
static V3 sky_lighting(V3 d, int sky)
{
    if (!sky) return v3(0.0f, 0.0f, 0.0f);
    const V3 white = v3(1.0f, 1.0f, 1.0f);
    const V3 blue = v3(0.05f, 0.45f, 1.0f);
    const V3 down = vscale(v3(0.2f, 0.6f, 1.0f), 0.125f);
    const V3 inner = vlerp(blue, white, om_powf(fmaxf(d.y, 0.0f), 0.75f));
    const V3 l = vlerp(inner, down, fminf(fmaxf(-d.y * 0.5f + 0.5f, 0.0f), 1.0f));
    return vscale(l, 0.5f);
}

/* ------------------------------------------------------------------------ */
/* Path loop                                                                  */
/* ------------------------------------------------------------------------ */
typedef struct {
    int64_t ext_rays, shadow_rays;
    /* optional recorders of every query (8 floats per ray) */
    float* ext_out; int64_t ext_cap;
    float* sh_out; int64_t sh_cap;
} Counters;

static void record_ray(float* out, int64_t cap, int64_t k, V3 o, float tmin, V3 d, float tmax)
{
    if (!out || k >= cap) return;
    float* r = out + 8 * k;
    r[0] = o.x; r[1] = o.y; r[2] = o.z; r[3] = tmin; r[4] = d.x; r[5] = d.y; r[6] = d.z; r[7] = tmax;
}

static int path_mode(const or_scene* s)
{
    return (s->flags & OR_REFERENCE_TRAVERSAL) ? (OR_TIE_FIRST_FOUND | OR_SLAB_REFERENCE)
                                               : (OR_TIE_LOWEST_INDEX | OR_SLAB_STANDARD);
}

static int closest(const or_scene* s, V3 ro, V3 rd, float tMin, Isect* out)
{
    /* Trace's closest hit: tMin is INTERSECT_EPS(depth), also the SDF tolerance */
    const TraceResult r = traverse(s, ro, rd, tMin, INFINITY, 0, path_mode(s), tMin);
    if (r.obj < 0) return 0;
    memset(out, 0, sizeof(*out));
    out->obj = r.obj;
    isect_object(s, r.obj, ro, rd, tMin, out);
    out->obj = r.obj;
    out->light = s->o[r.obj].light_index;
    return 1;
}

/* AnyHitSegmentBVH (intersection.cuh:372-397) */
/* ------------------------------------------------------------------------ */
/* Heterogeneous participating medium (extension; no reference counterpart:   */
/* the reference's Henyey-Greenstein helpers, sample.cuh:110-145, are unused). */
/* Same arithmetic, in the same order, as the device code: delta tracking     */
/* (Woodcock) for free flights, ratio tracking for shadow transmittance,      */
/* Henyey-Greenstein by CDF inversion, lowbias32 counter-based uniforms.      */
/* ------------------------------------------------------------------------ */
static uint32_t lowbias32(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
typedef struct { uint32_t seed, n; } HashRng;
static float hash_next(HashRng* h)
{
    const uint32_t v = lowbias32(h->seed ^ lowbias32(h->n++ * 0x9E3779B9u + 0x632BE5ABu));
    return ((float)(v >> 8) + 0.5f) * (1.0f / 16777216.0f);
}
static uint32_t medium_frame_key(uint64_t seed, uint64_t frame0)
{
    uint32_t h = lowbias32((uint32_t)seed ^ 0x6D2B79F5u);
    h = lowbias32(h ^ (uint32_t)(seed >> 32));
    h = lowbias32(h ^ (uint32_t)frame0);
    return lowbias32(h ^ (uint32_t)(frame0 >> 32));
}
static uint32_t medium_seed(uint32_t key, uint32_t sample, uint32_t pixel, uint32_t depth, uint32_t salt)
{
    uint32_t h = lowbias32(key ^ sample);
    h = lowbias32(h ^ pixel);
    return lowbias32(h ^ (depth * 2u + salt));
}
static int clamp_index(int v, int hi) { return v < 0 ? 0 : (v > hi ? hi : v); }
/* trilinear between voxel centres, clamped at the faces */
static float medium_density(const or_scene* s, V3 p)
{
    const float gx = (p.x - s->m_bmin[0]) / (s->m_bmax[0] - s->m_bmin[0]) * (float)s->m_dims[0] - 0.5f;
    const float gy = (p.y - s->m_bmin[1]) / (s->m_bmax[1] - s->m_bmin[1]) * (float)s->m_dims[1] - 0.5f;
    const float gz = (p.z - s->m_bmin[2]) / (s->m_bmax[2] - s->m_bmin[2]) * (float)s->m_dims[2] - 0.5f;
    const float fx0 = floorf(gx), fy0 = floorf(gy), fz0 = floorf(gz);
    const float tx = gx - fx0, ty = gy - fy0, tz = gz - fz0;
    const int X = s->m_dims[0] - 1, Y = s->m_dims[1] - 1, Z = s->m_dims[2] - 1;
    const int x0 = clamp_index((int)fx0, X), x1 = clamp_index((int)fx0 + 1, X);
    const int y0 = clamp_index((int)fy0, Y), y1 = clamp_index((int)fy0 + 1, Y);
    const int z0 = clamp_index((int)fz0, Z), z1 = clamp_index((int)fz0 + 1, Z);
    const size_t sy = (size_t)s->m_dims[0], sz = (size_t)s->m_dims[0] * (size_t)s->m_dims[1];
    const float* g = s->m_grid;
    const float c000 = g[x0 + y0 * sy + z0 * sz], c100 = g[x1 + y0 * sy + z0 * sz];
    const float c010 = g[x0 + y1 * sy + z0 * sz], c110 = g[x1 + y1 * sy + z0 * sz];
    const float c001 = g[x0 + y0 * sy + z1 * sz], c101 = g[x1 + y0 * sy + z1 * sz];
    const float c011 = g[x0 + y1 * sy + z1 * sz], c111 = g[x1 + y1 * sy + z1 * sz];
    const float c00 = c000 * (1.0f - tx) + c100 * tx, c10 = c010 * (1.0f - tx) + c110 * tx;
    const float c01 = c001 * (1.0f - tx) + c101 * tx, c11 = c011 * (1.0f - tx) + c111 * tx;
    const float c0 = c00 * (1.0f - ty) + c10 * ty, c1 = c01 * (1.0f - ty) + c11 * ty;
    return c0 * (1.0f - tz) + c1 * tz;
}
static int medium_span(const or_scene* s, V3 o, V3 d, float tmax, float* t0, float* t1)
{
    const V3 inv = v3(inv_safe(d.x), inv_safe(d.y), inv_safe(d.z));
    const V3 a = vmul(vsub(v3(s->m_bmin[0], s->m_bmin[1], s->m_bmin[2]), o), inv);
    const V3 b = vmul(vsub(v3(s->m_bmax[0], s->m_bmax[1], s->m_bmax[2]), o), inv);
    const V3 lo = vmin3(a, b), hi = vmax3(a, b);
    *t0 = fmaxf(fmaxf(fmaxf(lo.x, lo.y), lo.z), 0.0f);
    *t1 = fminf(fminf(fminf(hi.x, hi.y), hi.z), tmax);
    return *t0 < *t1 && s->m_major > 0.0f;
}
#define OR_MEDIUM_MAX_STEPS 4096
static float delta_track(const or_scene* s, V3 o, V3 d, float tmax, HashRng* h)
{
    float t0, t1;
    if (!medium_span(s, o, d, tmax, &t0, &t1)) return -1.0f;
    float t = t0;
    for (int i = 0; i < OR_MEDIUM_MAX_STEPS; ++i) {
        t = t - om_logf(1.0f - hash_next(h) * 0.99999994f) / s->m_major;
        if (t >= t1) return -1.0f;
        const float sg = medium_density(s, vadd(o, vscale(d, t))) * s->m_sigma;
        if (hash_next(h) * s->m_major < sg) return t;
    }
    return -1.0f;
}
static float ratio_track(const or_scene* s, V3 o, V3 d, float tmax, HashRng* h)
{
    float t0, t1;
    if (!medium_span(s, o, d, tmax, &t0, &t1)) return 1.0f;
    float t = t0, tr = 1.0f;
    for (int i = 0; i < OR_MEDIUM_MAX_STEPS; ++i) {
        t = t - om_logf(1.0f - hash_next(h) * 0.99999994f) / s->m_major;
        if (t >= t1) break;
        tr = tr * (1.0f - medium_density(s, vadd(o, vscale(d, t))) * s->m_sigma / s->m_major);
        if (tr <= 0.0f) return 0.0f;
    }
    return tr;
}
static float hg_phase(float g, float cosT)
{
    const float den = 1.0f + g * g - 2.0f * g * cosT;
    return (1.0f - g * g) / (4.0f * 3.14159265358979f * den * sqrtf(den));
}
static V3 hg_sample(V3 d, float g, float u1, float u2)
{
    float cosT;
    if (fabsf(g) < 1e-3f) {
        cosT = 1.0f - 2.0f * u1;
    } else {
        const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
        cosT = (1.0f + g * g - sq * sq) / (2.0f * g);
    }
    cosT = fminf(fmaxf(cosT, -1.0f), 1.0f);
    const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
    float sp, cp;
    om_sincosf(2.0f * 3.14159265358979f * u2, &sp, &cp);
    const V3 a = fabsf(d.z) < 0.999f ? v3(0.0f, 0.0f, 1.0f) : v3(1.0f, 0.0f, 0.0f);
    const V3 t = vnormalize(cross3(a, d));
    const V3 b = cross3(d, t);
    return vnormalize(vadd(vadd(vscale(t, sinT * cp), vscale(b, sinT * sp)), vscale(d, cosT)));
}
/* transmittance of an unoccluded shadow segment, with the geometry of
 * segment_occluded (1 when the segment is too short to be traced) */
static float segment_transmittance(const or_scene* s, float eps_d, V3 src, V3 dst, uint32_t seed)
{
    V3 dir = vsub(dst, src);
    const float dist = len3(dir);
    if (dist <= 0.0f) return 1.0f;
    dir = vdivs(dir, dist);
    const float eps = eps_d * fmaxf(1.0f, fmaxf(len3(src), len3(dst)));
    const float tMax = fmaxf(0.0f, dist - eps);
    if (tMax <= 0.0f) return 1.0f;
    HashRng h;
    h.seed = seed; h.n = 0;
    return ratio_track(s, src, dir, tMax, &h);
}

int or_scene_set_medium(or_scene* s, const ar_medium_desc* m)
{
    free(s->m_grid);
    s->m_grid = NULL;
    s->has_medium = 0;
    if (!m) return 0;
    const size_t n = (size_t)m->dims[0] * (size_t)m->dims[1] * (size_t)m->dims[2];
    s->m_grid = (float*)malloc(n * sizeof(float));
    float mx = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        const float v = m->precision == 16 ? half_to_float(((const uint16_t*)m->density)[i]) : ((const float*)m->density)[i];
        s->m_grid[i] = v;
        mx = fmaxf(mx, v);
    }
    for (int a = 0; a < 3; ++a) {
        s->m_bmin[a] = m->bounds_min[a]; s->m_bmax[a] = m->bounds_max[a];
        s->m_albedo[a] = m->albedo[a]; s->m_dims[a] = m->dims[a];
    }
    s->m_sigma = m->sigma_t_max;
    s->m_g = m->g;
    s->m_major = m->sigma_t_max * mx;
    s->has_medium = 1;
    return 0;
}

float or_medium_density(const or_scene* s, const float* p3) { return medium_density(s, v3(p3[0], p3[1], p3[2])); }

void or_hg_sample(const float* d3, float g, const float* u2, int64_t n, float* out3)
{
    for (int64_t i = 0; i < n; ++i) {
        const V3 r = hg_sample(v3(d3[0], d3[1], d3[2]), g, u2[2 * i], u2[2 * i + 1]);
        out3[3 * i] = r.x; out3[3 * i + 1] = r.y; out3[3 * i + 2] = r.z;
    }
}

float or_hg_phase(float g, float cosT) { return hg_phase(g, cosT); }

void or_medium_track(const or_scene* s, const float* rays8, int64_t n, const uint32_t* seeds, int ratio, float* out)
{
    for (int64_t i = 0; i < n; ++i) {
        const float* r = rays8 + 8 * i;
        HashRng h;
        h.seed = seeds[i]; h.n = 0;
        const V3 o = v3(r[0], r[1], r[2]), d = v3(r[4], r[5], r[6]);
        out[i] = ratio ? ratio_track(s, o, d, r[7], &h) : delta_track(s, o, d, r[7], &h);
    }
}

static int segment_occluded(const or_scene* s, float eps_d, V3 src, V3 dst, Counters* cnt)
{
    V3 dir = vsub(dst, src);
    const float dist = len3(dir);
    if (dist <= 0.0f) return 0;
    dir = vdivs(dir, dist);
    const float eps = eps_d * fmaxf(1.0f, fmaxf(len3(src), len3(dst)));
    const float tMax = fmaxf(0.0f, dist - eps);
    if (tMax <= 0.0f) return 0;
    record_ray(cnt->sh_out, cnt->sh_cap, cnt->shadow_rays, src, 0.0f, dir, tMax);
    cnt->shadow_rays++;
    const TraceResult r = traverse(s, src, dir, 0.0f, tMax, 1, path_mode(s), eps_d);
    return r.obj >= 0;
}

/* ------------------------------------------------------------------------ */
/* Spectral mode (core/spectrum/ of the reference, USE_SPECTRUM_RENDERING)    */
/* ------------------------------------------------------------------------ */
/* offsets of the table block (ar_scene_set_spectral layout) */
enum { SP_CMF = 0, SP_D65 = 1263, SP_RGB_IN_W = 1684, SP_RGB_IN_B = 2708, SP_RGB_BLK_W = 2740,
       SP_RGB_BLK_B = 9908, SP_RGB_OUT_W = 10132, SP_LAM_BLK_W = 10260, SP_LAM_BLK_B = 17428,
       SP_LAM_OUT_W = 17652, SP_FLOATS = 17780, SP_LAMBDA_RES = 840 };
#define SP_PI 3.141592654f /* CUDART_PI_F */

/* D65Norm (ciexyz.cuh:67-82) */
static float sp_d65(const float* tab, float l)
{
    const float* d = tab + SP_D65;
    const float k = 1.0f / 10567.065f;
    if (l <= 360.0f) return d[0] * k;
    if (l >= 780.0f) return d[420] * k;
    const float x = l - 360.0f;
    const int i = (int)floorf(x);
    const float t = x - (float)i;
    return (d[i] + (d[i + 1] - d[i]) * t) * k;
}
/* LambdaToCIE1931_XYZ (ciexyz.cuh:522-541) */
static V3 sp_cmf(const float* tab, float l)
{
    const float* c = tab + SP_CMF;
    if (l <= 360.0f) return v3(c[0], c[1], c[2]);
    if (l >= 780.0f) return v3(c[1260], c[1261], c[1262]);
    const float u = (l - 360.0f) * (1.0f / 1.0f);
    const int i = (int)u;
    const float t = u - (float)i;
    const float* a = c + 3 * i;
    const float* b = a + 3;
    return v3(a[0] + (b[0] - a[0]) * t, a[1] + (b[1] - a[1]) * t, a[2] + (b[2] - a[2]) * t);
}
/* erfc: Numerical Recipes 6.2 rational approximation (fractional error < 1.2e-7) */
static float sp_erfc(float x)
{
    const float z = fabsf(x);
    const float t = 1.0f / (1.0f + 0.5f * z);
    const float p = -z * z - 1.26551223f +
                    t * (1.00002368f + t * (0.37409196f + t * (0.09678418f + t * (-0.18628806f +
                    t * (0.27886807f + t * (-1.13520398f + t * (1.48851587f + t * (-0.82215223f + t * 0.17087277f))))))));
    const float r = t * om_expf(p);
    return x >= 0.0f ? r : 2.0f - r;
}
/* ndtrif (sample_ciexyz.cuh:28-156): Acklam's inverse normal CDF + one Newton step */
static float sp_ndtri(float u)
{
    const float uu = fminf(fmaxf(u, 0.0f), 1.0f);
    const float pLow = 0.02425f, pHigh = 1.0f - 0.02425f;
    float x;
    if (uu < pLow || uu > pHigh) {
        const float q = uu < pLow ? sqrtf(-2.0f * om_logf(uu)) : sqrtf(-2.0f * om_logf(1.0f - uu));
        float num = fmaf(-7.784894002430293e-03f, q, -3.223964580411365e-01f);
        num = fmaf(num, q, -2.400758277161838e+00f);
        num = fmaf(num, q, -2.549732539343734e+00f);
        num = fmaf(num, q, 4.374664141464968e+00f);
        num = fmaf(num, q, 2.938163982698783e+00f);
        float den = fmaf(7.784695709041462e-03f, q, 3.224671290700398e-01f);
        den = fmaf(den, q, 2.445134137142996e+00f);
        den = fmaf(den, q, 3.754408661907416e+00f);
        den = fmaf(den, q, 1.0f);
        x = uu < pLow ? num / den : -num / den;
    } else {
        const float q = uu - 0.5f;
        const float r = q * q;
        float num = fmaf(-3.969683028665376e+01f, r, 2.209460984245205e+02f);
        num = fmaf(num, r, -2.759285104469687e+02f);
        num = fmaf(num, r, 1.383577518672690e+02f);
        num = fmaf(num, r, -3.066479806614716e+01f);
        num = fmaf(num, r, 2.506628277459239e+00f);
        num *= q;
        float den = fmaf(-5.447609879822406e+01f, r, 1.615858368580409e+02f);
        den = fmaf(den, r, -1.556989798598866e+02f);
        den = fmaf(den, r, 6.680131188771972e+01f);
        den = fmaf(den, r, -1.328068155288572e+01f);
        den = fmaf(den, r, 1.0f);
        x = num / den;
    }
    const float pdf = om_expf(fmaf(-0.5f, x * x, 0.0f)) * 0.3989422804014327f;
    const float cdf = 0.5f * sp_erfc(-x * 0.7071067811865476f);
    x -= (cdf - uu) / pdf;
    return x;
}
static float sp_clamp_l(float h) { return h < 360.0f ? 360.0f : (h > 780.0f ? 780.0f : h); }
/* single-lobe CMF fits (Wyman, Sloan, Shirley 2013; sample_ciexyz.cuh:243-279) */
static float sp_fx(float l)
{
    const float k1 = (l - 595.8f) / 33.33f, k2 = (l - 446.8f) / 19.44f;
    return 1.065f * om_expf(-0.5f * k1 * k1) + 0.366f * om_expf(-0.5f * k2 * k2);
}
static float sp_fy(float l) { const float k = (om_logf(l) - 6.3213077f) / 0.075f; return 1.014f * om_expf(-0.5f * k * k); }
static float sp_fz(float l) { const float k = (om_logf(l) - 6.1088030f) / 0.051f; return 1.839f * om_expf(-0.5f * k * k); }
/* SampleCIE1931 (sample_ciexyz.cuh:288-325) */
static void sp_sample(float r0, float r1, float r2, float* lambda, float* pdf)
{
    const float total = 0.1f + 1.0f + 1.0f + 1.0f;
    const float ur = 0.1f / total, xr = 1.0f / total, yr = 1.0f / total, zr = 1.0f / total;
    float l;
    if (r0 < ur) {
        l = r1 * (780.0f - 360.0f) + 360.0f;
    } else if (r0 < ur + xr) {
        float h;
        if (r1 < 0.8330258723493694f) {
            const float t0 = 7.4884543e-13f + r2 * (0.9999999836707862f - 7.4884543e-13f);
            h = 595.7999999999999545f + 33.3299999999999983f * sp_ndtri(t0);
        } else {
            const float t1 = 0.0000040030528583f + r2 * (1.0f - 0.0000040030528583f);
            h = 446.8000000000000114f + 19.4400000000000013f * sp_ndtri(t1);
        }
        l = sp_clamp_l(h);
    } else if (r0 < ur + xr + yr) {
        const float t = 0.0000000020798312f + r1 * (0.9999953206338883f - 0.0000000020798312f);
        l = sp_clamp_l(om_expf(6.3269327170812479f + 0.0750000000000000f * sp_ndtri(t)));
    } else {
        const float t = 0.0000049890553249f + r1 * (1.0f - 0.0000049890553249f);
        l = sp_clamp_l(om_expf(6.1114040395252154f + 0.0510000000000000f * sp_ndtri(t)));
    }
    const float pMix = ur * 1.0f / (780.0f - 360.0f) + xr * (sp_fx(l) / 106.81109281f) + yr * (sp_fy(l) / 106.34513640f) +
                       zr * (sp_fz(l) / 105.88243587f);
    *lambda = l;
    *pdf = fmaxf(pMix, 1e-16f);
}
/* IORFromAbbeNM / SigmaAFromTiltNM (spectrum.cuh:8-54) */
static float sp_ior(float l, float nd, float vd)
{
    if (!(l > 0.0f)) return nd;
    const float invF = 1.0f / 486.1327f, invC = 1.0f / 656.2725f, invD = 1.0f / 587.5618f;
    const float K = (vd > 0.0f) ? (nd - 1.0f) / (vd * (invF - invC)) : 0.0f;
    return nd + K * (1.0f / l - invD);
}
static float sp_sigma(float sA, float l, float tilt)
{
    const float invF = 1.0f / 486.1327f, invC = 1.0f / 656.2725f, invD = 1.0f / 587.5618f;
    const float u = 1.0f / fmaxf(l, 1.0e-6f);
    const float du = (u - invD) / (invF - invC);
    return fmaxf(0.0f, sA * (1.0f + 1.0f * tilt * du));
}
/* networks (spectrum_basis.cuh:2262-2459): residual width-32 MLPs, layers
 * accumulated in input order with fma (tensor::LinearRowMajor) */
static void sp_block(float* h, const float* W, const float* B)
{
    float t[32];
    for (int i = 0; i < 32; ++i) {
        float a = B[i];
        for (int j = 0; j < 32; ++j) a = fmaf(h[j], W[i * 32 + j], a);
        t[i] = fmaxf(a, 0.0f);
    }
    for (int i = 0; i < 32; ++i) h[i] = h[i] + t[i];
}
static void sp_out(const float* h, const float* W, float* o)
{
    for (int i = 0; i < 4; ++i) {
        float a = 0.0f;
        for (int j = 0; j < 32; ++j) a = fmaf(h[j], W[i * 32 + j], a);
        o[i] = a;
    }
}
static void sp_rgb_encode(const float* tab, float r, float g, float b, float* k)
{
    const float scale = fmaxf(fmaxf(r, g), b);
    const float inv = 1.0f / (scale + 0.001f);
    const float in[3] = {r, g, b};
    float sv[32], h[32];
    for (int c = 0; c < 3; ++c)
        for (int q = 0; q < 4; ++q) om_sincosf(in[c] * inv * SP_PI * (float)(q + 1), &sv[8 * c + q], &sv[8 * c + q + 4]);
    for (int q = 0; q < 4; ++q) om_sincosf(scale * SP_PI * (float)(q + 1), &sv[24 + q], &sv[28 + q]);
    for (int i = 0; i < 32; ++i) {
        float a = tab[SP_RGB_IN_B + i];
        for (int j = 0; j < 32; ++j) a = fmaf(sv[j], tab[SP_RGB_IN_W + i * 32 + j], a);
        h[i] = fmaxf(a, 0.0f);
    }
    for (int blk = 0; blk < 7; ++blk) sp_block(h, tab + SP_RGB_BLK_W + blk * 1024, tab + SP_RGB_BLK_B + blk * 32);
    sp_out(h, tab + SP_RGB_OUT_W, k);
    for (int i = 0; i < 4; ++i) k[i] *= scale;
}
static void sp_lambda_encode(const float* tab, float l, float* k)
{
    const float x = fminf(fmaxf((l - 360.0f) / (780.0f - 360.0f), 0.0f), 1.0f);
    float h[32];
    for (int q = 0; q < 16; ++q) om_sincosf(x * SP_PI * (float)(q + 1), &h[q], &h[q + 16]);
    for (int blk = 0; blk < 7; ++blk) sp_block(h, tab + SP_LAM_BLK_W + blk * 1024, tab + SP_LAM_BLK_B + blk * 32);
    sp_out(h, tab + SP_LAM_OUT_W, k);
}
/* QueryLambda / QueryRGBBasis / Interact (spectrum_lut.cuh:92-236) */
static void sp_linear(float g, int res, int* i0, int* i1, float* t)
{
    const float f = floorf(g);
    *i0 = (int)f;
    *i1 = *i0 + 1;
    if (*i1 >= res) *i1 = res - 1;
    *t = g - f;
    if (*i0 == *i1) *t = 0.0f;
}
static void sp_query_lambda(const or_scene* s, float l, float* k)
{
    float u = (l - 360.0f) / (780.0f - 360.0f);
    u = fminf(fmaxf(u, 0.0f), 1.0f);
    float g = u * (float)SP_LAMBDA_RES - 0.5f;
    g = fminf(fmaxf(g, 0.0f), (float)SP_LAMBDA_RES - 1.0f);
    int i0, i1;
    float t;
    sp_linear(g, SP_LAMBDA_RES, &i0, &i1, &t);
    const float w0 = 1.0f - t, w1 = t;
    for (int q = 0; q < 4; ++q) k[q] = s->lut_lam[4 * i0 + q] * w0 + s->lut_lam[4 * i1 + q] * w1;
}
static void sp_acc(const float* v, float w, float* o) { for (int q = 0; q < 4; ++q) o[q] = fmaf(w, v[q], o[q]); }
static void sp_query_rgb(const or_scene* s, V3 c, float* k)
{
    const int res = s->spec_res;
    const float mx = (float)res - 1.0f;
    const float gx = fminf(fmaxf(c.x * (float)res - 0.5f, 0.0f), mx);
    const float gy = fminf(fmaxf(c.y * (float)res - 0.5f, 0.0f), mx);
    const float gz = fminf(fmaxf(c.z * (float)res - 0.5f, 0.0f), mx);
    int x0, x1, y0, y1, z0, z1;
    float tx, ty, tz;
    sp_linear(gx, res, &x0, &x1, &tx);
    sp_linear(gy, res, &y0, &y1, &ty);
    sp_linear(gz, res, &z0, &z1, &tz);
    const float wx0 = 1.0f - tx, wx1 = tx, wy0 = 1.0f - ty, wy1 = ty, wz0 = 1.0f - tz, wz1 = tz;
    const float* L = s->lut_rgb;
    const size_t sy = (size_t)res, sz = (size_t)res * res;
    k[0] = k[1] = k[2] = k[3] = 0.0f;
    sp_acc(L + 4 * (x0 + y0 * sy + z0 * sz), wx0 * wy0 * wz0, k);
    sp_acc(L + 4 * (x1 + y0 * sy + z0 * sz), wx1 * wy0 * wz0, k);
    sp_acc(L + 4 * (x0 + y1 * sy + z0 * sz), wx0 * wy1 * wz0, k);
    sp_acc(L + 4 * (x1 + y1 * sy + z0 * sz), wx1 * wy1 * wz0, k);
    sp_acc(L + 4 * (x0 + y0 * sy + z1 * sz), wx0 * wy0 * wz1, k);
    sp_acc(L + 4 * (x1 + y0 * sy + z1 * sz), wx1 * wy0 * wz1, k);
    sp_acc(L + 4 * (x0 + y1 * sy + z1 * sz), wx0 * wy1 * wz1, k);
    sp_acc(L + 4 * (x1 + y1 * sy + z1 * sz), wx1 * wy1 * wz1, k);
}
static float sp_dot(const float* a, const float* b)
{
    float acc = 0.0f;
    for (int i = 0; i < 4; ++i) acc = fmaf(a[i], b[i], acc);
    return fminf(fmaxf(acc, 0.0f), 1.0f);
}
static float sp_interact(const or_scene* s, const float* lk, V3 rgb)
{
    const float lum = fmaxf(rgb.x, fmaxf(rgb.y, rgb.z));
    float k[4];
    if (lum > 1.0f) {
        sp_query_rgb(s, v3(rgb.x / lum, rgb.y / lum, rgb.z / lum), k);
        return sp_dot(k, lk) * lum;
    }
    sp_query_rgb(s, rgb, k);
    return sp_dot(k, lk);
}

/* Spectral tables and the lookup tables built from them (PrecomputeRGBLUTKernel /
 * PrecomputeLambdaLUTKernel, spectrum_lut.cuh:12-58). */
int or_scene_set_spectral(or_scene* s, const float* tables, size_t count, int res, int threads)
{
    if (count != SP_FLOATS || res < 2 || res > 512) return -1;
    free(s->spec_tab); free(s->lut_lam); free(s->lut_rgb);
    s->spec_tab = (float*)malloc(count * sizeof(float));
    memcpy(s->spec_tab, tables, count * sizeof(float));
    s->lut_lam = (float*)malloc(SP_LAMBDA_RES * 4 * sizeof(float));
    const size_t nrgb = (size_t)res * res * res;
    s->lut_rgb = (float*)malloc(nrgb * 4 * sizeof(float));
    s->spec_res = res;
    const float step = (780.0f - 360.0f) / (float)SP_LAMBDA_RES;
    for (int i = 0; i < SP_LAMBDA_RES; ++i) sp_lambda_encode(s->spec_tab, 360.0f + ((float)i + 0.5f) * step, s->lut_lam + 4 * i);
    const float invRes = 1.0f / (float)res;
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nthreads)
#endif
    for (int64_t v = 0; v < (int64_t)nrgb; ++v) {
        const int x = (int)(v % res), y = (int)((v / res) % res), z = (int)(v / ((int64_t)res * res));
        sp_rgb_encode(s->spec_tab, ((float)x + 0.5f) * invRes, ((float)y + 0.5f) * invRes, ((float)z + 0.5f) * invRes,
                      s->lut_rgb + 4 * v);
    }
    return 0;
}
void or_spectral_luts(const or_scene* s, float* lam, float* rgb)
{
    if (lam) memcpy(lam, s->lut_lam, SP_LAMBDA_RES * 4 * sizeof(float));
    if (rgb) memcpy(rgb, s->lut_rgb, (size_t)s->spec_res * s->spec_res * s->spec_res * 4 * sizeof(float));
}
void or_spectral_sample(const float* u3, int64_t n, float* lambda, float* pdf)
{
    for (int64_t i = 0; i < n; ++i) sp_sample(u3[3 * i], u3[3 * i + 1], u3[3 * i + 2], &lambda[i], &pdf[i]);
}
void or_spectral_encode(const float* tables, const float* rgb, const float* lambda, int64_t n, float* rgb_k, float* lam_k)
{
    for (int64_t i = 0; i < n; ++i) {
        if (rgb) sp_rgb_encode(tables, rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2], rgb_k + 4 * i);
        if (lambda) sp_lambda_encode(tables, lambda[i], lam_k + 4 * i);
    }
}
/* Interact at wavelengths lambda[i] of colours rgb[i] through the scene's tables;
 * also D65Norm and the colour matching functions there. */
void or_spectral_interact(const or_scene* s, const float* lambda, const float* rgb, int64_t n, float* resp, float* d65,
                          float* xyz)
{
    for (int64_t i = 0; i < n; ++i) {
        float lk[4];
        sp_query_lambda(s, lambda[i], lk);
        resp[i] = sp_interact(s, lk, v3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
        d65[i] = sp_d65(s->spec_tab, lambda[i]);
        const V3 c = sp_cmf(s->spec_tab, lambda[i]);
        xyz[3 * i] = c.x; xyz[3 * i + 1] = c.y; xyz[3 * i + 2] = c.z;
    }
}

/* the path's wavelength and the values that follow from it */
typedef struct { int on; float lambda, pdf, d65; float lk[4]; } Spec;

/* the hit's G-buffer at the path's wavelength (EvaluateMaterial, spectral) */
static void sp_apply(const or_scene* s, const Spec* sp, Isect* ic, const ar_material* m)
{
    const float a = sp_interact(s, sp->lk, ic->albedo);
    const float e = sp_interact(s, sp->lk, ic->emissive);
    ic->albedo = v3(a, a, a);
    ic->emissive = v3(e, e, e);
    ic->ior = sp_ior(sp->lambda, ic->ior, m->abbe_number);
    ic->sigma_a = sp_sigma(ic->sigma_a, sp->lambda, m->tilt_number);
    ic->spectral = 1;
}

typedef struct { V3 radiance; int segments, nee_rays, nee_mask; int hits[AR_DEBUG_MAX_HITS]; } PathOut;

/* CalculateRadiance<bUseBVH=true, bUseNEE, bUsePathGuiding=false>, RGB
 * (render.cuh:460-999), with camera_inside = intersection::Overlap at the
 * camera position (render.cuh:536-538). */
static void calculate_radiance(const or_scene* s, const ar_render_params* p, int camera_inside,
                               Rng* g, V3 ro, V3 rd, PathOut* po, Counters* cnt,
                               uint32_t mkey, uint32_t sample, uint32_t pixel)
{
    int nonDelta = 0;
    Spec sp;
    memset(&sp, 0, sizeof(sp));
    sp.d65 = 1.0f;
    if (p->spectral && s->spec_tab) {  /* SampleCIE1931(Rand3(seed)) (render.cuh:467-473) */
        const float r0 = rng1(g), r1 = rng1(g), r2 = rng1(g);
        sp.on = 1;
        sp_sample(r0, r1, r2, &sp.lambda, &sp.pdf);
        sp_query_lambda(s, sp.lambda, sp.lk);
        sp.d65 = sp_d65(s->spec_tab, sp.lambda);
    }
    rd = vnormalize(rd);
    V3 radiance = v3(0.0f, 0.0f, 0.0f);
    V3 mask = v3(1.0f, 1.0f, 1.0f);
    V3 cro = ro, crd = rd;
    Media media;
    media.inside = camera_inside; media.vloc = ro; media.obj = -1; media.depth = 0;
    int prevDidNEE = 0;
    float prevPdf = 0.0f;
    V3 prevPos = v3(0.0f, 0.0f, 0.0f);
    po->segments = 0; po->nee_rays = 0; po->nee_mask = 0;
    for (int k = 0; k < AR_DEBUG_MAX_HITS; ++k) po->hits[k] = -1;
    for (int depth = 0; depth < p->max_depth; depth++) {
        /* ---- Trace (render.cuh:75-163), depth argument = nonDeltaDepth ---- */
        const float eps = s->eps_tab[nonDelta < 8 ? nonDelta : 8];
        Isect ic;
        memset(&ic, 0, sizeof(ic));
        ic.obj = -1; ic.light = -1;
        int hit;
        record_ray(cnt->ext_out, cnt->ext_cap, cnt->ext_rays, cro, eps, crd, INFINITY);
        cnt->ext_rays++;
        if (media.inside && media.obj >= 0 &&
            (s->o[media.obj].type != AR_OBJ_TRIANGLE || (s->flags & OR_TRIANGLE_SOLO_MEDIA))) {
            /* solo trace (intersection.cuh:185-193) */
            Isect t;
            memset(&t, 0, sizeof(t));
            t.obj = -1;
            hit = isect_object(s, media.obj, cro, crd, eps, &t) && !(t.dist < eps);
            if (hit) { ic = t; ic.obj = media.obj; ic.light = s->o[media.obj].light_index; }
            else { memset(&ic, 0, sizeof(ic)); ic.obj = -1; ic.light = -1; }
        } else {
            hit = closest(s, cro, crd, eps, &ic);
        }
        if (s->has_medium && !media.inside) {
            /* free flight in the medium up to the surface (extension) */
            HashRng hr;
            hr.seed = medium_seed(mkey, sample, pixel, (uint32_t)depth, 0u); hr.n = 0;
            const float tc = delta_track(s, cro, crd, hit ? ic.dist : INFINITY, &hr);
            if (tc >= 0.0f) {
                if (po->segments < AR_DEBUG_MAX_HITS) po->hits[po->segments] = -2;
                po->segments++;
                const V3 pos = vadd(cro, vscale(crd, tc));
                const float u1 = rng1(g), u2 = rng1(g);
                const V3 next = hg_sample(crd, s->m_g, u1, u2);
                const float pdf = hg_phase(s->m_g, dot3(crd, next));
                V3 alb = v3(s->m_albedo[0], s->m_albedo[1], s->m_albedo[2]);
                if (sp.on) { const float a = sp_interact(s, sp.lk, alb); alb = v3(a, a, a); }
                const V3 brdf = vscale(alb, pdf);
                const float lum = sp.on ? mask.x : luminance3(mask);
                const float useNEERate = sqrtf(saturatef_(lum));
                int neeValid = 0;
                if (p->use_nee && nonDelta < 10 && rng1(g) < useNEERate) {
                    LSmp ls = sample_light(s, pos, g, p->tri_light_nee);
                    if (sp.on) { const float e = sp_interact(s, sp.lk, ls.emis); ls.emis = v3(e, e, e); }
                    if (ls.valid) {
                        const float pATotal = fmaxf(1e-20f, ls.pA * ls.pFacet);
                        const V3 lu = vsub(ls.p, pos);
                        const float d2 = fmaxf(dot3(lu, lu), 1.0e-12f);
                        const V3 ld = vscale(lu, om_rsqrtf(d2));
                        po->nee_rays++;
                        if (depth < 32) po->nee_mask |= (int)(1u << depth);
                        const float epsS = s->eps_tab[depth < 8 ? depth : 8];
                        if (segment_occluded(s, epsS, pos, ls.p, cnt)) {
                            neeValid = 1;
                        } else {
                            const float cosY = fmaxf(0.0f, dot3(ls.n, vneg(ld)));
                            if (cosY > 0.0f) {
                                const V3 f = vscale(alb, hg_phase(s->m_g, dot3(crd, ld)));
                                const float G = cosY / d2;
                                const V3 contrib = vscale(vmul(f, ls.emis), G / pATotal);
                                neeValid = 1;
                                const float pL = area_to_solid_angle(pos, ls.p, ls.n, ls.pFacet * ls.pA);
                                const float pB = hg_phase(s->m_g, dot3(crd, ld));
                                const float w = power_heuristic(pL, pB);
                                const float tr = segment_transmittance(
                                    s, epsS, pos, ls.p, medium_seed(mkey, sample, pixel, (uint32_t)depth, 1u) & ~1u);
                                radiance = vadd(radiance, vscale(vscale(vmul(mask, vscale(contrib, w)), sp.d65), tr));
                            }
                        }
                    }
                }
                prevDidNEE = neeValid;
                prevPdf = pdf;
                prevPos = pos;
                const V3 contrib = v3(brdf.x / fmaxf(pdf, 1e-12f), brdf.y / fmaxf(pdf, 1e-12f), brdf.z / fmaxf(pdf, 1e-12f));
                float q = 1.0f;
                if (nonDelta >= p->rr_depth) {
                    const float mx = sp.on ? mask.x : max3f(mask);
                    const float basic = clampf_(lum * 0.5f + mx * 0.5f, 0.05f, 0.95f);
                    q = lerpf_(basic, 1.0f, 0.0f);
                    if (rng1(g) > q) break;
                }
                mask = vmul(mask, contrib);
                mask = vdivs(mask, q);
                cro = pos;
                crd = next;
                media.vloc = pos;
                nonDelta++;
                continue;
            }
        }
        if (po->segments < AR_DEBUG_MAX_HITS) po->hits[po->segments] = hit ? ic.obj : -1;
        po->segments++;
        SCtx sc;
        sctx_init(&sc);
        int model = -1;
        if (!hit && media.inside) {
            sc.miss_thin = 1;
            ic.obj = media.obj; /* traceResult.intersectionContext_.objectIndex_ */
            sc.media.vloc = cro;  /* hitLocalPosition_ = rayOrigin */
        }
        if (hit) {
            model = s->o[ic.obj].mat.shading_model;
            if (sp.on) sp_apply(s, &sp, &ic, &s->o[ic.obj].mat);
            const SCtx sb = sample_bsdf(g, model, crd, &ic, &media);
            sc = sb;
            sc.media.obj = ic.obj;
            sc.media.depth = media.depth + 1;
            sc.brdf = eval_bsdf_cos(model, crd, sc.next, &ic, &media);
        } else {
            sc.brdf = v3(1.0f, 1.0f, 1.0f);
            sc.delta = 0;
            sc.next = crd;
            sc.pdf = 1.0f;
            sc.emis = sky_lighting(crd, p->sky);
            if (sp.on) { const float e = sp_interact(s, sp.lk, sc.emis); sc.emis = v3(e, e, e); }
            sc.media.inside = 0;
        }
        {
            /* offset, always one Rand1 (render.cuh:156-160) */
            const float offEps = eps * fmaxf(1.0f, len3(ic.pos));
            const float sg = signf_(dot3(ic.nrm, sc.next));
            const float r = rng1(g);
            ic.pos = vadd(ic.pos, vscale(vscale(vscale(ic.nrm, sg), offEps), r + 0.5f));
        }
        media = sc.media;
        /* ---- emission (render.cuh:648-723) ---- */
        if (!hit) {
            if (!sc.miss_thin) radiance = vadd(radiance, vscale(vmul(mask, sc.emis), sp.d65));
        } else if (ic.light >= 0) {
            float misW = 1.0f;
            if (p->use_nee && depth > 0 && prevDidNEE) {
                const float pB = fmaxf(prevPdf, 0.0f);
                const float pL = pdf_light_from_hit(s, ic.obj, prevPos, ic.pos, ic.nrm, p->tri_light_nee);
                if (pL >= 0.0f && pB > 0.0f) misW = power_heuristic(pB, pL);
            }
            radiance = vadd(radiance, vscale(vscale(vmul(mask, sc.emis), sp.d65), misW));
        }
        if ((!hit && !sc.miss_thin) || sc.terminate) break;
        /* ---- NEE (render.cuh:766-827) ---- */
        if (!sc.miss_thin) {
            const float lum = sp.on ? mask.x : luminance3(mask);
            const float useNEERate = sqrtf(saturatef_(lum));
            int neeValid = 0;
            if (p->use_nee && nonDelta < 10 && !sc.delta && !media.inside && rng1(g) < useNEERate) {
                LSmp ls = sample_light(s, ic.pos, g, p->tri_light_nee);
                if (sp.on) { const float e = sp_interact(s, sp.lk, ls.emis); ls.emis = v3(e, e, e); }
                if (ls.valid) {
                    const float pATotal = fmaxf(1e-20f, ls.pA * ls.pFacet);
                    const V3 lu = vsub(ls.p, ic.pos);
                    const float d2 = fmaxf(dot3(lu, lu), 1.0e-12f);
                    const V3 ld = vscale(lu, om_rsqrtf(d2));
                    po->nee_rays++;
                    if (depth < 32) po->nee_mask |= (int)(1u << depth);
                    const int occ = segment_occluded(s, s->eps_tab[depth < 8 ? depth : 8], ic.pos, ls.p, cnt);
                    if (occ) {
                        neeValid = 1;
                    } else {
                        const float cosX = fmaxf(0.0f, dot3(ic.nrm, ld));
                        const float cosY = fmaxf(0.0f, dot3(ls.n, vneg(ld)));
                        if (cosX <= 0.0f || cosY <= 0.0f) {
                            neeValid = 0;
                        } else {
                            Media none;
                            memset(&none, 0, sizeof(none));
                            none.obj = -1;
                            const V3 f = eval_bsdf_cos(model, crd, ld, &ic, &none);
                            const float G = cosY / d2;
                            const V3 contrib = vscale(vmul(f, ls.emis), G / pATotal);
                            neeValid = 1;
                            const float pL = area_to_solid_angle(ic.pos, ls.p, ls.n, ls.pFacet * ls.pA);
                            const float pB = fmaxf(bsdf_pdf(model, &ic, ic.nrm, crd, ld), 0.0f);
                            const float w = power_heuristic(pL, pB);
                            const float tr = s->has_medium
                                ? segment_transmittance(s, s->eps_tab[depth < 8 ? depth : 8], ic.pos, ls.p,
                                                        medium_seed(mkey, sample, pixel, (uint32_t)depth, 1u) & ~1u)
                                : 1.0f;
                            radiance = vadd(radiance, vscale(vscale(vmul(mask, vscale(contrib, w)), sp.d65), tr));
                        }
                    }
                }
            }
            prevDidNEE = neeValid;
            prevPdf = sc.pdf;
            prevPos = ic.pos;
        }
        const V3 contrib = v3(sc.brdf.x / fmaxf(sc.pdf, 1e-12f), sc.brdf.y / fmaxf(sc.pdf, 1e-12f),
                              sc.brdf.z / fmaxf(sc.pdf, 1e-12f));
        float q = 1.0f;
        if (nonDelta >= p->rr_depth) {
            const float lum = sp.on ? mask.x : luminance3(mask);
            const float mx = sp.on ? mask.x : max3f(mask);
            const float basic = clampf_(lum * 0.5f + mx * 0.5f, 0.05f, 0.95f);
            q = lerpf_(basic, 1.0f, media.inside ? 0.99f : 0.0f);
            if (rng1(g) > q) break;
        }
        mask = vmul(mask, contrib);
        mask = vdivs(mask, q);
        cro = ic.pos;
        crd = sc.next;
        if (!sc.delta) nonDelta++;
    }
    /* checkNanInf + clamp (render.cuh:966-969), max(0, .) (scene.cu:238); spectral:
     * lambdaXYZ * radiance / pdf, linear CIE XYZ */
    V3 v = v3(fix_nan_inf(radiance.x), fix_nan_inf(radiance.y), fix_nan_inf(radiance.z));
    if (sp.on) {
        const V3 c = sp_cmf(s->spec_tab, sp.lambda);
        const float r = fix_nan_inf(radiance.x);
        v = v3((c.x * r) / sp.pdf, (c.y * r) / sp.pdf, (c.z * r) / sp.pdf);
    }
    V3 out = v3(clampf_(v.x, 0.0f, 1.0e3f), clampf_(v.y, 0.0f, 1.0e3f), clampf_(v.z, 0.0f, 1.0e3f));
    po->radiance = vmaxs(out, 0.0f);
}

/* intersection::Overlap (intersection.cuh:399-414): the first object that
 * contains p, or -1 */
static int overlap_index(const or_scene* s, V3 p)
{
    for (int i = 0; i < s->n; ++i) {
        const OObj* o = &s->o[i];
        if (o->type == AR_OBJ_CUBE) {
            const V3 l = mmul(&o->w2o, vsub(p, o->center));
            const V3 mn = vneg(o->extent), mx = o->extent;
            if (mn.x < l.x && mn.y < l.y && mn.z < l.z && mx.x > l.x && mx.y > l.y && mx.z > l.z) return i;
        } else if (o->type == AR_OBJ_SPHERE) {
            const V3 l = mmul(&o->w2o, vsub(p, o->center));
            const float r = max3f(o->extent);
            if (dot3(l, l) < r * r) return i;
        } else if (o->type == AR_OBJ_SDF) {
            /* OverlapSDFObject (sdf_base.cuh:166-177) */
            if (sdf_eval(o, to_unit(mmul(&o->w2o, vsub(p, o->center)), o->extent)) <= 0.0f) return i;
        }
    }
    return -1;
}

/* at the camera position */
static int camera_overlap(const or_scene* s, V3 p) { return overlap_index(s, p) >= 0; }

/* RenderCamera ray generation (scene.cu:213-230), field of view as parameter */
void or_camera_ray(const ar_camera* cam, int i, int j, float jx, float jy, float* ray8)
{
    const float u = ((float)i + jx) / (float)cam->width;
    const float v = ((float)j + jy) / (float)cam->height;
    const float ndcx = u * 2.0f - 1.0f;
    const float ndcy = (float)((1.0 - (double)v) * 2.0 - 1.0);
    const float fov = cam->fov_y_deg * 3.1415926f / 180.0f;
    const float aspect = (float)cam->width / fmaxf(1.0f, (float)cam->height);
    const float tanHalfY = om_tanf(0.5f * fov);
    const float tanHalfX = tanHalfY * aspect;
    const float sx = ndcx * tanHalfX;
    const float sy = ndcy * tanHalfY;
    const V3 cd = from_ar(cam->direction);
    const V3 right = vnormalize(cross3(cd, v3(0.0f, 1.0f, 0.0f)));
    const V3 up = vnormalize(cross3(cd, right));
    const V3 d = vnormalize(vadd(vadd(cd, vscale(right, sx)), vscale(up, sy)));
    ray8[0] = cam->position.x; ray8[1] = cam->position.y; ray8[2] = cam->position.z; ray8[3] = 0.0f;
    ray8[4] = d.x; ray8[5] = d.y; ray8[6] = d.z; ray8[7] = INFINITY;
}

int64_t or_render_paths(const or_scene* s, const ar_camera* cam, const ar_render_params* p,
                        const float* tape, int per_path, ar_path_record* rec, int threads)
{
    const int64_t W = cam->width, H = cam->height, S = p->spp;
    const int inside = camera_overlap(s, from_ar(cam->position));
    const uint32_t mkey = medium_frame_key(p->seed, (uint64_t)p->frame_offset);
    int64_t overflow = 0;
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : overflow) num_threads(nthreads)
#endif
    for (int64_t k = 0; k < W * H * S; ++k) {
        const int i = (int)(k % W), j = (int)((k / W) % H);
        const uint32_t smp = (uint32_t)(k / (W * H)), pix = (uint32_t)(k % (W * H));
        Rng g;
        g.tape = tape + k * per_path; g.limit = per_path; g.pos = 0; g.overflow = 0; g.state = 0;
        const float jx = rng1(&g), jy = rng1(&g);
        float ray[8];
        or_camera_ray(cam, i, j, jx, jy, ray);
        PathOut po;
        Counters cnt;
        memset(&cnt, 0, sizeof(cnt));
        calculate_radiance(s, p, inside, &g, v3(ray[0], ray[1], ray[2]), v3(ray[4], ray[5], ray[6]), &po, &cnt,
                           mkey, smp, pix);
        ar_path_record* r = &rec[k];
        memset(r, 0, sizeof(*r));
        r->radiance[0] = po.radiance.x; r->radiance[1] = po.radiance.y; r->radiance[2] = po.radiance.z;
        r->segments = po.segments;
        r->uniforms = g.pos;
        r->nee_rays = po.nee_rays;
        r->nee_depth_mask = po.nee_mask;
        for (int h = 0; h < AR_DEBUG_MAX_HITS; ++h) r->hit_object[h] = po.hits[h];
        if (g.overflow) overflow++;
    }
    return overflow;
}

void or_render_image(const or_scene* s, const ar_camera* cam, const ar_render_params* p,
                     int64_t pb, int64_t pe, int64_t step, double* accum, int64_t* ext, int64_t* shadow, int threads)
{
    const int64_t W = cam->width;
    const int inside = camera_overlap(s, from_ar(cam->position));
    const uint32_t mkey = medium_frame_key(p->seed, (uint64_t)p->frame_offset);
    int64_t e = 0, sh = 0;
    if (step < 1) step = 1;
    const int64_t count = (pe - pb + step - 1) / step;
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : e, sh) num_threads(nthreads)
#endif
    for (int64_t k = 0; k < count; ++k) {
        const int64_t pix = pb + k * step;
        const int i = (int)(pix % W), j = (int)(pix / W);
        double acc[3] = {0.0, 0.0, 0.0};
        Counters cnt;
        memset(&cnt, 0, sizeof(cnt));
        for (int smp = 0; smp < p->spp; ++smp) {
            Rng g;
            g.tape = NULL; g.limit = 0; g.pos = 0; g.overflow = 0;
            g.state = p->seed ^ ((uint64_t)pix * 0x9e3779b97f4a7c15ull) ^ ((uint64_t)(smp + p->frame_offset) << 40);
            const float jx = rng1(&g), jy = rng1(&g);
            float ray[8];
            or_camera_ray(cam, i, j, jx, jy, ray);
            PathOut po;
            calculate_radiance(s, p, inside, &g, v3(ray[0], ray[1], ray[2]), v3(ray[4], ray[5], ray[6]), &po, &cnt,
                               mkey, (uint32_t)smp, (uint32_t)pix);
            acc[0] += po.radiance.x; acc[1] += po.radiance.y; acc[2] += po.radiance.z;
        }
        accum[3 * pix + 0] += acc[0]; accum[3 * pix + 1] += acc[1]; accum[3 * pix + 2] += acc[2];
        e += cnt.ext_rays; sh += cnt.shadow_rays;
    }
    if (ext) *ext = e;
    if (shadow) *shadow = sh;
}

float or_sinf(float x) { return om_sinf(x); }
float or_cosf(float x) { return om_cosf(x); }
float or_expf(float x) { return om_expf(x); }
float or_logf(float x) { return om_logf(x); }
float or_powf(float x, float y) { return om_powf(x, y); }

int64_t or_collect_rays(const or_scene* s, const ar_camera* cam, const ar_render_params* p, int64_t pb, int64_t pe,
                        float* ext, int64_t ext_cap, int64_t* n_ext, float* sh, int64_t sh_cap, int64_t* n_sh)
{
    const int64_t W = cam->width;
    const int inside = camera_overlap(s, from_ar(cam->position));
    const uint32_t mkey = medium_frame_key(p->seed, (uint64_t)p->frame_offset);
    Counters cnt;
    memset(&cnt, 0, sizeof(cnt));
    cnt.ext_out = ext; cnt.ext_cap = ext_cap; cnt.sh_out = sh; cnt.sh_cap = sh_cap;
    for (int64_t pix = pb; pix < pe; ++pix) {
        const int i = (int)(pix % W), j = (int)(pix / W);
        for (int smp = 0; smp < p->spp; ++smp) {
            Rng g;
            g.tape = NULL; g.limit = 0; g.pos = 0; g.overflow = 0;
            g.state = p->seed ^ ((uint64_t)pix * 0x9e3779b97f4a7c15ull) ^ ((uint64_t)(smp + p->frame_offset) << 40);
            const float jx = rng1(&g), jy = rng1(&g);
            float ray[8];
            or_camera_ray(cam, i, j, jx, jy, ray);
            PathOut po;
            calculate_radiance(s, p, inside, &g, v3(ray[0], ray[1], ray[2]), v3(ray[4], ray[5], ray[6]), &po, &cnt,
                               mkey, (uint32_t)smp, (uint32_t)pix);
        }
    }
    *n_ext = cnt.ext_rays < ext_cap ? cnt.ext_rays : ext_cap;
    *n_sh = cnt.shadow_rays < sh_cap ? cnt.shadow_rays : sh_cap;
    return cnt.ext_rays + cnt.shadow_rays;
}

/* ------------------------------------------------------------------------ */
/* Per-query exports used to pin the restatement against the reference       */
/* ------------------------------------------------------------------------ */
void or_trace_detail(const or_scene* s, const float* rays, int64_t n, int mode, int32_t* hit_object, float* hit_t,
                     float* pos, float* nrm, int32_t* inside, int threads)
{
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        const V3 ro = v3(q[0], q[1], q[2]), rd = v3(q[4], q[5], q[6]);
        const TraceResult r = traverse(s, ro, rd, q[3], q[7], 0, mode, s->eps_tab[0]);
        hit_object[i] = r.obj;
        hit_t[i] = r.obj >= 0 ? r.t : q[7];
        Isect c;
        memset(&c, 0, sizeof(c));
        if (r.obj >= 0) isect_object(s, r.obj, ro, rd, s->eps_tab[0], &c);
        pos[3 * i + 0] = c.pos.x; pos[3 * i + 1] = c.pos.y; pos[3 * i + 2] = c.pos.z;
        nrm[3 * i + 0] = c.nrm.x; nrm[3 * i + 1] = c.nrm.y; nrm[3 * i + 2] = c.nrm.z;
        inside[i] = r.obj >= 0 ? c.inside : 0;
    }
}

void or_segments_occluded(const or_scene* s, const float* seg6, const int32_t* depth, int64_t n, int mode,
                          int32_t* occluded, int threads)
{
#ifdef _OPENMP
    const int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        const float* q = seg6 + 6 * i;
        const V3 src = v3(q[0], q[1], q[2]), dst = v3(q[3], q[4], q[5]);
        const int d = depth[i] < 8 ? (depth[i] < 0 ? 0 : depth[i]) : 8;
        V3 dir = vsub(dst, src);
        const float dist = len3(dir);
        occluded[i] = 0;
        if (dist <= 0.0f) continue;
        dir = vdivs(dir, dist);
        const float eps = s->eps_tab[d] * fmaxf(1.0f, fmaxf(len3(src), len3(dst)));
        const float tMax = fmaxf(0.0f, dist - eps);
        if (tMax <= 0.0f) continue;
        occluded[i] = traverse(s, src, dir, 0.0f, tMax, 1, mode, s->eps_tab[d]).obj >= 0;
    }
}

void or_overlap(const or_scene* s, const float* p3, int64_t n, int32_t* object_index)
{
    for (int64_t i = 0; i < n; ++i) object_index[i] = overlap_index(s, v3(p3[3 * i], p3[3 * i + 1], p3[3 * i + 2]));
}

float or_bsdf_pdf(int model, const ar_material* m, const float* N, const float* ray_dir, const float* L)
{
    Isect c;
    memset(&c, 0, sizeof(c));
    gbuffer_material(&c, m);
    return bsdf_pdf(model, &c, v3(N[0], N[1], N[2]), v3(ray_dir[0], ray_dir[1], ray_dir[2]), v3(L[0], L[1], L[2]));
}

float or_power_heuristic(float a, float b) { return power_heuristic(a, b); }

/* ------------------------------------------------------------------------ */
/* Output epilogue: Tonemap kernel (scene.cu:180-199), curves of tonemap.cuh  */
/* ------------------------------------------------------------------------ */
static M3 rows3(V3 a, V3 b, V3 c) { M3 m; m.x = a; m.y = b; m.z = c; return m; }
static V3 vmax0(V3 a) { return v3(fmaxf(0.0f, a.x), fmaxf(0.0f, a.y), fmaxf(0.0f, a.z)); }

/* Gamma (tonemap.cuh:6-9) */
static V3 tone_gamma(V3 c)
{
    const float e = 1.0f / 2.2f;
    return v3(om_powf(c.x, e), om_powf(c.y, e), om_powf(c.z, e));
}

/* XYZ2SRGBLinearD65 (tonemap.cuh:119-130) */
static V3 xyz_to_srgb(V3 xyz)
{
    const M3 m = rows3(v3(3.2406f, -1.5372f, -0.4986f), v3(-0.9689f, 1.8758f, 0.0415f), v3(0.0557f, -0.204f, 1.057f));
    return vmax0(mmul(&m, xyz));
}

/* ACES (tonemap.cuh:11-117) */
static V3 tone_aces(V3 col)
{
    const M3 ap1_xyz = rows3(v3(0.6624541811f, 0.1340042065f, 0.1561876870f), v3(0.2722287168f, 0.6740817658f, 0.0536895174f),
                             v3(-0.0055746495f, 0.0040607335f, 1.0103391003f));
    const M3 srgb_ap0 = rows3(v3(0.4397010f, 0.3829780f, 0.1773350f), v3(0.0897923f, 0.8134230f, 0.0967616f),
                              v3(0.0175440f, 0.1115440f, 0.8707040f));
    const M3 ap0_ap1 = rows3(v3(1.4514393161f, -0.2365107469f, -0.2149285693f), v3(-0.0765537734f, 1.1762296998f, -0.0996759264f),
                             v3(0.0083161484f, -0.0060324498f, 0.9977163014f));
    const M3 xyz_ap1 = rows3(v3(1.6410233797f, -0.3248032942f, -0.2364246952f), v3(-0.6636628587f, 1.6153315917f, 0.0167563477f),
                             v3(0.0117218943f, -0.0082844420f, 0.9883948585f));
    const M3 d60_d65 = rows3(v3(0.98722400f, -0.00611327f, 0.0159533f), v3(-0.00759836f, 1.00186000f, 0.0053302f),
                             v3(0.00307257f, -0.00509595f, 1.0816800f));
    const M3 xyz_709 = rows3(v3(3.2409699419f, -1.5373831776f, -0.4986107603f), v3(-0.9692436363f, 1.8759675015f, 0.0415550574f),
                             v3(0.0556300797f, -0.2039769589f, 1.0569715142f));
    const V3 y_of = v3(0.272229f, 0.674082f, 0.0536895f);
    const V3 ap0 = mmul(&srgb_ap0, col);
    V3 cg = mmul(&ap0_ap1, ap0);
    float y = dot3(cg, y_of);
    cg = vlerp(v3(y, y, y), cg, 0.96f);
    const float a = 278.5085f, b = 10.7772f, c = 293.6045f, d = 88.7122f, e = 80.6889f;
    V3 post;
    post.x = (cg.x * (cg.x * a + b)) / (cg.x * (cg.x * c + d) + e);
    post.y = (cg.y * (cg.y * a + b)) / (cg.y * (cg.y * c + d) + e);
    post.z = (cg.z * (cg.z * a + b)) / (cg.z * (cg.z * c + d) + e);
    V3 xyz = mmul(&ap1_xyz, post);
    const float dv = fmaxf(dot3(xyz, v3(1.0f, 1.0f, 1.0f)), 1.0e-4f);
    V3 xyY = v3(xyz.x / dv, xyz.y / dv, xyz.y);
    xyY.z = fminf(fmaxf(xyY.z, 0.0f), 65504.0f);
    xyY.z = om_powf(xyY.z, 0.9811f);
    const float m = xyY.z / fmaxf(xyY.y, 1e-4f);
    xyz = v3(xyY.x, xyY.z, (1.0f - xyY.x - xyY.y));
    xyz.x *= m;
    xyz.z *= m;
    V3 cv = mmul(&xyz_ap1, xyz);
    y = dot3(cv, y_of);
    cv = vlerp(v3(y, y, y), cv, 0.93f);
    const V3 x1 = mmul(&ap1_xyz, cv);
    const V3 x2 = mmul(&d60_d65, x1);
    return tone_gamma(vmax0(mmul(&xyz_709, x2)));
}

static float sat_(float v) { return (v != v) ? 0.0f : fminf(fmaxf(v, 0.0f), 1.0f); }

void or_tonemap(const float* rgb, int64_t n, int tone, float exposure, int xyz_input, uint32_t* out)
{
    for (int64_t i = 0; i < n; ++i) {
        V3 v = v3(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        if (xyz_input) v = xyz_to_srgb(v);
        v = vscale(v, exposure);
        if (tone == 1) v = tone_gamma(v);
        else if (tone == 2) v = tone_aces(v);
        const uint32_t r = (uint32_t)(255.0f * sat_(v.x)), g = (uint32_t)(255.0f * sat_(v.y)), b = (uint32_t)(255.0f * sat_(v.z));
        out[i] = 0xff000000u | (r << 16) | (g << 8) | b;
    }
}

void or_object_isect(const or_scene* s, int32_t obj, const float* rays, int64_t n, int32_t depth, float* t, float* pos,
                     float* nrm)
{
    const float eps_d = s->eps_tab[depth < 8 ? (depth < 0 ? 0 : depth) : 8];
    for (int64_t i = 0; i < n; ++i) {
        const float* q = rays + 8 * i;
        Isect c;
        memset(&c, 0, sizeof(c));
        c.obj = obj;
        const int h = isect_object(s, obj, v3(q[0], q[1], q[2]), v3(q[4], q[5], q[6]), eps_d, &c);
        t[i] = h ? c.dist : -1.0f;
        pos[3 * i] = h ? c.pos.x : 0.0f; pos[3 * i + 1] = h ? c.pos.y : 0.0f; pos[3 * i + 2] = h ? c.pos.z : 0.0f;
        nrm[3 * i] = h ? c.nrm.x : 0.0f; nrm[3 * i + 1] = h ? c.nrm.y : 0.0f; nrm[3 * i + 2] = h ? c.nrm.z : 0.0f;
    }
}

void or_volume_grid(const or_scene* s, int32_t v, float* out)
{
    if (v < 0 || v >= s->nvol) return;
    for (int i = 0; i < s->n; ++i)
        if (s->o[i].vol == s->vols[v]) {
            const size_t n = (size_t)s->o[i].dims[0] * s->o[i].dims[1] * s->o[i].dims[2];
            memcpy(out, s->vols[v], n * sizeof(float));
            return;
        }
}

/* ------------------------------------------------------------------------ */
/* Screen-space denoiser (core/denoise/)                                     */
/* ------------------------------------------------------------------------ */
/* IEEE binary16 <-> binary32 through _Float16 (round to nearest even). */
static inline float dn_h2f(uint16_t h) { _Float16 v; memcpy(&v, &h, 2); return (float)v; }
static inline uint16_t dn_f2h(float f) { _Float16 v = (_Float16)f; uint16_t h; memcpy(&h, &v, 2); return h; }
/* half - half rounded once to half, as __hsub: the exact difference in double */
static inline float dn_hsub(uint16_t a, uint16_t b)
{
    const _Float16 d = (_Float16)((double)dn_h2f(a) - (double)dn_h2f(b));
    return (float)d;
}

#define DN_MODELS 5 /* MAT_MAX + 1 (core/render/object.cuh:45-52) */

/* RecordShadingModel (core/denoise/denoise.cuh:86-104) */
static void dn_record_model(ar_screen_gbuffer* g, int model)
{
    if (g->frames == 0)
        for (int i = 0; i < DN_MODELS; ++i) g->shading_model[i] = 0;
    const float affix = 1.0f / (float)(g->frames + 1u);
    const float pre = (float)g->frames / (float)(g->frames + 1u);
    for (int i = 0; i < DN_MODELS; ++i) g->shading_model[i] = dn_f2h(dn_h2f(g->shading_model[i]) * pre);
    g->shading_model[model] = dn_f2h(dn_h2f(g->shading_model[model]) + affix);
}

/* RecordScreenGBuffer (core/denoise/denoise.cuh:106-166) */
static void dn_record_gbuffer(ar_screen_gbuffer* g, const float* h)
{
    if (h[10] != 0.0f) {
        int model = (int)h[9];
        if (model < 0) model = 0;
        if (model > DN_MODELS - 2) model = DN_MODELS - 2;
        if (g->valid_frames == 0) {
            for (int c = 0; c < 3; ++c) g->albedo[c] = g->normal[c] = 0;
            g->metallic = g->roughness = 0;
            g->depth = 0.0f;
        }
        const float affix = 1.0f / (float)(g->valid_frames + 1u);
        const float pre = (float)g->valid_frames / (float)(g->valid_frames + 1u);
        for (int c = 0; c < 3; ++c) {
            g->albedo[c] = dn_f2h(dn_h2f(g->albedo[c]) * pre);
            g->normal[c] = dn_f2h(dn_h2f(g->normal[c]) * pre);
        }
        g->metallic = dn_f2h(dn_h2f(g->metallic) * pre);
        g->roughness = dn_f2h(dn_h2f(g->roughness) * pre);
        g->depth = g->depth * pre;
        for (int c = 0; c < 3; ++c) {
            g->albedo[c] = dn_f2h(dn_h2f(g->albedo[c]) + affix * h[c]);
            g->normal[c] = dn_f2h(dn_h2f(g->normal[c]) + affix * h[3 + c]);
        }
        g->metallic = dn_f2h(dn_h2f(g->metallic) + affix * h[6]);
        g->roughness = dn_f2h(dn_h2f(g->roughness) + affix * h[7]);
        g->depth = g->depth + affix * h[8];
        ++g->valid_frames;
        dn_record_model(g, model);
    } else {
        dn_record_model(g, DN_MODELS - 1);
    }
    ++g->frames;
}

/* RecordScreenStatisticBuffer (core/denoise/denoise_statistic.cuh:37-69),
 * BoxCox05's powf(x, 0.5f) as sqrtf(x) */
static void dn_record_stats(ar_screen_stats* s, const float* x)
{
    const uint32_t n0 = s->num, n1 = n0 + 1u;
    s->num = n1;
    const float invN1 = 1.0f / (float)n1;
    for (int c = 0; c < 3; ++c) {
        const float bc = (sqrtf(fmaxf(x[c], 0.0f)) - 1.0f) * 2.0f;
        const float delta = bc - s->mean[c];
        const float dn = delta * invN1;
        const double m2 = (double)s->m2_div_n[c] * (double)n0 + (double)(delta * (delta - dn));
        const float d2 = delta * delta, dn2 = dn * dn;
        const double m3 = ((double)s->m3_div_n[c] * (double)n0 - 3.0 * ((double)dn * m2)) + (double)(delta * (d2 - dn2));
        s->mean[c] = s->mean[c] + dn;
        s->m2_div_n[c] = (float)(m2 / (double)n1);
        s->m3_div_n[c] = (float)(m3 / (double)n1);
    }
}

void or_dn_record(const float* hits, const float* samples, int64_t n, ar_screen_gbuffer* gbuffer,
                  ar_screen_stats* stats)
{
    for (int64_t i = 0; i < n; ++i) {
        if (gbuffer) dn_record_gbuffer(gbuffer + i, hits + 12 * i);
        if (stats) dn_record_stats(stats + i, samples + 3 * i);
    }
}

/* Per-pixel terms of ComputeTStatistic (denoise.cuh:278-302) and of
 * ComputeWelchNu (denoise.cuh:326-339), counts in 32-bit unsigned arithmetic. */
typedef struct { float vth[3], theta[3], u[3], l[3]; } DnT;
static DnT dn_tstat(const ar_screen_stats* s)
{
    DnT r;
    const uint32_t nm1 = (s->num - 1u) > 1u ? (s->num - 1u) : 1u;
    const double num = (double)s->num;
    const double invNm1 = 1.0 / (double)nm1;
    for (int c = 0; c < 3; ++c) {
        const float vb = (float)((double)s->m2_div_n[c] * num * invNm1);
        r.vth[c] = (float)((double)vb / num);
        r.theta[c] = s->mean[c] + s->m3_div_n[c] / 6.0f / vb;
        r.u[c] = vb / (float)s->num;
        r.l[c] = r.u[c] * r.u[c] / (float)nm1;
    }
    return r;
}

/* LookupTQuantile005(floorToInt(nu)) with a saturating conversion (NaN -> 0) */
static int dn_t_index(float nu)
{
    if (!(nu >= 1.0f)) return 0;
    if (nu >= 1024.0f) return 1023;
    return (int)floorf(nu) - 1;
}

/* ComputeSVGFWeight (denoise.cuh:185-245) */
static float dn_svgf(const ar_screen_gbuffer* a, const ar_screen_gbuffer* b)
{
    const float kAlb = 1.0f / (2.0f * 1.0f * 1.0f), kNrm = 1.0f / (2.0f * 0.5f * 0.5f);
    const float kDep = 1.0f / (2.0f * 0.25f * 0.25f), kMet = 1.0f / (2.0f * 0.5f * 0.5f);
    const float kRgh = 1.0f / (2.0f * 0.5f * 0.5f), kShd = 1.0f / (2.0f * 0.1f * 0.1f);
    float w = 0.0f;
    {
        const V3 d1 = vsub(v3(dn_h2f(a->albedo[0]), dn_h2f(a->albedo[1]), dn_h2f(a->albedo[2])),
                           v3(dn_h2f(b->albedo[0]), dn_h2f(b->albedo[1]), dn_h2f(b->albedo[2])));
        w += dot3(d1, d1) * kAlb;
    }
    {
        const V3 na = vnormalize(v3(dn_h2f(a->normal[0]), dn_h2f(a->normal[1]), dn_h2f(a->normal[2])));
        const V3 nb = vnormalize(v3(dn_h2f(b->normal[0]), dn_h2f(b->normal[1]), dn_h2f(b->normal[2])));
        const float d = 1.0f - dot3(na, nb);
        w += d * d * kNrm;
    }
    {
        const float denom = fmaxf(fmaxf(a->depth, b->depth), 1.0e-6f);
        const float d = (a->depth - b->depth) / denom;
        w += d * d * kDep;
    }
    const float dm = dn_hsub(a->metallic, b->metallic);
    w += dm * dm * kMet;
    const float dr = dn_hsub(a->roughness, b->roughness);
    w += dr * dr * kRgh;
    float l1 = 0.0f;
    for (int i = 0; i < DN_MODELS; ++i) l1 += fabsf(dn_hsub(a->shading_model[i], b->shading_model[i]));
    const float tv = 0.5f * l1;
    w += tv * tv * kShd;
    return om_expf(-w);
}

/* ComputeTStatisticFinal (denoise.cuh:341-356), A = center */
static float dn_ttest(const DnT* A, const DnT* B, const float* tq)
{
    int pass = 1;
    for (int c = 0; c < 3; ++c) {
        const float t = A->theta[c] - B->theta[c];
        const float t2 = t * t;
        const float W = (t2 + B->vth[c]) / fmaxf(t2 + A->vth[c] + B->vth[c], 1.0e-6f);
        const float T = sqrtf(0.5f / (1.0f - W) - 1.0f);
        const float up = A->u[c] + B->u[c];
        const float nu = up * up / (A->l[c] + B->l[c]);
        pass = pass && (T < tq[dn_t_index(nu)]);
    }
    return pass ? 1.0f : 0.0f;
}

/* Bilateral16x16<7> (denoise.cuh:359-443) over the whole image; t_quantiles:
 * the 1024-entry table of the 0.9975 Student t quantile. */
void or_dn_bilateral(const float* hdr, float* out, const ar_screen_gbuffer* gb, const ar_screen_stats* st, int width,
                     int height, const float* t_quantiles)
{
    const int R = 7;
    const float kSpatial = 1.0f / (2.0f * 2.0f * 2.0f);
    const int64_t np = (int64_t)width * height;
    DnT* ts = (DnT*)malloc(sizeof(DnT) * (size_t)np);
    for (int64_t p = 0; p < np; ++p) ts[p] = dn_tstat(st + p);
#pragma omp parallel for schedule(dynamic, 4)
    for (int oy = 0; oy < height; ++oy) {
        for (int ox = 0; ox < width; ++ox) {
            const int64_t ci = (int64_t)oy * width + ox;
            float acc[3], s[3];
            for (int c = 0; c < 3; ++c) acc[c] = 0.0f + om_logf(hdr[3 * ci + c] + 1.0f) * 1.0e-6f;
            float wsum = 0.0f + 1.0e-6f;
            for (int j = -R; j <= R; ++j) {
                int ny = oy + j;
                ny = ny < 0 ? 0 : (ny > height - 1 ? height - 1 : ny);
                for (int i = -R; i <= R; ++i) {
                    int nx = ox + i;
                    nx = nx < 0 ? 0 : (nx > width - 1 ? width - 1 : nx);
                    const int64_t ni = (int64_t)ny * width + nx;
                    float weight = dn_svgf(gb + ci, gb + ni) * om_expf((float)(-(i * i + j * j)) * kSpatial) *
                                   dn_ttest(ts + ci, ts + ni, t_quantiles);
                    if (weight != weight) weight = 0.0f; /* zero normal of a pixel that never hit */
                    if (weight == 0.0f) continue;
                    for (int c = 0; c < 3; ++c) s[c] = om_logf(hdr[3 * ni + c] + 1.0f);
                    for (int c = 0; c < 3; ++c) acc[c] = acc[c] + s[c] * weight;
                    wsum = wsum + weight;
                }
            }
            for (int c = 0; c < 3; ++c) out[3 * ci + c] = fmaxf(om_expf(acc[c] / wsum) - 1.0f, 0.0f);
        }
    }
    free(ts);
}
