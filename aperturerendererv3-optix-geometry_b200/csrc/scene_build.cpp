// scene_build.cpp -- scene ingest, SAH BVH, collapse to 8-wide quantised
// nodes.  Host code, compiled with -ffp-contract=off (see detmath.h).
//
// The reference keeps one 432-byte SceneObject per primitive and re-transforms
// triangle vertices on every test (intersection.cuh:27-29).  Here the transform
// is applied once, with the same expression, and the leaf records carry the
// world-space v0, e1 = v1 - v0 and e2 = v2 - v0 -- bit-identical operands of the
// reference's Moller-Trumbore test.  The BVH is not the reference's: SAH (exact
// sweep for small ranges, 256 bins above) over triangle-bound centroids (the
// reference bins SceneObject centres, which for a mesh are all the mesh
// position -- scene_helper.h:488-545 -- and degenerate into one leaf per mesh),
// max 4 primitives per leaf, collapsed along an SAH-optimal plan (dynamic
// programming over the binary tree) into 8-wide nodes whose child boxes are
// quantised to 8 bits per plane relative to a power-of-two grid that starts one
// step below the children's union, rounded outwards and padded by one grid step
// on both sides, so the decoded box contains the exact one with a margin of a
// grid step that absorbs the rounding of the kernel's plane decode.
#include "scene_build.h"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <stdexcept>
#include <string>
#include <unordered_map>

#include "sdf.cuh"

namespace ar {

namespace {

f3 from_ar(const ar_vec3& a) { return mk(a.x, a.y, a.z); }

bool finite3(const ar_vec3& a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

m3 mat_mul(const m3& a, const m3& m)
{
    const f3 c0 = mk(m.x.x, m.y.x, m.z.x);
    const f3 c1 = mk(m.x.y, m.y.y, m.z.y);
    const f3 c2 = mk(m.x.z, m.y.z, m.z.z);
    m3 r;
    r.x = mk(dot(a.x, c0), dot(a.x, c1), dot(a.x, c2));
    r.y = mk(dot(a.y, c0), dot(a.y, c1), dot(a.y, c2));
    r.z = mk(dot(a.z, c0), dot(a.z, c1), dot(a.z, c2));
    return r;
}

struct Bounds {
    f3 lo = mk(FLT_MAX, FLT_MAX, FLT_MAX);
    f3 hi = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    void grow(const Bounds& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    void grow(f3 p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    float area() const
    {
        const float dx = std::max(0.0f, hi.x - lo.x), dy = std::max(0.0f, hi.y - lo.y), dz = std::max(0.0f, hi.z - lo.z);
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
    bool empty() const { return lo.x > hi.x; }
};

float axis(f3 v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

struct BNode {
    Bounds b;
    int left = -1, right = -1;
    int begin = 0, count = 0;
    bool leaf() const { return left < 0; }
};

constexpr int kMaxLeaf = 4;
constexpr int kBins = 256;
// Ranges of at most kSweepMax primitives are split by the exact SAH sweep over
// the centroid order on each axis, larger ones by 256-bin SAH.  The cost of a
// split is kTraversalCost + (A_l n_l + A_r n_r) / A, a leaf's its primitive
// count: on the 1M-triangle sphere field, 0.25 (small leaves, mostly one
// triangle) traced 3 % faster than 1, and 2-5 (larger leaves) 4-6 % slower --
// a visit of an 8-wide node costs several triangle tests.
constexpr int kSweepMax = 64;
constexpr float kTraversalCost = 0.25f;
// Collapse costs (per unit of surface area): a wide-node visit and a
// primitive test.  On the 1M-triangle sphere field the greedy collapse
// (expand the child of largest area until 8 slots) left 3.8 of 8 slots used
// per node; this plan fills 5.9 and traces 2 % faster.  A cheaper primitive
// (0.3, 0.15: leaves of merged subtrees, 7.8 slots) was 1-3 % slower than
// greedy; 1, 3 and 10 within 0.2 % of each other.
constexpr float kCollapseNode = 1.0f;
constexpr float kCollapsePrim = 3.0f;

// SAH-optimal collapse of the binary tree into 8-wide nodes (dynamic
// programming over the binary nodes, after Ylitie, Karras and Laine 2017):
// C(n, i) is the least cost of subtree n spread over at most i child slots of
// the wide node above it, C(n, 1) the cheaper of n as one leaf slot (at most
// kMaxLeaf primitives, A(n) * p(n) * kCollapsePrim) and n as a wide node of
// its own (A(n) * kCollapseNode + D(n, 8)), with D(n, j) the best split of j
// slots between n's two children.
struct CollapsePlan {
    const std::vector<BNode>& bn;
    std::vector<float> cost;          // [node * 9 + i], i = 1..8
    std::vector<int8_t> how;          // [node * 9 + i]: -1 as with i - 1 slots; i = 1: 0 leaf, 1 wide node; else 2 split
    std::vector<int8_t> split;        // [node * 9 + i]: slots of the left child in D(n, i)
    std::vector<int> prims, first;

    explicit CollapsePlan(const std::vector<BNode>& b) : bn(b)
    {
        const size_t n = bn.size();
        cost.assign(n * 9, FLT_MAX);
        how.assign(n * 9, 0);
        split.assign(n * 9, 0);
        prims.assign(n, 0);
        first.assign(n, 0);
        std::vector<float> dist(9);
        std::vector<int8_t> dsplit(9);
        for (int64_t v = static_cast<int64_t>(n) - 1; v >= 0; --v) {   // children (larger indices) first
            const BNode& b = bn[v];
            const float area = b.b.area();
            float* c = &cost[v * 9];
            if (b.leaf()) {
                prims[v] = b.count;
                first[v] = b.begin;
                for (int i = 1; i <= 8; ++i) {
                    c[i] = area * static_cast<float>(b.count) * kCollapsePrim;
                    how[v * 9 + i] = 0;
                }
                continue;
            }
            prims[v] = prims[b.left] + prims[b.right];
            first[v] = first[b.left];
            // D(v, j): j slots split between the children
            for (int j = 2; j <= 8; ++j) {
                float best = FLT_MAX;
                int8_t bk = 1;
                for (int k = 1; k < j; ++k) {
                    const float t = cost[b.left * 9 + k] + cost[b.right * 9 + (j - k)];
                    if (t < best) { best = t; bk = static_cast<int8_t>(k); }
                }
                dist[j] = best;
                dsplit[j] = bk;
            }
            const float asLeaf = prims[v] <= kMaxLeaf ? area * static_cast<float>(prims[v]) * kCollapsePrim : FLT_MAX;
            const float asNode = area * kCollapseNode + dist[8];
            c[1] = std::min(asLeaf, asNode);
            how[v * 9 + 1] = asLeaf <= asNode ? 0 : 1;
            split[v * 9 + 8] = dsplit[8];   // the slot split of v as a wide node, D(v, 8)
            for (int i = 2; i <= 8; ++i) {
                if (c[i - 1] <= dist[i]) { c[i] = c[i - 1]; how[v * 9 + i] = -1; }
                else { c[i] = dist[i]; how[v * 9 + i] = 2; split[v * 9 + i] = dsplit[i]; }
            }
        }
    }

    struct Slot { int node; bool leaf; };

    // the child slots of subtree v spread over at most i slots
    void forest(int v, int i, std::vector<Slot>& out) const
    {
        if (bn[v].leaf()) {
            out.push_back({v, true});
            return;
        }
        while (i > 1 && how[v * 9 + i] == -1) --i;
        if (i == 1) {
            out.push_back({v, how[v * 9 + 1] == 0});
            return;
        }
        const int k = split[v * 9 + i];
        forest(bn[v].left, k, out);
        forest(bn[v].right, i - k, out);
    }

    // the child slots of v as a wide node
    void children(int v, std::vector<Slot>& out) const
    {
        const int k = split[v * 9 + 8];
        forest(bn[v].left, k, out);
        forest(bn[v].right, 8 - k, out);
    }
};


struct BinaryBuilder {
    const std::vector<Bounds>& pb;
    const std::vector<f3>& pc;
    std::vector<int>& idx;
    std::vector<BNode> nodes;

    BinaryBuilder(const std::vector<Bounds>& b, const std::vector<f3>& c, std::vector<int>& i) : pb(b), pc(c), idx(i) {}

    int build(int begin, int end)
    {
        const int ni = static_cast<int>(nodes.size());
        nodes.emplace_back();
        Bounds bb, cb;
        for (int i = begin; i < end; ++i) { bb.grow(pb[idx[i]]); cb.grow(pc[idx[i]]); }
        nodes[ni].b = bb;
        const int count = end - begin;
        if (count <= 1) { nodes[ni].begin = begin; nodes[ni].count = count; return ni; }
        const float parentArea = std::max(bb.area(), 1e-30f);
        int mid = -1;
        if (count <= kSweepMax) {
            // exact SAH: every split position of the centroid order on each axis
            float bestCost = FLT_MAX;
            int bestAxis = -1, bestPos = -1;
            std::vector<int> ord(idx.begin() + begin, idx.begin() + end);
            std::vector<float> rightArea(count);
            for (int a = 0; a < 3; ++a) {
                std::sort(ord.begin(), ord.end(), [&](int p, int q) {
                    const float cp = axis(pc[p], a), cq = axis(pc[q], a);
                    return cp < cq || (cp == cq && p < q);
                });
                Bounds run;
                for (int i = count - 1; i > 0; --i) { run.grow(pb[ord[i]]); rightArea[i] = run.area(); }
                Bounds left;
                for (int i = 0; i < count - 1; ++i) {
                    left.grow(pb[ord[i]]);
                    const float cost = kTraversalCost + (left.area() * static_cast<float>(i + 1) +
                                                         rightArea[i + 1] * static_cast<float>(count - i - 1)) /
                                                            parentArea;
                    if (cost < bestCost) { bestCost = cost; bestAxis = a; bestPos = i + 1; }
                }
            }
            if (count <= kMaxLeaf && static_cast<float>(count) <= bestCost) {
                nodes[ni].begin = begin; nodes[ni].count = count; return ni;
            }
            const int a = bestAxis;
            std::sort(idx.begin() + begin, idx.begin() + end, [&](int p, int q) {
                const float cp = axis(pc[p], a), cq = axis(pc[q], a);
                return cp < cq || (cp == cq && p < q);
            });
            mid = begin + bestPos;
        } else {   // binned SAH on all three axes
            float bestCost = FLT_MAX;
            int bestAxis = -1, bestBin = -1;
            for (int a = 0; a < 3; ++a) {
                const float cmin = axis(cb.lo, a), cmax = axis(cb.hi, a);
                if (!(cmax > cmin)) continue;
                const float scale = static_cast<float>(kBins) / (cmax - cmin);
                Bounds bins[kBins];
                int cnt[kBins] = {0};
                for (int i = begin; i < end; ++i) {
                    int b = static_cast<int>((axis(pc[idx[i]], a) - cmin) * scale);
                    b = std::min(std::max(b, 0), kBins - 1);
                    bins[b].grow(pb[idx[i]]);
                    cnt[b]++;
                }
                float rightArea[kBins];
                int rightCnt[kBins];
                Bounds run;
                int rc = 0;
                for (int b = kBins - 1; b > 0; --b) {
                    if (cnt[b]) run.grow(bins[b]);
                    rc += cnt[b];
                    rightArea[b] = rc ? run.area() : 0.0f;
                    rightCnt[b] = rc;
                }
                Bounds left;
                int lc = 0;
                for (int b = 0; b < kBins - 1; ++b) {
                    if (cnt[b]) left.grow(bins[b]);
                    lc += cnt[b];
                    const int nr = rightCnt[b + 1];
                    if (lc == 0 || nr == 0) continue;
                    const float cost = kTraversalCost + (left.area() * lc + rightArea[b + 1] * nr) / parentArea;
                    if (cost < bestCost) { bestCost = cost; bestAxis = a; bestBin = b; }
                }
            }
            if (bestAxis >= 0) {
                if (count <= kMaxLeaf && static_cast<float>(count) <= bestCost) {
                    nodes[ni].begin = begin; nodes[ni].count = count; return ni;
                }
                const float cmin = axis(cb.lo, bestAxis), cmax = axis(cb.hi, bestAxis);
                const float scale = static_cast<float>(kBins) / (cmax - cmin);
                auto it = std::partition(idx.begin() + begin, idx.begin() + end, [&](int p) {
                    int b = static_cast<int>((axis(pc[p], bestAxis) - cmin) * scale);
                    b = std::min(std::max(b, 0), kBins - 1);
                    return b <= bestBin;
                });
                mid = static_cast<int>(it - idx.begin());
                if (mid == begin || mid == end) mid = -1;
            }
        }
        if (mid < 0) {
            if (count <= kMaxLeaf) { nodes[ni].begin = begin; nodes[ni].count = count; return ni; }
            mid = begin + count / 2;  // coincident centroids: split by position in the list
        }
        const int l = build(begin, mid);
        const int r = build(mid, end);
        nodes[ni].left = l;
        nodes[ni].right = r;
        return ni;
    }
};

// smallest e such that extent / 2^e <= 250 and 2^e >= 2^-21 * magnitude
int grid_exponent(float lo, float hi)
{
    const double ext = static_cast<double>(hi) - static_cast<double>(lo);
    const double mag = std::max(std::fabs(static_cast<double>(lo)), std::fabs(static_cast<double>(hi)));
    int e_min = -126;
    if (mag > 0.0) {
        int me;
        std::frexp(mag, &me);
        e_min = std::max(e_min, me - 21);
    }
    int e = e_min;
    if (ext > 0.0) {
        int ee;
        std::frexp(ext / 250.0, &ee);  // ext/250 < 2^ee
        e = std::max(e, ee);
    }
    if (e > 126) throw std::domain_error("scene coordinates too large for the quantised BVH");
    return e;
}

float pow2f(int e) { return std::ldexp(1.0f, e); }

void quantise(float origin, float scale, float lo, float hi, uint8_t* qlo, uint8_t* qhi)
{
    long ql = static_cast<long>(std::floor((static_cast<double>(lo) - origin) / scale)) - 1;
    long qh = static_cast<long>(std::ceil((static_cast<double>(hi) - origin) / scale)) + 1;
    ql = std::max(0L, ql);
    qh = std::min(255L, qh);
    // the kernel decodes fmaf(q, scale, origin); make both planes conservative
    while (ql > 0 && std::fma(static_cast<float>(ql), scale, origin) > lo) --ql;
    while (qh < 255 && std::fma(static_cast<float>(qh), scale, origin) < hi) ++qh;
    if (std::fma(static_cast<float>(ql), scale, origin) > lo || std::fma(static_cast<float>(qh), scale, origin) < hi)
        throw std::domain_error("BVH quantisation could not enclose a child box");
    *qlo = static_cast<uint8_t>(ql);
    *qhi = static_cast<uint8_t>(qh);
}

}  // namespace

void euler_matrices(f3 deg, m3* o2w, m3* w2o)
{
    const float k = 3.14159265358979f / 180.0f;
    const float ax = deg.x * k, ay = deg.y * k, az = deg.z * k;
    m3 rx, ry, rz;
    float c = std::cos(ax), s = std::sin(ax);
    rx.x = mk(1, 0, 0); rx.y = mk(0, c, -s); rx.z = mk(0, s, c);
    c = std::cos(ay); s = std::sin(ay);
    ry.x = mk(c, 0, s); ry.y = mk(0, 1, 0); ry.z = mk(-s, 0, c);
    c = std::cos(az); s = std::sin(az);
    rz.x = mk(c, -s, 0); rz.y = mk(s, c, 0); rz.z = mk(0, 0, 1);
    const m3 yx = mat_mul(ry, rx);
    *o2w = mat_mul(rz, yx);
    w2o->x = mk(o2w->x.x, o2w->y.x, o2w->z.x);
    w2o->y = mk(o2w->x.y, o2w->y.y, o2w->z.y);
    w2o->z = mk(o2w->x.z, o2w->y.z, o2w->z.z);
}

// Volumes as they will be uploaded: the caller's values (float or half), or
// the torus fill of FillSDFVolume computed here, on the host, so that the
// camera-inside test can read the same grid.
void ingest_volumes(HostScene& hs, const ar_sdf_volume* vols, size_t nv)
{
    if (nv > 0 && vols == nullptr) throw std::invalid_argument("volumes is NULL");
    for (size_t v = 0; v < nv; ++v) {
        const ar_sdf_volume& sv = vols[v];
        const std::string tag = "volume " + std::to_string(v) + ": ";
        if (sv.dims[0] < 1 || sv.dims[1] < 1 || sv.dims[2] < 1 || sv.dims[0] > 4096 || sv.dims[1] > 4096 ||
            sv.dims[2] > 4096)
            throw std::invalid_argument(tag + "dims must be in 1..4096");
        if (sv.precision != 32 && sv.precision != 16) throw std::invalid_argument(tag + "precision must be 32 or 16");
        const size_t count = static_cast<size_t>(sv.dims[0]) * sv.dims[1] * sv.dims[2];
        if (count > (size_t(1) << 31)) throw std::invalid_argument(tag + "more than 2^31 values");
        HostVolume hv;
        for (int k = 0; k < 3; ++k) hv.dims[k] = sv.dims[k];
        hv.fp16 = sv.precision == 16;
        hv.voxel_size_max = voxel_size_max(hv.dims);
        hv.bytes.resize(count * (hv.fp16 ? 2 : 4));
        if (sv.data) {
            std::memcpy(hv.bytes.data(), sv.data, hv.bytes.size());
        } else {
            if (sv.fill_kind != AR_SDF_TORUS) throw std::invalid_argument(tag + "unknown fill_kind");
            float* f = reinterpret_cast<float*>(hv.bytes.data());
            __half* h = reinterpret_cast<__half*>(hv.bytes.data());
            size_t i = 0;
            for (int z = 0; z < hv.dims[2]; ++z)
                for (int y = 0; y < hv.dims[1]; ++y)
                    for (int x = 0; x < hv.dims[0]; ++x, ++i) {
                        const float d = torus_fill_value(x, y, z, hv.dims, sv.fill_info[0], sv.fill_info[1]);
                        if (hv.fp16) h[i] = __float2half_rn(d);
                        else f[i] = d;
                    }
        }
        hs.volumes.push_back(std::move(hv));
    }
}

HostScene build_scene(const ar_object_desc* objs, size_t n, const ar_sdf_volume* vols, size_t nv)
{
    if (n > 0 && objs == nullptr) throw std::invalid_argument("objects is NULL");
    if (n >= (1u << 30)) throw std::invalid_argument("too many objects");
    HostScene hs;
    ingest_volumes(hs, vols, nv);
    hs.objects.resize(n);
    std::unordered_map<std::string, int32_t> matIndex;
    std::vector<Bounds> pbounds;
    std::vector<f3> pcent;
    std::vector<PrimRec> precs;
    pbounds.reserve(n);
    pcent.reserve(n);
    precs.reserve(n);
    float lightTotal = 0.0f;
    for (size_t i = 0; i < n; ++i) {
        const ar_object_desc& d = objs[i];
        if (d.type < AR_OBJ_CUBE || d.type > AR_OBJ_TRIANGLE)
            throw std::invalid_argument("object " + std::to_string(i) + ": invalid type");
        if (d.type == AR_OBJ_SDF) {
            if (d.sdf.kind != AR_SDF_TORUS && d.sdf.kind != AR_SDF_VOLUME)
                throw std::invalid_argument("object " + std::to_string(i) + ": invalid sdf.kind");
            if (d.sdf.kind == AR_SDF_VOLUME && (d.sdf.volume < 0 || static_cast<size_t>(d.sdf.volume) >= nv))
                throw std::invalid_argument("object " + std::to_string(i) + ": sdf.volume out of range");
            if (!(d.extent.x != 0.0f && d.extent.y != 0.0f && d.extent.z != 0.0f))
                throw std::invalid_argument("object " + std::to_string(i) + ": SDF box extent must be non-zero");
        }
        if (d.material.shading_model < AR_MAT_DIFFUSE || d.material.shading_model > AR_MAT_GGX)
            throw std::invalid_argument("object " + std::to_string(i) + ": invalid shading model");
        if (!finite3(d.center) || !finite3(d.extent) || !finite3(d.rotation_deg))
            throw std::invalid_argument("object " + std::to_string(i) + ": non-finite transform");
        // material (de-duplicated)
        MaterialRec mr;
        std::memset(&mr, 0, sizeof(mr));
        mr.model = d.material.shading_model;
        mr.albedo[0] = d.material.albedo.x; mr.albedo[1] = d.material.albedo.y; mr.albedo[2] = d.material.albedo.z;
        mr.emissive[0] = d.material.emissive.x; mr.emissive[1] = d.material.emissive.y; mr.emissive[2] = d.material.emissive.z;
        mr.specular = d.material.specular; mr.metallic = d.material.metallic; mr.roughness = d.material.roughness;
        mr.ior = d.material.ior; mr.sigma_a = d.material.sigma_a;
        mr.abbe = d.material.abbe_number; mr.tilt = d.material.tilt_number;
        std::string key(reinterpret_cast<const char*>(&mr), sizeof(mr));
        auto it = matIndex.find(key);
        int32_t mi;
        if (it == matIndex.end()) {
            mi = static_cast<int32_t>(hs.materials.size());
            hs.materials.push_back(mr);
            matIndex.emplace(std::move(key), mi);
        } else {
            mi = it->second;
        }
        ObjInfo& oi = hs.objects[i];
        oi.type = d.type;
        oi.material = mi;
        oi.light = -1;
        oi.aux = -1;
        const f3 center = from_ar(d.center);
        const f3 extent = vabs(from_ar(d.extent));  // SceneObject ctor: extent_(abs(extent))
        m3 o2w, w2o;
        euler_matrices(from_ar(d.rotation_deg), &o2w, &w2o);
        float area = 0.0f;
        Bounds bb;
        if (d.type == AR_OBJ_TRIANGLE) {
            for (int v = 0; v < 3; ++v)
                if (!finite3(d.tri[v].position) || !finite3(d.tri[v].normal))
                    throw std::invalid_argument("object " + std::to_string(i) + ": non-finite vertex");
            // intersection.cuh:27-29 / 75-77
            const f3 p0 = mul(o2w, from_ar(d.tri[0].position)) + center;
            const f3 p1 = mul(o2w, from_ar(d.tri[1].position)) + center;
            const f3 p2 = mul(o2w, from_ar(d.tri[2].position)) + center;
            TriShade ts;
            std::memset(&ts, 0, sizeof(ts));
            const f3 n0 = mul(o2w, from_ar(d.tri[0].normal));
            const f3 n1 = mul(o2w, from_ar(d.tri[1].normal));
            const f3 n2 = mul(o2w, from_ar(d.tri[2].normal));
            ts.n0[0] = n0.x; ts.n0[1] = n0.y; ts.n0[2] = n0.z;
            ts.n1[0] = n1.x; ts.n1[1] = n1.y; ts.n1[2] = n1.z;
            ts.n2[0] = n2.x; ts.n2[1] = n2.y; ts.n2[2] = n2.z;
            oi.aux = static_cast<int32_t>(hs.trishade.size());
            hs.trishade.push_back(ts);
            hs.triangles++;
            // SceneObject::GetArea for triangles (object.cuh:294-299), object space
            const f3 e1o = from_ar(d.tri[1].position) - from_ar(d.tri[0].position);
            const f3 e2o = from_ar(d.tri[2].position) - from_ar(d.tri[0].position);
            area = 0.5f * length(cross(e1o, e2o));
            if (d.visible) {
                PrimRec pr;
                std::memset(&pr, 0, sizeof(pr));
                const f3 e1 = p1 - p0, e2 = p2 - p0;
                pr.v0[0] = p0.x; pr.v0[1] = p0.y; pr.v0[2] = p0.z; pr.object = static_cast<int32_t>(i);
                pr.e1[0] = e1.x; pr.e1[1] = e1.y; pr.e1[2] = e1.z; pr.kind = kPrimTriangle;
                pr.e2[0] = e2.x; pr.e2[1] = e2.y; pr.e2[2] = e2.z;
                bb.grow(p0); bb.grow(p1); bb.grow(p2);
                pbounds.push_back(bb);
                pcent.push_back(mk(0.5f * (bb.lo.x + bb.hi.x), 0.5f * (bb.lo.y + bb.hi.y), 0.5f * (bb.lo.z + bb.hi.z)));
                precs.push_back(pr);
            }
        } else {
            Analytic an;
            std::memset(&an, 0, sizeof(an));
            an.center[0] = center.x; an.center[1] = center.y; an.center[2] = center.z;
            an.extent[0] = extent.x; an.extent[1] = extent.y; an.extent[2] = extent.z;
            an.radius = max3(extent);
            const float* mo = &o2w.x.x;
            const float* mw = &w2o.x.x;
            for (int k = 0; k < 9; ++k) { an.o2w[k] = mo[k]; an.w2o[k] = mw[k]; }
            oi.aux = static_cast<int32_t>(hs.analytic.size());
            hs.analytic.push_back(an);
            if (d.type == AR_OBJ_SDF) {
                SdfRec sr;
                std::memset(&sr, 0, sizeof(sr));
                sr.object = static_cast<int32_t>(i);
                sr.analytic = oi.aux;
                sr.kind = d.sdf.kind == AR_SDF_TORUS ? kSdfTorus : kSdfVolume;
                for (int k = 0; k < 4; ++k) sr.info[k] = d.sdf.info[k];
                if (sr.kind == kSdfVolume) {
                    const HostVolume& hv = hs.volumes[static_cast<size_t>(d.sdf.volume)];
                    for (int k = 0; k < 3; ++k) sr.dims[k] = hv.dims[k];
                    sr.fp16 = hv.fp16 ? 1 : 0;
                    sr.voxel_size_max = hv.voxel_size_max;
                    sr.pad[0] = d.sdf.volume;   // resolved to a device pointer at upload
                }
                oi.aux = static_cast<int32_t>(hs.sdf.size());
                hs.sdf.push_back(sr);
                // SceneObject::GetArea of OBJ_SDF is the box's (object.cuh:278-285); not a BVH primitive
                area = 8.0f * (extent.x * extent.y + extent.x * extent.z + extent.y * extent.z);
            } else if (d.type == AR_OBJ_CUBE) {
                // UpdateProxy (object.cuh:312-323) then a relative pad for rounding
                const f3 axx = mul(o2w, mk(1, 0, 0)), ayy = mul(o2w, mk(0, 1, 0)), azz = mul(o2w, mk(0, 0, 1));
                f3 h;
                h.x = std::fabs(axx.x) * extent.x + std::fabs(ayy.x) * extent.y + std::fabs(azz.x) * extent.z;
                h.y = std::fabs(axx.y) * extent.x + std::fabs(ayy.y) * extent.y + std::fabs(azz.y) * extent.z;
                h.z = std::fabs(axx.z) * extent.x + std::fabs(ayy.z) * extent.y + std::fabs(azz.z) * extent.z;
                bb.lo = center - h; bb.hi = center + h;
                const float ex = std::max(std::max(std::fabs(d.extent.x), std::fabs(d.extent.y)), std::fabs(d.extent.z));
                area = 8.0f * (extent.x * extent.y + extent.x * extent.z + extent.y * extent.z);
                (void)ex;
            } else {
                const float r = max3(extent);
                bb.lo = center - mk(r, r, r); bb.hi = center + mk(r, r, r);
                const float rr = std::fabs(extent.x);
                area = 4.0f * kPi * rr * rr;
            }
            if (d.type != AR_OBJ_SDF) {  // SDF objects are tested after the BVH, not in it
                const float pad = 1e-5f * (max3(vabs(center)) + max3(extent)) + 1e-30f;
                bb.lo = bb.lo - mk(pad, pad, pad);
                bb.hi = bb.hi + mk(pad, pad, pad);
                PrimRec pr;
                std::memset(&pr, 0, sizeof(pr));
                pr.object = static_cast<int32_t>(i);
                pr.kind = kPrimAnalytic;
                pbounds.push_back(bb);
                pcent.push_back(center);
                precs.push_back(pr);
            }
        }
        if (d.material.shading_model == AR_MAT_LIGHT) {
            // triangle lights: world-space vertices for the optional triangle NEE sampler
            float4_ t0 = {0, 0, 0, 0}, t1 = {0, 0, 0, 0}, t2 = {0, 0, 0, 0};
            if (d.type == AR_OBJ_TRIANGLE) {
                const f3 p0 = mul(o2w, from_ar(d.tri[0].position)) + center;
                const f3 e1 = (mul(o2w, from_ar(d.tri[1].position)) + center) - p0;
                const f3 e2 = (mul(o2w, from_ar(d.tri[2].position)) + center) - p0;
                const float wa = 0.5f * length(cross(e1, e2));
                t0 = {p0.x, p0.y, p0.z, wa};
                t1 = {e1.x, e1.y, e1.z, 0.0f};
                t2 = {e2.x, e2.y, e2.z, 0.0f};
            }
            hs.light_tri.push_back(t0);
            hs.light_tri.push_back(t1);
            hs.light_tri.push_back(t2);
            // scene.cu:1060-1076
            oi.light = static_cast<int32_t>(hs.light_object.size());
            const float w = std::max(area * luminance(from_ar(d.material.emissive)), 1.0e-20f);
            hs.light_object.push_back(static_cast<int32_t>(i));
            hs.light_prob.push_back(w);
            lightTotal += w;
        }
    }
    for (float& p : hs.light_prob) p = p / lightTotal;

    // ---------------- binary SAH BVH
    const int np = static_cast<int>(precs.size());
    if (np == 0) return hs;
    std::vector<int> idx(np);
    for (int i = 0; i < np; ++i) idx[i] = i;
    BinaryBuilder bb(pbounds, pcent, idx);
    bb.nodes.reserve(2 * static_cast<size_t>(np));
    bb.build(0, np);
    const std::vector<BNode>& bn = bb.nodes;

    // ---------------- collapse to 8-wide along the SAH-optimal plan, breadth
    // first so that the internal children of a node are contiguous
    const CollapsePlan plan(bn);
    struct Item { int wide; int bnode; };
    std::deque<Item> q;
    hs.nodes.emplace_back();
    q.push_back({0, 0});
    std::vector<int> nInternal;
    std::vector<std::vector<int>> internalChildren;
    while (!q.empty()) {
        const Item it = q.front();
        q.pop_front();
        std::vector<CollapsePlan::Slot> slots;
        if (bn[it.bnode].leaf()) slots.push_back({it.bnode, true});
        else plan.children(it.bnode, slots);
        std::vector<int> ch;
        for (const auto& sl : slots) ch.push_back(sl.node);
        WideNode w;
        std::memset(&w, 0, sizeof(w));
        Bounds u;
        for (int c : ch) u.grow(bn[c].b);
        const int ex = grid_exponent(u.lo.x, u.hi.x);
        const int ey = grid_exponent(u.lo.y, u.hi.y);
        const int ez = grid_exponent(u.lo.z, u.hi.z);
        const float sx = pow2f(ex), sy = pow2f(ey), sz = pow2f(ez);
        // the grid starts one step below the union, so that the lowest child
        // planes get the same one-step padding as every other plane
        w.ox = u.lo.x - sx; w.oy = u.lo.y - sy; w.oz = u.lo.z - sz;
        w.exps = static_cast<uint32_t>(ex + 127) | (static_cast<uint32_t>(ey + 127) << 8) | (static_cast<uint32_t>(ez + 127) << 16);
        w.child_base = static_cast<uint32_t>(hs.nodes.size());
        w.prim_base = static_cast<uint32_t>(hs.prims.size());
        uint8_t meta[8];
        std::memset(meta, kMetaEmpty, sizeof(meta));
        int rank = 0, poff = 0;
        for (size_t k = 0; k < ch.size(); ++k) {
            const BNode& c = bn[ch[k]];
            quantise(w.ox, sx, c.b.lo.x, c.b.hi.x, &w.qlo_x[k], &w.qhi_x[k]);
            quantise(w.oy, sy, c.b.lo.y, c.b.hi.y, &w.qlo_y[k], &w.qhi_y[k]);
            quantise(w.oz, sz, c.b.lo.z, c.b.hi.z, &w.qlo_z[k], &w.qhi_z[k]);
            if (slots[k].leaf) {
                const int cnt = plan.prims[ch[k]], beg = plan.first[ch[k]];
                if (cnt < 1 || cnt > kMaxLeaf) throw std::runtime_error("bad leaf size");
                meta[k] = static_cast<uint8_t>(((cnt - 1) << 5) | poff);
                for (int p = 0; p < cnt; ++p) hs.prims.push_back(precs[idx[beg + p]]);
                poff += cnt;
            } else {
                meta[k] = static_cast<uint8_t>(kMetaInternal | rank);
                q.push_back({static_cast<int>(hs.nodes.size()), ch[k]});
                hs.nodes.emplace_back();
                rank++;
            }
        }
        for (size_t k = ch.size(); k < 8; ++k) {
            w.qlo_x[k] = w.qlo_y[k] = w.qlo_z[k] = 255;
            w.qhi_x[k] = w.qhi_y[k] = w.qhi_z[k] = 0;
        }
        w.meta_lo = static_cast<uint32_t>(meta[0]) | (static_cast<uint32_t>(meta[1]) << 8) |
                    (static_cast<uint32_t>(meta[2]) << 16) | (static_cast<uint32_t>(meta[3]) << 24);
        w.meta_hi = static_cast<uint32_t>(meta[4]) | (static_cast<uint32_t>(meta[5]) << 8) |
                    (static_cast<uint32_t>(meta[6]) << 16) | (static_cast<uint32_t>(meta[7]) << 24);
        if (rank == 0) w.child_base = 0;
        hs.nodes[it.wide] = w;
        if (static_cast<int>(nInternal.size()) <= it.wide) { nInternal.resize(it.wide + 1); internalChildren.resize(it.wide + 1); }
        nInternal[it.wide] = rank;
        for (int r = 0; r < rank; ++r) internalChildren[it.wide].push_back(static_cast<int>(w.child_base) + r);
    }
    // exact worst-case stack depth: along any root path, each node pushes its
    // hit internal children except the one it descends into
    nInternal.resize(hs.nodes.size());
    internalChildren.resize(hs.nodes.size());
    std::vector<int> bound(hs.nodes.size(), 0), depth(hs.nodes.size(), 1);
    for (int wi = static_cast<int>(hs.nodes.size()) - 1; wi >= 0; --wi) {
        int b = 0, dmax = 0;
        for (int c : internalChildren[wi]) { b = std::max(b, bound[c]); dmax = std::max(dmax, depth[c]); }
        bound[wi] = (nInternal[wi] > 0 ? nInternal[wi] - 1 : 0) + b;
        depth[wi] = 1 + dmax;
    }
    hs.stack_bound = bound[0];
    hs.wide_depth = depth[0];
    return hs;
}

}  // namespace ar
