// guiding.cuh -- path guiding (core/guiding of the reference, used by its
// interactive renderer: CalculateRadiance<..., bUsePathGuiding>,
// core/render/render.cuh:545-640, SceneRenderer update scene.cu:583-744).
//
// What it keeps from the reference (core/guiding/*.cuh, config.cuh:30-70):
//   * a probe per (voxel of PATH_GUIDING_RESOLUTION_UNIT = 0.05 world units,
//     icosahedron face of the reflected ray direction): 20 faces;
//   * a probe is an 8x8 equal-area octahedral map (Clarberg 2008) of RGB
//     incident radiance with its mip chain 4x4, 2x2, 1x1 (85 texels); texels
//     are clamped to >= 1e-5 before the mips are built;
//   * sampling descends the mips choosing children by their weight
//     dot(texel, query) (query = the path throughput colour normalised), then
//     picks a point in the leaf texel; pdf = (w_leaf / w_avg) / (4 pi);
//     hemisphere variants add the mirror direction's density (reflection
//     about the normal);
//   * paths take the probe's sample with probability alpha = 0.5 * min(1,
//     frame / 64)^0.5 and weight by the mixture (1 - alpha) p_bsdf + alpha p_probe,
//     in the BSDF pdf of MIS as well;
//   * samples: the RGB radiance arriving at the first 5 non-delta vertices
//     along their sampled direction, luminance in [1e-5, 1e5], accumulated per
//     texel (times the 4 pi Jacobian) and merged into the probe as a running
//     mean over at most 10^6 samples.
// What is B200-first instead of a port: probes live in a fixed pool indexed
// by an open-addressing hash table of 64-bit (voxel, face) keys built on the
// GPU with atomicCAS (no thrust sort/unique, no growing indirection volume,
// no host synchronisation); the incident radiance of a vertex is read off the
// path's radiance record at retirement (radiance gathered after the next
// event over the throughput that reached it) instead of per-vertex arrays in
// registers.
#pragma once

#include <cmath>
#include <cstdint>

#include "detmath.h"

namespace ar {

constexpr int kPgRes = 8;                 // leaf resolution (PATH_GUIDING_RESOLUTION_LEVEL 4)
constexpr int kPgTexels = 85;             // 64 + 16 + 4 + 1
constexpr int kPgStride = 88;             // float4 texels per probe (padded)
constexpr int kPgFaces = 20;
constexpr int kPgCollect = 5;             // PATH_GUIDING_COLLECT_DEPTH
constexpr int kPgEvents = kPgCollect + 1; // recorded events per pixel (the last closes the previous vertex)
constexpr float kPgUnit = 0.05f;          // PATH_GUIDING_RESOLUTION_UNIT
constexpr float kPgMinBrightness = 1.0e-5f;
constexpr float kPgMaxBrightness = 1.0e5f;
constexpr unsigned long long kPgMaxCount = 1000000ull;
constexpr uint64_t kPgEmpty = ~0ull;
constexpr int kPgMaxProbe = 32;           // hash-table probe sequence bound

__host__ __device__ __forceinline__ int pg_level_offset(int level)   // texel offset of mip level
{
    return level == 0 ? 0 : (level == 1 ? 64 : (level == 2 ? 80 : 84));
}

// Equal-area octahedral map of the unit square onto the sphere and back
// (Clarberg, "Fast equal-area mapping of the (hemi)sphere using SIMD", JGT 2008).
__host__ __device__ __forceinline__ f3 pg_uv_to_dir(float su, float sv)
{
    const float u = 2.0f * su - 1.0f, v = 2.0f * sv - 1.0f;
    const float au = fabsf(u), av = fabsf(v);
    const float d = 1.0f - (au + av);
    const float r = 1.0f - fabsf(d);
    const float phi = r > 0.0f ? ((av - au) / r + 1.0f) * 0.78539816339744831f : 0.0f;
    const float z = copysignf(1.0f - r * r, d);
    const float s = r * sqrtf(fmaxf(0.0f, 2.0f - r * r));
    float sp, cp;
#ifdef __CUDA_ARCH__
    sincosf(phi, &sp, &cp);
#else
    sp = sinf(phi);
    cp = cosf(phi);
#endif
    return mk(copysignf(cp * s, u), copysignf(sp * s, v), z);
}

__host__ __device__ __forceinline__ void pg_dir_to_uv(f3 w, float* su, float* sv)
{
    const float r = sqrtf(fmaxf(0.0f, 1.0f - fabsf(w.z)));
    const float psi = atan2f(fabsf(w.y), fabsf(w.x)) * 0.63661977236758134f;   // in [0, 1]
    float v = psi * r, u = r - v;
    if (w.z < 0.0f) {
        const float t = u;
        u = 1.0f - v;
        v = 1.0f - t;
    }
    u = copysignf(u, w.x);
    v = copysignf(v, w.y);
    *su = fminf(fmaxf(0.5f * (u + 1.0f), 0.0f), 1.0f);
    *sv = fminf(fmaxf(0.5f * (v + 1.0f), 0.0f), 1.0f);
}

__host__ __device__ __forceinline__ f3 pg_mirror(f3 w, f3 n) { return w - n * (2.0f * dot(n, w)); }

// (voxel, face) -> 64-bit key: 19-bit two's-complement voxel coordinates and
// the face index.
__host__ __device__ __forceinline__ uint64_t pg_key(f3 p, f3 dir, const float* faces)
{
    const int x = static_cast<int>(floorf(p.x * (1.0f / kPgUnit)));
    const int y = static_cast<int>(floorf(p.y * (1.0f / kPgUnit)));
    const int z = static_cast<int>(floorf(p.z * (1.0f / kPgUnit)));
    const f3 d = normalize(dir);
    int best = 0;
    float bd = -1e30f;
    for (int f = 0; f < kPgFaces; ++f) {
        const float v = d.x * faces[3 * f] + d.y * faces[3 * f + 1] + d.z * faces[3 * f + 2];
        if (v > bd) { bd = v; best = f; }
    }
    const uint64_t m = (1ull << 19) - 1ull;
    return (static_cast<uint64_t>(static_cast<uint32_t>(x)) & m) | ((static_cast<uint64_t>(static_cast<uint32_t>(y)) & m) << 19) |
           ((static_cast<uint64_t>(static_cast<uint32_t>(z)) & m) << 38) | (static_cast<uint64_t>(best) << 57);
}

__host__ __device__ __forceinline__ uint32_t pg_hash(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return static_cast<uint32_t>(k);
}

// Device state of the guiding structure.
struct GuideView {
    uint64_t* keys;          // hash table keys (kPgEmpty = free)
    int32_t* slots;          // probe index of each key (-1 until assigned)
    uint32_t table_mask;     // table size - 1
    float4* probes;          // capacity x kPgStride texels (running means, mips)
    float4* accum;           // capacity x 64 leaf sums of the current frame
    unsigned long long* counts;      // samples merged per probe (capped)
    unsigned int* frame_counts;      // samples of the current frame per probe
    int32_t* touched;        // probes that received samples this frame
    int32_t* counters;       // [0] probes allocated, [1] touched, [2] samples, [3] dropped,
                             // [4] [5] samples and dropped of the last update
    int32_t capacity;
    float alpha;             // guiding probability of this frame
    const float* faces;      // 20 unit face normals (x, y, z)
    // per-pixel event records of the frame (interactive frames: one path per pixel)
    float4* events;          // npix x kPgEvents x 3: (key lo bits, key hi bits, guidable, -), (dir, -), (T, -)
    float4* event_lb;        // npix x kPgEvents: radiance gathered before the event
    int32_t* event_count;    // npix
    float4* samples;         // sample records: (key lo, key hi, -, -), (dir, -), (rgb, -)
    int32_t sample_cap;
};

// Probe index of a key, or -1 (no probe for it yet, or the table is full).
__host__ __device__ __forceinline__ int pg_lookup(const GuideView& g, uint64_t key)
{
    uint32_t h = pg_hash(key) & g.table_mask;
    for (int i = 0; i < kPgMaxProbe; ++i) {
        const uint64_t k = g.keys[h];
        if (k == key) return g.slots[h];
        if (k == kPgEmpty) return -1;
        h = (h + 1) & g.table_mask;
    }
    return -1;
}

__host__ __device__ __forceinline__ float pg_w(const float4& t, f3 q) { return t.x * q.x + t.y * q.y + t.z * q.z; }

// OctahedronPDF: density of a full-sphere probe sample in direction w.
__host__ __device__ __forceinline__ float pg_pdf(const float4* probe, f3 w, f3 q)
{
    float su, sv;
    pg_dir_to_uv(w, &su, &sv);
    const int ix = min(kPgRes - 1, max(0, static_cast<int>(floorf(su * kPgRes))));
    const int iy = min(kPgRes - 1, max(0, static_cast<int>(floorf(sv * kPgRes))));
    const float wl = pg_w(probe[iy * kPgRes + ix], q);
    const float wa = pg_w(probe[pg_level_offset(3)], q);
    const float inv4pi = 0.07957747154594767f;
    if (!(wa > 0.0f)) return inv4pi;
    return fmaxf((wl / wa) * inv4pi, 1.0e-12f);
}

// OctahedronHemispherePDF: sample on the sphere, mirrored into the hemisphere of n.
__host__ __device__ __forceinline__ float pg_hemi_pdf(const float4* probe, f3 w, f3 n, f3 q)
{
    if (dot(w, n) <= 0.0f) return 0.0f;
    return pg_pdf(probe, w, q) + pg_pdf(probe, pg_mirror(w, n), q);
}

// SampleOctahedronHemisphere with uniforms u[0..2] (mip descent: levels 3 -> 1
// choose among 4 children each) and u[3], u[4] (point in the leaf texel).
__host__ __device__ __forceinline__ f3 pg_sample_hemi(const float4* probe, f3 n, f3 q, const float* u, float* pdf)
{
    int cx = 0, cy = 0;
    float pt = 1.0f;
    for (int level = 3; level > 0; --level) {
        const int res = kPgRes >> level;
        const float sum = 4.0f * pg_w(probe[pg_level_offset(level) + cy * res + cx], q);
        const int nx = cx << 1, ny = cy << 1;
        const int cres = kPgRes >> (level - 1);
        const float r = u[3 - level];
        if (!(sum > 0.0f)) {
            const int pick = min(3, static_cast<int>(r * 4.0f));
            cx = nx + (pick & 1);
            cy = ny + (pick >> 1);
            pt *= 0.25f;
        } else {
            float cdf = 0.0f;
            int chosen = 3;
            float wsel = 0.0f;
            for (int c = 0; c < 4; ++c) {   // children in the order (0,0) (0,1) (1,0) (1,1) of (x, y)
                const int ox = c >> 1, oy = c & 1;
                const float wc = pg_w(probe[pg_level_offset(level - 1) + (ny + oy) * cres + nx + ox], q) / sum;
                cdf += wc;
                if (r <= cdf || c == 3) { chosen = c; wsel = wc; break; }
            }
            cx = nx + (chosen >> 1);
            cy = ny + (chosen & 1);
            pt *= wsel;
        }
    }
    const float su = fminf(fmaxf((static_cast<float>(cx) + (1.0f - u[3])) / kPgRes, 0.0f), 1.0f);
    const float sv = fminf(fmaxf((static_cast<float>(cy) + (1.0f - u[4])) / kPgRes, 0.0f), 1.0f);
    f3 w = pg_uv_to_dir(su, sv);
    float p = fmaxf(pt * (kPgRes * kPgRes) * 0.07957747154594767f, 1.0e-12f);
    const f3 mirror = pg_mirror(w, n);
    p += pg_pdf(probe, mirror, q);
    if (dot(w, n) < 0.0f) w = mirror;
    *pdf = p;
    return w;
}

// alpha of a frame: lerp(0, 0.5, min(1, frame / 64)^0.5) (render.cuh:198-203)
inline float pg_alpha(int64_t frame)
{
    const double t = frame <= 0 ? 0.0 : (frame >= 64 ? 1.0 : static_cast<double>(frame) / 64.0);
    return static_cast<float>(0.5 * std::sqrt(t));
}

// Host launchers (guiding.cu).
cudaError_t pg_update(const GuideView& g, int sm_count, cudaStream_t st);
cudaError_t pg_clear(const GuideView& g, size_t table_size, cudaStream_t st);
void pg_face_normals(float* out60);
cudaError_t pg_eval(const float4* probes, const int32_t* probe_of, const float* n3, const float* q3, const float* u5,
                    const float* e3, const float* p3, int64_t n, const float* faces, float* dir3, float* pdf,
                    float* epdf, unsigned long long* key, cudaStream_t st);

}  // namespace ar
