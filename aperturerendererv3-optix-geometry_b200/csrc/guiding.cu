// guiding.cu -- the per-frame update of the path-guiding probes, all on the
// GPU: insert the frame's (voxel, face) keys into the hash table (probes
// allocated from a fixed pool), add each sample's RGB radiance (times the
// 4 pi Jacobian of the equal-area map) to its leaf texel, and merge the
// touched probes' sums into their running means and mip chains
// (reference: core/guiding/guiding.cuh:70-517, scene.cu:583-744, which does
// the same with thrust sort/unique/copy_if and a host-synchronised growing
// indirection volume).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "guiding.cuh"

namespace ar {

namespace {

__device__ __forceinline__ uint64_t sample_key(const float4* s) { return (static_cast<uint64_t>(__float_as_uint(s[0].y)) << 32) | __float_as_uint(s[0].x); }

__global__ void k_pg_insert(GuideView g)
{
    const int n = min(g.counters[2], g.sample_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t key = sample_key(g.samples + 3 * static_cast<int64_t>(i));
        uint32_t h = pg_hash(key) & g.table_mask;
        for (int j = 0; j < kPgMaxProbe; ++j) {
            const unsigned long long prev = atomicCAS(reinterpret_cast<unsigned long long*>(g.keys + h),
                                                      static_cast<unsigned long long>(kPgEmpty),
                                                      static_cast<unsigned long long>(key));
            if (prev == kPgEmpty) {   // this thread owns the new key: give it a probe
                const int idx = atomicAdd(&g.counters[0], 1);
                g.slots[h] = idx < g.capacity ? idx : -1;
                break;
            }
            if (prev == key) break;
            h = (h + 1) & g.table_mask;
        }
    }
}

__global__ void k_pg_accumulate(GuideView g)
{
    const int n = min(g.counters[2], g.sample_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4* s = g.samples + 3 * static_cast<int64_t>(i);
        const int idx = pg_lookup(g, sample_key(s));
        if (idx < 0) {
            atomicAdd(&g.counters[3], 1);
            continue;
        }
        float su, sv;
        pg_dir_to_uv(mk(s[1].x, s[1].y, s[1].z), &su, &sv);
        const int ix = min(kPgRes - 1, max(0, static_cast<int>(floorf(su * kPgRes))));
        const int iy = min(kPgRes - 1, max(0, static_cast<int>(floorf(sv * kPgRes))));
        const float J = 12.566370614359172f;   // equal-area map: d omega / d uv = 4 pi
        float4* t = g.accum + static_cast<int64_t>(idx) * (kPgRes * kPgRes) + iy * kPgRes + ix;
        atomicAdd(&t->x, s[2].x * J);
        atomicAdd(&t->y, s[2].y * J);
        atomicAdd(&t->z, s[2].z * J);
        if (atomicAdd(&g.frame_counts[idx], 1u) == 0u) g.touched[atomicAdd(&g.counters[1], 1)] = idx;
    }
}

// one warp per touched probe: running mean, clamp, mips (GenerateMipmaps)
__global__ void k_pg_merge(GuideView g)
{
    const int warps = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int n = g.counters[1];
    for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += warps) {
        const int idx = g.touched[w];
        float4* p = g.probes + static_cast<int64_t>(idx) * kPgStride;
        float4* a = g.accum + static_cast<int64_t>(idx) * (kPgRes * kPgRes);
        const unsigned long long cO = g.counts[idx];
        const unsigned long long cN = g.frame_counts[idx];
        const double inv = 1.0 / static_cast<double>(cO + cN);
        const double keep = static_cast<double>(cO) * inv;
        for (int k = lane; k < kPgRes * kPgRes; k += 32) {
            const float4 o = p[k], s = a[k];
            float4 m;
            m.x = fmaxf(static_cast<float>(static_cast<double>(o.x) * keep + static_cast<double>(s.x) * inv), kPgMinBrightness);
            m.y = fmaxf(static_cast<float>(static_cast<double>(o.y) * keep + static_cast<double>(s.y) * inv), kPgMinBrightness);
            m.z = fmaxf(static_cast<float>(static_cast<double>(o.z) * keep + static_cast<double>(s.z) * inv), kPgMinBrightness);
            m.w = 0.0f;
            p[k] = m;
            a[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        __syncwarp();
        // mip levels 1 (4x4), 2 (2x2), 3 (1x1): averages of 2x2 children
        for (int level = 1; level < 4; ++level) {
            const int res = kPgRes >> level, cres = res << 1;
            const int off = pg_level_offset(level), coff = pg_level_offset(level - 1);
            if (lane < res * res) {
                const int x = lane % res, y = lane / res;
                const float4 c0 = p[coff + (2 * y) * cres + 2 * x], c1 = p[coff + (2 * y) * cres + 2 * x + 1];
                const float4 c2 = p[coff + (2 * y + 1) * cres + 2 * x], c3 = p[coff + (2 * y + 1) * cres + 2 * x + 1];
                p[off + y * res + x] = make_float4((c0.x + c1.x + c2.x + c3.x) * 0.25f, (c0.y + c1.y + c2.y + c3.y) * 0.25f,
                                                   (c0.z + c1.z + c2.z + c3.z) * 0.25f, 0.0f);
            }
            __syncwarp();
        }
        if (lane == 0) {
            g.counts[idx] = min(kPgMaxCount, cO + cN);
            g.frame_counts[idx] = 0u;
        }
    }
}

__global__ void k_pg_reset_frame(GuideView g)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {   // keep the frame's sample counts, clear the rest
        g.counters[4] = g.counters[2];
        g.counters[5] = g.counters[3];
        g.counters[1] = 0;
        g.counters[2] = 0;
        g.counters[3] = 0;
    }
}

}  // namespace

cudaError_t pg_update(const GuideView& g, int sm_count, cudaStream_t st)
{
    const int grid = std::max(1, sm_count * 4);
    k_pg_insert<<<grid, 256, 0, st>>>(g);
    k_pg_accumulate<<<grid, 256, 0, st>>>(g);
    k_pg_merge<<<grid, 256, 0, st>>>(g);
    k_pg_reset_frame<<<1, 1, 0, st>>>(g);
    return cudaGetLastError();
}

cudaError_t pg_clear(const GuideView& g, size_t table_size, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(g.keys, 0xFF, table_size * sizeof(uint64_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.slots, 0xFF, table_size * sizeof(int32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.probes, 0, static_cast<size_t>(g.capacity) * kPgStride * sizeof(float4), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.accum, 0, static_cast<size_t>(g.capacity) * kPgRes * kPgRes * sizeof(float4), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.counts, 0, static_cast<size_t>(g.capacity) * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.frame_counts, 0, static_cast<size_t>(g.capacity) * sizeof(unsigned int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g.counters, 0, 6 * sizeof(int32_t), st);
    return e;
}

// Unit normals of the 20 faces of the regular icosahedron with vertices
// (0, +-1, +-phi) and their cyclic permutations: the normalised centroids of
// the vertex triples at mutual distance 2, in lexicographic triple order.
// Probe math of the queries of ar_guide_probe_eval: one thread per query.
__global__ void k_pg_eval(const float4* probes, const int32_t* probe_of, const float* n3, const float* q3,
                          const float* u5, const float* e3, const float* p3, int64_t n, const float* faces,
                          float* dir3, float* pdf, float* epdf, unsigned long long* key)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float4* pr = probes + static_cast<int64_t>(probe_of[i]) * kPgStride;
        const f3 nrm = mk(n3[3 * i], n3[3 * i + 1], n3[3 * i + 2]);
        const f3 q = mk(q3[3 * i], q3[3 * i + 1], q3[3 * i + 2]);
        const f3 e = mk(e3[3 * i], e3[3 * i + 1], e3[3 * i + 2]);
        float u[5];
        for (int k = 0; k < 5; ++k) u[k] = u5[5 * i + k];
        float p = 0.0f;
        const f3 w = pg_sample_hemi(pr, nrm, q, u, &p);
        dir3[3 * i] = w.x; dir3[3 * i + 1] = w.y; dir3[3 * i + 2] = w.z;
        pdf[i] = p;
        epdf[i] = pg_hemi_pdf(pr, e, nrm, q);
        key[i] = pg_key(mk(p3[3 * i], p3[3 * i + 1], p3[3 * i + 2]), e, faces);
    }
}

cudaError_t pg_eval(const float4* probes, const int32_t* probe_of, const float* n3, const float* q3, const float* u5,
                    const float* e3, const float* p3, int64_t n, const float* faces, float* dir3, float* pdf,
                    float* epdf, unsigned long long* key, cudaStream_t st)
{
    const int grid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4096));
    if (grid > 0) k_pg_eval<<<grid, 256, 0, st>>>(probes, probe_of, n3, q3, u5, e3, p3, n, faces, dir3, pdf, epdf, key);
    return cudaGetLastError();
}

// The 20 face normals of the regular icosahedron in the reference's face
// numbering (FaceNormal20FromIndex, core/guiding/guiding_bin.cuh:40-66), which
// probe keys carry.  Each face is given by the signs of its normal's x, y, z:
// three non-zero signs are a face on a cube diagonal, (+-1, +-1, +-1) / sqrt 3;
// a zero at axis k puts the long component phi^2 / sqrt(1 + phi^4) on axis
// (k + 1) % 3 and the short one 1 / sqrt(1 + phi^4) on axis (k + 2) % 3.
// Values are computed in double and rounded once.
void pg_face_normals(float* out60)
{
    static const signed char sgn[kPgFaces][3] = {
        {-1, 1, 1}, {0, 1, 1},   {0, 1, -1},  {-1, 1, -1}, {-1, 1, 0},  {1, 1, 1},    {-1, 0, 1},
        {-1, -1, 0}, {-1, 0, -1}, {1, 1, -1},  {1, -1, 1},  {0, -1, 1},  {0, -1, -1},  {1, -1, -1},
        {1, -1, 0},  {1, 0, 1},   {-1, -1, 1}, {-1, -1, -1}, {1, 0, -1}, {1, 1, 0}};
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    const double len = std::sqrt(1.0 + phi * phi * phi * phi);
    const double diag = 1.0 / std::sqrt(3.0), lng = phi * phi / len, shrt = 1.0 / len;
    for (int f = 0; f < kPgFaces; ++f) {
        int zero = -1;
        for (int a = 0; a < 3; ++a)
            if (sgn[f][a] == 0) zero = a;
        double v[3];
        if (zero < 0) {
            for (int a = 0; a < 3; ++a) v[a] = sgn[f][a] * diag;
        } else {
            v[zero] = 0.0;
            v[(zero + 1) % 3] = sgn[f][(zero + 1) % 3] * lng;
            v[(zero + 2) % 3] = sgn[f][(zero + 2) % 3] * shrt;
        }
        for (int a = 0; a < 3; ++a) out60[3 * f + a] = static_cast<float>(v[a]);
    }
}

}  // namespace ar
