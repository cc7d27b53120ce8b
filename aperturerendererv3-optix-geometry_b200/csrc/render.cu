// render.cu -- sm_100a kernels of the wavefront path tracer and the ray queries.
//
// Built with --fmad=false: every floating-point expression rounds exactly as
// the reference's source reads (see detmath.h); fused multiply-adds appear only
// where written as fmaf (the BVH box planes).
#include <curand_kernel.h>

#include "render_kernels.h"
#include "wavefront.cuh"

namespace ar {

// ------------------------------------------------------------------ helpers
struct Rng {
    curandStateXORWOW_t st;
    int used;
    __device__ __forceinline__ float next()
    {
        ++used;
        return curand_uniform(&st);  // Rand1 (random.cuh:41-44)
    }
};

__device__ __forceinline__ void rng_load(const PathSoA& P, int slot, Rng& r)
{
    const uint4 a = P.rng0[slot];
    const uint2 b = P.rng1[slot];
    r.st.d = a.x; r.st.v[0] = a.y; r.st.v[1] = a.z; r.st.v[2] = a.w; r.st.v[3] = b.x; r.st.v[4] = b.y;
    r.st.boxmuller_flag = 0; r.st.boxmuller_flag_double = 0;
    r.st.boxmuller_extra = 0.0f; r.st.boxmuller_extra_double = 0.0;
    r.used = 0;
}
__device__ __forceinline__ void rng_store(const PathSoA& P, int slot, const Rng& r)
{
    P.rng0[slot] = make_uint4(r.st.d, r.st.v[0], r.st.v[1], r.st.v[2]);
    P.rng1[slot] = make_uint2(r.st.v[3], r.st.v[4]);
    if (P.ucount) P.ucount[slot] += r.used;
}

__device__ __forceinline__ f3 xyz(float4 a) { return mk(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated queue append: one atomic per warp, slots ordered by lane.
__device__ __forceinline__ void warp_append(int32_t* counter, int32_t* queue, bool pred, int32_t value)
{
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (m == 0) return;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (static_cast<int>(lane_id()) == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(m | (1u << leader), base, leader);
    if (pred) queue[base + __popc(m & ((1u << lane_id()) - 1u))] = value;
}

__device__ __forceinline__ void warp_count(unsigned long long* counter, bool pred)
{
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (m && static_cast<int>(lane_id()) == __ffs(active) - 1) atomicAdd(counter, static_cast<unsigned long long>(__popc(m)));
}

// reference pixel index of InitRand (random.cuh:31-39) for 8x4 blocks
__device__ __forceinline__ unsigned long long ref_pixel_index(int i, int j, int grid_x)
{
    const int tx = i & 7, ty = j & 3, bxi = i >> 3, byi = j >> 2;
    return static_cast<unsigned long long>(tx + ty * 8) + 32ull * static_cast<unsigned long long>(bxi + byi * grid_x);
}

// ------------------------------------------------------------------ ray queries

__device__ __forceinline__ uint32_t* lane_stack(uint32_t* smem)
{
    return smem + (threadIdx.x >> 5) * (kStackShared * 32) + lane_id();
}
__device__ __forceinline__ uint32_t* thread_overflow(uint32_t* base)
{
    return base + (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kStackOverflow;
}

struct RaysIO {
    const float4* rays;
    int32_t* out_obj;
    float* out_t;
    __device__ __forceinline__ int load(const SceneView&, int k, RayState& r)
    {
        const float4 a = rays[2 * static_cast<int64_t>(k)], b = rays[2 * static_cast<int64_t>(k) + 1];
        ray_begin(r, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w);
        return k;
    }
    __device__ __forceinline__ void store(const SceneView&, int k, const RayState& r)
    {
        out_obj[k] = r.best.obj;
        if (out_t) out_t[k] = r.best.t;
    }
};

template <bool kAny>
__global__ void __launch_bounds__(kTraceBlock) k_trace_rays(SceneView s, RaysIO io, int n, PoolCtl* ctl,
                                                            uint32_t* ovf, int* err)
{
    extern __shared__ uint32_t smem[];
    traverse_queue<kAny>(s, io, n, &ctl->fetch_rays, lane_stack(smem), thread_overflow(ovf), err, nullptr);
}

// ------------------------------------------------------------------ RNG
// curand_init(GLOBAL_SEED, pixelIndex, TOTAL_FRAME_INDEX * 2^32) (random.cuh:35-38)
__global__ void k_rng_init(FrameParams fp, uint4* base0, uint2* base1)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= fp.npix) return;
    const int i = p % fp.width, j = p / fp.width;
    curandStateXORWOW_t st;
    curand_init(fp.seed, ref_pixel_index(i, j, fp.grid_x), fp.frame0 << 32, &st);
    base0[p] = make_uint4(st.d, st.v[0], st.v[1], st.v[2]);
    base1[p] = make_uint2(st.v[3], st.v[4]);
}

// out[(s * npix + p) * per_path + k] = k-th uniform of pixel p at sample s
__global__ void k_rng_tape(FrameParams fp, int spp, int per_path, float* out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= fp.npix) return;
    const int i = p % fp.width, j = p / fp.width;
    for (int s = 0; s < spp; ++s) {
        curandStateXORWOW_t st;
        curand_init(fp.seed, ref_pixel_index(i, j, fp.grid_x), (fp.frame0 + static_cast<uint64_t>(s)) << 32, &st);
        float* o = out + (static_cast<int64_t>(s) * fp.npix + p) * per_path;
        for (int k = 0; k < per_path; ++k) o[k] = curand_uniform(&st);
    }
}

// ------------------------------------------------------------------ path pool
__global__ void k_pool_init(PathSoA P, PoolCtl* ctl, int pool, int64_t total)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < pool) P.freeq[i] = i;
    if (i == 0) {
        ctl->qcount[0] = 0;
        ctl->qcount[1] = 0;
        ctl->shadow_count = 0;
        ctl->retire_count = 0;
        ctl->fetch_ext = 0;
        ctl->fetch_shadow = 0;
        ctl->fetch_rays = 0;
        ctl->free_count = pool;
        ctl->plan_new = 0;
        ctl->plan_src = 0;
        ctl->gen_next = 0;
        ctl->plan_first = 0;
        ctl->retired = 0;
        ctl->total = total;
    }
}

// Start of an iteration: decide how many new samples enter the pool (at most
// one per pixel per iteration, so the per-pixel random state is advanced in
// sample order), and reset the queues this iteration fills.
__global__ void k_plan(PoolCtl* ctl, int cur, int npix)
{
    const int64_t remaining = ctl->total - ctl->gen_next;
    int n = min(ctl->free_count, npix);
    if (static_cast<int64_t>(n) > remaining) n = static_cast<int>(remaining);
    ctl->plan_new = n;
    ctl->plan_src = ctl->free_count - n;
    ctl->free_count -= n;
    ctl->plan_first = ctl->gen_next;
    ctl->gen_next += n;
    ctl->qcount[1 - cur] = 0;
    ctl->shadow_count = 0;
    ctl->retire_count = 0;
    ctl->fetch_ext = 0;
    ctl->fetch_shadow = 0;
}

// RenderCamera (scene.cu:213-230) + CalculateRadiance prologue (render.cuh:520-539)
// for sample g = s * npix + p, in a free slot; appended to the extension queue.
__global__ void k_regen(FrameParams fp, PathSoA P, PoolCtl* ctl, int cur, uint4* base0, uint2* base1,
                        ar_path_record* rec)
{
    const int n = ctl->plan_new;
    const int src = ctl->plan_src;
    const int64_t first = ctl->plan_first;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool act = i < n;
        int slot = 0;
        if (act) {
            slot = P.freeq[src + i];
            const int64_t g = first + i;
            const int sidx = static_cast<int>(g / fp.npix);
            const int p = static_cast<int>(g - static_cast<int64_t>(sidx) * fp.npix);
            const int px = p % fp.width, py = p / fp.width;
            Rng r;
            {
                const uint4 a = base0[p];
                const uint2 b = base1[p];
                r.st.d = a.x; r.st.v[0] = a.y; r.st.v[1] = a.z; r.st.v[2] = a.w; r.st.v[3] = b.x; r.st.v[4] = b.y;
                r.st.boxmuller_flag = 0; r.st.boxmuller_flag_double = 0;
                r.st.boxmuller_extra = 0.0f; r.st.boxmuller_extra_double = 0.0;
                r.used = 0;
                // advance the per-pixel state to the next frame: offset + 2^32
                curandStateXORWOW_t nx = r.st;
                skipahead(1ull << 32, &nx);
                base0[p] = make_uint4(nx.d, nx.v[0], nx.v[1], nx.v[2]);
                base1[p] = make_uint2(nx.v[3], nx.v[4]);
            }
            const float jx = r.next();
            const float jy = r.next();
            const float u = (static_cast<float>(px) + jx) / static_cast<float>(fp.width);
            const float v = (static_cast<float>(py) + jy) / static_cast<float>(fp.height);
            const float ndcx = u * 2.0f - 1.0f;
            const float ndcy = static_cast<float>((1.0 - static_cast<double>(v)) * 2.0 - 1.0);
            const float sx = ndcx * fp.tan_half_x;
            const float sy = ndcy * fp.tan_half_y;
            const f3 cd = mk(fp.cam_d[0], fp.cam_d[1], fp.cam_d[2]);
            const f3 right = mk(fp.right[0], fp.right[1], fp.right[2]);
            const f3 up = mk(fp.up[0], fp.up[1], fp.up[2]);
            const f3 dir0 = normalize(cd + right * sx + up * sy);
            const f3 dir = normalize(dir0);  // CalculateRadiance: rayDirection = normalize(rayDirection)
            const f3 o = mk(fp.cam_o[0], fp.cam_o[1], fp.cam_o[2]);
            P.o[slot] = f4(o, 0.0f);
            P.d[slot] = f4(dir, 0.0f);
            P.mask[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
            P.rad[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (rec) {
#pragma unroll
                for (int k = 0; k < AR_DEBUG_MAX_HITS; ++k) rec[g].hit_object[k] = -1;
            }
            P.info[slot] = make_int4(p, 0, sidx, fp.camera_inside ? kFlagInside : 0);
            P.prev[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            P.media[slot] = make_float4(o.x, o.y, o.z, __int_as_float(-1));
            P.rng0[slot] = make_uint4(r.st.d, r.st.v[0], r.st.v[1], r.st.v[2]);
            P.rng1[slot] = make_uint2(r.st.v[3], r.st.v[4]);
            if (P.ucount) P.ucount[slot] = r.used;
        }
        warp_append(&ctl->qcount[cur], P.q[cur], act, slot);
    }
}

// ------------------------------------------------------------------ extend
// INTERSECT_EPS(d) for d = 0..8 (config.cuh:3), computed on the host with the
// fixed exp of detmath.h and uploaded once (set_intersect_eps).
__constant__ float c_eps_tab[9];

cudaError_t set_intersect_eps(const float* tab9)
{
    return cudaMemcpyToSymbol(c_eps_tab, tab9, 9 * sizeof(float));
}

struct ExtendIO {
    PathSoA P;
    const int32_t* q;
    __device__ __forceinline__ int load(const SceneView& s, int k, RayState& r)
    {
        const int slot = q[k];
        const f3 o = xyz(P.o[slot]), d = xyz(P.d[slot]);
        const int4 info = P.info[slot];
        const float e = c_eps_tab[min(info.y >> 16, 8)];
        const int mobj = __float_as_int(P.media[slot].w);
        if ((info.w & kFlagInside) && mobj >= 0 && s.objects[mobj].type != AR_OBJ_TRIANGLE) {
            // solo trace of the medium's object (render.cuh:91-94, intersection.cuh:185-193)
            const float t = isect_analytic_t(s, mobj, o, d);
            P.hit[slot] = (t >= 0.0f && !(t < e)) ? make_int4(mobj, -1, __float_as_int(t), 0) : make_int4(-1, -1, 0, 0);
            return -1;
        }
        ray_begin(r, o, d, e, INFINITY);
        return slot;
    }
    __device__ __forceinline__ void store(const SceneView&, int slot, const RayState& r)
    {
        P.hit[slot] = r.best.obj >= 0 ? make_int4(r.best.obj, r.best.prim, __float_as_int(r.best.t), 0)
                                      : make_int4(-1, -1, 0, 0);
    }
};

// Trace's closest-hit query (render.cuh:86-99) for every queued path.
__global__ void __launch_bounds__(kTraceBlock) k_extend(SceneView s, PathSoA P, int cur, PoolCtl* ctl,
                                                        unsigned long long* stats, uint32_t* ovf, int* err)
{
    extern __shared__ uint32_t smem[];
    const int n = ctl->qcount[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&stats[0], static_cast<unsigned long long>(n));
    ExtendIO io;
    io.P = P;
    io.q = P.q[cur];
    traverse_queue<false>(s, io, n, &ctl->fetch_ext, lane_stack(smem), thread_overflow(ovf), err, &stats[2]);
}

// ------------------------------------------------------------------ shading helpers
struct GB {
    f3 albedo, emissive;
    float specular, metallic, roughness, ior, sigma_a;
};

__device__ __forceinline__ GB load_gb(const MaterialRec& m)
{
    GB g;
    g.albedo = mk(m.albedo[0], m.albedo[1], m.albedo[2]);
    g.emissive = mk(m.emissive[0], m.emissive[1], m.emissive[2]);
    g.specular = m.specular; g.metallic = m.metallic; g.roughness = m.roughness; g.ior = m.ior; g.sigma_a = m.sigma_a;
    return g;
}

// BuildTangentBasis / BuildTangentBasisRandom (vector.cuh:264-283)
__device__ __forceinline__ void tangent_basis(f3 n, f3& t, f3& b)
{
    const f3 a = (fabsf(n.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    t = normalize(cross(a, n));
    b = cross(n, t);
}
__device__ __forceinline__ void tangent_basis_random(f3 n, f3& t, f3& b, float e)
{
    const f3 a = (fabsf(n.z) < 0.999f) ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    const f3 t0 = normalize(cross(a, n));
    const f3 b0 = cross(n, t0);
    float sn, cs;
    sincos_det(e * kPi * 2.0f, &sn, &cs);
    t = t0 * cs + b0 * sn;
    b = t0 * (-sn) + b0 * cs;
}
// SampleCosineWeightedHemisphere + ConcentricSampleDisk (sample.cuh:63-108)
__device__ __forceinline__ f3 sample_cosine(float e0, float e1, float e2, f3 n, float& pdf)
{
    f3 T, B;
    tangent_basis_random(n, T, B, e2);
    const float sx = 2.0f * e0 - 1.0f;
    const float sy = 2.0f * e1 - 1.0f;
    float x = 0.0f, y = 0.0f;
    if (!(sx == 0.0f && sy == 0.0f)) {
        float r, phi;
        if (fabsf(sx) > fabsf(sy)) { r = sx; phi = (kPi / 4.0f) * (sy / fmaxf(fabsf(sx), 1e-20f)); }
        else { r = sy; phi = (kPi / 2.0f) - (kPi / 4.0f) * (sx / fmaxf(fabsf(sy), 1e-20f)); }
        float sn, cs;
        sincos_det(phi, &sn, &cs);
        x = r * cs; y = r * sn;
    }
    const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
    const f3 dir = T * x + B * y + n * z;
    pdf = z / kPi;
    return normalize(dir);
}
__device__ __forceinline__ float fresnel_exact(float cosI, float cosT, float eta)
{
    const float invE = 1.0f / eta;
    const float rPar = (invE * cosI - cosT) / (invE * cosI + cosT);
    const float rPerp = (cosI - invE * cosT) / (cosI + invE * cosT);
    return 0.5f * (rPar * rPar + rPerp * rPerp);
}
__device__ __forceinline__ float ggx_d(float alpha, float NoH)
{
    const float a2 = alpha * alpha;
    const float d = NoH * NoH * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxf(kPi * d * d, 1e-12f);
}
__device__ __forceinline__ float ggx_g_corr(float alpha, float NoL, float NoV)
{
    const float a2 = alpha * alpha;
    const float gv = NoL * sqrtf(a2 + (1.0f - a2) * NoV * NoV);
    const float gl = NoV * sqrtf(a2 + (1.0f - a2) * NoL * NoL);
    const float den = gv + gl;
    return (den > 0.0f) ? (2.0f * NoL * NoV) / den : 0.0f;
}
__device__ __forceinline__ void ggx_params(const GB& g, float& alpha, float& kD, f3& F0)
{
    alpha = g.roughness * g.roughness;
    const float f0d = 0.08f * clampf(g.specular, 0.0f, 1.0f);
    F0 = lerp3(mk(f0d, f0d, f0d), g.albedo, g.metallic);
    kD = 1.0f - g.metallic;
}
// SampleGGXBoundedVNDF (sample.cuh:179-222)
__device__ __forceinline__ f3 sample_ggx_vndf(f3 V, f3 N, float alpha, float r0, float r1, float r2, float& pdf)
{
    f3 X, Y;
    tangent_basis_random(N, X, Y, r2);
    const float XoV = dot(X, V), YoV = dot(Y, V), NoV = dot(N, V);
    const f3 localV = mk(XoV, YoV, NoV);
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const f3 lstd = mk(XoV * alpha, YoV * alpha, NoV) / sqrtf(a2 + (1.0f - a2) * NoV2);
    const float phi = 2.0f * kPi * r0;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float b = NoV > 0 ? k * lstd.z : lstd.z;
    const float z = fmaf(1.0f - r1, 1.0f + b, -b);
    const float sinT = sqrtf(saturate(1.0f - z * z));
    float sp, cp;
    sincos_det(phi, &sp, &cp);
    const f3 ostd = mk(sinT * cp, sinT * sp, z);
    const f3 mstd = lstd + ostd;
    const f3 lh = normalize(mk(mstd.x * alpha, mstd.y * alpha, mstd.z));
    const f3 ll = reflect(-localV, lh);
    const f3 dir = X * ll.x + Y * ll.y + N * ll.z;
    const float ndf = ggx_d(alpha, lh.z);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    pdf = ndf / (2.0f * (k * NoV + t));
    return dir;
}
// GGXBoundedVNDF_PDF (sample.cuh:224-248)
__device__ __forceinline__ float ggx_vndf_pdf(f3 V, f3 N, f3 L, float alpha)
{
    const float NoV = dot(N, V), NoL = dot(N, L);
    if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
    const f3 H = normalize(V + L);
    const float NoV2 = fminf(1.0f, NoV * NoV);
    const float a2 = alpha * alpha;
    const float sv = 1.0f + sqrtf(1.0f - NoV2);
    const float s2 = sv * sv;
    const float k = (1.0f - a2) * s2 / (s2 + a2 * NoV2);
    const float NoH = fmaxf(0.0f, dot(N, H));
    const float ndf = ggx_d(alpha, NoH);
    const float len2 = (1.0f - NoV2) * a2;
    const float t = sqrtf(len2 + NoV2);
    return fmaxf(ndf / (2.0f * (k * NoV + t)), 1e-12f);
}

// EvaluateBSDFWithCos, RGB (material.cuh:48-175)
__device__ __forceinline__ f3 eval_bsdf_cos(int model, f3 rayDir, f3 L, f3 N, f3 pos, const GB& g, bool inside, f3 vloc)
{
    const float NoL = fmaxf(0.0f, dot(N, L));
    if (model == AR_MAT_DIFFUSE) return g.albedo * (NoL / kPi);
    if (model == AR_MAT_GGX) {
        const f3 V = normalize(-rayDir);
        const float NoV = fmaxf(0.0f, dot(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return mk(0.0f, 0.0f, 0.0f);
        float alpha, kD;
        f3 F0;
        ggx_params(g, alpha, kD, F0);
        // GGXLambert_BRDF (brdf.cuh:96-112)
        const f3 Hn = normalize(V + L);
        const float NoH = fmaxf(0.0f, dot(N, Hn));
        const float LoH = fmaxf(0.0f, dot(L, Hn));
        const float c = clampf(1.0f - LoH, 0.0f, 1.0f);
        const float c5 = c * c * c * c * c;
        const f3 F = mk(F0.x + (1.0f - F0.x) * c5, F0.y + (1.0f - F0.y) * c5, F0.z + (1.0f - F0.z) * c5);
        const float D = ggx_d(alpha, NoH);
        const float G = ggx_g_corr(alpha, NoL, NoV);
        f3 spec = mk(0.0f, 0.0f, 0.0f);
        if (NoL > 0.0f) spec = ((F * D) * G) / fmaxf(4.0f * NoV, 1e-7f);
        const f3 omF = mk(1.0f - F.x, 1.0f - F.y, 1.0f - F.z);
        const f3 diff = ((omF * kD) * g.albedo) * (NoL / kPi);
        return spec + diff;
    }
    if (model == AR_MAT_GLASS) {
        const float IOR = g.ior;
        f3 tr = mk(1.0f, 1.0f, 1.0f);
        if (inside) {
            // BeerLambert (brdf.cuh:15-18)
            const float dd = length(vloc - pos);
            const f3 al = vmin(vmaxs(g.albedo, 1.0e-12f), mk(1.0f, 1.0f, 1.0f));
            const float ds = dd * g.sigma_a;
            tr = mk(exp_det(ds * log_det(al.x)), exp_det(ds * log_det(al.y)), exp_det(ds * log_det(al.z)));
        }
        const f3 nIn = (dot(N, rayDir) > 0.0f) ? -N : N;
        const float eta = inside ? IOR : 1.0f / IOR;
        const float cosI = -dot(nIn, rayDir);
        const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
        const float k = 1.0f - sin2I * (eta * eta);
        if (k <= 0.0f) return tr * 0.99f;
        const float cosT = sqrtf(k);
        const float Fr = fresnel_exact(cosI, cosT, eta);
        const f3 R = reflect(rayDir, nIn);
        const f3 T = refract(rayDir, nIn, eta);
        const float dR = dot(L, R), dT = dot(L, T);
        if (dR >= dT) return tr * Fr;
        const float weight = (eta * eta) * (fabsf(cosT) / fmaxf(1e-6f, cosI));
        return (tr * (1.0f - Fr)) * weight;
    }
    return mk(0.0f, 0.0f, 0.0f);
}

// BSDF_PDF, RGB (material.cuh:332-387)
__device__ __forceinline__ float bsdf_pdf(int model, const GB& g, f3 N, f3 rayDir, f3 L)
{
    const f3 V = -rayDir;
    const float NoL = fmaxf(0.0f, dot(N, L));
    if (model == AR_MAT_DIFFUSE) return NoL > 0.0f ? (NoL * (1.0f / kPi)) : 0.0f;
    if (model == AR_MAT_GGX) {
        const float NoV = fmaxf(0.0f, dot(N, V));
        if (NoV <= 0.0f || NoL <= 0.0f) return 0.0f;
        float alpha, kD;
        f3 F0;
        ggx_params(g, alpha, kD, F0);
        const float pSpec = clampf(luminance(F0), 0.1f, 0.9f);
        const float pdfSpec = ggx_vndf_pdf(V, N, L, alpha);
        const float pdfDiff = NoL * (1.0f / kPi);
        return fmaxf(0.0f, pSpec * pdfSpec + (1.0f - pSpec) * pdfDiff);
    }
    return 0.0f;
}

__device__ __forceinline__ float power_heuristic(float pA, float pB)
{
    const float a = pA * pA, b = pB * pB;
    return a / fmaxf(1e-24f, a + b);
}

__device__ __forceinline__ float area_to_solid_angle(f3 sp, f3 lp, f3 ln, float pA)
{
    const f3 s2l = lp - sp;
    const float d2 = fmaxf(dot(s2l, s2l), 1e-20f);
    const f3 dir = s2l * rsqrt_ieee(d2);
    const float cosY = fmaxf(0.0f, dot(ln, -dir));
    if (cosY <= 0.0f) return 0.0f;
    return pA * (d2 / cosY);
}

struct Box6 {
    f3 fn[6], fc[6];
    float s1[6], s2[6], area[6];
    f3 ux, uy, uz;
};
__device__ __forceinline__ void box_facets(const Analytic& an, Box6& b)
{
    const m3 M = load_m3(an.o2w);
    b.ux = normalize(mk(M.x.x, M.y.x, M.z.x));
    b.uy = normalize(mk(M.x.y, M.y.y, M.z.y));
    b.uz = normalize(mk(M.x.z, M.y.z, M.z.z));
    const f3 c = mk(an.center[0], an.center[1], an.center[2]);
    const f3 e = mk(an.extent[0], an.extent[1], an.extent[2]);
    b.fn[0] = b.ux; b.fn[1] = -b.ux; b.fn[2] = b.uy; b.fn[3] = -b.uy; b.fn[4] = b.uz; b.fn[5] = -b.uz;
    b.fc[0] = c + b.ux * e.x; b.fc[1] = c - b.ux * e.x;
    b.fc[2] = c + b.uy * e.y; b.fc[3] = c - b.uy * e.y;
    b.fc[4] = c + b.uz * e.z; b.fc[5] = c - b.uz * e.z;
    b.s1[0] = e.y; b.s1[1] = e.y; b.s1[2] = e.x; b.s1[3] = e.x; b.s1[4] = e.x; b.s1[5] = e.x;
    b.s2[0] = e.z; b.s2[1] = e.z; b.s2[2] = e.z; b.s2[3] = e.z; b.s2[4] = e.y; b.s2[5] = e.y;
#pragma unroll
    for (int f = 0; f < 6; ++f) b.area[f] = 4.0f * b.s1[f] * b.s2[f];
}
__device__ __forceinline__ float facing_weight(f3 fn, f3 fc, f3 sp, float area)
{
    const f3 l2s = normalize(sp - fc);
    return area * fmaxf(0.0f, dot(fn, l2s));
}

// NEEPDFOmegaFromHit (nee.cuh:64-151, 254-271, 313-327)
__device__ float pdf_light_from_hit(const SceneView& s, int obj, f3 sp, f3 lp, f3 ln)
{
    const ObjInfo oi = s.objects[obj];
    const float sel = s.light_prob[oi.light];
    if (oi.type == AR_OBJ_CUBE) {
        const Analytic& an = s.analytic[oi.aux];
        Box6 b;
        box_facets(an, b);
        int hitFacet = -1;
        for (int f = 0; f < 6; ++f) if (dot(b.fn[f], ln) > 0.999f) { hitFacet = f; break; }
        if (hitFacet < 0) {
            float best = 1e30f;
            for (int f = 0; f < 6; ++f) {
                const float dd = fabsf(dot(b.fn[f], lp - b.fc[f]));
                if (dd < best) { best = dd; hitFacet = f; }
            }
        }
        float sum = 0.0f, wHit = 0.0f, aHit = 0.0f;
        for (int f = 0; f < 6; ++f) {
            const float w = facing_weight(b.fn[f], b.fc[f], sp, b.area[f]);
            sum += w;
            if (f == hitFacet) { wHit = w; aHit = b.area[f]; }
        }
        if (sum <= 0.0f || wHit <= 0.0f) return 0.0f;
        const float pA = sel * (1.0f / aHit) * (wHit / sum);
        return area_to_solid_angle(sp, lp, ln, pA);
    }
    if (oi.type == AR_OBJ_SPHERE) {
        const Analytic& an = s.analytic[oi.aux];
        const f3 c = mk(an.center[0], an.center[1], an.center[2]);
        const float R = an.radius;
        const float dist = length(sp - c);
        if (dist <= R) return 0.0f;
        const float cosC = clampf(R / dist, 0.0f, 1.0f);
        const float areaCap = 2.0f * kPi * R * R * (1.0f - cosC);
        if (areaCap <= 1e-20f) return 0.0f;
        return area_to_solid_angle(sp, lp, ln, sel / areaCap);
    }
    return 0.0f;
}

struct LightSample {
    f3 p, n, emis;
    float pFacet, pA;
    bool valid;
};

// NEESampleLight (nee.cuh:330-377) with the box and sphere samplers
__device__ LightSample sample_light(const SceneView& s, f3 sp, Rng& g)
{
    LightSample ls;
    ls.valid = false;
    if (s.num_lights <= 0) return ls;
    int pick = s.num_lights - 1;
    float pprob = 0.0f;
    {
        const float rr = g.next();
        float acc = 0.0f;
        for (int l = 0; l < s.num_lights; ++l) {
            const float p = s.light_prob[l];
            acc += p;
            if (rr < acc) { pick = l; pprob = p; break; }
        }
    }
    const int lobj = s.light_object[pick];
    const ObjInfo oi = s.objects[lobj];
    const MaterialRec& mr = s.materials[oi.material];
    if (oi.type == AR_OBJ_CUBE) {
        const Analytic& an = s.analytic[oi.aux];
        Box6 b;
        box_facets(an, b);
        int vi[6];
        float vw[6];
        int nv = 0;
        float wsum = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const float w = facing_weight(b.fn[f], b.fc[f], sp, b.area[f]);
            if (w > 0.0f) { vi[nv] = f; vw[nv] = w; wsum += w; ++nv; }
        }
        if (nv == 0) return ls;
        int slot = 0, fi = vi[0];
        {
            const float r = g.next() * wsum;
            float acc = 0.0f;
            for (int k = 0; k < nv; ++k) {
                acc += vw[k];
                if (r <= acc) { slot = k; fi = vi[k]; break; }
            }
        }
        const float u1 = 2.0f * g.next() - 1.0f;
        const float u2 = 2.0f * g.next() - 1.0f;
        const f3 ft = (fi < 2) ? b.uy : b.ux;
        const f3 fb = (fi < 4) ? b.uz : b.uy;
        ls.p = b.fc[fi] + ft * (u1 * b.s1[fi]) + fb * (u2 * b.s2[fi]);
        ls.n = b.fn[fi];
        ls.emis = mk(mr.emissive[0], mr.emissive[1], mr.emissive[2]);
        ls.pFacet = 1.0f * (vw[slot] / wsum);
        ls.pA = 1.0f / b.area[fi];
        ls.valid = true;
    } else if (oi.type == AR_OBJ_SPHERE) {
        const Analytic& an = s.analytic[oi.aux];
        const f3 c = mk(an.center[0], an.center[1], an.center[2]);
        const float R = an.radius;
        const f3 p2c = sp - c;
        const float dist = length(p2c);
        if (dist <= R) return ls;
        const f3 axis = p2c / dist;
        const float cosC = clampf(R / dist, 0.0f, 1.0f);
        const float areaCap = 2.0f * kPi * R * R * (1.0f - cosC);
        const float u = g.next();
        const float vphi = g.next();
        const float cosT = lerpf(cosC, 1.0f, u);
        const float sinT = sqrtf(fmaxf(0.0f, 1.0f - cosT * cosT));
        const float phi = 2.0f * kPi * vphi;
        f3 t, b;
        tangent_basis(axis, t, b);
        float sn, cs;
        sincos_det(phi, &sn, &cs);
        const f3 n = t * (cs * sinT) + b * (sn * sinT) + axis * cosT;
        ls.p = c + n * R;
        ls.n = n;
        ls.emis = mk(mr.emissive[0], mr.emissive[1], mr.emissive[2]);
        ls.pFacet = 1.0f;
        ls.pA = 1.0f / areaCap;
        ls.valid = true;
    } else {
        return ls;
    }
    ls.pFacet = ls.pFacet * pprob;
    return ls;
}

// SkyLighting (render.cuh:58-73)
__device__ __forceinline__ f3 sky_lighting(f3 d, int sky)
{
    if (!sky) return mk(0.0f, 0.0f, 0.0f);
    const f3 white = mk(1.0f, 1.0f, 1.0f);
    const f3 blue = mk(0.05f, 0.45f, 1.0f);
    const f3 down = mk(0.2f, 0.6f, 1.0f) * 0.125f;
    const f3 inner = lerp3(blue, white, pow_det(fmaxf(d.y, 0.0f), 0.75f));
    return lerp3(inner, down, fminf(fmaxf(-d.y * 0.5f + 0.5f, 0.0f), 1.0f)) * 0.5f;
}

// ------------------------------------------------------------------ shade
// One iteration of the CalculateRadiance loop body (render.cuh:541-908) up to
// the shadow query: Trace's material evaluation and hit offset, emission with
// MIS, light sampling for NEE, throughput and Russian roulette.
__global__ void __launch_bounds__(kShadeBlock) k_shade(SceneView s, FrameParams fp, PathSoA P, int cur, PoolCtl* ctl,
                                                       ar_path_record* rec)
{
    const int n = ctl->qcount[cur];
    const int32_t* q = P.q[cur];
    for (int qi0 = blockIdx.x * blockDim.x; qi0 < n; qi0 += gridDim.x * blockDim.x) {
        const int qi = qi0 + threadIdx.x;
        const bool active = qi < n;
        bool cont = false, shadow = false;
        int slot = 0;
        if (active) {
            slot = q[qi];
            int4 info = P.info[slot];
            const int depth = info.y & 0xFFFF;
            int nonDelta = info.y >> 16;
            const int64_t ri = static_cast<int64_t>(info.z) * fp.npix + info.x;
            int flags = info.w & 0xFF;
            int mdepth = info.w >> 8;
            const float4 o4 = P.o[slot], d4 = P.d[slot];
            const f3 crd = xyz(d4);
            const f3 cro = xyz(o4);
            f3 mask = xyz(P.mask[slot]);
            f3 radiance = xyz(P.rad[slot]);
            float4 md = P.media[slot];
            const bool inside = (flags & kFlagInside) != 0;
            const f3 vloc = xyz(md);
            const int mobj = __float_as_int(md.w);
            const int4 hr = P.hit[slot];
            const bool hit = hr.x >= 0;
            const float eps = c_eps_tab[min(nonDelta, 8)];
            Rng g;
            rng_load(P, slot, g);
            if (rec && depth < AR_DEBUG_MAX_HITS) rec[ri].hit_object[depth] = hit ? hr.x : -1;
            if (rec) rec[ri].segments = depth + 1;
            // ---- intersection details (re-run of the accepted test)
            f3 pos = mk(0.0f, 0.0f, 0.0f), nrm = mk(0.0f, 0.0f, 0.0f);
            GB gb;
            int model = -1, light = -1;
            if (hit) {
                const ObjInfo oi = s.objects[hr.x];
                model = s.materials[oi.material].model;
                gb = load_gb(s.materials[oi.material]);
                light = oi.light;
                if (oi.type == AR_OBJ_TRIANGLE) {
                    const PrimRec& pr = s.prims[hr.y];
                    const f3 v0 = mk(pr.v0[0], pr.v0[1], pr.v0[2]);
                    const f3 e1 = mk(pr.e1[0], pr.e1[1], pr.e1[2]);
                    const f3 e2 = mk(pr.e2[0], pr.e2[1], pr.e2[2]);
                    const f3 h = cross(crd, e2);
                    const float a = dot(e1, h);
                    const float f = __frcp_rn(a);
                    const f3 sv = cro - v0;
                    const float u = f * dot(sv, h);
                    const f3 qv = cross(sv, e1);
                    const float v = f * dot(crd, qv);
                    const float t = __int_as_float(hr.z);
                    pos = cro + crd * t;
                    const float w = 1.0f - u - v;
                    const TriShade& ts = s.trishade[oi.aux];
                    const f3 n0 = mk(ts.n0[0], ts.n0[1], ts.n0[2]);
                    const f3 n1 = mk(ts.n1[0], ts.n1[1], ts.n1[2]);
                    const f3 n2 = mk(ts.n2[0], ts.n2[1], ts.n2[2]);
                    const f3 ni = normalize(n0 * w + n1 * u + n2 * v);
                    nrm = dot(crd, ni) > 0.0f ? -ni : ni;
                } else if (oi.type == AR_OBJ_CUBE) {
                    isect_cube<true>(s.analytic[oi.aux], cro, crd, &pos, &nrm);
                } else {
                    isect_sphere<true>(s.analytic[oi.aux], cro, crd, &pos, &nrm);
                }
            }
            // ---- SampleContext (material.cuh:19-37, 177-330, 389-425)
            f3 next = mk(0.0f, 0.0f, 0.0f), emis = mk(0.0f, 0.0f, 0.0f), brdf = mk(0.0f, 0.0f, 0.0f);
            float pdf = 1.0f;
            bool terminate = false, delta = false, missThin = false;
            bool nInside = false;
            f3 nvloc = mk(0.0f, 0.0f, 0.0f);
            int nmobj = -1, nmdepth = 0;
            if (!hit && inside) {
                missThin = true;
                nvloc = cro;
            }
            if (hit) {
                const f3 N = nrm;
                if (model == AR_MAT_DIFFUSE) {
                    const float e0 = g.next(), e1 = g.next(), e2 = g.next();
                    next = sample_cosine(e0, e1, e2, N, pdf);
                    emis = gb.emissive;
                    nInside = inside; nvloc = pos;
                } else if (model == AR_MAT_LIGHT) {
                    pdf = 1.0f; emis = gb.emissive; terminate = true;
                } else if (model == AR_MAT_GLASS) {
                    delta = true;
                    const float eta = inside ? gb.ior : 1.0f / gb.ior;
                    const f3 nIn = (dot(N, crd) > 0.0f) ? -N : N;
                    const float cosI = -dot(nIn, crd);
                    const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
                    const float k = 1.0f - sin2I * (eta * eta);
                    if (k <= 0.0f) {
                        if (mdepth < 1024) { next = reflect(crd, nIn); nInside = inside; }
                        else { next = crd; nInside = !inside; }
                        pdf = 1.0f; nvloc = pos;
                    } else {
                        const float cosT = sqrtf(k);
                        const float Fr = fresnel_exact(cosI, cosT, eta);
                        if (g.next() < Fr) { next = reflect(crd, nIn); pdf = Fr; nInside = inside; }
                        else { next = refract(crd, nIn, eta); pdf = 1.0f - Fr; nInside = !inside; }
                        nvloc = pos;
                    }
                } else if (model == AR_MAT_GGX) {
                    emis = gb.emissive;
                    const f3 V = -crd;
                    const float NoV = fmaxf(0.0f, dot(N, V));
                    if (NoV <= 0.0f) {
                        terminate = true;
                    } else {
                        float alpha, kD;
                        f3 F0;
                        ggx_params(gb, alpha, kD, F0);
                        const float pSpec = clampf(luminance(F0), 0.1f, 0.9f);
                        const float uu = g.next();
                        const float e0 = g.next(), e1 = g.next(), e2 = g.next();
                        if (uu < pSpec) {
                            float ps;
                            const f3 L = sample_ggx_vndf(V, N, alpha, e0, e1, e2, ps);
                            const float NoL = fmaxf(0.0f, dot(N, L));
                            if (NoL <= 0.0f) {
                                terminate = true;
                            } else {
                                next = L; pdf = pSpec * ps + (1.0f - pSpec) * (NoL / kPi);
                                nInside = inside; nvloc = pos;
                            }
                        } else {
                            float pd;
                            const f3 L = sample_cosine(e0, e1, e2, N, pd);
                            const float pspec = ggx_vndf_pdf(V, N, L, alpha);
                            next = L; pdf = pSpec * pspec + (1.0f - pSpec) * pd;
                            nInside = inside; nvloc = pos;
                        }
                    }
                }
                nmobj = hr.x;
                nmdepth = mdepth + 1;
                brdf = eval_bsdf_cos(model, crd, next, N, pos, gb, inside, vloc);
            } else {
                brdf = mk(1.0f, 1.0f, 1.0f);
                delta = false;
                next = crd;
                pdf = 1.0f;
                emis = sky_lighting(crd, fp.sky);
                nInside = false;
            }
            {   // hit offset, always one uniform (render.cuh:156-160)
                const float offEps = eps * fmaxf(1.0f, length(pos));
                const float sg = signf(dot(nrm, next));
                const float r = g.next();
                pos = pos + ((nrm * sg) * offEps) * (r + 0.5f);
            }
            // media state after this segment
            const bool mInside = nInside;
            // ---- emission (render.cuh:648-723)
            if (!hit) {
                if (!missThin) radiance = radiance + mask * emis;
            } else if (light >= 0) {
                float misW = 1.0f;
                if (fp.use_nee && depth > 0 && (flags & kFlagPrevNEE)) {
                    const float4 pv = P.prev[slot];
                    const float pB = fmaxf(pv.w, 0.0f);
                    const float pL = pdf_light_from_hit(s, hr.x, xyz(pv), pos, nrm);
                    if (pL >= 0.0f && pB > 0.0f) misW = power_heuristic(pB, pL);
                }
                radiance = radiance + (mask * emis) * misW;
            }
            const bool brk = (!hit && !missThin) || terminate;
            f3 pending = mk(0.0f, 0.0f, 0.0f);
            bool cosOK = false;
            if (!brk) {
                // ---- NEE (render.cuh:766-827)
                if (!missThin) {
                    const float lum = luminance(mask);
                    const float rate = sqrtf(saturate(lum));
                    int newPrev = 0;
                    if (fp.use_nee && nonDelta < 10 && !delta && !mInside && g.next() < rate) {
                        const LightSample ls = sample_light(s, pos, g);
                        if (ls.valid) {
                            const float pATotal = fmaxf(1e-20f, ls.pA * ls.pFacet);
                            const f3 lu = ls.p - pos;
                            const float d2 = fmaxf(dot(lu, lu), 1.0e-12f);
                            const f3 ld = lu * rsqrt_ieee(d2);
                            const float cosX = fmaxf(0.0f, dot(nrm, ld));
                            const float cosY = fmaxf(0.0f, dot(ls.n, -ld));
                            if (cosX > 0.0f && cosY > 0.0f) {
                                cosOK = true;
                                const f3 fcos = eval_bsdf_cos(model, crd, ld, nrm, pos, gb, false, mk(0.0f, 0.0f, 0.0f));
                                const float G = cosY / d2;
                                const f3 contrib = (fcos * ls.emis) * (G / pATotal);
                                const float pL = area_to_solid_angle(pos, ls.p, ls.n, ls.pFacet * ls.pA);
                                const float pB = fmaxf(bsdf_pdf(model, gb, nrm, crd, ld), 0.0f);
                                pending = mask * (contrib * power_heuristic(pL, pB));
                            }
                            shadow = true;
                            P.sseg0[slot] = f4(pos, c_eps_tab[min(depth, 8)]);
                            P.sseg1[slot] = f4(ls.p, 0.0f);
                            if (rec) {
                                rec[ri].nee_rays += 1;
                                if (depth < 32) rec[ri].nee_depth_mask |= static_cast<int32_t>(1u << depth);
                            }
                        }
                    }
                    flags = (flags & ~kFlagPrevNEE) | (newPrev ? kFlagPrevNEE : 0);
                    P.prev[slot] = f4(pos, pdf);
                }
                // ---- throughput and Russian roulette (render.cuh:829-907)
                const f3 contrib = mk(brdf.x / fmaxf(pdf, 1e-12f), brdf.y / fmaxf(pdf, 1e-12f), brdf.z / fmaxf(pdf, 1e-12f));
                float qrr = 1.0f;
                bool survived = true;
                if (nonDelta >= fp.rr_depth) {
                    const float lum = luminance(mask);
                    const float mx = max3(mask);
                    const float basic = clampf(lum * 0.5f + mx * 0.5f, 0.05f, 0.95f);
                    qrr = lerpf(basic, 1.0f, mInside ? 0.99f : 0.0f);
                    if (g.next() > qrr) survived = false;
                }
                if (survived) {
                    mask = mask * contrib;
                    mask = mask / qrr;
                    if (!delta) nonDelta++;
                    cont = depth + 1 < fp.max_depth;
                    P.o[slot] = f4(pos, 0.0f);
                    P.d[slot] = f4(next, 0.0f);
                    P.mask[slot] = f4(mask, 0.0f);
                }
            }
            flags = (flags & ~(kFlagInside | kFlagNeeCosOK | kFlagMissThin)) | (mInside ? kFlagInside : 0) |
                    (cosOK ? kFlagNeeCosOK : 0) | (missThin ? kFlagMissThin : 0);
            P.rad[slot] = f4(radiance, 0.0f);
            P.nee[slot] = f4(pending, 0.0f);
            P.media[slot] = make_float4(nvloc.x, nvloc.y, nvloc.z, __int_as_float(nmobj));
            P.info[slot] = make_int4(info.x, (depth + 1) | (nonDelta << 16), info.z, flags | (nmdepth << 8));
            rng_store(P, slot, g);
        }
        warp_append(&ctl->qcount[1 - cur], P.q[1 - cur], cont, slot);
        warp_append(&ctl->shadow_count, P.qs, shadow, slot);
        warp_append(&ctl->retire_count, P.qr, active && !cont, slot);
    }
}

// ------------------------------------------------------------------ shadow
// SegmentTrace -> AnyHitSegmentBVH (render.cuh:167-183, intersection.cuh:372-397)
// and the remainder of NEE (render.cuh:242-343): the pending term is added when
// the segment is unoccluded, and previousDidNEE_ becomes "occluded or cos > 0".
struct ShadowIO {
    PathSoA P;
    unsigned long long traced;
    __device__ __forceinline__ void finish(int slot, bool occ)
    {
        int4 info = P.info[slot];
        const bool cosOK = (info.w & kFlagNeeCosOK) != 0;
        if (!occ && cosOK) {
            const float4 r = P.rad[slot], pn = P.nee[slot];
            P.rad[slot] = make_float4(r.x + pn.x, r.y + pn.y, r.z + pn.z, 0.0f);
        }
        info.w = (info.w & ~kFlagPrevNEE) | ((occ || cosOK) ? kFlagPrevNEE : 0);
        P.info[slot] = info;
    }
    __device__ __forceinline__ int load(const SceneView&, int k, RayState& r)
    {
        const int slot = P.qs[k];
        const float4 a = P.sseg0[slot], b = P.sseg1[slot];
        const f3 src = xyz(a), dst = xyz(b);
        f3 dir = dst - src;
        const float dist = length(dir);
        if (dist > 0.0f) {
            dir = dir / dist;
            const float eps = a.w * fmaxf(1.0f, fmaxf(length(src), length(dst)));
            const float tMax = fmaxf(0.0f, dist - eps);
            if (tMax > 0.0f) {
                ray_begin(r, src, dir, 0.0f, tMax);
                ++traced;
                return slot;
            }
        }
        finish(slot, false);
        return -1;
    }
    __device__ __forceinline__ void store(const SceneView&, int slot, const RayState& r) { finish(slot, r.best.obj >= 0); }
};

__global__ void __launch_bounds__(kTraceBlock) k_shadow(SceneView s, PathSoA P, PoolCtl* ctl,
                                                        unsigned long long* stats, uint32_t* ovf, int* err)
{
    extern __shared__ uint32_t smem[];
    const int n = ctl->shadow_count;
    ShadowIO io;
    io.P = P;
    io.traced = 0;
    traverse_queue<true>(s, io, n, &ctl->fetch_shadow, lane_stack(smem), thread_overflow(ovf), err, &stats[4]);
    unsigned long long c = io.traced;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane_id() == 0 && c) atomicAdd(&stats[1], c);
}

// ------------------------------------------------------------------ finish
// checkNanInf + clamp (render.cuh:969), max(0, .) (scene.cu:238), FP64 sum.
__device__ __forceinline__ float fix_nan_inf(float x)
{
    if (isnan_(x)) return 0.0f;
    if (isinf_(x)) return x > 0.0f ? 0.0f : -0.0f;
    return x;
}
// Paths that ended this iteration (after their last shadow query): FP64 sum
// into the pixel, slot back onto the free stack.
__global__ void k_retire(FrameParams fp, PathSoA P, PoolCtl* ctl, double* accum, ar_path_record* rec)
{
    const int n = ctl->retire_count;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->retired += n;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + threadIdx.x;
        const bool act = i < n;
        int slot = 0;
        if (act) {
            slot = P.qr[i];
            const float4 r = P.rad[slot];
            const float x = fmaxf(clampf(fix_nan_inf(r.x), 0.0f, 1.0e3f), 0.0f);
            const float y = fmaxf(clampf(fix_nan_inf(r.y), 0.0f, 1.0e3f), 0.0f);
            const float z = fmaxf(clampf(fix_nan_inf(r.z), 0.0f, 1.0e3f), 0.0f);
            const int4 info = P.info[slot];
            double* a = accum + 3 * static_cast<int64_t>(info.x);
            atomicAdd(a + 0, static_cast<double>(x));
            atomicAdd(a + 1, static_cast<double>(y));
            atomicAdd(a + 2, static_cast<double>(z));
            if (rec) {
                const int64_t ri = static_cast<int64_t>(info.z) * fp.npix + info.x;
                rec[ri].radiance[0] = x; rec[ri].radiance[1] = y; rec[ri].radiance[2] = z;
                rec[ri].uniforms = P.ucount ? P.ucount[slot] : 0;
            }
        }
        warp_append(&ctl->free_count, P.freeq, act, slot);
    }
}

__global__ void k_mean(const double* accum, int64_t n, double inv, float* out)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) out[i] = static_cast<float>(accum[i] * inv);
}

__global__ void k_add(const double* src, int64_t n, double* dst)
{
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) dst[i] += src[i];
}

// ------------------------------------------------------------------ launchers
constexpr size_t kTraceSmem = static_cast<size_t>(kStackShared) * kTraceBlock * 4;

int trace_grid(int sm_count)
{
    static int blocks = 0;
    if (blocks == 0) {
        int b0 = 1, b1 = 1, b2 = 1, b3 = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_extend, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_shadow, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_trace_rays<false>, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_trace_rays<true>, kTraceBlock, kTraceSmem);
        cudaGetLastError();
        blocks = max(1, max(max(b0, b1), max(b2, b3)));
    }
    return blocks * sm_count;
}

cudaError_t launch_trace_rays(const SceneView& s, const float4* rays, int n, int any, int32_t* obj, float* t,
                              PoolCtl* ctl, uint32_t* ovf, int* err, int grid, cudaStream_t st)
{
    RaysIO io;
    io.rays = rays;
    io.out_obj = obj;
    io.out_t = t;
    if (any) k_trace_rays<true><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
    else k_trace_rays<false><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
    return cudaGetLastError();
}

cudaError_t launch_rng_init(const FrameParams& fp, uint4* b0, uint2* b1, cudaStream_t st)
{
    k_rng_init<<<(fp.npix + 255) / 256, 256, 0, st>>>(fp, b0, b1);
    return cudaGetLastError();
}

cudaError_t launch_rng_tape(const FrameParams& fp, int spp, int per_path, float* out, cudaStream_t st)
{
    k_rng_tape<<<(fp.npix + 127) / 128, 128, 0, st>>>(fp, spp, per_path, out);
    return cudaGetLastError();
}

cudaError_t launch_pool_init(const PathSoA& P, PoolCtl* ctl, int pool, int64_t total, cudaStream_t st)
{
    k_pool_init<<<(pool + 255) / 256, 256, 0, st>>>(P, ctl, pool, total);
    return cudaGetLastError();
}

cudaError_t launch_iterations(const SceneView& s, const FrameParams& fp, const PathSoA& P, PoolCtl* ctl, uint4* b0,
                              uint2* b1, unsigned long long* stats, uint32_t* ovf, int* err, double* accum,
                              ar_path_record* rec, int iterations, int* cur, int grid_trace, int grid_other,
                              cudaStream_t st, int64_t* launches, LaunchTimers* tm)
{
    for (int it = 0; it < iterations; ++it) {
        const int c = *cur;
        k_plan<<<1, 1, 0, st>>>(ctl, c, fp.npix);
        k_regen<<<grid_other, kShadeBlock, 0, st>>>(fp, P, ctl, c, b0, b1, rec);
        const bool te = tm && tm->n_extend < tm->cap;
        if (te) cudaEventRecord(tm->extend_ev[2 * tm->n_extend], st);
        k_extend<<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, P, c, ctl, stats, ovf, err);
        if (te) cudaEventRecord(tm->extend_ev[2 * tm->n_extend++ + 1], st);
        k_shade<<<grid_other, kShadeBlock, 0, st>>>(s, fp, P, c, ctl, rec);
        const bool ts = tm && tm->n_shadow < tm->cap;
        if (ts) cudaEventRecord(tm->shadow_ev[2 * tm->n_shadow], st);
        k_shadow<<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, P, ctl, stats, ovf, err);
        if (ts) cudaEventRecord(tm->shadow_ev[2 * tm->n_shadow++ + 1], st);
        k_retire<<<grid_other, kShadeBlock, 0, st>>>(fp, P, ctl, accum, rec);
        *launches += 6;
        *cur = 1 - c;
    }
    return cudaGetLastError();
}

cudaError_t launch_mean(const double* accum, int64_t n, double inv, float* out, cudaStream_t st)
{
    k_mean<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(accum, n, inv, out);
    return cudaGetLastError();
}
cudaError_t launch_add(const double* src, int64_t n, double* dst, cudaStream_t st)
{
    k_add<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(src, n, dst);
    return cudaGetLastError();
}

}  // namespace ar
