// render.cu -- sm_100a kernels of the wavefront path tracer and the ray queries.
//
// Built with --fmad=false: every floating-point expression rounds exactly as
// the reference's source reads (see detmath.h); fused multiply-adds appear only
// where written as fmaf (the BVH box planes and the sampling polynomials).
#include <curand_kernel.h>

#include "render_kernels.h"
#include "shading.cuh"
#include "wavefront.cuh"
#include "xorwow_jump.h"

namespace ar {

cudaError_t set_intersect_eps(const float* tab9)
{
    return cudaMemcpyToSymbol(c_eps_tab, tab9, 9 * sizeof(float));
}

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ unsigned lanes_below() { return (1u << lane_id()) - 1u; }

// Warp-aggregated allocation: one atomic per warp, indices ordered by lane.
// Returns the caller's index, or -1 when pred is false.
__device__ __forceinline__ int warp_alloc(int32_t* counter, bool pred)
{
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (m == 0) return -1;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (static_cast<int>(lane_id()) == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(active, base, leader);
    return pred ? base + __popc(m & lanes_below()) : -1;
}

// Append `value` to bucket `bucket` of a bucketed queue (data[bucket * cap + i]);
// lanes of a warp with the same bucket share one atomic (__match_any_sync).
__device__ __forceinline__ void bucket_append(int32_t* counts, int32_t* data, int cap, int bucket, int32_t value)
{
    const unsigned active = __activemask();
    const unsigned same = __match_any_sync(active, bucket);
    const int leader = __ffs(same) - 1;
    int base = 0;
    if (static_cast<int>(lane_id()) == leader) base = atomicAdd(&counts[bucket], __popc(same));
    base = __shfl_sync(same, base, leader);
    data[static_cast<int64_t>(bucket) * cap + base + __popc(same & lanes_below())] = value;
}

// reference pixel index of InitRand (random.cuh:31-39) for 8x4 blocks
__device__ __forceinline__ unsigned long long ref_pixel_index(int i, int j, int grid_x)
{
    const int tx = i & 7, ty = j & 3, bxi = i >> 3, byi = j >> 2;
    return static_cast<unsigned long long>(tx + ty * 8) + 32ull * static_cast<unsigned long long>(bxi + byi * grid_x);
}

__device__ __forceinline__ uint32_t* lane_stack(uint32_t* smem)
{
    return smem + (threadIdx.x >> 5) * (kStackShared * 32) + lane_id();
}
__device__ __forceinline__ uint32_t* thread_overflow(uint32_t* base)
{
    return base + (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kStackOverflow;
}

__device__ __forceinline__ int ibits(float f) { return __float_as_int(f); }
// pool buffer `c` without dynamic indexing of the kernel-parameter array
__device__ __forceinline__ PathRec* pool_of(const PathBuffers& B, int c) { return c ? B.pool[1] : B.pool[0]; }
__device__ __forceinline__ float4* aux_of(const PathBuffers& B, int c) { return c ? B.aux[1] : B.aux[0]; }
__device__ __forceinline__ float fbits(int i) { return __int_as_float(i); }

// ------------------------------------------------------------------ ray queries
template <bool kSdf>
struct RaysIO {
    const float4* rays;
    int32_t* out_obj;
    float* out_t;
    int any;
    __device__ __forceinline__ int load(const SceneView&, int k, RayState& r)
    {
        const float4 a = rays[2 * static_cast<int64_t>(k)], b = rays[2 * static_cast<int64_t>(k) + 1];
        ray_begin(r, mk(a.x, a.y, a.z), mk(b.x, b.y, b.z), a.w, b.w);
        return k;
    }
    __device__ __forceinline__ void store(const SceneView& s, int k, const RayState& r)
    {
        int32_t obj = r.best.obj;
        float t = r.best.t;
        if (kSdf && s.num_sdf > 0) {  // standalone queries use the depth-0 tolerance
            if (!any) sdf_closest(s, r.o, r.d, r.tmin, kEpsDepth0, &t, &obj);
            else if (obj < 0) obj = sdf_any(s, r.o, r.d, r.tmin, t, kEpsDepth0);
        }
        out_obj[k] = obj;
        if (out_t) out_t[k] = t;
    }
};

template <bool kAny, bool kSdf>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_trace_rays(SceneView s, RaysIO<kSdf> io, int n, PoolCtl* ctl,
                                                            uint32_t* ovf, int* err)
{
    extern __shared__ uint32_t smem[];
    traverse_queue<kAny>(s, io, n, &ctl->fetch_rays, lane_stack(smem), thread_overflow(ovf), err, nullptr);
}

// ------------------------------------------------------------------ RNG
// curand_init(GLOBAL_SEED, pixelIndex, TOTAL_FRAME_INDEX * 2^32) (random.cuh:35-38)
// Every pixel's state of InitRand: curand_init(seed, s, frame0 * 2^32) with s
// its reference pixel index.  One thread per 8x4 pixel block, i.e. per run of
// 32 consecutive s: curand_init for the block's first pixel, then each next
// pixel's register as A^(2^67) times the previous one (subsequences are 2^67
// draws apart; the Weyl counter moves by 362437 * 2^67 = 0 mod 2^32), which
// replaces 31 of every 32 general skip-aheads by a table jump.
__global__ void k_rng_init(FrameParams fp, uint4* base0, uint2* base1, const uint32_t* __restrict__ jump67)
{
    __shared__ uint32_t jt[kJumpWords];
    for (int k = threadIdx.x; k < kJumpWords; k += blockDim.x) jt[k] = jump67[k];
    __syncthreads();
    const int grid_y = (fp.height + 3) / 4;
    const int nblk = fp.grid_x * grid_y;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += gridDim.x * blockDim.x) {
        curandStateXORWOW_t st;
        curand_init(fp.seed, 32ull * static_cast<unsigned long long>(b), fp.frame0 << 32, &st);
        uint32_t v[5] = {st.v[0], st.v[1], st.v[2], st.v[3], st.v[4]};
        const int bx = b % fp.grid_x, by = b / fp.grid_x;
        for (int w = 0; w < 32; ++w) {   // w = tx + 8 ty: ref_pixel_index order within the block
            if (w > 0) xorwow_jump(v, jt);   // A^(2^67): the next subsequence
            const int i = 8 * bx + (w & 7), j = 4 * by + (w >> 3);
            if (i < fp.width && j < fp.height) {
                const int p = j * fp.width + i;
                base0[p] = make_uint4(st.d, v[0], v[1], v[2]);
                base1[p] = make_uint2(v[3], v[4]);
            }
        }
    }
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

__device__ __forceinline__ void rng_from(Rng& r, uint4 a, uint4 b)
{
    r.st.d = a.x; r.st.v[0] = a.y; r.st.v[1] = a.z; r.st.v[2] = a.w; r.st.v[3] = b.x; r.st.v[4] = b.y;
    r.st.boxmuller_flag = 0; r.st.boxmuller_flag_double = 0;
    r.st.boxmuller_extra = 0.0f; r.st.boxmuller_extra_double = 0.0;
    r.used = 0;
}

// ------------------------------------------------------------------ path pool
__global__ void k_pool_init(PoolCtl* ctl, int64_t total)
{
    ctl->count[0] = 0;
    ctl->count[1] = 0;
    for (int b = 0; b < 8; ++b) ctl->shade_count[b] = 0;
    ctl->shadow_count = 0;
    ctl->retire_count = 0;
    ctl->fetch_ext = 0;
    ctl->fetch_shadow = 0;
    ctl->fetch_rays = 0;
    ctl->plan_new = 0;
    ctl->plan_base = 0;
    ctl->gen_next = 0;
    ctl->plan_first = 0;
    ctl->retired = 0;
    ctl->total = total;
}

// Start of an iteration: the current pool holds the paths that survived the
// previous one; top it up with new samples (at most one per pixel, so the
// per-pixel random state advances in sample order) and reset the queues this
// iteration fills.
__global__ void k_plan(PoolCtl* ctl, int cur, int npix, int capacity)
{
    const int64_t remaining = ctl->total - ctl->gen_next;
    const int ncont = ctl->count[cur];
    int n = min(capacity - ncont, npix);
    if (static_cast<int64_t>(n) > remaining) n = static_cast<int>(remaining);
    ctl->plan_new = n;
    ctl->plan_base = ncont;
    ctl->count[cur] = ncont + n;
    ctl->plan_first = ctl->gen_next;
    ctl->gen_next += n;
    ctl->count[1 - cur] = 0;
    for (int b = 0; b < 8; ++b) ctl->shade_count[b] = 0;
    ctl->shadow_count = 0;
    ctl->retire_count = 0;
    ctl->fetch_ext = 0;
    ctl->fetch_shadow = 0;
}

// RenderCamera (scene.cu:213-230) + CalculateRadiance prologue (render.cuh:520-539)
// for sample g = s * npix + p, written to the current pool behind the survivors.
__global__ void k_regen(FrameParams fp, PathBuffers B, PoolCtl* ctl, int cur, uint4* base0, uint2* base1,
                        const uint32_t* __restrict__ jump_table, ar_path_record* rec)
{
    __shared__ uint32_t jt[kJumpWords];
    for (int k = threadIdx.x; k < kJumpWords; k += blockDim.x) jt[k] = jump_table[k];
    __syncthreads();
    const int n = ctl->plan_new;
    const int base = ctl->plan_base;
    const int64_t first = ctl->plan_first;
    PathRec* pool = pool_of(B, cur);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int64_t g = first + i;
        const int sidx = static_cast<int>(g / fp.npix);
        const int p = static_cast<int>(g - static_cast<int64_t>(sidx) * fp.npix);
        const int px = p % fp.width, py = p / fp.width;
        const uint4 a = base0[p];
        const uint2 b = base1[p];
        Rng r;
        rng_from(r, a, make_uint4(b.x, b.y, 0u, 0u));
        {   // advance the per-pixel state to the next frame: offset + 2^32
            uint32_t nv[5] = {a.y, a.z, a.w, b.x, b.y};
            xorwow_jump(nv, jt);
            base0[p] = make_uint4(a.x, nv[0], nv[1], nv[2]);
            base1[p] = make_uint2(nv[3], nv[4]);
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
        if (rec) {
#pragma unroll
            for (int k = 0; k < AR_DEBUG_MAX_HITS; ++k) rec[g].hit_object[k] = -1;
        }
        PathRec pr;
        pr.o = f4(o, fbits(0));
        pr.d = f4(dir, fbits(fp.camera_inside ? kFlagInside : 0));
        pr.mask = make_float4(1.0f, 1.0f, 1.0f, fbits(p));
        if (fp.spectral) {  // CalculateRadiance starts with SampleCIE1931(Rand3(seed)) (render.cuh:467)
            const float r0 = r.next(), r1 = r.next(), r2 = r.next();
            const LambdaSample ls = sample_cie1931(r0, r1, r2);
            if (fp.spectral == 4) {   // hero wavelength + 3 rotations: throughputs 1, hero in the side record
                pr.mask = make_float4(1.0f, 1.0f, 1.0f, fbits(p));
                aux_of(B, cur)[base + i] = make_float4(1.0f, 0.0f, ls.lambda, 0.0f);
            } else {
                pr.mask = make_float4(1.0f, ls.lambda, ls.pdf, fbits(p));
            }
        }
        pr.rad = make_float4(0.0f, 0.0f, 0.0f, fbits(sidx));
        pr.rng0 = make_uint4(r.st.d, r.st.v[0], r.st.v[1], r.st.v[2]);
        pr.rng1 = make_uint4(r.st.v[3], r.st.v[4], static_cast<uint32_t>(-1), static_cast<uint32_t>(r.used));
        pr.prev = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        pr.vloc = make_float4(o.x, o.y, o.z, 0.0f);
        pool[base + i] = pr;
    }
}

// ------------------------------------------------------------------ extend
// Free-flight sampling in the medium along the extension segment [0, tmax):
// the distance of the first real collision, or -1 (out of line: only scenes
// with a medium reach it).
__device__ __noinline__ float medium_collision(const SceneView& s, const PathRec& pr, f3 o, f3 d, float tmax,
                                               uint32_t key)
{
    HashRng h;
    h.seed = medium_seed(key, static_cast<uint32_t>(ibits(pr.rad.w)), static_cast<uint32_t>(ibits(pr.mask.w)),
                         static_cast<uint32_t>(ibits(pr.o.w) & 0xFFFF), 0u);
    h.n = 0;
    return delta_track(s.medium, o, d, tmax, h);
}

template <bool kExt>
struct ExtendIO {
    const PathRec* pool;
    int4* hit;
    int32_t* shade_count;
    int32_t* qsh;
    int cap;
    uint32_t medium_key;  // medium_frame_key of the render
    // queue the path for shading, bucketed by what it hit (render.cuh:97-118)
    __device__ __forceinline__ void to_shade(const SceneView& s, int k, int obj)
    {
        const int bucket = obj >= 0 ? s.materials[s.objects[obj].material].model + 1 : (obj == kHitMedium ? kModelMedium + 1 : 0);
        bucket_append(shade_count, qsh, cap, bucket, k);
    }
    __device__ __forceinline__ int load(const SceneView& s, int k, RayState& r)
    {
        const float4 o4 = pool[k].o, d4 = pool[k].d;
        const f3 o = xyz(o4), d = xyz(d4);
        const float e = c_eps_tab[min(ibits(o4.w) >> 16, 8)];
        if (ibits(d4.w) & kFlagInside) {
            const int mobj = static_cast<int>(pool[k].rng1.z);
            if (mobj >= 0 && s.objects[mobj].type != AR_OBJ_TRIANGLE) {
                // solo trace of the medium's object (render.cuh:91-94, intersection.cuh:185-193)
                const float t = (kExt && s.objects[mobj].type == AR_OBJ_SDF) ? sdf_solo_t(s, mobj, o, d, e)
                                                                             : isect_analytic_t(s, mobj, o, d);
                const bool h = t >= 0.0f && !(t < e);
                hit[k] = h ? make_int4(mobj, -1, ibits(t), 0) : make_int4(-1, -1, 0, 0);
                to_shade(s, k, h ? mobj : -1);
                return -1;
            }
        }
        ray_begin(r, o, d, e, INFINITY);
        return k;
    }
    __device__ __forceinline__ void store(const SceneView& s, int k, const RayState& r)
    {
        int32_t obj = r.best.obj, prim = r.best.prim;
        float t = r.best.t;
        if (kExt && s.num_sdf > 0) {
            const int32_t before = obj;
            sdf_closest(s, r.o, r.d, r.tmin, c_eps_tab[min(ibits(pool[k].o.w) >> 16, 8)], &t, &obj);
            if (obj != before) prim = -1;
        }
        if (kExt && s.has_medium && !(ibits(pool[k].d.w) & kFlagInside)) {
            const float tc = medium_collision(s, pool[k], r.o, r.d, obj >= 0 ? t : INFINITY, medium_key);
            if (tc >= 0.0f) { obj = kHitMedium; prim = -1; t = tc; }
        }
        hit[k] = obj >= 0 || obj == kHitMedium ? make_int4(obj, prim, ibits(t), 0) : make_int4(-1, -1, 0, 0);
        to_shade(s, k, obj);
    }
};

// Trace's closest-hit query (render.cuh:86-99) for every path of the pool,
// then (extension) free-flight sampling in the participating medium.
template <bool kExt>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_extend(SceneView s, PathBuffers B, int cur, PoolCtl* ctl,
                                                        unsigned long long* stats, uint32_t* ovf, int* err,
                                                        uint32_t medium_key)
{
    extern __shared__ uint32_t smem[];
    ExtendIO<kExt> io;
    io.medium_key = medium_key;
    io.pool = pool_of(B, cur);
    io.hit = B.hit;
    io.shade_count = ctl->shade_count;
    io.qsh = B.qsh;
    io.cap = B.capacity;
    const int n = ctl->count[cur];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&stats[0], static_cast<unsigned long long>(n));
    traverse_queue<false>(s, io, n, &ctl->fetch_ext, lane_stack(smem), thread_overflow(ovf), err, &stats[2]);
}

// ------------------------------------------------------------------ shade
// G-buffer of an RGB material at one wavelength (EvaluateMaterial, spectral).
__device__ __forceinline__ GB gb_at(const GB& rgb, const SpectralView& sv, const float4& lk, float lambda)
{
    GB g = rgb;
    const float a = interact(sv.lut_rgb, sv.res, lk, rgb.albedo);
    const float e = interact(sv.lut_rgb, sv.res, lk, rgb.emissive);
    g.albedo = mk(a, a, a);
    g.emissive = mk(e, e, e);
    g.ior = ior_abbe(lambda, rgb.ior, rgb.abbe);
    g.sigma_a = sigma_tilt(rgb.sigma_a, lambda, rgb.tilt);
    g.spectral = true;
    return g;
}

// One iteration of the CalculateRadiance loop body (render.cuh:541-908) up to
// the shadow query: Trace's material evaluation and hit offset, emission with
// MIS, light sampling for NEE, throughput and Russian roulette.  kModel is the
// shading model of every path of this launch's bucket, -1 = miss.
template <int kModel, bool kExt, int kSpec, bool kNrc, bool kGuide>
__global__ void __launch_bounds__(kShadeBlock) k_shade(SceneView s, FrameParams fp, PathBuffers B, int cur,
                                                       PoolCtl* ctl, ar_path_record* rec)
{
    const int bucket = kModel + 1;
    const int n = ctl->shade_count[bucket];
    const int32_t* q = B.qsh + static_cast<int64_t>(bucket) * B.capacity;
    const PathRec* pool = pool_of(B, cur);
    PathRec* next_pool = pool_of(B, 1 - cur);
    for (int qi = blockIdx.x * blockDim.x + threadIdx.x; qi < n; qi += gridDim.x * blockDim.x) {
        const int k = q[qi];
        const PathRec pr = pool[k];
        const int depth = ibits(pr.o.w) & 0xFFFF;
        int nonDelta = ibits(pr.o.w) >> 16;
        int flags = ibits(pr.d.w) & 0xFF;
        const int mdepth = ibits(pr.d.w) >> 8;
        const int pixel = ibits(pr.mask.w);
        const int sidx = ibits(pr.rad.w);
        const int64_t ri = static_cast<int64_t>(sidx) * fp.npix + pixel;
        const f3 crd = xyz(pr.d);
        const f3 cro = xyz(pr.o);
        f3 mask = xyz(pr.mask);
        f3 radiance = xyz(pr.rad);
        // spectral: scalar throughput and radiance broadcast to the three lanes
        // of the RGB arithmetic, the wavelength's basis and D65 weight
        float lambda = 0.0f, lpdf = 0.0f, d65 = 1.0f;
        float4 lk = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (kSpec == 1) {
            lambda = pr.mask.y;
            lpdf = pr.mask.z;
            mask = mk(pr.mask.x, pr.mask.x, pr.mask.x);
            radiance = mk(pr.rad.x, pr.rad.x, pr.rad.x);
            lk = query_lambda(fp.spec.lut_lam, lambda);
            d65 = d65_norm(fp.spec.tables, lambda);
        }
        f3 d65v = mk(d65, d65, d65);
        // four wavelengths (extension): lanes x, y, z of the RGB arithmetic carry
        // wavelengths 0-2, the *3 scalars wavelength 3; directions follow the hero (0)
        float mask3 = 0.0f, rad3 = 0.0f, d65_3 = 0.0f;
        float lam4[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        float4 lk4[4];
        if (kSpec == 4) {
            const float4 ax = aux_of(B, cur)[k];
            lambda = ax.z;
            mask3 = ax.x;
            rad3 = ax.y;
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                lam4[w] = rotate_lambda(lambda, w);
                lk4[w] = query_lambda(fp.spec.lut_lam, lam4[w]);
            }
            lk = lk4[0];
            d65v = mk(d65_norm(fp.spec.tables, lam4[0]), d65_norm(fp.spec.tables, lam4[1]), d65_norm(fp.spec.tables, lam4[2]));
            d65_3 = d65_norm(fp.spec.tables, lam4[3]);
        }
        const bool inside = (flags & kFlagInside) != 0;
        const f3 vloc = xyz(pr.vloc);
        const f3 maskIn = mask, radIn = radiance;   // path guiding: values at arrival
        const int4 hr = B.hit[k];
        constexpr bool kMed = kModel == kModelMedium;  // collisions in the participating medium
        constexpr bool hit = kModel >= 0 && !kMed;
        const float eps = c_eps_tab[min(nonDelta, 8)];
        Rng g;
        rng_from(g, pr.rng0, pr.rng1);
        if (rec && depth < AR_DEBUG_MAX_HITS) rec[ri].hit_object[depth] = hit || kMed ? hr.x : -1;
        if (rec) rec[ri].segments = depth + 1;
        // ---- intersection details (re-run of the accepted test)
        f3 pos = mk(0.0f, 0.0f, 0.0f), nrm = mk(0.0f, 0.0f, 0.0f);
        GB gb, gbr;
        int light = -1;
        if (hit) {
            const ObjInfo oi = s.objects[hr.x];
            gb = load_gb(s.materials[oi.material]);
            gbr = gb;
            if (kSpec) {  // EvaluateMaterial / SampleBSDF at the path's wavelength (material.cuh)
                const float a = interact(fp.spec.lut_rgb, fp.spec.res, lk, gb.albedo);
                const float e = interact(fp.spec.lut_rgb, fp.spec.res, lk, gb.emissive);
                gb.albedo = mk(a, a, a);
                gb.emissive = mk(e, e, e);
                gb.ior = ior_abbe(lambda, gb.ior, gb.abbe);
                gb.sigma_a = sigma_tilt(gb.sigma_a, lambda, gb.tilt);
                gb.spectral = true;
            }
            light = oi.light;
            if (oi.type == AR_OBJ_TRIANGLE) {
                const PrimRec& prim = s.prims[hr.y];
                const f3 v0 = mk(prim.v0[0], prim.v0[1], prim.v0[2]);
                const f3 e1 = mk(prim.e1[0], prim.e1[1], prim.e1[2]);
                const f3 e2 = mk(prim.e2[0], prim.e2[1], prim.e2[2]);
                const f3 h = cross(crd, e2);
                const float a = dot(e1, h);
                const float f = __frcp_rn(a);
                const f3 sv = cro - v0;
                const float u = f * dot(sv, h);
                const f3 qv = cross(sv, e1);
                const float v = f * dot(crd, qv);
                const float t = fbits(hr.z);
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
            } else if (kExt && oi.type == AR_OBJ_SDF) {
                sdf_surface_of(s, oi.aux, cro, crd, fbits(hr.z), eps, &pos, &nrm);
            } else {
                isect_sphere<true>(s.analytic[oi.aux], cro, crd, &pos, &nrm);
            }
        }
        if (kMed) pos = cro + crd * fbits(hr.z);  // no surface: the normal stays zero
        // denoiser guide buffer: the primary hit (RecordScreenGBuffer at depth 0, render.cuh:640-643)
        if (fp.dn.gbuf && depth == 0) {
            if (hit) record_gbuffer(fp.dn.gbuf + pixel, true, gb.albedo, nrm, gb.metallic, gb.roughness, fbits(hr.z), kModel);
            else record_gbuffer(fp.dn.gbuf + pixel, false, nrm, nrm, 0.0f, 0.0f, 0.0f, 0);
        }
        // ---- learned radiance cache (extension): path spread (Mueller et al. 2021,
        // a = (sum_i sqrt(|x_i-1 - x_i|^2 / (p_i |cos_i|)))^2 against
        // a0 = |x_0 - x_1|^2 / (4 pi |cos_1|)), training vertices, termination
        bool nrcQuery = false;
        float nrcS = 0.0f, nrcA = 0.0f;
        NrcVertex nv;
        if (kNrc) {
            nrcS = __uint_as_float(pr.rng1.w);
            nrcA = pr.vloc.w;
            if (hit && !inside && kModel != AR_MAT_LIGHT && kModel != AR_MAT_GLASS) {
                const float tt = fbits(hr.z);
                const float cosT = fmaxf(fabsf(dot(nrm, crd)), 1e-4f);
                if (depth == 0) {
                    nrcA = tt / sqrtf(4.0f * kPi * cosT);
                    nrcS = 0.0f;
                } else {
                    nrcS = nrcS + tt / sqrtf(fmaxf(pr.prev.w, 1e-12f) * cosT);
                }
                nv.p = make_float4(pos.x, pos.y, pos.z, fbits(pixel));
                nv.d = make_float4(-crd.x, -crd.y, -crd.z, kModel == AR_MAT_GGX ? gb.roughness : 1.0f);
                // four wavelengths: the hero wavelength rides in n.w, the features
                // keep the material's RGB albedo
                nv.n = make_float4(nrm.x, nrm.y, nrm.z, kSpec == 4 ? lambda : 0.0f);
                const f3 alb = kSpec ? gbr.albedo : gb.albedo;
                nv.a = make_float4(alb.x, alb.y, alb.z, 0.0f);
                int slot;
                if (sidx == 0 && nrc_train_slot(fp.nrc, pixel, &slot)) {   // sample 0 of a training pixel
                    const int kv = fp.nrc.slot_count[slot];
                    if (kv < fp.nrc.max_train_vertices) {
                        NrcTrainVertex tv;
                        tv.v = nv;
                        tv.t = f4(mask, kSpec == 4 ? mask3 : 0.0f);
                        tv.lb = f4(radiance, kSpec == 4 ? rad3 : 0.0f);
                        fp.nrc.train_vertices[static_cast<int64_t>(slot) * fp.nrc.max_train_vertices + kv] = tv;
                        fp.nrc.slot_count[slot] = kv + 1;
                    }
                } else if (depth >= 1 && nrcS > sqrtf(fp.nrc.spread_c) * nrcA) {
                    nrcQuery = true;
                }
            }
        }
        // ---- SampleContext (material.cuh:19-37, 177-330, 389-425)
        f3 next = mk(0.0f, 0.0f, 0.0f), emis = mk(0.0f, 0.0f, 0.0f), brdf = mk(0.0f, 0.0f, 0.0f);
        float pdf = 1.0f;
        bool terminate = false, delta = false, missThin = false;
        bool nInside = false;
        f3 nvloc = mk(0.0f, 0.0f, 0.0f);
        int nmobj = -1, nmdepth = 0;
        f3 malb = mk(0.0f, 0.0f, 0.0f);  // medium: single-scatter albedo
        float emis3 = 0.0f, brdf3 = 0.0f, malb3 = 0.0f;  // wavelength 3 (four-wavelength mode)
        bool dispersed = false;
        if (!hit && !kMed && inside) {
            missThin = true;
            nvloc = cro;
        }
        if (hit) {
            const f3 N = nrm;
            if (kModel == AR_MAT_DIFFUSE) {
                const float e0 = g.next(), e1 = g.next(), e2 = g.next();
                next = sample_cosine(e0, e1, e2, N, pdf);
                emis = gb.emissive;
                nInside = inside; nvloc = pos;
            } else if (kModel == AR_MAT_LIGHT) {
                pdf = 1.0f; emis = gb.emissive; terminate = true;
            } else if (kModel == AR_MAT_GLASS) {
                delta = true;
                const float eta = inside ? gb.ior : 1.0f / gb.ior;
                const f3 nIn = (dot(N, crd) > 0.0f) ? -N : N;
                const float cosI = -dot(nIn, crd);
                const float sin2I = fmaxf(0.0f, 1.0f - cosI * cosI);
                const float kk = 1.0f - sin2I * (eta * eta);
                if (kk <= 0.0f) {
                    if (mdepth < 1024) { next = reflect(crd, nIn); nInside = inside; }
                    else { next = crd; nInside = !inside; }
                    pdf = 1.0f; nvloc = pos;
                } else {
                    const float cosT = sqrtf(kk);
                    const float Fr = fresnel_exact(cosI, cosT, eta);
                    if (g.next() < Fr) { next = reflect(crd, nIn); pdf = Fr; nInside = inside; }
                    else { next = refract(crd, nIn, eta); pdf = 1.0f - Fr; nInside = !inside; }
                    nvloc = pos;
                }
            } else if (kModel == AR_MAT_GGX) {
                emis = gb.emissive;
                const f3 V = -crd;
                const float NoV = fmaxf(0.0f, dot(N, V));
                if (NoV <= 0.0f) {
                    terminate = true;
                } else {
                    float alpha, kD;
                    f3 F0;
                    ggx_params(gb, alpha, kD, F0);
                    const float pSpec = ggx_pspec(gb, F0);
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
            brdf = eval_bsdf_cos(kModel, crd, next, N, pos, gb, inside, vloc);
            if (kSpec == 4) {
                if (kModel != AR_MAT_GLASS) {
                    emis = mk(interact(fp.spec.lut_rgb, fp.spec.res, lk4[0], gbr.emissive),
                              interact(fp.spec.lut_rgb, fp.spec.res, lk4[1], gbr.emissive),
                              interact(fp.spec.lut_rgb, fp.spec.res, lk4[2], gbr.emissive));
                    emis3 = interact(fp.spec.lut_rgb, fp.spec.res, lk4[3], gbr.emissive);
                }
                if (kModel == AR_MAT_GLASS && gbr.abbe > 0.0f && !(flags & kFlagHeroOnly)) {
                    // dispersive glass: the other wavelengths cannot follow the hero's
                    // direction; the path continues with the hero alone (its weight
                    // becomes that of a single-wavelength sample)
                    dispersed = true;
                } else if (kModel != AR_MAT_LIGHT && !(flags & kFlagHeroOnly)) {
                    const float b1 = eval_bsdf_cos(kModel, crd, next, N, pos, gb_at(gbr, fp.spec, lk4[1], lam4[1]), inside, vloc).x;
                    const float b2 = eval_bsdf_cos(kModel, crd, next, N, pos, gb_at(gbr, fp.spec, lk4[2], lam4[2]), inside, vloc).x;
                    brdf3 = eval_bsdf_cos(kModel, crd, next, N, pos, gb_at(gbr, fp.spec, lk4[3], lam4[3]), inside, vloc).x;
                    brdf = mk(brdf.x, b1, b2);
                }
            }
        } else if (kMed) {
            // Henyey-Greenstein scattering; phase / pdf = 1, throughput weight = albedo
            const float u1 = g.next(), u2 = g.next();
            next = hg_sample(crd, s.medium.g, u1, u2);
            pdf = hg_phase(s.medium.g, dot(crd, next));
            malb = mk(s.medium.albedo[0], s.medium.albedo[1], s.medium.albedo[2]);
            if (kSpec == 4) {
                const f3 rgb = malb;
                malb = mk(interact(fp.spec.lut_rgb, fp.spec.res, lk4[0], rgb), interact(fp.spec.lut_rgb, fp.spec.res, lk4[1], rgb),
                          interact(fp.spec.lut_rgb, fp.spec.res, lk4[2], rgb));
                malb3 = interact(fp.spec.lut_rgb, fp.spec.res, lk4[3], rgb);
                brdf3 = malb3 * pdf;
            } else if (kSpec) {
                const float a = interact(fp.spec.lut_rgb, fp.spec.res, lk, malb);
                malb = mk(a, a, a);
            }
            brdf = malb * pdf;
            nInside = false;
            nvloc = pos;
            nmobj = static_cast<int>(pr.rng1.z);
            nmdepth = mdepth;
        } else {
            brdf = mk(1.0f, 1.0f, 1.0f);
            next = crd;
            pdf = 1.0f;
            emis = sky_lighting(crd, fp.sky);
            if (kSpec == 4) {
                const f3 rgb = emis;
                emis = mk(interact(fp.spec.lut_rgb, fp.spec.res, lk4[0], rgb), interact(fp.spec.lut_rgb, fp.spec.res, lk4[1], rgb),
                          interact(fp.spec.lut_rgb, fp.spec.res, lk4[2], rgb));
                emis3 = interact(fp.spec.lut_rgb, fp.spec.res, lk4[3], rgb);
                brdf3 = 1.0f;
            } else if (kSpec) {
                const float e = interact(fp.spec.lut_rgb, fp.spec.res, lk, emis);
                emis = mk(e, e, e);
            }
            nInside = false;
        }
        // ---- path guiding (render.cuh:555-640): mix the probe's hemisphere
        // density into the BSDF's, or sample the probe with probability alpha
        int gProbe = -1;
        bool guidable = false;
        f3 gq = mk(0.0f, 0.0f, 0.0f);
        uint64_t gKey = 0;
        if (kGuide && hit && (kModel == AR_MAT_DIFFUSE || kModel == AR_MAT_GGX) && !inside && !terminate) {
            guidable = true;
            gKey = pg_key(pos, reflect(crd, nrm), fp.guide.faces);
            gProbe = pg_lookup(fp.guide, gKey);
            if (gProbe >= 0) {
                const f3 mq = vmaxs(mask, 1.0e-6f);
                gq = mq / (mq.x + mq.y + mq.z + 1.0e-6f);
                const float4* P = fp.guide.probes + static_cast<int64_t>(gProbe) * kPgStride;
                const float pP = pg_hemi_pdf(P, next, nrm, gq);
                const float a = fp.guide.alpha;
                if (pdf > 1.0e-12f && pP > 1.0e-12f) {
                    if (g.next() < a) {
                        float u[5];
#pragma unroll
                        for (int t = 0; t < 5; ++t) u[t] = g.next();
                        float pg;
                        const f3 w = pg_sample_hemi(P, nrm, gq, u, &pg);
                        if (dot(w, nrm) > 1.0e-12f) {
                            const float pBs = bsdf_pdf(kModel, gb, nrm, crd, w);
                            next = w;
                            brdf = eval_bsdf_cos(kModel, crd, w, nrm, pos, gb, inside, vloc);
                            pdf = (1.0f - a) * fmaxf(pBs, 1.0e-12f) + a * pg;
                        } else {
                            gProbe = -1;
                        }
                    } else {
                        pdf = (1.0f - a) * pdf + a * pP;
                    }
                } else {
                    gProbe = -1;
                }
            }
        }
        if (!kMed) {   // hit offset, always one uniform (render.cuh:156-160)
            const float offEps = eps * fmaxf(1.0f, length(pos));
            const float sg = signf(dot(nrm, next));
            const float r = g.next();
            pos = pos + ((nrm * sg) * offEps) * (r + 0.5f);
        }
        const bool mInside = nInside;  // media state after this segment
        // ---- emission (render.cuh:648-723)
        if (!hit && !kMed) {
            if (!missThin) {
                radiance = radiance + (mask * emis) * d65v;
                if (kSpec == 4) rad3 = rad3 + (mask3 * emis3) * d65_3;
            }
        } else if (hit && light >= 0 && !nrcQuery) {
            float misW = 1.0f;
            if (fp.use_nee && depth > 0 && (flags & kFlagPrevNEE)) {
                const float pB = fmaxf(pr.prev.w, 0.0f);
                const float pL = pdf_light_from_hit(s, hr.x, xyz(pr.prev), pos, nrm, fp.tri_light_nee != 0);
                if (pL >= 0.0f && pB > 0.0f) misW = power_heuristic(pB, pL);
            }
            radiance = radiance + ((mask * emis) * d65v) * misW;
            if (kSpec == 4) rad3 = rad3 + ((mask3 * emis3) * d65_3) * misW;
        }
        const bool brk = (!hit && !kMed && !missThin) || terminate || nrcQuery;
        bool cont = false, shadow = false, cosOK = false;
        f3 pending = mk(0.0f, 0.0f, 0.0f), lightP = mk(0.0f, 0.0f, 0.0f);
        float pend3 = 0.0f;
        float4 prevOut = pr.prev;
        if (!brk) {
            // ---- NEE (render.cuh:766-827)
            if (!missThin) {
                const float lum = kSpec == 4 ? 0.25f * (mask.x + mask.y + mask.z + mask3)
                                             : (kSpec ? mask.x : luminance(mask));
                const float rate = sqrtf(saturate(lum));
                if (fp.use_nee && nonDelta < 10 && !delta && !mInside && g.next() < rate) {
                    LightSample ls = sample_light(s, pos, g, fp.tri_light_nee != 0);
                    const f3 lsRgb = ls.emis;
                    if (kSpec) {
                        const float e = interact(fp.spec.lut_rgb, fp.spec.res, lk, ls.emis);
                        ls.emis = mk(e, e, e);
                    }
                    if (ls.valid) {
                        const float pATotal = fmaxf(1e-20f, ls.pA * ls.pFacet);
                        const f3 lu = ls.p - pos;
                        const float d2 = fmaxf(dot(lu, lu), 1.0e-12f);
                        const f3 ld = lu * rsqrt_ieee(d2);
                        const float cosX = kMed ? 1.0f : fmaxf(0.0f, dot(nrm, ld));
                        const float cosY = fmaxf(0.0f, dot(ls.n, -ld));
                        if (cosX > 0.0f && cosY > 0.0f) {
                            cosOK = true;
                            const f3 fcos = kMed ? malb * hg_phase(s.medium.g, dot(crd, ld))
                                                 : eval_bsdf_cos(kModel, crd, ld, nrm, pos, gb, false, mk(0.0f, 0.0f, 0.0f));
                            const float G = cosY / d2;
                            const f3 contrib = (fcos * ls.emis) * (G / pATotal);
                            const float pL = area_to_solid_angle(pos, ls.p, ls.n, ls.pFacet * ls.pA);
                            float pB = kMed ? hg_phase(s.medium.g, dot(crd, ld))
                                            : fmaxf(bsdf_pdf(kModel, gb, nrm, crd, ld), 0.0f);
                            if (kGuide && gProbe >= 0) {
                                const float a = fp.guide.alpha;
                                pB = (1.0f - a) * pB +
                                     a * pg_hemi_pdf(fp.guide.probes + static_cast<int64_t>(gProbe) * kPgStride, ld, nrm, gq);
                            }
                            const float wmis = power_heuristic(pL, pB);
                            pending = (mask * (contrib * wmis)) * d65v;
                            if (kSpec == 4) {
                                const float G4 = G / pATotal;
                                float f1, f2, f3v;
                                if (kMed) {
                                    const float ph = hg_phase(s.medium.g, dot(crd, ld));
                                    f1 = malb.y * ph; f2 = malb.z * ph; f3v = malb3 * ph;
                                } else {
                                    const f3 z0 = mk(0.0f, 0.0f, 0.0f);
                                    f1 = eval_bsdf_cos(kModel, crd, ld, nrm, pos, gb_at(gbr, fp.spec, lk4[1], lam4[1]), false, z0).x;
                                    f2 = eval_bsdf_cos(kModel, crd, ld, nrm, pos, gb_at(gbr, fp.spec, lk4[2], lam4[2]), false, z0).x;
                                    f3v = eval_bsdf_cos(kModel, crd, ld, nrm, pos, gb_at(gbr, fp.spec, lk4[3], lam4[3]), false, z0).x;
                                }
                                const f3 c3 = mk(contrib.x,
                                                 (f1 * interact(fp.spec.lut_rgb, fp.spec.res, lk4[1], lsRgb)) * G4,
                                                 (f2 * interact(fp.spec.lut_rgb, fp.spec.res, lk4[2], lsRgb)) * G4);
                                pending = (mask * (c3 * wmis)) * d65v;
                                pend3 = (mask3 * (((f3v * interact(fp.spec.lut_rgb, fp.spec.res, lk4[3], lsRgb)) * G4) * wmis)) * d65_3;
                            }
                        }
                        shadow = true;
                        lightP = ls.p;
                        if (rec) {
                            rec[ri].nee_rays += 1;
                            if (depth < 32) rec[ri].nee_depth_mask |= static_cast<int32_t>(1u << depth);
                        }
                    }
                }
                // previousDidNEE_ is decided by the shadow query when one is cast
                flags &= ~kFlagPrevNEE;
                prevOut = f4(pos, (kNrc && delta) ? INFINITY : pdf);
            }
            // ---- throughput and Russian roulette (render.cuh:829-907)
            const f3 contrib = mk(brdf.x / fmaxf(pdf, 1e-12f), brdf.y / fmaxf(pdf, 1e-12f), brdf.z / fmaxf(pdf, 1e-12f));
            float qrr = 1.0f;
            bool survived = true;
            if (nonDelta >= fp.rr_depth) {
                const float lum = kSpec == 4 ? 0.25f * (mask.x + mask.y + mask.z + mask3)
                                             : (kSpec ? mask.x : luminance(mask));
                const float mx = kSpec == 4 ? fmaxf(max3(mask), mask3) : (kSpec ? mask.x : max3(mask));
                const float basic = clampf(lum * 0.5f + mx * 0.5f, 0.05f, 0.95f);
                qrr = lerpf(basic, 1.0f, mInside ? 0.99f : 0.0f);
                if (g.next() > qrr) survived = false;
            }
            if (survived) {
                mask = mask * contrib;
                mask = mask / qrr;
                if (kSpec == 4) {
                    mask3 = (mask3 * (brdf3 / fmaxf(pdf, 1e-12f))) / qrr;
                    if (dispersed) {   // hero alone from here: weight sum_j p(lambda_j) / p(lambda_0)
                        const float ps = pdf_cie1931(lam4[0]) + pdf_cie1931(lam4[1]) + pdf_cie1931(lam4[2]) + pdf_cie1931(lam4[3]);
                        mask = mk(mask.x * (ps / pdf_cie1931(lam4[0])), 0.0f, 0.0f);
                        mask3 = 0.0f;
                        flags |= kFlagHeroOnly;
                    }
                }
                if (!delta) nonDelta++;
                cont = depth + 1 < fp.max_depth;
            }
        }
        flags = (flags & ~kFlagInside) | (mInside ? kFlagInside : 0);
        if (kGuide) {   // this event of the pixel's path, for the probes' samples at retirement
            const int ne = fp.guide.event_count[pixel];
            if (ne < kPgEvents) {
                float4* ev = fp.guide.events + (static_cast<int64_t>(pixel) * kPgEvents + ne) * 3;
                ev[0] = make_float4(__uint_as_float(static_cast<uint32_t>(gKey)), __uint_as_float(static_cast<uint32_t>(gKey >> 32)),
                                    (guidable && cont) ? 1.0f : 0.0f, 0.0f);
                ev[1] = f4(next, 0.0f);
                ev[2] = f4(maskIn, 0.0f);
                fp.guide.event_lb[static_cast<int64_t>(pixel) * kPgEvents + ne] = f4(radIn, 0.0f);
                fp.guide.event_count[pixel] = ne + 1;
            }
        }
        const uint32_t used = pr.rng1.w + static_cast<uint32_t>(g.used);
        int target;
        const int j = warp_alloc(&ctl->count[1 - cur], cont);
        const int r = warp_alloc(&ctl->retire_count, !cont);
        if (kNrc) {   // the path ends here; the cache supplies the rest
            const int qi = warp_alloc(fp.nrc.query_count, nrcQuery);
            if (nrcQuery && qi < fp.nrc.query_cap) {
                NrcQuery qq;
                qq.v = nv;
                qq.t = f4(mask, kSpec == 4 ? mask3 : 0.0f);
                fp.nrc.queries[qi] = qq;
            }
        }
        if (cont) {
            PathRec out;
            out.o = f4(pos, fbits((depth + 1) | (nonDelta << 16)));
            out.d = f4(next, fbits(flags | (nmdepth << 8)));
            out.mask = kSpec == 1 ? make_float4(mask.x, lambda, lpdf, fbits(pixel)) : f4(mask, fbits(pixel));
            out.rad = kSpec == 1 ? make_float4(radiance.x, 0.0f, 0.0f, fbits(sidx)) : f4(radiance, fbits(sidx));
            if (kSpec == 4) aux_of(B, 1 - cur)[j] = make_float4(mask3, rad3, lambda, 0.0f);
            out.rng0 = make_uint4(g.st.d, g.st.v[0], g.st.v[1], g.st.v[2]);
            out.rng1 = make_uint4(g.st.v[3], g.st.v[4], static_cast<uint32_t>(nmobj), kNrc ? __float_as_uint(nrcS) : used);
            out.prev = prevOut;
            out.vloc = f4(nvloc, kNrc ? nrcA : 0.0f);
            next_pool[j] = out;
            target = j;
        } else {
            RetireRec out;
            out.rad = f4(radiance, fbits(pixel));
            out.meta = make_int4(sidx, static_cast<int>(used), ibits(lambda), ibits(kSpec == 4 ? rad3 : lpdf));
            B.retire[r] = out;
            target = ~r;
        }
        const int m = warp_alloc(&ctl->shadow_count, shadow);
        if (shadow) {
            ShadowRec sr;
            sr.src = f4(pos, c_eps_tab[min(depth, 8)]);
            sr.dst = f4(lightP, fbits(target));
            const uint32_t mseed = kExt && s.has_medium
                ? medium_seed(fp.medium_key, static_cast<uint32_t>(sidx), static_cast<uint32_t>(pixel), static_cast<uint32_t>(depth), 1u) & ~1u
                : 0u;
            sr.nee = f4(pending, fbits(static_cast<int>(mseed | (cosOK ? 1u : 0u))));
            if (kSpec == 4) B.shadow3[m] = pend3;
            B.shadow[m] = sr;
        }
    }
}

// ------------------------------------------------------------------ shadow
// Transmittance of the medium along an unoccluded shadow segment (out of line).
__device__ __noinline__ float shadow_transmittance(const SceneView& s, f3 o, f3 d, float tmax, uint32_t seed)
{
    HashRng h;
    h.seed = seed;
    h.n = 0;
    return ratio_track(s.medium, o, d, tmax, h);
}

// SegmentTrace -> AnyHitSegmentBVH (render.cuh:167-183, intersection.cuh:372-397)
// and the remainder of NEE (render.cuh:242-343): the pending term is added when
// the segment is unoccluded, and previousDidNEE_ becomes "occluded or cos > 0".
template <bool kExt>
struct ShadowIO {
    const ShadowRec* rec;
    PathRec* next_pool;
    RetireRec* retire;
    float4* next_aux;         // four-wavelength mode: side records of the next pool
    const float* pend3;       // four-wavelength mode: pending radiance of wavelength 3
    int spec4;
    unsigned long long traced;
    __device__ __forceinline__ void finish(int m, bool occ, float tr = 1.0f)
    {
        const float4 dst = rec[m].dst;
        float4 nee = rec[m].nee;
        const int target = ibits(dst.w);
        const bool cosOK = (ibits(nee.w) & 1) != 0;
        const bool add = !occ && cosOK;
        if (kExt) { nee.x *= tr; nee.y *= tr; nee.z *= tr; }  // medium transmittance
        if (target >= 0) {
            PathRec& p = next_pool[target];
            if (add) {
                const float4 r = p.rad;
                p.rad = make_float4(r.x + nee.x, r.y + nee.y, r.z + nee.z, r.w);
                if (spec4) next_aux[target].y += pend3[m] * (kExt ? tr : 1.0f);
            }
            if (occ || cosOK) {
                const float4 d = p.d;
                p.d = make_float4(d.x, d.y, d.z, fbits(ibits(d.w) | kFlagPrevNEE));
            }
        } else if (add) {
            RetireRec& p = retire[~target];
            const float4 r = p.rad;
            p.rad = make_float4(r.x + nee.x, r.y + nee.y, r.z + nee.z, r.w);
            if (spec4) p.meta.w = __float_as_int(__int_as_float(p.meta.w) + pend3[m] * (kExt ? tr : 1.0f));
        }
    }
    __device__ __forceinline__ int load(const SceneView&, int m, RayState& r)
    {
        const float4 a = rec[m].src, b = rec[m].dst;
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
                return m;
            }
        }
        finish(m, false);
        return -1;
    }
    __device__ __forceinline__ void store(const SceneView& s, int m, const RayState& r)
    {
        bool occ = r.best.obj >= 0;
        if (kExt && !occ && s.num_sdf > 0) occ = sdf_any(s, r.o, r.d, 0.0f, r.best.t, rec[m].src.w) >= 0;
        float tr = 1.0f;
        if (kExt && !occ && s.has_medium) tr = shadow_transmittance(s, r.o, r.d, r.best.t, static_cast<uint32_t>(ibits(rec[m].nee.w)) & ~1u);
        finish(m, occ, tr);
    }
};

template <bool kExt>
__global__ void __launch_bounds__(kTraceBlock, kTraceMinBlocks) k_shadow(SceneView s, PathBuffers B, int cur, PoolCtl* ctl,
                                                        unsigned long long* stats, uint32_t* ovf, int* err, int spec4)
{
    extern __shared__ uint32_t smem[];
    const int n = ctl->shadow_count;
    ShadowIO<kExt> io;
    io.rec = B.shadow;
    io.next_pool = pool_of(B, 1 - cur);
    io.retire = B.retire;
    io.next_aux = aux_of(B, 1 - cur);
    io.pend3 = B.shadow3;
    io.spec4 = spec4;
    io.traced = 0;
    traverse_queue<true>(s, io, n, &ctl->fetch_shadow, lane_stack(smem), thread_overflow(ovf), err, &stats[4]);
    unsigned long long c = io.traced;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane_id() == 0 && c) atomicAdd(&stats[1], c);
}

// ------------------------------------------------------------------ retire
// checkNanInf + clamp (render.cuh:969), max(0, .) (scene.cu:238), FP64 sum.
__device__ __forceinline__ float fix_nan_inf(float x)
{
    if (isnan_(x)) return 0.0f;
    if (isinf_(x)) return x > 0.0f ? 0.0f : -0.0f;
    return x;
}

__global__ void k_retire(FrameParams fp, PathBuffers B, PoolCtl* ctl, double* accum, ar_path_record* rec)
{
    const int n = ctl->retire_count;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->retired += n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const RetireRec rr = B.retire[i];
        f3 v = xyz(rr.rad);
        if (fp.spectral == 4) {
            // four wavelengths: sum_i XYZ(lambda_i) L_i / sum_j p(lambda_j), the
            // one-sample estimator of the rotation set (balance heuristic over
            // which member was the hero)
            const float h = fbits(rr.meta.z);
            const float L[4] = {fix_nan_inf(rr.rad.x), fix_nan_inf(rr.rad.y), fix_nan_inf(rr.rad.z), fix_nan_inf(fbits(rr.meta.w))};
            float ps = 0.0f;
            f3 acc = mk(0.0f, 0.0f, 0.0f);
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const float lw = rotate_lambda(h, w);
                ps += pdf_cie1931(lw);
                acc = acc + cmf_xyz(fp.spec.tables, lw) * L[w];
            }
            v = acc / ps;
        } else if (fp.spectral) {  // lambdaXYZ * radiance / pdf (render.cuh:966), linear CIE XYZ
            const float lam = fbits(rr.meta.z), lpdf = fbits(rr.meta.w);
            const float r = fix_nan_inf(rr.rad.x);
            const f3 c = cmf_xyz(fp.spec.tables, lam);
            v = mk((c.x * r) / lpdf, (c.y * r) / lpdf, (c.z * r) / lpdf);
        } else {
            v = mk(fix_nan_inf(v.x), fix_nan_inf(v.y), fix_nan_inf(v.z));
        }
        const float x = fmaxf(clampf(v.x, 0.0f, 1.0e3f), 0.0f);
        const float y = fmaxf(clampf(v.y, 0.0f, 1.0e3f), 0.0f);
        const float z = fmaxf(clampf(v.z, 0.0f, 1.0e3f), 0.0f);
        const int pixel = ibits(rr.rad.w);
        // denoiser moments of the clamped sample (RecordScreenStatisticBuffer, render.cuh:988-991)
        if (fp.dn.stat) record_stats(fp.dn.stat + pixel, mk(x, y, z));
        int slot;
        if (fp.nrc.enabled && rr.meta.x == 0 && nrc_train_slot(fp.nrc, pixel, &slot)) {
            // training targets: radiance gathered after each recorded vertex,
            // divided by the throughput that reached it
            const int nvtx = fp.nrc.slot_count[slot];
            const f3 L = mk(fix_nan_inf(rr.rad.x), fix_nan_inf(rr.rad.y), fix_nan_inf(rr.rad.z));
            if (fp.nrc.spectral == 4) {
                // four wavelengths: a target per wavelength, negative (left out of the
                // loss) where no throughput reached the vertex (hero-only after dispersion),
                const float L3 = fix_nan_inf(fbits(rr.meta.w));
                for (int k = 0; k < nvtx; ++k) {
                    const NrcTrainVertex tv = fp.nrc.train_vertices[static_cast<int64_t>(slot) * fp.nrc.max_train_vertices + k];
                    if (!nrc_vertex_finite(tv.v)) continue;   // a non-finite input would poison the whole step
                    const float Lw[4] = {L.x, L.y, L.z, L3};
                    const float T[4] = {tv.t.x, tv.t.y, tv.t.z, tv.t.w};
                    const float B4[4] = {tv.lb.x, tv.lb.y, tv.lb.z, tv.lb.w};
                    // relative to the D65 weight of the wavelength (the cache's output scale)
                    float tg[4];
#pragma unroll
                    for (int w = 0; w < 4; ++w)
                        tg[w] = T[w] > 1e-6f ? fminf(fmaxf(((Lw[w] - B4[w]) / T[w]) /
                                                               d65_norm(fp.spec.tables, rotate_lambda(tv.v.n.w, w)),
                                                           0.0f),
                                                     1.0e3f)
                                             : -1.0f;
                    const int si = atomicAdd(fp.nrc.sample_count, 1);
                    if (si < fp.nrc.sample_cap) {
                        NrcSample sm;
                        sm.v = tv.v;
                        sm.v.p.w = tg[0];
                        sm.v.n.w = tg[1];
                        sm.v.a.w = tg[2];
                        sm.x = make_float4(tg[3], tv.v.n.w, 0.0f, 0.0f);
                        fp.nrc.samples[si] = sm;
                    }
                }
            }
            for (int k = 0; k < (fp.nrc.spectral == 4 ? 0 : nvtx); ++k) {
                const NrcTrainVertex tv = fp.nrc.train_vertices[static_cast<int64_t>(slot) * fp.nrc.max_train_vertices + k];
                if (!nrc_vertex_finite(tv.v)) continue;
                const f3 tgt = mk(tv.t.x > 1e-6f ? (L.x - tv.lb.x) / tv.t.x : 0.0f,
                                  tv.t.y > 1e-6f ? (L.y - tv.lb.y) / tv.t.y : 0.0f,
                                  tv.t.z > 1e-6f ? (L.z - tv.lb.z) / tv.t.z : 0.0f);
                const int si = atomicAdd(fp.nrc.sample_count, 1);
                if (si < fp.nrc.sample_cap) {
                    NrcSample sm;
                    sm.v = tv.v;
                    sm.v.p.w = fminf(fmaxf(tgt.x, 0.0f), 1.0e3f);
                    sm.v.n.w = fminf(fmaxf(tgt.y, 0.0f), 1.0e3f);
                    sm.v.a.w = fminf(fmaxf(tgt.z, 0.0f), 1.0e3f);
                    sm.x = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    fp.nrc.samples[si] = sm;
                }
            }
        }
        if (fp.guiding) {
            // incident radiance along each guidable vertex's sampled direction:
            // radiance gathered from the next event on over the throughput that reached it
            const int ne = fp.guide.event_count[pixel];
            const f3 L = mk(fix_nan_inf(rr.rad.x), fix_nan_inf(rr.rad.y), fix_nan_inf(rr.rad.z));
            for (int e = 0; e + 1 < ne; ++e) {
                const float4* ev = fp.guide.events + (static_cast<int64_t>(pixel) * kPgEvents + e) * 3;
                const float4 h = ev[0];
                if (h.z == 0.0f) continue;
                const float4 tn = fp.guide.events[(static_cast<int64_t>(pixel) * kPgEvents + e + 1) * 3 + 2];
                const float4 lb = fp.guide.event_lb[static_cast<int64_t>(pixel) * kPgEvents + e + 1];
                const f3 inc = mk(tn.x > 1e-8f ? fmaxf((L.x - lb.x) / tn.x, 0.0f) : 0.0f,
                                  tn.y > 1e-8f ? fmaxf((L.y - lb.y) / tn.y, 0.0f) : 0.0f,
                                  tn.z > 1e-8f ? fmaxf((L.z - lb.z) / tn.z, 0.0f) : 0.0f);
                const float strength = fminf(luminance(inc), kPgMaxBrightness);
                if (!(strength >= kPgMinBrightness)) continue;
                const int si = atomicAdd(&fp.guide.counters[2], 1);
                if (si < fp.guide.sample_cap) {
                    float4* o = fp.guide.samples + 3 * static_cast<int64_t>(si);
                    o[0] = make_float4(h.x, h.y, 0.0f, 0.0f);
                    o[1] = ev[1];
                    o[2] = f4(inc, 0.0f);
                }
            }
            fp.guide.event_count[pixel] = 0;
        }
        double* a = accum + 3 * static_cast<int64_t>(pixel);
        atomicAdd(a + 0, static_cast<double>(x));
        atomicAdd(a + 1, static_cast<double>(y));
        atomicAdd(a + 2, static_cast<double>(z));
        if (rec) {
            const int64_t ri = static_cast<int64_t>(rr.meta.x) * fp.npix + pixel;
            rec[ri].radiance[0] = x; rec[ri].radiance[1] = y; rec[ri].radiance[2] = z;
            rec[ri].uniforms = rr.meta.y;
        }
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
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_extend<false>, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_shadow<false>, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_trace_rays<false, false>, kTraceBlock, kTraceSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b3, k_trace_rays<true, false>, kTraceBlock, kTraceSmem);
        cudaGetLastError();
        blocks = max(1, max(max(b0, b1), max(b2, b3)));
    }
    return blocks * sm_count;
}

cudaError_t launch_trace_rays(const SceneView& s, const float4* rays, int n, int any, int32_t* obj, float* t,
                              PoolCtl* ctl, uint32_t* ovf, int* err, int grid, cudaStream_t st)
{
    if (s.num_sdf > 0) {
        RaysIO<true> io;
        io.rays = rays;
        io.out_obj = obj;
        io.out_t = t;
        io.any = any ? 1 : 0;
        if (any) k_trace_rays<true, true><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
        else k_trace_rays<false, true><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
    } else {
        RaysIO<false> io;
        io.rays = rays;
        io.out_obj = obj;
        io.out_t = t;
        io.any = any ? 1 : 0;
        if (any) k_trace_rays<true, false><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
        else k_trace_rays<false, false><<<grid, kTraceBlock, kTraceSmem, st>>>(s, io, n, ctl, ovf, err);
    }
    return cudaGetLastError();
}

cudaError_t launch_rng_init(const FrameParams& fp, uint4* b0, uint2* b1, const uint32_t* jump67, cudaStream_t st)
{
    const int nblk = fp.grid_x * ((fp.height + 3) / 4);
    k_rng_init<<<(nblk + 127) / 128, 128, 0, st>>>(fp, b0, b1, jump67);
    return cudaGetLastError();
}

cudaError_t launch_rng_tape(const FrameParams& fp, int spp, int per_path, float* out, cudaStream_t st)
{
    k_rng_tape<<<(fp.npix + 127) / 128, 128, 0, st>>>(fp, spp, per_path, out);
    return cudaGetLastError();
}

cudaError_t launch_pool_init(PoolCtl* ctl, int64_t total, cudaStream_t st)
{
    k_pool_init<<<1, 1, 0, st>>>(ctl, total);
    return cudaGetLastError();
}

// The five per-material shading launches of one iteration.
template <bool kExt, int kSpec, bool kNrc, bool kGuide = false>
void launch_shade(const SceneView& s, const FrameParams& fp, const PathBuffers& B, int c, PoolCtl* ctl,
                  ar_path_record* rec, int grid, cudaStream_t st)
{
    k_shade<-1, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
    k_shade<AR_MAT_DIFFUSE, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
    k_shade<AR_MAT_LIGHT, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
    k_shade<AR_MAT_GLASS, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
    k_shade<AR_MAT_GGX, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
    if (kExt && s.has_medium)
        k_shade<kModelMedium, kExt, kSpec, kNrc, kGuide><<<grid, kShadeBlock, 0, st>>>(s, fp, B, c, ctl, rec);
}

cudaError_t launch_iterations(const SceneView& s, const FrameParams& fp, const PathBuffers& B, PoolCtl* ctl,
                              uint4* b0, uint2* b1, const uint32_t* jump_table, unsigned long long* stats,
                              uint32_t* ovf, int* err, double* accum, ar_path_record* rec, int iterations, int* cur,
                              int grid_trace, int grid_other, cudaStream_t st, int64_t* launches, LaunchTimers* tm)
{
    const bool ext = s.num_sdf > 0 || s.has_medium;
    for (int it = 0; it < iterations; ++it) {
        const int c = *cur;
        k_plan<<<1, 1, 0, st>>>(ctl, c, fp.npix, B.capacity);
        k_regen<<<grid_other, kShadeBlock, 0, st>>>(fp, B, ctl, c, b0, b1, jump_table, rec);
        const bool te = tm && tm->n_extend < tm->cap;
        if (te) cudaEventRecord(tm->extend_ev[2 * tm->n_extend], st);
        if (ext) k_extend<true><<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, B, c, ctl, stats, ovf, err, fp.medium_key);
        else k_extend<false><<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, B, c, ctl, stats, ovf, err, fp.medium_key);
        if (te) cudaEventRecord(tm->extend_ev[2 * tm->n_extend++ + 1], st);
        if (fp.spectral == 4 && fp.nrc.enabled) {
            if (ext) launch_shade<true, 4, true>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 4, true>(s, fp, B, c, ctl, rec, grid_other, st);
        } else if (fp.spectral == 4) {
            if (ext) launch_shade<true, 4, false>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 4, false>(s, fp, B, c, ctl, rec, grid_other, st);
        } else if (fp.spectral) {
            if (ext) launch_shade<true, 1, false>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 1, false>(s, fp, B, c, ctl, rec, grid_other, st);
        } else if (fp.guiding) {
            if (ext) launch_shade<true, 0, false, true>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 0, false, true>(s, fp, B, c, ctl, rec, grid_other, st);
        } else if (fp.nrc.enabled) {
            if (ext) launch_shade<true, 0, true>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 0, true>(s, fp, B, c, ctl, rec, grid_other, st);
        } else {
            if (ext) launch_shade<true, 0, false>(s, fp, B, c, ctl, rec, grid_other, st);
            else launch_shade<false, 0, false>(s, fp, B, c, ctl, rec, grid_other, st);
        }
        const bool ts = tm && tm->n_shadow < tm->cap;
        if (ts) cudaEventRecord(tm->shadow_ev[2 * tm->n_shadow], st);
        const int spec4 = fp.spectral == 4 ? 1 : 0;
        if (ext) k_shadow<true><<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, B, c, ctl, stats, ovf, err, spec4);
        else k_shadow<false><<<grid_trace, kTraceBlock, kTraceSmem, st>>>(s, B, c, ctl, stats, ovf, err, spec4);
        if (ts) cudaEventRecord(tm->shadow_ev[2 * tm->n_shadow++ + 1], st);
        k_retire<<<grid_other, kShadeBlock, 0, st>>>(fp, B, ctl, accum, rec);
        *launches += s.has_medium ? 11 : 10;
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
