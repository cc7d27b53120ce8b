// nrc_tc.cu -- radiance-cache inference on the 5th-generation tensor cores:
// tcgen05.mma (M = 128 rows per tile, kind::f16 with bf16 operands, fp32
// accumulators in tensor memory), one elected thread issuing the MMAs of a
// layer, completion through tcgen05.commit on an mbarrier, and the epilogue
// of each layer (ReLU, bf16 pack, or exp at the output) from tcgen05.ld:
// thread t of a 128-thread tile group owns row t of the tile, so it reads its
// 64 accumulator columns from TMEM lane t and writes the next layer's A
// operand row back to shared memory.  Inference runs two tiles per CTA.
//
// Operands live in shared memory in the canonical K-major layout of
// tcgen05.cuh.
//
// Every wait is bounded: a CTA whose MMA does not complete within the limit
// sets the error word, skips the rest of its work, and still frees its
// tensor memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "nrc.cuh"
#include "tcgen05.cuh"

namespace ar {

namespace {

constexpr int kTcRows = 128;                       // rows per CTA tile (M)
constexpr int kTcThreads = 128;
constexpr int kTcCols = 64;                        // TMEM columns allocated (fp32 accumulators)
constexpr int kTcWBytes = 5 * kNrcHid * kNrcIn * 2 + kNrcOut * kNrcIn * 2;   // 43008
constexpr int kTcABytes = kTcRows * kNrcIn * 2;                               // 16384
constexpr int kTcSmem = kTcWBytes + kTcABytes + 64;
constexpr int kTcInferSmem = kTcWBytes + 2 * kTcABytes + 64;                  // two tiles per CTA
constexpr uint32_t kTcSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t pack2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// the network input of one vertex as 32 bf16 pairs (layout of encode_row in nrc.cu)
__device__ void tc_encode(const NrcNet& net, const NrcVertex& v, bool valid, uint32_t* r32)
{
    if (!valid) {
#pragma unroll
        for (int k = 0; k < 32; ++k) r32[k] = 0u;
        return;
    }
    float u[3];
    nrc_unit_pos(net.grid, v.p, u);
#pragma unroll 1
    for (int l = 0; l < kNrcMaxLevels; ++l) {
        float f0 = 0.0f, f1 = 0.0f;
        if (l < net.grid.levels) {
            uint32_t idx[8];
            float w[8];
            nrc_level_corners(net.grid, l, u[0], u[1], u[2], idx, w);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const float2 h = __half22float2(__ldg(net.table + idx[c]));
                f0 += w[c] * h.x;
                f1 += w[c] * h.y;
            }
        }
        r32[l] = pack2(f0, f1);
    }
    float sh[16];
    nrc_sh16(v.d.x, v.d.y, v.d.z, sh);
#pragma unroll
    for (int k = 0; k < 8; ++k) r32[16 + k] = pack2(sh[2 * k], sh[2 * k + 1]);
    r32[24] = pack2(v.d.w, v.a.x);
    r32[25] = pack2(v.a.y, v.a.z);
    r32[26] = pack2(v.n.x * 0.5f + 0.5f, v.n.y * 0.5f + 0.5f);
    r32[27] = pack2(v.n.z * 0.5f + 0.5f, 1.0f);
#pragma unroll
    for (int k = 28; k < 32; ++k) r32[k] = 0u;
}

// Two halves of 128 threads run two query tiles side by side, each with its
// own A operand, mbarrier, 64 tensor-memory columns and named barrier: one
// half's hash-grid gathers and epilogues overlap the other half's MMAs.
__global__ void __launch_bounds__(2 * kTcRows, 2) k_nrc_infer_tc(NrcNet net, const NrcQuery* __restrict__ q,
                                                               const int32_t* count, int cap, double* accum,
                                                               float* out_rgb, int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sW = smem;                                  // 6 weight operands, canonical layout
    const int half = threadIdx.x >> 7;                         // which tile of the pair
    const int t = threadIdx.x & (kTcRows - 1), warp = threadIdx.x >> 5;
    unsigned char* sA = smem + kTcWBytes + half * kTcABytes;   // this half's 128 x 64 activation operand
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kTcWBytes + 2 * kTcABytes) + half;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTcWBytes + 2 * kTcABytes + 16);

    // weights [out][in] -> canonical K-major chunks
    for (int e = threadIdx.x; e < kTcWBytes / 16; e += 2 * kTcRows) {
        const int l = min(e / (kNrcHid * 8), kNrcLayers - 1);
        const int local = e - l * (kNrcHid * 8);
        const int R = nrc_w_rows(l);
        const int r = local / 8, kc = local % 8;
        const uint4 v = *reinterpret_cast<const uint4*>(net.w + nrc_w_offset(l) + r * kNrcIn + kc * 8);
        *reinterpret_cast<uint4*>(sW + l * (kNrcHid * kNrcIn * 2) + tc_chunk_offset(R, r, kc)) = v;
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     : : "r"(smem_addr(tmem_slot)), "r"(2 * kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot + static_cast<uint32_t>(half * kTcCols);     // this half's columns
    const uint32_t taddr = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);  // lanes of this warp's rows
    const uint32_t aBase = smem_addr(sA), wBase = smem_addr(sW), mb = smem_addr(mbar);
    uint32_t phase = 0;
    bool failed = false;

    const int n = min(*count, cap);
    for (int tile = 2 * blockIdx.x + half; tile * kTcRows < n && !failed; tile += 2 * gridDim.x) {
        const int row = tile * kTcRows + t;
        const bool valid = row < n;
        NrcQuery qq;
        if (valid) qq = q[row];
        {
            uint32_t r32[32];
            tc_encode(net, qq.v, valid, r32);
#pragma unroll
            for (int kc = 0; kc < 8; ++kc)
                *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) =
                    make_uint4(r32[4 * kc], r32[4 * kc + 1], r32[4 * kc + 2], r32[4 * kc + 3]);
        }
        float out[3] = {0.0f, 0.0f, 0.0f};
        for (int l = 0; l < kNrcLayers && !failed; ++l) {
            const int N = nrc_w_rows(l);
            // generic-proxy writes of the A operand -> visible to the tensor core
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            half_sync(half);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (t == 0) {
                const uint32_t wl = wBase + static_cast<uint32_t>(l * (kNrcHid * kNrcIn * 2));
                const uint32_t idesc = tc_idesc(kTcRows, N);
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const uint64_t da = tc_desc(aBase + static_cast<uint32_t>(2 * s * kTcRows * 16), kTcRows * 16, 128);
                    const uint64_t db = tc_desc(wl + static_cast<uint32_t>(2 * s * N * 16), static_cast<uint32_t>(N * 16), 128);
                    tc_mma(tmem, da, db, idesc, s > 0 ? 1u : 0u);
                }
                tc_commit(mb);
            }
            uint32_t spins = 0;
            bool late = false;
            while (!mbar_try_wait(mb, phase)) {
                if (++spins >= kTcSpinLimit) { late = true; break; }
            }
            phase ^= 1u;
            failed = half_sync_or(half, late);   // the same decision in every thread of the half
            if (failed) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t v[64];
            tc_ld64(taddr, v);
            if (l < kNrcLayers - 1) {
#pragma unroll
                for (int kc = 0; kc < 8; ++kc) {
                    uint32_t p[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        p[j] = pack2(fmaxf(__uint_as_float(v[8 * kc + 2 * j]), 0.0f), fmaxf(__uint_as_float(v[8 * kc + 2 * j + 1]), 0.0f));
                    *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) = make_uint4(p[0], p[1], p[2], p[3]);
                }
            } else if (net.spectral) {   // four wavelengths: the path's XYZ from the 16 spectral bins
                float e[kNrcBins];
#pragma unroll
                for (int b = 0; b < kNrcBins; ++b) e[b] = expf(fminf(__uint_as_float(v[b]), 15.0f));
                if (valid && accum) {
                    const f3 c = nrc_spectral_xyz(net.tables, e, qq.v.n.w, qq.t);
                    out[0] = c.x; out[1] = c.y; out[2] = c.z;
                }
                if (valid && out_rgb)
                    for (int b = 0; b < kNrcBins; ++b) out_rgb[kNrcBins * static_cast<int64_t>(row) + b] = e[b];
            } else {
                out[0] = expf(fminf(__uint_as_float(v[0]), 15.0f));
                out[1] = expf(fminf(__uint_as_float(v[1]), 15.0f));
                out[2] = expf(fminf(__uint_as_float(v[2]), 15.0f));
            }
        }
        if (failed) break;
        if (valid && net.spectral) {   // out holds the XYZ contribution already
            if (accum) {
                const int64_t pix = __float_as_int(qq.v.p.w);
                atomicAdd(&accum[3 * pix + 0], nrc_contrib(out[0]));
                atomicAdd(&accum[3 * pix + 1], nrc_contrib(out[1]));
                atomicAdd(&accum[3 * pix + 2], nrc_contrib(out[2]));
            }
        } else if (valid) {
            if (accum) {
                const int64_t pix = __float_as_int(qq.v.p.w);
                atomicAdd(&accum[3 * pix + 0], nrc_contrib(qq.t.x * out[0]));
                atomicAdd(&accum[3 * pix + 1], nrc_contrib(qq.t.y * out[1]));
                atomicAdd(&accum[3 * pix + 2], nrc_contrib(qq.t.z * out[2]));
            }
            if (out_rgb) {
                out_rgb[3 * static_cast<int64_t>(row) + 0] = out[0];
                out_rgb[3 * static_cast<int64_t>(row) + 1] = out[1];
                out_rgb[3 * static_cast<int64_t>(row) + 2] = out[2];
            }
        }
    }
    if (failed) {
        // A layer's MMAs did not complete within the wait limit and may still be
        // writing this CTA's tensor-memory columns: wait for that commit once more
        // (bounded) before the columns are released to other CTAs.  Error bit 2
        // marks every output of the launch as invalid.
        uint32_t spins = 0;
        while (!mbar_try_wait(mb, phase ^ 1u) && ++spins < 4u * kTcSpinLimit) {
        }
        atomicOr(err, 2);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(*tmem_slot), "r"(2 * kTcCols) : "memory");
}

// ------------------------------------------------------------------ training
// Weights of the forward pass ([out][in] per layer) or of the backward pass
// (the transposes [in][out]; layer 5 [64][16]) into canonical K-major B
// operands: hidden layers at l * 8192 bytes (64 rows x 8 chunks), the output
// layer at 40960 (forward: 16 rows x 8 chunks; backward: 64 rows x 2 chunks).
__device__ void tc_stage_weights(const __nv_bfloat16* w, bool backward, unsigned char* sW)
{
    for (int e = threadIdx.x; e < kTcWBytes / 16; e += blockDim.x) {
        const int l = min(e / (kNrcHid * 8), kNrcLayers - 1);
        const int local = e - l * (kNrcHid * 8);
        int R, r, kc, K;
        if (l < kNrcLayers - 1) {
            R = kNrcHid; K = kNrcIn; r = local / 8; kc = local % 8;
        } else if (!backward) {
            R = kNrcOut; K = kNrcIn; r = local / 8; kc = local % 8;
        } else {
            R = kNrcIn; K = kNrcOut; r = local / 2; kc = local % 2;
        }
        const uint4 v = *reinterpret_cast<const uint4*>(w + nrc_w_offset(l) + r * K + kc * 8);
        *reinterpret_cast<uint4*>(sW + l * (kNrcHid * kNrcIn * 2) + tc_chunk_offset(R, r, kc)) = v;
    }
}

// The training forward pass of a batch on the tensor cores: the layers of
// k_nrc_infer_tc, storing the input and every hidden activation (bf16,
// [rows][64] per layer) and the 16 raw outputs ([rows][16] fp32) for the
// backward pass, as k_nrc_train_fwd (nrc.cu) does.
__global__ void __launch_bounds__(kTcThreads, 1) k_nrc_train_fwd_tc(NrcNet net, const NrcSample* __restrict__ smp,
                                                                   const int32_t* count, int first, int batch,
                                                                   NrcTrainBuffers T, int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sW = smem;
    unsigned char* sA = smem + kTcWBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kTcWBytes + kTcABytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTcWBytes + kTcABytes + 16);
    const int t = threadIdx.x, warp = t >> 5;
    tc_stage_weights(net.w, false, sW);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     : : "r"(smem_addr(tmem_slot)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
    const uint32_t aBase = smem_addr(sA), wBase = smem_addr(sW), mb = smem_addr(mbar);
    uint32_t phase = 0;
    bool failed = false;
    const int nv = max(0, min(batch, *count - first));
    for (int tile = blockIdx.x; tile * kTcRows < batch && !failed; tile += gridDim.x) {
        const int row = tile * kTcRows + t;
        const bool valid = row < nv;
        const bool keep = row < batch;
        NrcSample sm;
        if (valid) sm = smp[first + row];
        {
            uint32_t r32[32];
            tc_encode(net, sm.v, valid, r32);
            uint4* dst = reinterpret_cast<uint4*>(T.acts + static_cast<int64_t>(row) * kNrcIn);
#pragma unroll
            for (int kc = 0; kc < 8; ++kc) {
                const uint4 v = make_uint4(r32[4 * kc], r32[4 * kc + 1], r32[4 * kc + 2], r32[4 * kc + 3]);
                *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) = v;
                if (keep) dst[kc] = v;
            }
        }
        for (int l = 0; l < kNrcLayers && !failed; ++l) {
            const int N = nrc_w_rows(l);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (t == 0) {
                const uint32_t wl = wBase + static_cast<uint32_t>(l * (kNrcHid * kNrcIn * 2));
                const uint32_t idesc = tc_idesc(kTcRows, N);
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const uint64_t da = tc_desc(aBase + static_cast<uint32_t>(2 * s * kTcRows * 16), kTcRows * 16, 128);
                    const uint64_t db = tc_desc(wl + static_cast<uint32_t>(2 * s * N * 16), static_cast<uint32_t>(N * 16), 128);
                    tc_mma(tmem, da, db, idesc, s > 0 ? 1u : 0u);
                }
                tc_commit(mb);
            }
            uint32_t spins = 0;
            bool late = false;
            while (!mbar_try_wait(mb, phase)) {
                if (++spins >= kTcSpinLimit) { late = true; break; }
            }
            phase ^= 1u;
            failed = __syncthreads_or(late ? 1 : 0) != 0;
            if (failed) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t v[64];
            tc_ld64(taddr, v);
            if (l < kNrcLayers - 1) {
                uint4* dst = reinterpret_cast<uint4*>(T.acts + (static_cast<int64_t>(l + 1) * batch + row) * kNrcIn);
#pragma unroll
                for (int kc = 0; kc < 8; ++kc) {
                    uint32_t p[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        p[j] = pack2(fmaxf(__uint_as_float(v[8 * kc + 2 * j]), 0.0f), fmaxf(__uint_as_float(v[8 * kc + 2 * j + 1]), 0.0f));
                    const uint4 q4 = make_uint4(p[0], p[1], p[2], p[3]);
                    *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) = q4;
                    if (keep) dst[kc] = q4;
                }
            } else if (keep) {
                float4* r = reinterpret_cast<float4*>(T.raw) + 4 * static_cast<int64_t>(row);
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    r[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]), __uint_as_float(v[4 * q + 2]),
                                       __uint_as_float(v[4 * q + 3]));
            }
        }
    }
    if (failed) {
        uint32_t spins = 0;
        while (!mbar_try_wait(mb, phase ^ 1u) && ++spins < 4u * kTcSpinLimit) {
        }
        atomicOr(err, 4);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(kTcCols) : "memory");
}

// The training backward pass on the tensor cores (k_nrc_train_bwd, nrc.cu):
// thread t owns row t of a 128-row tile; the loss gradient of its 16 raw
// outputs (nrc_output_grad) is the first A operand (K = 16); each layer l =
// 5..0 is one product with the transposed weights (N = 64) in tensor memory,
// then the row is masked by the ReLU of the stored activation l, rounded to
// bf16, stored as the pre-activation gradient of layer l - 1 and written back
// as the next A operand; layer 0 gives the input gradient, whose 32 hash-grid
// columns are stored in fp32.
__global__ void __launch_bounds__(kTcThreads, 1) k_nrc_train_bwd_tc(NrcNet net, const NrcSample* __restrict__ smp,
                                                                   const int32_t* count, int first, int batch,
                                                                   NrcTrainBuffers T, int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sW = smem;
    unsigned char* sA = smem + kTcWBytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kTcWBytes + kTcABytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kTcWBytes + kTcABytes + 16);
    const int t = threadIdx.x, warp = t >> 5;
    tc_stage_weights(net.wt, true, sW);
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     : : "r"(smem_addr(tmem_slot)), "r"(kTcCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16);
    const uint32_t aBase = smem_addr(sA), wBase = smem_addr(sW), mb = smem_addr(mbar);
    uint32_t phase = 0;
    bool failed = false;
    const int nv = max(0, min(batch, *count - first));
    const float norm = nv > 0 ? 1.0f / ((net.spectral ? 4.0f : 3.0f) * static_cast<float>(nv)) : 0.0f;
    float loss_acc = 0.0f;
    for (int tile = blockIdx.x; tile * kTcRows < batch && !failed; tile += gridDim.x) {
        const int row = tile * kTcRows + t;
        const bool keep = row < batch;
        {
            float d[kNrcBins];
#pragma unroll
            for (int b = 0; b < kNrcBins; ++b) d[b] = 0.0f;
            if (row < nv) {
                const NrcSample sm = smp[first + row];
                const float4* rr = reinterpret_cast<const float4*>(T.raw) + 4 * static_cast<int64_t>(row);
                float raw[kNrcBins];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 v = rr[q];
                    raw[4 * q] = v.x; raw[4 * q + 1] = v.y; raw[4 * q + 2] = v.z; raw[4 * q + 3] = v.w;
                }
                loss_acc += nrc_output_grad(net.spectral, sm, raw, norm, d);
            }
            uint4* dz5 = reinterpret_cast<uint4*>(T.dz + (static_cast<int64_t>(5) * batch + row) * kNrcIn);
#pragma unroll
            for (int kc = 0; kc < 2; ++kc) {
                uint32_t p[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) p[j] = pack2(d[8 * kc + 2 * j], d[8 * kc + 2 * j + 1]);
                const uint4 q4 = make_uint4(p[0], p[1], p[2], p[3]);
                *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) = q4;
                if (keep) dz5[kc] = q4;
            }
        }
        for (int l = kNrcLayers - 1; l >= 0 && !failed; --l) {
            const int ksteps = l == kNrcLayers - 1 ? 1 : 4;   // K = 16 (output gradient) or 64
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (t == 0) {
                const uint32_t wl = wBase + static_cast<uint32_t>(l * (kNrcHid * kNrcIn * 2));
                const uint32_t idesc = tc_idesc(kTcRows, kNrcIn);
                for (int s = 0; s < ksteps; ++s) {
                    const uint64_t da = tc_desc(aBase + static_cast<uint32_t>(2 * s * kTcRows * 16), kTcRows * 16, 128);
                    const uint64_t db = tc_desc(wl + static_cast<uint32_t>(2 * s * kNrcIn * 16), kNrcIn * 16, 128);
                    tc_mma(tmem, da, db, idesc, s > 0 ? 1u : 0u);
                }
                tc_commit(mb);
            }
            uint32_t spins = 0;
            bool late = false;
            while (!mbar_try_wait(mb, phase)) {
                if (++spins >= kTcSpinLimit) { late = true; break; }
            }
            phase ^= 1u;
            failed = __syncthreads_or(late ? 1 : 0) != 0;
            if (failed) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t v[64];
            tc_ld64(taddr, v);
            if (l == 0) {   // gradient of the input: the 32 hash-grid columns, fp32
                if (keep) {
                    float4* dx = reinterpret_cast<float4*>(T.dx + static_cast<int64_t>(row) * 32);
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        dx[q] = make_float4(__uint_as_float(v[4 * q]), __uint_as_float(v[4 * q + 1]),
                                            __uint_as_float(v[4 * q + 2]), __uint_as_float(v[4 * q + 3]));
                }
                break;
            }
            // through the ReLU of activation l: the pre-activation gradient of layer l - 1
            const uint4* H = reinterpret_cast<const uint4*>(T.acts + (static_cast<int64_t>(l) * batch + row) * kNrcIn);
            uint4* DZ = reinterpret_cast<uint4*>(T.dz + (static_cast<int64_t>(l - 1) * batch + row) * kNrcIn);
#pragma unroll
            for (int kc = 0; kc < 8; ++kc) {
                const uint4 h4 = keep ? H[kc] : make_uint4(0u, 0u, 0u, 0u);
                const uint32_t hw[4] = {h4.x, h4.y, h4.z, h4.w};
                uint32_t p[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    __nv_bfloat162 hb;
                    *reinterpret_cast<uint32_t*>(&hb) = hw[j];
                    const float2 h = __bfloat1622float2(hb);
                    const float g0 = h.x > 0.0f ? __uint_as_float(v[8 * kc + 2 * j]) : 0.0f;
                    const float g1 = h.y > 0.0f ? __uint_as_float(v[8 * kc + 2 * j + 1]) : 0.0f;
                    p[j] = pack2(g0, g1);
                }
                const uint4 q4 = make_uint4(p[0], p[1], p[2], p[3]);
                *reinterpret_cast<uint4*>(sA + tc_chunk_offset(kTcRows, t, kc)) = q4;
                if (keep) DZ[kc] = q4;
            }
        }
    }
    if (failed) {
        uint32_t spins = 0;
        while (!mbar_try_wait(mb, phase ^ 1u) && ++spins < 4u * kTcSpinLimit) {
        }
        atomicOr(err, 8);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if ((t & 31) == 0 && loss_acc != 0.0f) atomicAdd(T.loss, loss_acc);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(kTcCols) : "memory");
}

}  // namespace

cudaError_t nrc_infer_tc(const NrcNet& net, const NrcQuery* q, const int32_t* count, int cap, double* accum,
                         float* out_rgb, int* err, int sm_count, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_nrc_infer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcInferSmem);
    if (e != cudaSuccess) return e;
    const int tiles = (cap + kTcRows - 1) / kTcRows;
    const int grid = std::max(1, std::min((tiles + 1) / 2, sm_count * 2));
    k_nrc_infer_tc<<<grid, 2 * kTcRows, kTcInferSmem, st>>>(net, q, count, cap, accum, out_rgb, err);
    return cudaGetLastError();
}

}  // namespace ar

namespace ar {

cudaError_t nrc_train_fwd_bwd_tc(const NrcNet& net, const NrcSample* samples, const int32_t* count, int first,
                                 int batch, const NrcTrainBuffers& T, int* err, int sm_count, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_nrc_train_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_nrc_train_bwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
    if (e != cudaSuccess) return e;
    const int tiles = (batch + kTcRows - 1) / kTcRows;
    const int grid = std::max(1, std::min(tiles, sm_count * 2));
    k_nrc_train_fwd_tc<<<grid, kTcThreads, kTcSmem, st>>>(net, samples, count, first, batch, T, err);
    k_nrc_train_bwd_tc<<<grid, kTcThreads, kTcSmem, st>>>(net, samples, count, first, batch, T, err);
    return cudaGetLastError();
}

}  // namespace ar
