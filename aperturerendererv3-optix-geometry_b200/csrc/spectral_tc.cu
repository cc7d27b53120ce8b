// spectral_tc.cu -- the RGB lookup table of the spectral mode built on the
// 5th-generation tensor cores (PrecomputeRGBLUTKernel,
// core/spectrum/spectrum_lut.cuh:12-38, evaluates the reference's RGB
// spectrum-basis network -- 32 sin/cos input features, an input layer and 7
// residual blocks of width 32 with ReLU, a 4-wide output -- at every voxel
// centre of the unit colour cube; 512^3 voxels in the reference).
//
// A tile is 128 voxels, one per thread; every layer is one 128 x 32 x 32
// matrix product on tcgen05.mma (kind::f16) with fp32 accumulators in tensor
// memory.  A CTA of 256 threads runs two tiles side by side.  The MMA takes bf16 operands, so fp32 accuracy comes from splitting
// both operands into three bf16 terms, x = x0 + x1 + x2 (x0 = bf16(x),
// x1 = bf16(x - x0), x2 = bf16(x - x0 - x1): 24 significant bits), and
// accumulating the six products whose order is at most 2 (x2 w0, x1 w1,
// x0 w2, x1 w0, x0 w1, x0 w0, smallest first).  The activations stay fp32 in
// the registers of the row's thread between layers (bias, ReLU, residual sum
// from tcgen05.ld); only the next layer's split operand goes back to shared
// memory.  Entries differ from the SIMT build (one thread per voxel, fmaf in
// input order) by the summation order and the dropped products of order 3
// and above: a few fp32 ulps, measured by ar_spectral_rgb_lut.
//
// Every wait is bounded; a CTA whose MMA does not complete within the limit
// sets the error word, waits once more for its commit, frees its tensor
// memory and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "render_kernels.h"
#include "spectral.cuh"
#include "tcgen05.cuh"

namespace ar {

namespace {

constexpr int kLutRows = 128;                                 // voxels per CTA tile (M)
constexpr int kLutLayers = 2 + kSpecBlocks;                   // input, 7 blocks, output
constexpr int kLutN = 32;                                     // width of the hidden layers
constexpr int kLutNOut = 16;                                  // output layer N (4 used)
constexpr int kLutK = 32;
constexpr int kLutWLayer = kLutN * kLutK * 2;                 // bytes of one bf16 weight split (hidden)
constexpr int kLutWOut = kLutNOut * kLutK * 2;
constexpr int kLutWBytes = 3 * ((kLutLayers - 1) * kLutWLayer + kLutWOut);   // three splits
constexpr int kLutABytes = kLutRows * kLutK * 2;              // one bf16 split of the activations
constexpr int kLutSmem = kLutWBytes + 6 * kLutABytes + 64;   // weights, two tiles' A operands, barriers
constexpr int kLutCols = 32;                                  // TMEM columns (fp32 accumulators)
constexpr uint32_t kLutSpinLimit = 1u << 22;

// byte offset of split j of layer l's weights
__host__ __device__ constexpr int lut_w_offset(int l, int j)
{
    return j * ((kLutLayers - 1) * kLutWLayer + kLutWOut) + l * kLutWLayer;
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16* t)
{
    t[0] = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(t[0]);
    t[1] = __float2bfloat16_rn(r1);
    t[2] = __float2bfloat16_rn(r1 - __bfloat162float(t[1]));
}

// row t's 32 fp32 values as the three bf16 splits of the A operand
__device__ __forceinline__ void store_row(unsigned char* sA, int t, const float* h)
{
#pragma unroll
    for (int kc = 0; kc < kLutK / 8; ++kc) {
        __nv_bfloat16 v[3][8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            __nv_bfloat16 s3[3];
            split3(h[8 * kc + e], s3);
            v[0][e] = s3[0];
            v[1][e] = s3[1];
            v[2][e] = s3[2];
        }
#pragma unroll
        for (int j = 0; j < 3; ++j)
            *reinterpret_cast<uint4*>(sA + j * kLutABytes + tc_chunk_offset(kLutRows, t, kc)) =
                *reinterpret_cast<const uint4*>(v[j]);
    }
}

}  // namespace

namespace {

// Two halves of 128 threads run two tiles side by side: each half has its own
// A operand, mbarrier and 32 tensor-memory columns and synchronises on a named
// barrier of its own, so one half's epilogue (tcgen05.ld, bias, ReLU, split,
// store) overlaps the other half's MMAs.  The weights are shared.
__global__ void __launch_bounds__(2 * kLutRows) k_lut_rgb_tc(const float* __restrict__ tab, int res,
                                                             float4* __restrict__ lut, int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* sW = smem;
    const int half = threadIdx.x >> 7;                 // which tile of the pair
    const int t = threadIdx.x & (kLutRows - 1);        // row within the tile
    const int warp = threadIdx.x >> 5;
    unsigned char* sA = smem + kLutWBytes + half * 3 * kLutABytes;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kLutWBytes + 6 * kLutABytes) + half;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kLutWBytes + 6 * kLutABytes + 16);

    // weights [out][in] of every layer as three bf16 splits, B operands (N rows x K)
    for (int e = threadIdx.x; e < kLutLayers * kLutN * kLutK; e += 2 * kLutRows) {
        const int l = e / (kLutN * kLutK), rem = e - l * (kLutN * kLutK);
        const int n = rem / kLutK, k = rem - n * kLutK;
        const int R = l == kLutLayers - 1 ? kLutNOut : kLutN;
        if (n >= R) continue;
        float w;
        if (l == 0) w = tab[kTabRgbInW + n * kLutK + k];
        else if (l < kLutLayers - 1) w = tab[kTabRgbBlkW + (l - 1) * 1024 + n * kLutK + k];
        else w = n < kSpecKernel ? tab[kTabRgbOutW + n * kLutK + k] : 0.0f;
        __nv_bfloat16 s3[3];
        split3(w, s3);
        for (int j = 0; j < 3; ++j)
            *reinterpret_cast<__nv_bfloat16*>(sW + lut_w_offset(l, j) + tc_chunk_offset(R, n, k / 8) + (k % 8) * 2) =
                s3[j];
    }
    if (t == 0) {   // thread 0 of each half: its mbarrier
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_addr(mbar)), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     : : "r"(smem_addr(tmem_slot)), "r"(2 * kLutCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot + static_cast<uint32_t>(half * kLutCols);   // this half's columns
    const uint32_t taddr = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16);  // lanes of this warp's rows
    const uint32_t aBase = smem_addr(sA), wBase = smem_addr(sW), mb = smem_addr(mbar);
    uint32_t phase = 0;
    bool failed = false;
    const int64_t total = static_cast<int64_t>(res) * res * res;
    const float invRes = 1.0f / static_cast<float>(res);
    for (int64_t tile = 2 * static_cast<int64_t>(blockIdx.x) + half; tile * kLutRows < total && !failed;
         tile += 2 * static_cast<int64_t>(gridDim.x)) {
        const int64_t vx = tile * kLutRows + t;
        const bool valid = vx < total;
        const int64_t v = valid ? vx : total - 1;
        const int x = static_cast<int>(v % res), y = static_cast<int>((v / res) % res);
        const int z = static_cast<int>(v / (static_cast<int64_t>(res) * res));
        // RGBEncode's input features (spectrum_basis.cuh:2273-2300), as rgb_encode
        const float in[3] = {(static_cast<float>(x) + 0.5f) * invRes, (static_cast<float>(y) + 0.5f) * invRes,
                             (static_cast<float>(z) + 0.5f) * invRes};
        const float scale = fmaxf(fmaxf(in[0], in[1]), in[2]);
        const float inv = 1.0f / (scale + 0.001f);
        float h[kLutK];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k)
                sincos_det(in[c] * inv * kSpecPi * static_cast<float>(k + 1), &h[8 * c + k], &h[8 * c + k + 4]);
#pragma unroll
        for (int k = 0; k < 4; ++k) sincos_det(scale * kSpecPi * static_cast<float>(k + 1), &h[24 + k], &h[28 + k]);
        float out[kSpecKernel] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (int l = 0; l < kLutLayers && !failed; ++l) {
            const int N = l == kLutLayers - 1 ? kLutNOut : kLutN;
            store_row(sA, t, h);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            half_sync(half);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (t == 0) {
                const uint32_t idesc = tc_idesc(kLutRows, N);
                const int pa[6] = {2, 1, 0, 1, 0, 0}, pw[6] = {0, 1, 2, 0, 1, 0};   // smallest products first
#pragma unroll
                for (int ks = 0; ks < kLutK / 16; ++ks)
#pragma unroll
                    for (int p = 0; p < 6; ++p) {
                        const uint64_t da = tc_desc(aBase + static_cast<uint32_t>(pa[p] * kLutABytes + 2 * ks * kLutRows * 16),
                                                    kLutRows * 16, 128);
                        const uint64_t db = tc_desc(wBase + static_cast<uint32_t>(lut_w_offset(l, pw[p]) + 2 * ks * N * 16),
                                                    static_cast<uint32_t>(N * 16), 128);
                        tc_mma(tmem, da, db, idesc, (ks > 0 || p > 0) ? 1u : 0u);
                    }
                tc_commit(mb);
            }
            uint32_t spins = 0;
            bool late = false;
            while (!mbar_try_wait(mb, phase)) {
                if (++spins >= kLutSpinLimit) { late = true; break; }
            }
            phase ^= 1u;
            failed = half_sync_or(half, late);   // the same decision in every thread of the half
            if (failed) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            uint32_t acc[kLutN];
            tc_ld32(taddr, acc);
            if (l == 0) {
#pragma unroll
                for (int i = 0; i < kLutN; ++i) h[i] = fmaxf(__uint_as_float(acc[i]) + __ldg(tab + kTabRgbInB + i), 0.0f);
            } else if (l < kLutLayers - 1) {
                const float* B = tab + kTabRgbBlkB + (l - 1) * 32;
#pragma unroll
                for (int i = 0; i < kLutN; ++i) h[i] = h[i] + fmaxf(__uint_as_float(acc[i]) + __ldg(B + i), 0.0f);
            } else {
#pragma unroll
                for (int i = 0; i < kSpecKernel; ++i) out[i] = __uint_as_float(acc[i]) * scale;
            }
        }
        if (failed) break;
        if (valid) lut[vx] = make_float4(out[0], out[1], out[2], out[3]);
    }
    if (failed) {   // the timed-out MMAs may still write tensor memory: wait for their commit once more
        uint32_t spins = 0;
        while (!mbar_try_wait(mb, phase ^ 1u) && ++spins < 4u * kLutSpinLimit) {
        }
        atomicOr(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(*tmem_slot), "r"(2 * kLutCols) : "memory");
}

}  // namespace

cudaError_t launch_spectral_rgb_lut_tc(const float* tab, int res, float4* lut, int* err, int sm_count,
                                       cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_lut_rgb_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kLutSmem);
    if (e != cudaSuccess) return e;
    const int64_t total = static_cast<int64_t>(res) * res * res;
    const int64_t tiles = (total + kLutRows - 1) / kLutRows;
    const int grid = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((tiles + 1) / 2, int64_t(sm_count) * 2)));
    k_lut_rgb_tc<<<grid, 2 * kLutRows, kLutSmem, st>>>(tab, res, lut, err);
    return cudaGetLastError();
}

}  // namespace ar
