// nrc.cu -- kernels of the learned radiance cache: encoding, fused MLP
// inference, fused training forward and backward on bf16 tensor cores
// (mma.sync m16n8k16, fp32 accumulation, activations kept in registers from
// layer to layer), weight and hash-table gradients, Adam.
//
// Fragment layout of mma.sync.m16n8k16 (lane = 4 * group + t):
//   A 16x16 row-major: a0 (group, 2t..2t+1) a1 (group+8, 2t..) a2 (group, 2t+8..) a3 (group+8, 2t+8..)
//   B 16x8 "col":      b0 (k 2t..2t+1, n group) b1 (k 2t+8.., n group)
//   C 16x8:            c0 c1 (group, 2t..2t+1)  c2 c3 (group+8, 2t..2t+1)
// so the C tiles of columns 16s..16s+15 are, packed to bf16 pairs, exactly the
// A fragment of k-slice s of the next layer.  B fragments of W (stored
// [out][in], `in` contiguous) are 32-bit loads from shared memory rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "nrc.cuh"

namespace ar {

namespace {

constexpr int kWarps = kNrcBlock / 32;
// shared memory: forward weights [out][in] with kNrcWRow-element rows
constexpr int kFwdRows = 5 * kNrcHid + kNrcOut;               // 336
constexpr int kSmemW = kFwdRows * kNrcWRow * 2;               // 48384 B
// backward weights [in][out]: hidden layers rows of 72, output layer rows of 24
constexpr int kBwdRow5 = 24;
constexpr int kSmemWt = (5 * kNrcIn * kNrcWRow + kNrcIn * kBwdRow5) * 2;  // 49152 B
constexpr int kSmemIn = kWarps * kNrcWarpRows * kNrcWRow * 2;            // 18432 B
constexpr int kOutRow = 17;
constexpr int kSmemOut = kWarps * kNrcWarpRows * kOutRow * 4;            // 8704 B

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float2 unpack_bf16(uint32_t u)
{
    __nv_bfloat162 v;
    *reinterpret_cast<uint32_t*>(&v) = u;
    return __bfloat1622float2(v);
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Network input of one vertex into a bf16 shared-memory row (kNrcWRow wide).
__device__ void encode_row(const NrcNet& net, const NrcVertex& v, bool valid, __nv_bfloat16* row)
{
    uint32_t* r32 = reinterpret_cast<uint32_t*>(row);
    if (!valid) {
#pragma unroll
        for (int k = 0; k < kNrcIn / 2; ++k) r32[k] = 0u;
        return;
    }
    float u[3];
    nrc_unit_pos(net.grid, v.p, u);
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
        r32[l] = pack_bf16(f0, f1);
    }
    float sh[16];
    nrc_sh16(v.d.x, v.d.y, v.d.z, sh);
#pragma unroll
    for (int k = 0; k < 8; ++k) r32[16 + k] = pack_bf16(sh[2 * k], sh[2 * k + 1]);
    r32[24] = pack_bf16(v.d.w, v.a.x);
    r32[25] = pack_bf16(v.a.y, v.a.z);
    r32[26] = pack_bf16(v.n.x * 0.5f + 0.5f, v.n.y * 0.5f + 0.5f);
    r32[27] = pack_bf16(v.n.z * 0.5f + 0.5f, 1.0f);
#pragma unroll
    for (int k = 28; k < 32; ++k) r32[k] = 0u;
}

__device__ __forceinline__ void load_a(const __nv_bfloat16* s, int g, int t, uint32_t (*a)[4][4])
{
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const __nv_bfloat16* r0 = s + (16 * mt + g) * kNrcWRow + 16 * ks + 2 * t;
            const __nv_bfloat16* r1 = r0 + 8 * kNrcWRow;
            a[mt][ks][0] = ld32(r0);
            a[mt][ks][1] = ld32(r1);
            a[mt][ks][2] = ld32(r0 + 8);
            a[mt][ks][3] = ld32(r1 + 8);
        }
}

// The fused forward pass of one warp tile (32 rows): input rows in sIn, raw
// outputs (16 columns) to sOut.  With acts != nullptr the input and every
// hidden activation are stored (bf16, [rows][64] per layer) for the backward
// pass; rows >= nrows are not stored.
__device__ void forward_tile(const __nv_bfloat16* sW, const __nv_bfloat16* sIn, float* sOut, __nv_bfloat16* acts,
                             int64_t batch, int64_t row0, int64_t nrows)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint32_t a[2][4][4];
    load_a(sIn, g, t, a);
    if (acts) {   // layer-0 input: each lane copies its own row
        const int64_t r = row0 + lane;
        if (r < nrows) {
            const uint4* src = reinterpret_cast<const uint4*>(sIn + lane * kNrcWRow);
            uint4* dst = reinterpret_cast<uint4*>(acts + r * kNrcIn);
#pragma unroll
            for (int k = 0; k < 8; ++k) dst[k] = src[k];
        }
    }
    for (int l = 0; l < kNrcLayers - 1; ++l) {
        const __nv_bfloat16* W = sW + l * kNrcHid * kNrcWRow;
        float c[2][8][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int j = 0; j < 8; ++j) c[mt][j][0] = c[mt][j][1] = c[mt][j][2] = c[mt][j][3] = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const __nv_bfloat16* wr = W + (8 * j + g) * kNrcWRow + 16 * ks + 2 * t;
                const uint32_t b0 = ld32(wr), b1 = ld32(wr + 8);
                mma_bf16(c[0][j], a[0][ks], b0, b1);
                mma_bf16(c[1][j], a[1][ks], b0, b1);
            }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                a[mt][ks][0] = pack_bf16(fmaxf(c[mt][2 * ks][0], 0.0f), fmaxf(c[mt][2 * ks][1], 0.0f));
                a[mt][ks][1] = pack_bf16(fmaxf(c[mt][2 * ks][2], 0.0f), fmaxf(c[mt][2 * ks][3], 0.0f));
                a[mt][ks][2] = pack_bf16(fmaxf(c[mt][2 * ks + 1][0], 0.0f), fmaxf(c[mt][2 * ks + 1][1], 0.0f));
                a[mt][ks][3] = pack_bf16(fmaxf(c[mt][2 * ks + 1][2], 0.0f), fmaxf(c[mt][2 * ks + 1][3], 0.0f));
            }
        if (acts) {
            __nv_bfloat16* dst = acts + static_cast<int64_t>(l + 1) * batch * kNrcIn;
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int64_t r0 = row0 + 16 * mt + g, r1 = r0 + 8;
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    const int col = 16 * ks + 2 * t;
                    if (r0 < nrows) {
                        *reinterpret_cast<uint32_t*>(dst + r0 * kNrcIn + col) = a[mt][ks][0];
                        *reinterpret_cast<uint32_t*>(dst + r0 * kNrcIn + col + 8) = a[mt][ks][2];
                    }
                    if (r1 < nrows) {
                        *reinterpret_cast<uint32_t*>(dst + r1 * kNrcIn + col) = a[mt][ks][1];
                        *reinterpret_cast<uint32_t*>(dst + r1 * kNrcIn + col + 8) = a[mt][ks][3];
                    }
                }
            }
        }
    }
    // output layer: 16 columns
    const __nv_bfloat16* W = sW + 5 * kNrcHid * kNrcWRow;
    float c[2][2][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int j = 0; j < 2; ++j) c[mt][j][0] = c[mt][j][1] = c[mt][j][2] = c[mt][j][3] = 0.0f;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            const __nv_bfloat16* wr = W + (8 * j + g) * kNrcWRow + 16 * ks + 2 * t;
            const uint32_t b0 = ld32(wr), b1 = ld32(wr + 8);
            mma_bf16(c[0][j], a[0][ks], b0, b1);
            mma_bf16(c[1][j], a[1][ks], b0, b1);
        }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            float* o0 = sOut + (16 * mt + g) * kOutRow + 8 * j + 2 * t;
            float* o1 = o0 + 8 * kOutRow;
            o0[0] = c[mt][j][0]; o0[1] = c[mt][j][1];
            o1[0] = c[mt][j][2]; o1[1] = c[mt][j][3];
        }
}

__device__ void load_weights_fwd(const __nv_bfloat16* w, __nv_bfloat16* sW)
{
    for (int e = threadIdx.x; e < kFwdRows * (kNrcIn / 2); e += blockDim.x) {
        const int r = e / (kNrcIn / 2), c = e - r * (kNrcIn / 2);
        reinterpret_cast<uint32_t*>(sW + r * kNrcWRow)[c] = reinterpret_cast<const uint32_t*>(w + r * kNrcIn)[c];
    }
}

__device__ __forceinline__ float exp_out(float raw) { return nrc_exp_out(raw); }

// ------------------------------------------------------------------ inference
__global__ void __launch_bounds__(kNrcBlock) k_nrc_infer(NrcNet net, const NrcQuery* __restrict__ q,
                                                         const int32_t* count, int cap, double* accum, float* out_rgb)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* sIn = reinterpret_cast<__nv_bfloat16*>(smem + kSmemW) + warp * kNrcWarpRows * kNrcWRow;
    float* sOut = reinterpret_cast<float*>(smem + kSmemW + kSmemIn) + warp * kNrcWarpRows * kOutRow;
    load_weights_fwd(net.w, sW);
    __syncthreads();
    const int n = min(*count, cap);
    for (int tile = blockIdx.x * kWarps + warp; tile * kNrcWarpRows < n; tile += gridDim.x * kWarps) {
        const int i = tile * kNrcWarpRows + lane;
        const bool valid = i < n;
        NrcQuery qq;
        if (valid) qq = q[i];
        encode_row(net, qq.v, valid, sIn + lane * kNrcWRow);
        __syncwarp();
        forward_tile(sW, sIn, sOut, nullptr, 0, 0, 0);
        __syncwarp();
        if (valid && net.spectral) {   // four wavelengths: 16 spectral bins
            const float* o = sOut + lane * kOutRow;
            float e[kNrcBins];
#pragma unroll
            for (int b = 0; b < kNrcBins; ++b) e[b] = exp_out(o[b]);
            if (accum) {
                const int pix = __float_as_int(qq.v.p.w);
                const f3 c = nrc_spectral_xyz(net.tables, e, qq.v.n.w, qq.t);
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 0], nrc_contrib(c.x));
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 1], nrc_contrib(c.y));
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 2], nrc_contrib(c.z));
            }
            if (out_rgb)
                for (int b = 0; b < kNrcBins; ++b) out_rgb[kNrcBins * static_cast<int64_t>(i) + b] = e[b];
        } else if (valid) {
            const float* o = sOut + lane * kOutRow;
            const float L0 = exp_out(o[0]), L1 = exp_out(o[1]), L2 = exp_out(o[2]);
            if (accum) {
                const int pix = __float_as_int(qq.v.p.w);
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 0], nrc_contrib(qq.t.x * L0));
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 1], nrc_contrib(qq.t.y * L1));
                atomicAdd(&accum[3 * static_cast<int64_t>(pix) + 2], nrc_contrib(qq.t.z * L2));
            }
            if (out_rgb) {
                out_rgb[3 * static_cast<int64_t>(i) + 0] = L0;
                out_rgb[3 * static_cast<int64_t>(i) + 1] = L1;
                out_rgb[3 * static_cast<int64_t>(i) + 2] = L2;
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------ training
__device__ __forceinline__ int valid_rows(const int32_t* count, int first, int batch)
{
    return max(0, min(batch, *count - first));
}

__global__ void __launch_bounds__(kNrcBlock) k_nrc_train_fwd(NrcNet net, const NrcSample* __restrict__ smp,
                                                             const int32_t* count, int first, int batch,
                                                             NrcTrainBuffers T)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sW = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __nv_bfloat16* sIn = reinterpret_cast<__nv_bfloat16*>(smem + kSmemW) + warp * kNrcWarpRows * kNrcWRow;
    float* sOut = reinterpret_cast<float*>(smem + kSmemW + kSmemIn) + warp * kNrcWarpRows * kOutRow;
    load_weights_fwd(net.w, sW);
    __syncthreads();
    const int nv = valid_rows(count, first, batch);
    for (int tile = blockIdx.x * kWarps + warp; tile * kNrcWarpRows < batch; tile += gridDim.x * kWarps) {
        const int i = tile * kNrcWarpRows + lane;
        const bool valid = i < nv;
        NrcSample s;
        if (valid) s = smp[first + i];
        encode_row(net, s.v, valid, sIn + lane * kNrcWRow);
        __syncwarp();
        forward_tile(sW, sIn, sOut, T.acts, batch, static_cast<int64_t>(tile) * kNrcWarpRows, batch);
        __syncwarp();
        if (i < batch) {   // all 16 raw outputs (rgb uses 0-2)
            const float* o = sOut + lane * kOutRow;
            float4* r = reinterpret_cast<float4*>(T.raw) + 4 * static_cast<int64_t>(i);
#pragma unroll
            for (int q = 0; q < 4; ++q) r[q] = make_float4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
        }
        __syncwarp();
    }
}

// Backward pass of one warp tile.  Relative L2 loss per channel,
// (pred - target)^2 / (sg(pred)^2 + 0.01), averaged over valid rows and
// channels; its gradient times the loss scale flows back through exp, the
// output layer and the ReLU layers.  Stores the pre-activation gradients of
// every layer (bf16, [rows][64]) and the input gradient of the hash-grid
// features (fp32, [rows][32]).
__global__ void __launch_bounds__(kNrcBlock) k_nrc_train_bwd(NrcNet net, const NrcSample* __restrict__ smp,
                                                             const int32_t* count, int first, int batch,
                                                             NrcTrainBuffers T)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sWt = reinterpret_cast<__nv_bfloat16*>(smem);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    __nv_bfloat16* sIn = reinterpret_cast<__nv_bfloat16*>(smem + kSmemWt) + warp * kNrcWarpRows * kNrcWRow;
    // transposed weights: hidden layers [in][out] rows of 72, output layer [in][16] rows of 24
    for (int e = threadIdx.x; e < 5 * kNrcIn * (kNrcHid / 2); e += blockDim.x) {
        const int r = e / (kNrcHid / 2), c = e - r * (kNrcHid / 2);
        reinterpret_cast<uint32_t*>(sWt + r * kNrcWRow)[c] = reinterpret_cast<const uint32_t*>(net.wt + r * kNrcHid)[c];
    }
    __nv_bfloat16* sWt5 = sWt + 5 * kNrcIn * kNrcWRow;
    for (int e = threadIdx.x; e < kNrcIn * (kNrcOut / 2); e += blockDim.x) {
        const int r = e / (kNrcOut / 2), c = e - r * (kNrcOut / 2);
        reinterpret_cast<uint32_t*>(sWt5 + r * kBwdRow5)[c] =
            reinterpret_cast<const uint32_t*>(net.wt + nrc_w_offset(5) + r * kNrcOut)[c];
    }
    __syncthreads();
    const int nv = valid_rows(count, first, batch);
    const float norm = nv > 0 ? 1.0f / ((net.spectral ? 4.0f : 3.0f) * static_cast<float>(nv)) : 0.0f;
    float loss_acc = 0.0f;
    for (int tile = blockIdx.x * kWarps + warp; tile * kNrcWarpRows < batch; tile += gridDim.x * kWarps) {
        const int64_t row0 = static_cast<int64_t>(tile) * kNrcWarpRows;
        const int i = static_cast<int>(row0) + lane;
        // output gradient of this lane's row into its shared-memory row (16 columns)
        float d[kNrcBins];
#pragma unroll
        for (int b = 0; b < kNrcBins; ++b) d[b] = 0.0f;
        if (i < nv) {
            const NrcSample s = smp[first + i];
            const float4* rr = reinterpret_cast<const float4*>(T.raw) + 4 * static_cast<int64_t>(i);
            float raw[kNrcBins];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = rr[q];
                raw[4 * q] = v.x; raw[4 * q + 1] = v.y; raw[4 * q + 2] = v.z; raw[4 * q + 3] = v.w;
            }
            loss_acc += nrc_output_grad(net.spectral, s, raw, norm, d);
        }
        uint32_t* row = reinterpret_cast<uint32_t*>(sIn + lane * kNrcWRow);
#pragma unroll
        for (int k = 0; k < 8; ++k) row[k] = pack_bf16(d[2 * k], d[2 * k + 1]);
        if (i < batch) {   // output-layer gradient for the weight gradient (first 16 columns)
            uint4* dst = reinterpret_cast<uint4*>(T.dz + static_cast<int64_t>(5) * batch * kNrcIn + static_cast<int64_t>(i) * kNrcIn);
            const uint4* src = reinterpret_cast<const uint4*>(row);
            dst[0] = src[0];
            dst[1] = src[1];
        }
        __syncwarp();
        // A fragments of the output gradient: one k-slice of 16
        uint32_t a[2][4][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const __nv_bfloat16* r0 = sIn + (16 * mt + g) * kNrcWRow + 2 * t;
            const __nv_bfloat16* r1 = r0 + 8 * kNrcWRow;
            a[mt][0][0] = ld32(r0);
            a[mt][0][1] = ld32(r1);
            a[mt][0][2] = ld32(r0 + 8);
            a[mt][0][3] = ld32(r1 + 8);
        }
        for (int l = kNrcLayers - 1; l >= 0; --l) {
            const int kslices = l == kNrcLayers - 1 ? 1 : 4;
            const __nv_bfloat16* Wt = l == kNrcLayers - 1 ? sWt5 : sWt + l * kNrcIn * kNrcWRow;
            const int wrow = l == kNrcLayers - 1 ? kBwdRow5 : kNrcWRow;
            float c[2][8][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt)
#pragma unroll
                for (int j = 0; j < 8; ++j) c[mt][j][0] = c[mt][j][1] = c[mt][j][2] = c[mt][j][3] = 0.0f;
#pragma unroll
            for (int j = 0; j < 8; ++j)
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    if (ks < kslices) {
                        const __nv_bfloat16* wr = Wt + (8 * j + g) * wrow + 16 * ks + 2 * t;
                        const uint32_t b0 = ld32(wr), b1 = ld32(wr + 8);
                        mma_bf16(c[0][j], a[0][ks], b0, b1);
                        mma_bf16(c[1][j], a[1][ks], b0, b1);
                    }
                }
            if (l == 0) {   // gradient of the input: keep the 32 hash-grid columns
#pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    const int64_t r0 = row0 + 16 * mt + g, r1 = r0 + 8;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int col = 8 * j + 2 * t;
                        if (r0 < batch) *reinterpret_cast<float2*>(T.dx + r0 * 32 + col) = make_float2(c[mt][j][0], c[mt][j][1]);
                        if (r1 < batch) *reinterpret_cast<float2*>(T.dx + r1 * 32 + col) = make_float2(c[mt][j][2], c[mt][j][3]);
                    }
                }
                break;
            }
            // through the ReLU of activation l: gradient of the pre-activation of layer l-1
            const __nv_bfloat16* H = T.acts + static_cast<int64_t>(l) * batch * kNrcIn;
            __nv_bfloat16* DZ = T.dz + static_cast<int64_t>(l - 1) * batch * kNrcIn;
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int64_t r0 = row0 + 16 * mt + g, r1 = r0 + 8;
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = 8 * j + 2 * t;
                    const float2 h0 = r0 < batch ? unpack_bf16(ld32(H + r0 * kNrcIn + col)) : make_float2(0.0f, 0.0f);
                    const float2 h1 = r1 < batch ? unpack_bf16(ld32(H + r1 * kNrcIn + col)) : make_float2(0.0f, 0.0f);
                    c[mt][j][0] = h0.x > 0.0f ? c[mt][j][0] : 0.0f;
                    c[mt][j][1] = h0.y > 0.0f ? c[mt][j][1] : 0.0f;
                    c[mt][j][2] = h1.x > 0.0f ? c[mt][j][2] : 0.0f;
                    c[mt][j][3] = h1.y > 0.0f ? c[mt][j][3] : 0.0f;
                }
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    a[mt][ks][0] = pack_bf16(c[mt][2 * ks][0], c[mt][2 * ks][1]);
                    a[mt][ks][1] = pack_bf16(c[mt][2 * ks][2], c[mt][2 * ks][3]);
                    a[mt][ks][2] = pack_bf16(c[mt][2 * ks + 1][0], c[mt][2 * ks + 1][1]);
                    a[mt][ks][3] = pack_bf16(c[mt][2 * ks + 1][2], c[mt][2 * ks + 1][3]);
                    const int col = 16 * ks + 2 * t;
                    if (r0 < batch) {
                        *reinterpret_cast<uint32_t*>(DZ + r0 * kNrcIn + col) = a[mt][ks][0];
                        *reinterpret_cast<uint32_t*>(DZ + r0 * kNrcIn + col + 8) = a[mt][ks][2];
                    }
                    if (r1 < batch) {
                        *reinterpret_cast<uint32_t*>(DZ + r1 * kNrcIn + col) = a[mt][ks][1];
                        *reinterpret_cast<uint32_t*>(DZ + r1 * kNrcIn + col + 8) = a[mt][ks][3];
                    }
                }
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(0xFFFFFFFFu, loss_acc, o);
    if (lane == 0 && loss_acc != 0.0f) atomicAdd(T.loss, loss_acc);
}

// Weight gradients dW_l[o][i] = sum over rows of dz_l[row][o] * act_l[row][i],
// on the tensor cores: per block a chunk of kWgRows rows of both operands is
// staged in shared memory (rows padded to 72 bf16), each warp owns 16 output
// rows o and all 64 inputs i, and the A (dz transposed) and B (act) fragments
// come from ldmatrix.trans of the row-major tiles.  fp32 accumulators, one
// atomic per weight and block.
constexpr int kWgRows = 256;
constexpr int kSmemWg = 2 * kWgRows * kNrcWRow * 2;   // 73728 B

__device__ __forceinline__ void ldsm_x4_trans(const __nv_bfloat16* p, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                              uint32_t& r3)
{
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(a));
}

__global__ void __launch_bounds__(kNrcBlock) k_nrc_wgrad(NrcTrainBuffers T, int batch, float* wg)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __nv_bfloat16* sZ = reinterpret_cast<__nv_bfloat16*>(smem);                 // [kWgRows][72]: dz
    __nv_bfloat16* sX = sZ + kWgRows * kNrcWRow;                                 // [kWgRows][72]: act
    const int l = blockIdx.y;
    const int outs = nrc_w_rows(l);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int m0 = 16 * warp;                      // this warp's output rows
    const bool active = m0 < outs;
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
    const __nv_bfloat16* dzl = T.dz + static_cast<int64_t>(l) * batch * kNrcIn;
    const __nv_bfloat16* acl = T.acts + static_cast<int64_t>(l) * batch * kNrcIn;
    // ldmatrix row addresses: lane -> (8x8 matrix q = lane / 8, row r = lane % 8)
    const int q = lane >> 3, r = lane & 7;
    for (int r0 = blockIdx.x * kWgRows; r0 < batch; r0 += gridDim.x * kWgRows) {
        const int rows = min(kWgRows, batch - r0);
        __syncthreads();
        for (int e = threadIdx.x; e < kWgRows * (kNrcIn / 8); e += blockDim.x) {   // 16-byte pieces
            const int rr = e >> 3, c = (e & 7) * 8;
            uint4 z = make_uint4(0u, 0u, 0u, 0u), a = z;
            if (rr < rows) {
                const int64_t off = static_cast<int64_t>(r0 + rr) * kNrcIn + c;
                if (c < outs) z = *reinterpret_cast<const uint4*>(dzl + off);
                a = *reinterpret_cast<const uint4*>(acl + off);
            }
            *reinterpret_cast<uint4*>(sZ + rr * kNrcWRow + c) = z;
            *reinterpret_cast<uint4*>(sX + rr * kNrcWRow + c) = a;
        }
        __syncthreads();
        if (active) {
#pragma unroll 2
            for (int k0 = 0; k0 < kWgRows; k0 += 16) {
                // A = dz^T (16 outputs x 16 rows): matrices (m0, k0) (m0+8, k0) (m0, k0+8) (m0+8, k0+8)
                uint32_t a[4];
                ldsm_x4_trans(sZ + (k0 + ((q >> 1) << 3) + r) * kNrcWRow + m0 + ((q & 1) << 3), a[0], a[1], a[2], a[3]);
#pragma unroll
                for (int jp = 0; jp < 4; ++jp) {
                    // B = act (16 rows x 8 inputs) for n-tiles 2jp, 2jp+1: (k0, n) (k0+8, n) (k0, n+8) (k0+8, n+8)
                    uint32_t b0, b1, b2, b3;
                    ldsm_x4_trans(sX + (k0 + ((q & 1) << 3) + r) * kNrcWRow + 16 * jp + ((q >> 1) << 3), b0, b1, b2, b3);
                    mma_bf16(acc[2 * jp], a, b0, b1);
                    mma_bf16(acc[2 * jp + 1], a, b2, b3);
                }
            }
        }
    }
    if (!active) return;
    float* dst = wg + nrc_w_offset(l);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int col = 8 * j + 2 * t;
        atomicAdd(dst + (m0 + g) * kNrcIn + col, acc[j][0]);
        atomicAdd(dst + (m0 + g) * kNrcIn + col + 1, acc[j][1]);
        atomicAdd(dst + (m0 + g + 8) * kNrcIn + col, acc[j][2]);
        atomicAdd(dst + (m0 + g + 8) * kNrcIn + col + 1, acc[j][3]);
    }
}

// Hash-table gradients: the input gradient of each level's two features,
// spread over its 8 corners with the trilinear weights.
__global__ void k_nrc_hash_bwd(NrcNet net, const NrcSample* __restrict__ smp, const int32_t* count, int first,
                               int batch, NrcTrainBuffers T, float* tg)
{
    const int nv = valid_rows(count, first, batch);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv * net.grid.levels; i += gridDim.x * blockDim.x) {
        const int row = i / net.grid.levels, l = i - row * net.grid.levels;
        float u[3];
        nrc_unit_pos(net.grid, smp[first + row].v.p, u);
        uint32_t idx[8];
        float w[8];
        nrc_level_corners(net.grid, l, u[0], u[1], u[2], idx, w);
        const float2 d = *reinterpret_cast<const float2*>(T.dx + static_cast<int64_t>(row) * 32 + 2 * l);
        if (d.x == 0.0f && d.y == 0.0f) continue;
#pragma unroll
        for (int c = 0; c < 8; ++c)   // one vector atomic per corner (both features)
            atomicAdd(reinterpret_cast<float2*>(tg) + idx[c], make_float2(w[c] * d.x, w[c] * d.y));
    }
}

// Adam (Kingma and Ba 2015) on the MLP weights; publishes the bf16 copies in
// both layouts and clears the gradient.
__global__ void k_nrc_adam_mlp(float* p, float* m, float* v, float* gr, __nv_bfloat16* wbf, __nv_bfloat16* wtbf,
                               float lr_t, float b1, float b2, float eps, float inv_scale, int update)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kNrcParams; e += gridDim.x * blockDim.x) {
        float w = p[e];
        const float gg = gr[e] * inv_scale;
        if (update && gg - gg == 0.0f) {   // a non-finite gradient element skips its update
            const float mm = b1 * m[e] + (1.0f - b1) * gg;
            const float vv = b2 * v[e] + (1.0f - b2) * gg * gg;
            m[e] = mm;
            v[e] = vv;
            w -= lr_t * mm / (sqrtf(vv) + eps);
            p[e] = w;
        }
        if (update) gr[e] = 0.0f;
        const int l = min(e / (kNrcHid * kNrcIn), kNrcLayers - 1);
        const int local = e - nrc_w_offset(l);
        const int rows = nrc_w_rows(l);
        const int o = local / kNrcIn, i = local - o * kNrcIn;
        const __nv_bfloat16 b = __float2bfloat16_rn(w);
        wbf[e] = b;
        wtbf[nrc_w_offset(l) + i * rows + o] = b;
    }
}

// Adam on the hash tables, lazily: entries without gradient in this step keep
// their moments.  Publishes the half copy of updated entries.
__global__ void k_nrc_adam_table(float* p, float* m, float* v, float* gr, __half2* th, int64_t entries, float lr_t,
                                 float b1, float b2, float eps, float inv_scale, int update)
{
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < entries;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        float2 w = reinterpret_cast<float2*>(p)[e];
        if (update) {
            const float2 g2 = reinterpret_cast<float2*>(gr)[e];
            if (g2.x == 0.0f && g2.y == 0.0f) continue;
            float2 m2 = reinterpret_cast<float2*>(m)[e], v2 = reinterpret_cast<float2*>(v)[e];
            const float gx = g2.x * inv_scale, gy = g2.y * inv_scale;
            reinterpret_cast<float2*>(gr)[e] = make_float2(0.0f, 0.0f);
            if (!(gx - gx == 0.0f && gy - gy == 0.0f)) continue;   // non-finite: skip the entry's update
            m2.x = b1 * m2.x + (1.0f - b1) * gx;
            m2.y = b1 * m2.y + (1.0f - b1) * gy;
            v2.x = b2 * v2.x + (1.0f - b2) * gx * gx;
            v2.y = b2 * v2.y + (1.0f - b2) * gy * gy;
            w.x -= lr_t * m2.x / (sqrtf(v2.x) + eps);
            w.y -= lr_t * m2.y / (sqrtf(v2.y) + eps);
            reinterpret_cast<float2*>(m)[e] = m2;
            reinterpret_cast<float2*>(v)[e] = v2;
            reinterpret_cast<float2*>(p)[e] = w;
        }
        th[e] = __floats2half2_rn(w.x, w.y);
    }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x)
{
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float u01(uint32_t h) { return (static_cast<float>(h >> 8) + 0.5f) * (1.0f / 16777216.0f); }

// Initial state: tables U(-1e-4, 1e-4), weights He-uniform U(+-sqrt(6 / 64)).
__global__ void k_nrc_init(float* table, int64_t tfloats, float* w, uint32_t seed)
{
    const int64_t n = tfloats + kNrcParams;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < n;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const float u = u01(mix32(static_cast<uint32_t>(e) * 0x9E3779B9u ^ mix32(seed ^ static_cast<uint32_t>(e >> 32))));
        if (e < tfloats) table[e] = (2.0f * u - 1.0f) * 1e-4f;
        else w[e - tfloats] = (2.0f * u - 1.0f) * 0.30618622f;
    }
}

int blocks_for(int64_t n, int per, int cap) { return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, cap))); }

}  // namespace

cudaError_t nrc_publish(const NrcParams& P, cudaStream_t st)
{
    k_nrc_adam_mlp<<<blocks_for(kNrcParams, 256, 1024), 256, 0, st>>>(P.w_f32, P.w_m, P.w_v, P.w_g, P.w_bf, P.wt_bf,
                                                                       0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0);
    k_nrc_adam_table<<<blocks_for(P.table_floats / 2, 256, 4096), 256, 0, st>>>(
        P.table_f32, P.table_m, P.table_v, P.table_g, P.table_h, P.table_floats / 2, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0);
    return cudaGetLastError();
}

cudaError_t nrc_init_params(const NrcParams& P, uint64_t seed, cudaStream_t st)
{
    k_nrc_init<<<2048, 256, 0, st>>>(P.table_f32, P.table_floats, P.w_f32, static_cast<uint32_t>(seed ^ (seed >> 32)));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return nrc_publish(P, st);
}

static cudaError_t set_attrs()
{
    cudaError_t e = cudaFuncSetAttribute(k_nrc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemW + kSmemIn + kSmemOut);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_nrc_train_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemW + kSmemIn + kSmemOut);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_nrc_train_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemWt + kSmemIn);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_nrc_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemWg);
    return e;
}

cudaError_t nrc_infer(const NrcNet& net, const NrcQuery* q, const int32_t* count, int cap, double* accum,
                      float* out_rgb, int sm_count, cudaStream_t st)
{
    cudaError_t e = set_attrs();
    if (e != cudaSuccess) return e;
    const int tiles = (cap + kNrcWarpRows - 1) / kNrcWarpRows;
    const int grid = std::max(1, std::min((tiles + kWarps - 1) / kWarps, sm_count * 4));
    k_nrc_infer<<<grid, kNrcBlock, kSmemW + kSmemIn + kSmemOut, st>>>(net, q, count, cap, accum, out_rgb);
    return cudaGetLastError();
}

cudaError_t nrc_train_step(const NrcNet& net, const NrcParams& P, const NrcSample* samples, const int32_t* count,
                           int first, int batch, const NrcTrainBuffers& T, float lr, int step, int sm_count,
                           cudaStream_t st, bool apply, int* tc_err)
{
    cudaError_t e = set_attrs();
    if (e != cudaSuccess) return e;
    if (tc_err) {   // forward and backward on the tcgen05 tensor cores
        e = nrc_train_fwd_bwd_tc(net, samples, count, first, batch, T, tc_err, sm_count, st);
        if (e != cudaSuccess) return e;
    } else {
        const int tiles = (batch + kNrcWarpRows - 1) / kNrcWarpRows;
        const int grid = std::max(1, std::min((tiles + kWarps - 1) / kWarps, sm_count * 2));
        k_nrc_train_fwd<<<grid, kNrcBlock, kSmemW + kSmemIn + kSmemOut, st>>>(net, samples, count, first, batch, T);
        k_nrc_train_bwd<<<grid, kNrcBlock, kSmemWt + kSmemIn, st>>>(net, samples, count, first, batch, T);
    }
    k_nrc_wgrad<<<dim3(std::min((batch + kWgRows - 1) / kWgRows, 32), kNrcLayers), kNrcBlock, kSmemWg, st>>>(T, batch, P.w_g);
    k_nrc_hash_bwd<<<blocks_for(static_cast<int64_t>(batch) * net.grid.levels, 256, sm_count * 8), 256, 0, st>>>(
        net, samples, count, first, batch, T, P.table_g);
    if (!apply) return cudaGetLastError();   // gradients stay in P.w_g / P.table_g (scaled by kNrcLossScale)
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-15f;
    const double t = static_cast<double>(step);
    const float lr_t = static_cast<float>(lr * std::sqrt(1.0 - std::pow(b2, t)) / (1.0 - std::pow(b1, t)));
    k_nrc_adam_mlp<<<blocks_for(kNrcParams, 256, 1024), 256, 0, st>>>(P.w_f32, P.w_m, P.w_v, P.w_g, P.w_bf, P.wt_bf,
                                                                       lr_t, b1, b2, eps, 1.0f / kNrcLossScale, 1);
    k_nrc_adam_table<<<blocks_for(P.table_floats / 2, 256, sm_count * 16), 256, 0, st>>>(
        P.table_f32, P.table_m, P.table_v, P.table_g, P.table_h, P.table_floats / 2, lr_t, b1, b2, eps,
        1.0f / kNrcLossScale, 1);
    return cudaGetLastError();
}

}  // namespace ar
