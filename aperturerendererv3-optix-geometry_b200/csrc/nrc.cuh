// nrc.cuh -- the learned radiance cache (extension; the reference has none):
// a multiresolution hash-grid encoding of position (Mueller et al., "Instant
// neural graphics primitives", 2022), a degree-4 spherical-harmonics encoding
// of direction, roughness, diffuse albedo and normal, fed to a 64-wide MLP of
// 5 hidden ReLU layers and a 3-channel exp output (Mueller et al., "Real-time
// neural radiance caching for path tracing", 2021).  Weights and activations
// are bf16 with fp32 accumulation (mma.sync m16n8k16); the hash tables are
// half floats with fp32 master copies, Adam moments and gradients.
//
// Network input (64 values): [0, 32) hash-grid features (16 levels x 2),
// [32, 48) spherical harmonics of the outgoing direction, 48 roughness,
// [49, 52) albedo, [52, 55) normal * 0.5 + 0.5, 55 the constant 1 (the first
// layer's bias), [56, 64) zero.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "spectral.cuh"

namespace ar {

constexpr int kNrcIn = 64, kNrcHid = 64, kNrcOut = 16;
constexpr int kNrcLayers = 6;                       // 5 hidden transforms + output
constexpr int kNrcParams = 5 * kNrcHid * kNrcIn + kNrcOut * kNrcHid;  // 21504
constexpr int kNrcMaxLevels = 16;
constexpr int kNrcFeatures = 2;
constexpr int kNrcWarpRows = 32;                    // samples per warp tile (2 m16 tiles)
constexpr int kNrcBlock = 128;                      // 4 warps
constexpr int kNrcWRow = 72;                        // padded bf16 row of a weight matrix in shared memory
constexpr float kNrcLossScale = 128.0f;

// offset (elements) of layer l's weights in the packed [out][in] arrays
__host__ __device__ constexpr int nrc_w_offset(int l) { return l * kNrcHid * kNrcIn; }
__host__ __device__ constexpr int nrc_w_rows(int l) { return l == kNrcLayers - 1 ? kNrcOut : kNrcHid; }

// Hash grid geometry (host-computed).
struct NrcGrid {
    int32_t levels;
    uint32_t mask;                 // table entries per level - 1 (power of two)
    int32_t res[kNrcMaxLevels];    // grid resolution of each level
    int32_t dense[kNrcMaxLevels];  // 1: (res+1)^3 <= entries, direct indexing
    float bmin[3], inv_ext[3];     // scene box -> [0, 1]^3
};

// Four-wavelength mode: the 16 network outputs, through exp, are the outgoing
// spectral radiance at 16 wavelength bins of 26.25 nm over [360, 780] nm (bin
// centres 373.125 + 26.25 b), relative to the D65 weight d65_norm of the
// wavelength (the factor the tracer applies to emission, ~0.01), which keeps
// the targets near 1; a wavelength's value interpolates linearly between the
// two nearest centres (clamped to the first and last).
constexpr int kNrcBins = 16;
constexpr float kNrcLambda0 = 360.0f, kNrcBinWidth = 26.25f;

__host__ __device__ __forceinline__ void nrc_bin_weights(float lambda, int* b0, float* f)
{
    float x = (lambda - kNrcLambda0) / kNrcBinWidth - 0.5f;
    x = x > 0.0f ? x : 0.0f;   // not-a-number as bin 0
    x = x < static_cast<float>(kNrcBins - 1) ? x : static_cast<float>(kNrcBins - 1);
    int b = static_cast<int>(floorf(x));
    b = b < 0 ? 0 : (b > kNrcBins - 2 ? kNrcBins - 2 : b);
    *b0 = b;
    *f = x - static_cast<float>(b);
}

// The XYZ a four-wavelength path gets from a cache prediction: the hero
// wavelength's rotation set lambda_i, the predicted radiance L(lambda_i) from
// the exp'd bins e[16], the path's throughput T_i per wavelength, weighted as
// the path's own estimate sum_i XYZ(lambda_i) L_i / sum_j p(lambda_j).
__host__ __device__ __forceinline__ f3 nrc_spectral_xyz(const float* tables, const float* e, float hero, float4 T)
{
    const float t[4] = {T.x, T.y, T.z, T.w};
    float ps = 0.0f;
    f3 acc = mk(0.0f, 0.0f, 0.0f);
    for (int w = 0; w < 4; ++w) {
        const float lw = rotate_lambda(hero, w);
        ps += pdf_cie1931(lw);
        int b;
        float f;
        nrc_bin_weights(lw, &b, &f);
        const float L = ((1.0f - f) * e[b] + f * e[b + 1]) * d65_norm(tables, lw);
        acc = acc + cmf_xyz(tables, lw) * (t[w] * L);
    }
    return acc / ps;
}

// Device view of the network state.
struct NrcNet {
    NrcGrid grid;
    const __half2* table;          // levels x entries features (forward copy)
    const __nv_bfloat16* w;        // [out][in] per layer, packed
    const __nv_bfloat16* wt;       // [in][out] per layer, packed (backward)
    int32_t spectral;              // 0: RGB outputs 0-2; 4: four wavelengths, 16 spectral bins
    const float* tables;           // spectral tables of the scene (colour matching functions), mode 4
};

// One vertex as the cache sees it: 4 x float4 =
//   (pos.xyz, aux) (dir.xyz, roughness) (normal.xyz, aux) (albedo.xyz, aux)
struct NrcVertex {
    float4 p, d, n, a;
};

// Records that the path tracer writes for the cache.
struct NrcQuery {                  // a path terminated into the cache
    NrcVertex v;                   // v.p.w: pixel (int bits); four wavelengths: v.n.w hero wavelength
    float4 t;                      // throughput rgb, or of wavelengths 0-3
};
struct NrcTrainVertex {            // a vertex of a training path (v.n.w: hero wavelength, mode 4)
    NrcVertex v;
    float4 t;                      // throughput arriving at the vertex (rgb or wavelengths 0-3)
    float4 lb;                     // radiance gathered before the vertex
};
struct NrcSample {                 // a training sample: vertex + target radiance
    NrcVertex v;                   // target radiance r, g, b (wavelengths 0-2) in v.p.w, v.n.w, v.a.w
    float4 x;                      // four wavelengths: x.x target of wavelength 3, x.y hero wavelength;
                                   // a negative target (no throughput reached it) is left out of the loss
};

// Per-frame parameters of the cache inside the wavefront (FrameParams.nrc).
struct NrcFrame {
    int32_t enabled;
    int32_t spectral;              // 0 RGB, 4 four wavelengths (the cache's mode)
    int32_t stride, offset;        // sample 0 of pixel p trains when (p + offset) % stride == 0
    int32_t max_train_vertices;    // vertices recorded per training path
    float spread_c;                // terminate when spread^2 > c * a0
    int32_t query_cap, sample_cap, slots;
    NrcQuery* queries;
    int32_t* query_count;
    NrcTrainVertex* train_vertices;  // slots x max_train_vertices
    int32_t* slot_count;             // vertices recorded per slot
    NrcSample* samples;
    int32_t* sample_count;
};

__host__ __device__ __forceinline__ bool nrc_train_slot(const NrcFrame& f, int pixel, int* slot)
{
    const int q = pixel + f.offset;
    if (q % f.stride != 0) return false;
    *slot = q / f.stride;
    return *slot < f.slots;
}

__device__ __forceinline__ float nrc_exp_out(float raw) { return expf(fminf(raw, 15.0f)); }

// A cache contribution to a pixel, bounded as the tracer bounds a sample
// (RADIANCE_CLAMP 1e3 per channel, not-a-number as 0; render.cuh:966-969).
__device__ __forceinline__ double nrc_contrib(float v)
{
    return (v >= 0.0f) ? static_cast<double>(fminf(v, 1.0e3f)) : 0.0;
}

// Gradient (times the loss scale) of the training loss with respect to the 16
// raw outputs of one sample, and the sample's loss, normalised by `norm`.
// RGB: relative L2 per channel (pred - target)^2 / (sg(pred)^2 + 0.01) with
// pred = exp(raw); four wavelengths: the same per wavelength with pred the
// bins interpolated at the wavelength, targets below zero left out.
__device__ __forceinline__ float nrc_output_grad(int spectral, const NrcSample& s, const float* raw, float norm,
                                                 float* d)
{
    float loss = 0.0f;
#pragma unroll
    for (int b = 0; b < kNrcBins; ++b) d[b] = 0.0f;
    if (spectral) {
        float e[kNrcBins];
#pragma unroll
        for (int b = 0; b < kNrcBins; ++b) e[b] = nrc_exp_out(raw[b]);
        const float tg[4] = {s.v.p.w, s.v.n.w, s.v.a.w, s.x.x};
        for (int w = 0; w < 4; ++w) {
            if (tg[w] < 0.0f) continue;   // no throughput reached this wavelength
            int b;
            float f;
            nrc_bin_weights(rotate_lambda(s.x.y, w), &b, &f);
            const float pred = (1.0f - f) * e[b] + f * e[b + 1];
            const float den = pred * pred + 0.01f;
            const float diff = pred - tg[w];
            loss += diff * diff / den * norm;
            const float g = (2.0f * diff / den) * norm * kNrcLossScale;
            d[b] += g * (1.0f - f) * e[b];
            d[b + 1] += g * f * e[b + 1];
        }
    } else {
        const float tg[3] = {s.v.p.w, s.v.n.w, s.v.a.w};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float pred = nrc_exp_out(raw[c]);
            const float den = pred * pred + 0.01f;
            const float diff = pred - tg[c];
            loss += diff * diff / den * norm;
            d[c] = (2.0f * diff / den) * norm * pred * kNrcLossScale;
        }
    }
    return loss;
}

// Real spherical harmonics up to degree 3 (16 coefficients) of a unit
// direction, in the usual (l, m) order with the standard normalisation.
__host__ __device__ __forceinline__ void nrc_sh16(float x, float y, float z, float* o)
{
    const float xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.48860251190291987f * y;
    o[2] = 0.48860251190291987f * z;
    o[3] = -0.48860251190291987f * x;
    o[4] = 1.0925484305920792f * x * y;
    o[5] = -1.0925484305920792f * y * z;
    o[6] = 0.94617469575755997f * zz - 0.31539156525251999f;
    o[7] = -1.0925484305920792f * x * z;
    o[8] = 0.54627421529603959f * (xx - yy);
    o[9] = 0.59004358992664352f * y * (-3.0f * xx + yy);
    o[10] = 2.8906114426405538f * x * y * z;
    o[11] = 0.45704579946446572f * y * (1.0f - 5.0f * zz);
    o[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    o[13] = 0.45704579946446572f * x * (1.0f - 5.0f * zz);
    o[14] = 1.4453057213202769f * z * (xx - yy);
    o[15] = 0.59004358992664352f * x * (-xx + 3.0f * yy);
}

// Grid cell and trilinear weights of one level: 8 table indices (corner c =
// bit0 x, bit1 y, bit2 z) and their weights.  The spatial hash is the XOR of
// the integer coordinates times the primes 1, 2654435761, 805459861
// (Teschner et al. 2003, as instant-ngp uses it).
__host__ __device__ __forceinline__ void nrc_level_corners(const NrcGrid& g, int l, float px, float py, float pz,
                                                          uint32_t* idx, float* w)
{
    const int r = g.res[l];
    const float fx = px * static_cast<float>(r), fy = py * static_cast<float>(r), fz = pz * static_cast<float>(r);
    int ix = static_cast<int>(floorf(fx)), iy = static_cast<int>(floorf(fy)), iz = static_cast<int>(floorf(fz));
    ix = ix < 0 ? 0 : (ix > r - 1 ? r - 1 : ix);
    iy = iy < 0 ? 0 : (iy > r - 1 ? r - 1 : iy);
    iz = iz < 0 ? 0 : (iz > r - 1 ? r - 1 : iz);
    float tx = fx - static_cast<float>(ix), ty = fy - static_cast<float>(iy), tz = fz - static_cast<float>(iz);
    tx = tx < 0.0f ? 0.0f : (tx > 1.0f ? 1.0f : tx);
    ty = ty < 0.0f ? 0.0f : (ty > 1.0f ? 1.0f : ty);
    tz = tz < 0.0f ? 0.0f : (tz > 1.0f ? 1.0f : tz);
    const uint32_t stride = static_cast<uint32_t>(r + 1);
    for (int c = 0; c < 8; ++c) {
        const uint32_t cx = static_cast<uint32_t>(ix + (c & 1)), cy = static_cast<uint32_t>(iy + ((c >> 1) & 1)),
                       cz = static_cast<uint32_t>(iz + ((c >> 2) & 1));
        uint32_t h;
        if (g.dense[l]) h = cx + cy * stride + cz * stride * stride;
        else h = (cx * 1u) ^ (cy * 2654435761u) ^ (cz * 805459861u);
        idx[c] = (h & g.mask) + static_cast<uint32_t>(l) * (g.mask + 1u);
        w[c] = ((c & 1) ? tx : 1.0f - tx) * (((c >> 1) & 1) ? ty : 1.0f - ty) * (((c >> 2) & 1) ? tz : 1.0f - tz);
    }
}

__host__ __device__ __forceinline__ void nrc_unit_pos(const NrcGrid& g, const float4& p, float* u)
{
    u[0] = (p.x - g.bmin[0]) * g.inv_ext[0];
    u[1] = (p.y - g.bmin[1]) * g.inv_ext[1];
    u[2] = (p.z - g.bmin[2]) * g.inv_ext[2];
    for (int k = 0; k < 3; ++k) u[k] = u[k] > 0.0f ? (u[k] < 1.0f ? u[k] : 1.0f) : 0.0f;   // not-a-number as 0
}

// A recorded vertex the cache may train on: every input finite.
__host__ __device__ __forceinline__ bool nrc_vertex_finite(const NrcVertex& v)
{
    const float s = (v.p.x - v.p.x) + (v.p.y - v.p.y) + (v.p.z - v.p.z) + (v.d.x - v.d.x) + (v.d.y - v.d.y) +
                    (v.d.z - v.d.z) + (v.n.x - v.n.x) + (v.n.y - v.n.y) + (v.n.z - v.n.z) + (v.n.w - v.n.w) +
                    (v.a.x - v.a.x) + (v.a.y - v.a.y) + (v.a.z - v.a.z);
    return s == 0.0f;   // x - x is 0 for finite x, not-a-number for infinities and not-a-number
}

// Host launchers (nrc.cu).
struct NrcTrainBuffers {
    __nv_bfloat16* acts;     // kNrcLayers x [batch][64]: input and hidden activations
    float* raw;              // [batch][16] raw outputs (pre-exp): rgb in 0-2, or the 16 spectral bins
    __nv_bfloat16* dz;       // kNrcLayers x [batch][64]: gradients of the pre-activations (scaled)
    float* dx;               // [batch][32] gradient of the hash-grid features (scaled)
    float* loss;             // [1] sum of the relative L2 loss over the step
};

struct NrcParams {           // trainable state (fp32 master, moments, gradients)
    float* table_f32;
    float* table_m;
    float* table_v;
    float* table_g;
    __half2* table_h;        // forward copy
    float* w_f32;
    float* w_m;
    float* w_v;
    float* w_g;
    __nv_bfloat16* w_bf;
    __nv_bfloat16* wt_bf;
    int64_t table_floats;    // levels x entries x 2
};

cudaError_t nrc_init_params(const NrcParams& P, uint64_t seed, cudaStream_t st);
cudaError_t nrc_publish(const NrcParams& P, cudaStream_t st);   // bf16 / half copies of the fp32 masters
cudaError_t nrc_infer(const NrcNet& net, const NrcQuery* q, const int32_t* count, int cap, double* accum,
                      float* out_rgb, int sm_count, cudaStream_t st);
// The same inference on the tcgen05 tensor cores (nrc_tc.cu); *err gets bit 1
// when a CTA's MMA wait runs out.
cudaError_t nrc_infer_tc(const NrcNet& net, const NrcQuery* q, const int32_t* count, int cap, double* accum,
                         float* out_rgb, int* err, int sm_count, cudaStream_t st);
cudaError_t nrc_train_step(const NrcNet& net, const NrcParams& P, const NrcSample* samples, const int32_t* count,
                           int first, int batch, const NrcTrainBuffers& T, float lr, int step, int sm_count,
                           cudaStream_t st, bool apply = true, int* tc_err = nullptr);
// The training forward and backward passes on the tcgen05 tensor cores
// (nrc_tc.cu); *err gets bit 2 (forward) or 3 (backward) when an MMA wait runs out.
cudaError_t nrc_train_fwd_bwd_tc(const NrcNet& net, const NrcSample* samples, const int32_t* count, int first,
                                 int batch, const NrcTrainBuffers& T, int* err, int sm_count, cudaStream_t st);

}  // namespace ar
