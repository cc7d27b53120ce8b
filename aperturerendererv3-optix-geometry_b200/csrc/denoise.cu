// denoise.cu -- the screen-space denoiser's bilateral filter and frame
// recording from caller-supplied primary hits.
//
// k_dn_ttest and k_dn_filter replace denoise::Bilateral16x16<7>
// (core/denoise/denoise.cuh:359-443) in two passes.  A CTA of either pass
// handles a 32 x 8 tile and stages its 46 x 22 window (radius 7, coordinates
// clamped at the borders) once in shared memory as per-pixel terms, one warp
// per tile row, so a warp's 32 lanes read 32 consecutive words.  Pass 1
// evaluates the skewness-corrected Welch t-test of all 225 taps from the
// pixels' halves of ComputeTStatistic / ComputeWelchNu (12 words per staged
// pixel, four CTAs per SM) and writes a 225-bit mask per pixel; its square
// root is replaced by an exact threshold compare.  Pass 2 stages log(1 + c)
// and the guide values (14 words, three CTAs per SM) and sums the taps whose
// bit is set, in the reference's order; a failing tap has weight 0 and costs
// nothing.  Every term is computed with the reference's expressions and
// order of operations, so the weights are the reference's (with the fixed
// exp/log of detmath.h); the guide weight's half-precision differences round
// to half as the reference's device code does (__hsub).
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "../../include/aperture_b200.h"
#include "denoise.cuh"
#include "detmath.h"
#include "t_quantile_table.h"

namespace ar {

ar_status set_error(ar_status st, const std::string& msg);

namespace {

constexpr int kDnRadius = 7;
constexpr int kTileX = 32, kTileY = 8;
constexpr int kWinX = kTileX + 2 * kDnRadius, kWinY = kTileY + 2 * kDnRadius;
constexpr int kWin = kWinX * kWinY;
constexpr int kTaps = (2 * kDnRadius + 1) * (2 * kDnRadius + 1);

// FilterParams (denoise.cuh:13-32), the same float expressions
constexpr float kInvAlbedo = 1.0f / (2.0f * 1.0f * 1.0f);
constexpr float kInvNormal = 1.0f / (2.0f * 0.5f * 0.5f);
constexpr float kInvDepth = 1.0f / (2.0f * 0.25f * 0.25f);
constexpr float kInvMetallic = 1.0f / (2.0f * 0.5f * 0.5f);
constexpr float kInvRough = 1.0f / (2.0f * 0.5f * 0.5f);
constexpr float kInvShading = 1.0f / (2.0f * 0.1f * 0.1f);
constexpr float kInvSpatial = 1.0f / (2.0f * 2.0f * 2.0f);
constexpr float kCenterEps = 1.0e-6f;

// Shared-memory windows, structure of arrays (word w of pixel p at [w][p]).
// Pass 1 (t-test) stages the per-pixel terms of ComputeTStatistic and of
// ComputeWelchNu (denoise.cuh:278-339); pass 2 (weights) the guide values and
// log(1 + c).
enum : int {
    kVth0 = 0, kVth1, kVth2,      // varianceThetaHat
    kTh0, kTh1, kTh2,             // theta
    kU0, kU1, kU2,                // s^2 / n (Welch numerator term)
    kL0, kL1, kL2,                // (s^2 / n)^2 / max(n - 1, 1)
    kTWords
};
enum : int {
    kS0 = 0, kS1, kS2,            // log(1 + c)
    kA0, kA1, kA2,                // albedo
    kN0, kN1, kN2,                // normalised normal
    kDepth,
    kMR,                          // metallic | roughness << 16 (half bits)
    kSM01, kSM23, kSM4,           // shading-model shares (half bits)
    kGWords
};
constexpr int kMaskWords = (kTaps + 31) / 32;  // 225 tap bits per pixel
constexpr size_t kTSmem = (static_cast<size_t>(kTWords) * kWin + kTQuantiles) * sizeof(float);
constexpr size_t kGSmem = (static_cast<size_t>(kGWords) * kWin + kTaps) * sizeof(float);

__device__ __forceinline__ float hsub_f(uint32_t a, uint32_t b)
{
    return __half2float(__hsub(__ushort_as_half(static_cast<uint16_t>(a)), __ushort_as_half(static_cast<uint16_t>(b))));
}

// LookupTQuantile005(floorToInt(nu)) (t_quantile.cuh:15-27) with the device's
// saturating float-to-int conversion (NaN -> 0)
__device__ __forceinline__ int t_index(float nu)
{
    if (!(nu >= 1.0f)) return 0;
    if (nu >= 1024.0f) return kTQuantiles - 1;
    return static_cast<int>(floorf(nu)) - 1;
}

__device__ __forceinline__ int64_t window_pixel(int p, int gx0, int gy0, int width, int height)
{
    const int gx = min(max(gx0 + p % kWinX, 0), width - 1);
    const int gy = min(max(gy0 + p / kWinX, 0), height - 1);
    return static_cast<int64_t>(gy) * width + gx;
}

// ComputeTStatistic (denoise.cuh:278-302) and the per-pixel quotients of
// ComputeWelchNu (denoise.cuh:326-339); counts in 32-bit unsigned arithmetic
__device__ void stage_tstat(float* w, int p, const ar_screen_stats* st, int64_t idx)
{
    const ar_screen_stats s = st[idx];
    const double num = static_cast<double>(s.num);
    const double invNm1 = 1.0 / static_cast<double>(max(s.num - 1u, 1u));
    const float fnum = static_cast<float>(s.num);
    const float fnm1 = static_cast<float>(max(s.num - 1u, 1u));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float vb = static_cast<float>(static_cast<double>(s.m2_div_n[c]) * num * invNm1);
        w[(kVth0 + c) * kWin + p] = static_cast<float>(static_cast<double>(vb) / num);
        w[(kTh0 + c) * kWin + p] = s.mean[c] + s.m3_div_n[c] / 6.0f / vb;
        const float ua = vb / fnum;
        w[(kU0 + c) * kWin + p] = ua;
        w[(kL0 + c) * kWin + p] = ua * ua / fnm1;
    }
}

__device__ void stage_guide(float* w, int p, const float* hdr, const ar_screen_gbuffer* gb, int64_t idx)
{
    const ar_screen_gbuffer g = gb[idx];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        w[(kS0 + c) * kWin + p] = log_det(hdr[3 * idx + c] + 1.0f);  // SeparateSample (denoise.cuh:250-259)
        w[(kA0 + c) * kWin + p] = h2f(g.albedo[c]);
    }
    const f3 n = normalize(mk(h2f(g.normal[0]), h2f(g.normal[1]), h2f(g.normal[2])));
    w[kN0 * kWin + p] = n.x;
    w[kN1 * kWin + p] = n.y;
    w[kN2 * kWin + p] = n.z;
    w[kDepth * kWin + p] = g.depth;
    uint32_t* u = reinterpret_cast<uint32_t*>(w);
    u[kMR * kWin + p] = g.metallic | (static_cast<uint32_t>(g.roughness) << 16);
    u[kSM01 * kWin + p] = g.shading_model[0] | (static_cast<uint32_t>(g.shading_model[1]) << 16);
    u[kSM23 * kWin + p] = g.shading_model[2] | (static_cast<uint32_t>(g.shading_model[3]) << 16);
    u[kSM4 * kWin + p] = g.shading_model[4];
}

// Pass 1: ComputeTStatisticFinal (denoise.cuh:341-356) of every tap, center =
// A, as a 225-bit mask per pixel (bit (j + 7) * 15 + i + 7; word k of pixel p
// at mask[k * npix + p]).  The statistic T = sqrtf(x) is below the quantile
// exactly when 0 <= x < (smallest float whose square root reaches it), so the
// square root is not taken; the three channels are evaluated without branches.
__global__ void __launch_bounds__(kTileX * kTileY) k_dn_ttest(const ar_screen_stats* __restrict__ st,
                                                              uint32_t* __restrict__ mask, int width, int height)
{
    extern __shared__ float sm[];
    float* w = sm;
    float* thr = sm + static_cast<size_t>(kTWords) * kWin;
    const int tid = threadIdx.y * kTileX + threadIdx.x;
    for (int k = tid; k < kTQuantiles; k += kTileX * kTileY) thr[k] = kTQuantileSqrtThreshold[k];
    const int gx0 = blockIdx.x * kTileX - kDnRadius, gy0 = blockIdx.y * kTileY - kDnRadius;
    for (int p = tid; p < kWin; p += kTileX * kTileY) stage_tstat(w, p, st, window_pixel(p, gx0, gy0, width, height));
    __syncthreads();
    const int ox = blockIdx.x * kTileX + threadIdx.x, oy = blockIdx.y * kTileY + threadIdx.y;
    if (ox >= width || oy >= height) return;
    const int c = (threadIdx.y + kDnRadius) * kWinX + threadIdx.x + kDnRadius;
    float cv[kTWords];
#pragma unroll
    for (int k = 0; k < kTWords; ++k) cv[k] = w[k * kWin + c];
    const int64_t npix = static_cast<int64_t>(width) * height, pix = static_cast<int64_t>(oy) * width + ox;
    uint32_t bits = 0;  // the mask word being filled; taps run in increasing order
    int tap = 0;
#pragma unroll 1
    for (int j = -kDnRadius; j <= kDnRadius; ++j) {
#pragma unroll
        for (int i = -kDnRadius; i <= kDnRadius; ++i, ++tap) {
            const int q = c + j * kWinX + i;
            bool pass = true;
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) {
                const float vthB = w[(kVth0 + ch) * kWin + q];
                const float t = cv[kTh0 + ch] - w[(kTh0 + ch) * kWin + q];
                const float t2 = t * t;
                const float W = (t2 + vthB) / fmaxf(t2 + cv[kVth0 + ch] + vthB, 1.0e-6f);
                const float x = 0.5f / (1.0f - W) - 1.0f;
                const float up = cv[kU0 + ch] + w[(kU0 + ch) * kWin + q];
                const float nu = up * up / (cv[kL0 + ch] + w[(kL0 + ch) * kWin + q]);
                pass &= !(x < 0.0f) & (x < thr[t_index(nu)]);
            }
            bits |= static_cast<uint32_t>(pass) << (tap & 31);
            if ((tap & 31) == 31 || tap == kTaps - 1) {
                mask[(tap >> 5) * npix + pix] = bits;
                bits = 0;
            }
        }
    }
}

// Pass 2: the weighted mean of Bilateral16x16 (denoise.cuh:359-443) over the
// taps that passed the t-test, in the reference's order (rows, then columns).
__global__ void __launch_bounds__(kTileX * kTileY) k_dn_filter(const float* __restrict__ hdr, float* __restrict__ out,
                                                               const ar_screen_gbuffer* __restrict__ gb,
                                                               const uint32_t* __restrict__ mask, int width,
                                                               int height)
{
    extern __shared__ float sm[];
    float* w = sm;
    float* spatial = sm + static_cast<size_t>(kGWords) * kWin;
    const int tid = threadIdx.y * kTileX + threadIdx.x;
    for (int k = tid; k < kTaps; k += kTileX * kTileY) {
        const int j = k / (2 * kDnRadius + 1) - kDnRadius, i = k % (2 * kDnRadius + 1) - kDnRadius;
        spatial[k] = exp_det(static_cast<float>(-(i * i + j * j)) * kInvSpatial);
    }
    const int gx0 = blockIdx.x * kTileX - kDnRadius, gy0 = blockIdx.y * kTileY - kDnRadius;
    for (int p = tid; p < kWin; p += kTileX * kTileY)
        stage_guide(w, p, hdr, gb, window_pixel(p, gx0, gy0, width, height));
    __syncthreads();
    const int ox = blockIdx.x * kTileX + threadIdx.x, oy = blockIdx.y * kTileY + threadIdx.y;
    if (ox >= width || oy >= height) return;
    const int64_t npix = static_cast<int64_t>(width) * height, pix = static_cast<int64_t>(oy) * width + ox;
    const uint32_t* u = reinterpret_cast<const uint32_t*>(w);
    const int c = (threadIdx.y + kDnRadius) * kWinX + threadIdx.x + kDnRadius;
    float cv[kGWords];
#pragma unroll
    for (int k = 0; k < kGWords; ++k) cv[k] = w[k * kWin + c];
    const uint32_t cMR = __float_as_uint(cv[kMR]), cSM01 = __float_as_uint(cv[kSM01]);
    const uint32_t cSM23 = __float_as_uint(cv[kSM23]), cSM4 = __float_as_uint(cv[kSM4]);
    float acc0 = 0.0f + cv[kS0] * kCenterEps, acc1 = 0.0f + cv[kS1] * kCenterEps, acc2 = 0.0f + cv[kS2] * kCenterEps;
    float wsum = 0.0f + kCenterEps;
#pragma unroll 1
    for (int k = 0; k < kMaskWords; ++k) {
        uint32_t m = mask[k * npix + pix];
        while (m) {   // passing taps in increasing order: rows, then columns
            const int tap = 32 * k + __ffs(m) - 1;
            m &= m - 1u;
            const int j = tap / (2 * kDnRadius + 1) - kDnRadius, i = tap % (2 * kDnRadius + 1) - kDnRadius;
            const int q = c + j * kWinX + i;
            // ComputeSVGFWeight (denoise.cuh:185-245)
            float wt = 0.0f;
            {
                const float d0 = cv[kA0] - w[kA0 * kWin + q], d1 = cv[kA1] - w[kA1 * kWin + q];
                const float d2 = cv[kA2] - w[kA2 * kWin + q];
                wt += (d0 * d0 + d1 * d1 + d2 * d2) * kInvAlbedo;
            }
            {
                const float dv = cv[kN0] * w[kN0 * kWin + q] + cv[kN1] * w[kN1 * kWin + q] + cv[kN2] * w[kN2 * kWin + q];
                const float d = 1.0f - dv;
                wt += d * d * kInvNormal;
            }
            {
                const float db = w[kDepth * kWin + q];
                const float denom = fmaxf(fmaxf(cv[kDepth], db), 1.0e-6f);
                const float d = (cv[kDepth] - db) / denom;
                wt += d * d * kInvDepth;
            }
            const uint32_t nMR = u[kMR * kWin + q];
            const float dm = hsub_f(cMR, nMR);
            wt += dm * dm * kInvMetallic;
            const float dr = hsub_f(cMR >> 16, nMR >> 16);
            wt += dr * dr * kInvRough;
            {
                const uint32_t s01 = u[kSM01 * kWin + q], s23 = u[kSM23 * kWin + q], s4 = u[kSM4 * kWin + q];
                float l1 = 0.0f;
                l1 += fabsf(hsub_f(cSM01, s01));
                l1 += fabsf(hsub_f(cSM01 >> 16, s01 >> 16));
                l1 += fabsf(hsub_f(cSM23, s23));
                l1 += fabsf(hsub_f(cSM23 >> 16, s23 >> 16));
                l1 += fabsf(hsub_f(cSM4, s4));
                const float tv = 0.5f * l1;
                wt += tv * tv * kInvShading;
            }
            float weight = exp_det(-wt) * spatial[tap];
            if (isnan_(weight)) weight = 0.0f;  // zero normal of a pixel that never hit a surface
            if (weight == 0.0f) continue;
            acc0 = acc0 + w[kS0 * kWin + q] * weight;
            acc1 = acc1 + w[kS1 * kWin + q] * weight;
            acc2 = acc2 + w[kS2 * kWin + q] * weight;
            wsum = wsum + weight;
        }
    }
    // CompositeSample (denoise.cuh:261-270)
    float* o = out + 3 * pix;
    o[0] = fmaxf(exp_det(acc0 / wsum) - 1.0f, 0.0f);
    o[1] = fmaxf(exp_det(acc1 / wsum) - 1.0f, 0.0f);
    o[2] = fmaxf(exp_det(acc2 / wsum) - 1.0f, 0.0f);
}

__global__ void k_dn_record(const float* __restrict__ hits, const float* __restrict__ samples, int64_t n,
                            ar_screen_gbuffer* gb, ar_screen_stats* st)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (gb) {
            const float* h = hits + 12 * i;
            const int model = min(max(static_cast<int>(h[9]), 0), kDnModels - 2);
            record_gbuffer(gb + i, h[10] != 0.0f, mk(h[0], h[1], h[2]), mk(h[3], h[4], h[5]), h[6], h[7], h[8], model);
        }
        if (st) record_stats(st + i, mk(samples[3 * i], samples[3 * i + 1], samples[3 * i + 2]));
    }
}

ar_status dn_cuda_fail(cudaError_t e, const char* where)
{
    cudaGetLastError();
    return set_error(AR_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

bool have_device()
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return false;
    }
    return true;
}

}  // namespace

cudaError_t launch_dn_record(const float* hits, const float* samples, int64_t n, ar_screen_gbuffer* gb,
                             ar_screen_stats* st, cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    const int64_t want = (n + 255) / 256;
    const int grid = static_cast<int>(want < 148 * 16 ? want : 148 * 16);
    k_dn_record<<<grid, 256, 0, stream>>>(hits, samples, n, gb, st);
    return cudaGetLastError();
}

}  // namespace ar

extern "C" ar_status ar_denoise_record(const float* hits, const float* samples, size_t n, ar_screen_gbuffer* gbuffer,
                                       ar_screen_stats* stats, void* stream)
{
    using namespace ar;
    if (n == 0) return AR_OK;
    if (!gbuffer && !stats) return set_error(AR_ERR_INVALID_ARGUMENT, "gbuffer and stats are both NULL");
    if (gbuffer && !hits) return set_error(AR_ERR_INVALID_ARGUMENT, "hits is NULL");
    if (stats && !samples) return set_error(AR_ERR_INVALID_ARGUMENT, "samples is NULL");
    if (!have_device()) return set_error(AR_ERR_NO_DEVICE, "no CUDA device available");
    const cudaError_t e = launch_dn_record(hits, samples, static_cast<int64_t>(n), gbuffer, stats,
                                           static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? AR_OK : dn_cuda_fail(e, "k_dn_record launch");
}

extern "C" ar_status ar_denoise_bilateral(const float* hdr_in, float* hdr_out, const ar_screen_gbuffer* gbuffer,
                                          const ar_screen_stats* stats, int32_t width, int32_t height, void* stream)
{
    using namespace ar;
    if (!hdr_in || !hdr_out || !gbuffer || !stats) return set_error(AR_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (width <= 0 || height <= 0) return set_error(AR_ERR_INVALID_ARGUMENT, "width and height must be positive");
    if (hdr_in == hdr_out) return set_error(AR_ERR_INVALID_ARGUMENT, "hdr_out must not alias hdr_in");
    if (!have_device()) return set_error(AR_ERR_NO_DEVICE, "no CUDA device available");
    // the shared-memory opt-in is a per-device attribute of the kernels
    static std::atomic<uint64_t> attr_set{0};
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return dn_cuda_fail(e, "cudaGetDevice");
    const uint64_t bit = dev < 64 ? (uint64_t{1} << dev) : 0;
    if (!bit || !(attr_set.load() & bit)) {
        if ((e = cudaFuncSetAttribute(k_dn_ttest, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kTSmem))) != cudaSuccess ||
            (e = cudaFuncSetAttribute(k_dn_filter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kGSmem))) != cudaSuccess)
            return dn_cuda_fail(e, "cudaFuncSetAttribute");
        attr_set.fetch_or(bit);
    }
    // the tap mask between the passes: stream-ordered scratch, freed on the stream
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t mask_bytes = static_cast<size_t>(kMaskWords) * sizeof(uint32_t) * static_cast<size_t>(width) *
                              static_cast<size_t>(height);
    uint32_t* mask = nullptr;
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&mask), mask_bytes, st)) != cudaSuccess)
        return dn_cuda_fail(e, "cudaMallocAsync");
    const dim3 block(kTileX, kTileY);
    const dim3 grid((width + kTileX - 1) / kTileX, (height + kTileY - 1) / kTileY);
    k_dn_ttest<<<grid, block, kTSmem, st>>>(stats, mask, width, height);
    const cudaError_t e1 = cudaGetLastError();
    if (e1 == cudaSuccess) k_dn_filter<<<grid, block, kGSmem, st>>>(hdr_in, hdr_out, gbuffer, mask, width, height);
    const cudaError_t e2 = cudaGetLastError();
    const cudaError_t e3 = cudaFreeAsync(mask, st);
    if (e1 != cudaSuccess) return dn_cuda_fail(e1, "k_dn_ttest launch");
    if (e2 != cudaSuccess) return dn_cuda_fail(e2, "k_dn_filter launch");
    if (e3 != cudaSuccess) return dn_cuda_fail(e3, "cudaFreeAsync");
    return AR_OK;
}
