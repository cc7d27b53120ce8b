// spectral.cu -- building the spectral lookup tables on the GPU.
//
// k_lut_lambda evaluates the wavelength network at the 840 bin centres of
// 360-780 nm, k_lut_rgb the RGB network at the res^3 voxel centres of the unit
// colour cube (PrecomputeLambdaLUTKernel / PrecomputeRGBLUTKernel,
// core/spectrum/spectrum_lut.cuh:12-58).  One thread per entry; the 32-wide
// residual network runs from registers with its weights read through the
// read-only cache (every thread of a warp reads the same weight).
#include <cuda_runtime.h>

#include "render_kernels.h"
#include "spectral.cuh"

namespace ar {

namespace {

__global__ void __launch_bounds__(128) k_lut_lambda(const float* __restrict__ tab, float4* __restrict__ lut)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kLambdaLutRes) return;
    const float step = (kLamMax - kLamMin) / static_cast<float>(kLambdaLutRes);
    const float lambda = kLamMin + (static_cast<float>(i) + 0.5f) * step;
    float k[kSpecKernel];
    lambda_encode(tab, lambda, k);
    lut[i] = make_float4(k[0], k[1], k[2], k[3]);
}

__global__ void __launch_bounds__(128) k_lut_rgb(const float* __restrict__ tab, int res, float4* __restrict__ lut)
{
    const int64_t total = static_cast<int64_t>(res) * res * res;
    const float invRes = 1.0f / static_cast<float>(res);
    for (int64_t v = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; v < total;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(v % res);
        const int y = static_cast<int>((v / res) % res);
        const int z = static_cast<int>(v / (static_cast<int64_t>(res) * res));
        float k[kSpecKernel];
        rgb_encode(tab, (static_cast<float>(x) + 0.5f) * invRes, (static_cast<float>(y) + 0.5f) * invRes,
                   (static_cast<float>(z) + 0.5f) * invRes, k);
        lut[v] = make_float4(k[0], k[1], k[2], k[3]);
    }
}

}  // namespace

cudaError_t launch_spectral_luts(const float* tab, int res, float4* lut_lam, float4* lut_rgb, int sm_count,
                                 cudaStream_t st)
{
    k_lut_lambda<<<(kLambdaLutRes + 127) / 128, 128, 0, st>>>(tab, lut_lam);
    const int64_t total = static_cast<int64_t>(res) * res * res;
    const int64_t want = (total + 127) / 128;
    const int grid = static_cast<int>(want < int64_t(sm_count) * 64 ? want : int64_t(sm_count) * 64);
    k_lut_rgb<<<grid, 128, 0, st>>>(tab, res, lut_rgb);
    return cudaGetLastError();
}

}  // namespace ar
