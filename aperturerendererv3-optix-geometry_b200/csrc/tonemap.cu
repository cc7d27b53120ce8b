// tonemap.cu -- ar_tonemap: the output epilogue (linear radiance -> BGRA8).
//
// One thread per pixel, grid-stride: 12 bytes in, 4 bytes out, a few hundred
// FLOPs for ACES -- an HBM-bound elementwise kernel.  Host buffers are staged
// through device buffers owned by the call.
#include <cuda_runtime.h>

#include <string>

#include "../../include/aperture_b200.h"
#include "tonemap.cuh"

namespace ar {

ar_status set_error(ar_status st, const std::string& msg);

namespace {

__global__ void __launch_bounds__(256) k_tonemap(const float* __restrict__ rgb, int64_t n, int tone, float exposure,
                                                 int xyz_input, uint32_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const f3 v = mk(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        out[i] = tonemap_pixel(v, tone, exposure, xyz_input);
    }
}

struct Staging {
    float* rgb = nullptr;
    uint32_t* out = nullptr;
    ~Staging()
    {
        if (rgb) cudaFree(rgb);
        if (out) cudaFree(out);
    }
};

ar_status cuda_fail(cudaError_t e, const char* where)
{
    cudaGetLastError();
    return set_error(e == cudaErrorMemoryAllocation ? AR_ERR_OUT_OF_MEMORY : AR_ERR_CUDA,
                     std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace ar

extern "C" ar_status ar_tonemap(const float* rgb, size_t n, int32_t tone_type, float exposure, int32_t xyz_input,
                                uint32_t* bgra, int32_t mem_kind, void* stream)
{
    using namespace ar;
    if (n == 0) return AR_OK;
    if (!rgb || !bgra) return set_error(AR_ERR_INVALID_ARGUMENT, "rgb/bgra is NULL");
    if (tone_type < 0 || tone_type > 2) return set_error(AR_ERR_INVALID_ARGUMENT, "tone_type must be 0, 1 or 2");
    if (mem_kind != AR_MEM_HOST && mem_kind != AR_MEM_DEVICE) return set_error(AR_ERR_INVALID_ARGUMENT, "bad mem_kind");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_error(AR_ERR_NO_DEVICE, "no CUDA device available");
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Staging tmp;
    const float* in = rgb;
    uint32_t* out = bgra;
    cudaError_t e = cudaSuccess;
    if (mem_kind == AR_MEM_HOST) {
        if ((e = cudaMalloc(&tmp.rgb, n * 3 * sizeof(float))) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        if ((e = cudaMalloc(&tmp.out, n * sizeof(uint32_t))) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
        if ((e = cudaMemcpyAsync(tmp.rgb, rgb, n * 3 * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync");
        in = tmp.rgb;
        out = tmp.out;
    }
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (static_cast<int64_t>(n) + 255) / 256;
    const int grid = static_cast<int>(want < int64_t(sms) * 8 ? want : int64_t(sms) * 8);
    k_tonemap<<<grid, 256, 0, st>>>(in, static_cast<int64_t>(n), tone_type, exposure, xyz_input, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_tonemap launch");
    if (mem_kind == AR_MEM_HOST) {
        if ((e = cudaMemcpyAsync(bgra, tmp.out, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    }
    return AR_OK;
}

extern "C" ar_status ar_tone_curve(const float* rgb3, int32_t tone_type, float* out3)
{
    using namespace ar;
    if (!rgb3 || !out3) return set_error(AR_ERR_INVALID_ARGUMENT, "rgb3/out3 is NULL");
    if (tone_type < 0 || tone_type > 2) return set_error(AR_ERR_INVALID_ARGUMENT, "tone_type must be 0, 1 or 2");
    f3 v = mk(rgb3[0], rgb3[1], rgb3[2]);
    if (tone_type == 1) v = tone_gamma(v);
    else if (tone_type == 2) v = tone_aces(v);
    out3[0] = v.x;
    out3[1] = v.y;
    out3[2] = v.z;
    return AR_OK;
}
