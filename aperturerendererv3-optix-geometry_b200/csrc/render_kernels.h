// render_kernels.h -- host-side launchers of the sm_100a kernels (render.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "wavefront.cuh"

namespace ar {

constexpr int kTraceBlock = 128;  // threads per traversal block (4 warps)
constexpr int kTraceMinBlocks = 8;  // resident blocks per SM the traversal kernels are built for (<= 64 registers)
constexpr int kShadeBlock = 256;

// Upload INTERSECT_EPS(0..8) to the current device.
cudaError_t set_intersect_eps(const float* tab9);
// Blocks of the persistent traversal kernels: occupancy limit x SM count.
int trace_grid(int sm_count);
cudaError_t launch_trace_rays(const SceneView& s, const float4* rays, int n, int any, int32_t* obj, float* t,
                              PoolCtl* ctl, uint32_t* ovf, int* err, int grid, cudaStream_t st);
cudaError_t launch_rng_init(const FrameParams& fp, uint4* b0, uint2* b1, const uint32_t* jump67, cudaStream_t st);
cudaError_t launch_rng_tape(const FrameParams& fp, int spp, int per_path, float* out, cudaStream_t st);

// Optional event pairs around every traversal launch: ev[2k], ev[2k+1].
struct LaunchTimers {
    cudaEvent_t* extend_ev = nullptr;
    cudaEvent_t* shadow_ev = nullptr;
    int cap = 0;        // event pairs available per kind
    int n_extend = 0;   // pairs recorded
    int n_shadow = 0;
};

cudaError_t launch_pool_init(PoolCtl* ctl, int64_t total, cudaStream_t st);
// `iterations` rounds of plan -> regen -> extend -> shade (per material) -> shadow -> retire.
cudaError_t launch_iterations(const SceneView& s, const FrameParams& fp, const PathBuffers& B, PoolCtl* ctl,
                              uint4* b0, uint2* b1, const uint32_t* jump_table, unsigned long long* stats,
                              uint32_t* ovf, int* err, double* accum, ar_path_record* rec, int iterations, int* cur,
                              int grid_trace, int grid_other, cudaStream_t st, int64_t* launches, LaunchTimers* tm);
// Spectral lookup tables from the network weights in `tab` (device memory).
cudaError_t launch_spectral_luts(const float* tab, int res, float4* lut_lam, float4* lut_rgb, int sm_count,
                                 cudaStream_t st);
// The RGB table alone on the tensor cores (spectral_tc.cu); *err gets bit 0
// when a CTA's MMA wait runs out.
cudaError_t launch_spectral_rgb_lut_tc(const float* tab, int res, float4* lut, int* err, int sm_count,
                                       cudaStream_t st);
cudaError_t launch_mean(const double* accum, int64_t n, double inv, float* out, cudaStream_t st);
cudaError_t launch_add(const double* src, int64_t n, double* dst, cudaStream_t st);

}  // namespace ar
