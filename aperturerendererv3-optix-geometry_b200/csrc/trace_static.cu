// trace_static.cu -- ar_trace_rays_static: ray queries that allocate nothing.
//
// Some callers cannot call cudaMalloc at the moment they need a ray query: a
// host that hands the library a fixed memory budget and forbids further device
// allocation, a real-time thread that must not take the allocator's locks, or
// code that runs while another part of the process is capturing a CUDA graph
// (cudaMalloc is not allowed then).  ar_trace_rays allocates a workspace on
// first use; this entry point instead keeps its scratch -- two counters and the
// traversal-stack overflow slabs of its persistent threads -- in one file-scope
// __device__ array of kStaticScratchBytes (16 MiB), which every GPU that loads
// the library holds until the process exits.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.  Every call shares the array, so calls
// whose work overlaps on the GPU race with each other; issue them on one
// stream or otherwise serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <string>

#include "../../include/aperture_b200.h"
#include "render_kernels.h"
#include "traverse.cuh"

namespace ar {

// internal accessors of the scene handle and the error string (capi.cu)
bool scene_view_of(const ar_scene* s, SceneView* v, int* device, int* sm_count);
ar_status set_error(ar_status st, const std::string& msg);

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr size_t kStaticHeaderBytes = 256;  // [0] work counter, [1] error word
constexpr size_t kSlabBytes = static_cast<size_t>(kStackOverflow) * 4;
constexpr int kStaticMaxBlocks =
    static_cast<int>((kStaticScratchBytes - kStaticHeaderBytes) / (kSlabBytes * kTraceBlock));

static __device__ __align__(256) unsigned char g_trace_scratch[kStaticScratchBytes];

template <bool kSdf>
struct StaticRaysIO {
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
        if (kSdf && s.num_sdf > 0) {
            if (!any) sdf_closest(s, r.o, r.d, r.tmin, kEpsDepth0, &t, &obj);
            else if (obj < 0) obj = sdf_any(s, r.o, r.d, r.tmin, t, kEpsDepth0);
        }
        out_obj[k] = obj;
        if (out_t) out_t[k] = t;
    }
};

template <bool kAny, bool kSdf>
__global__ void __launch_bounds__(kTraceBlock) k_trace_rays_static(SceneView s, StaticRaysIO<kSdf> io, int n,
                                                                   unsigned char* scratch)
{
    extern __shared__ uint32_t smem[];
    int* fetch = reinterpret_cast<int*>(scratch);
    int* err = fetch + 1;
    uint32_t* ovf = reinterpret_cast<uint32_t*>(scratch + kStaticHeaderBytes) +
                    (static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x) * kStackOverflow;
    uint32_t* stack = smem + (threadIdx.x >> 5) * (kStackShared * 32) + (threadIdx.x & 31u);
    traverse_queue<kAny>(s, io, n, fetch, stack, ovf, err, nullptr);
}

std::mutex g_setup_mutex;
unsigned char* g_scratch_of_device[256] = {};
int g_blocks_of_device[256] = {};

}  // namespace
}  // namespace ar

extern "C" ar_status ar_trace_rays_static(const ar_scene* scene, const float* rays, size_t n, int32_t any_hit,
                                          int32_t* hit_object, float* hit_t, void* stream)
{
    using namespace ar;
    SceneView view;
    int device = 0, sms = 0;
    if (!scene_view_of(scene, &view, &device, &sms)) return set_error(AR_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (n == 0) return AR_OK;
    if (!rays || !hit_object) return set_error(AR_ERR_INVALID_ARGUMENT, "rays/hit_object is NULL");
    if (reinterpret_cast<uintptr_t>(rays) & 15u)
        return set_error(AR_ERR_INVALID_ARGUMENT, "ray buffer must be 16-byte aligned device memory");
    if (device < 0 || device >= 256) return set_error(AR_ERR_UNSUPPORTED, "device index above 255");
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        return set_error(AR_ERR_CUDA, "cudaGetDevice failed");
    }
    if (prev != device && cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return set_error(AR_ERR_CUDA, "cudaSetDevice failed");
    }
    struct Restore {
        int prev, dev;
        ~Restore() { if (prev != dev) cudaSetDevice(prev); }
    } restore{prev, device};
    unsigned char* scratch;
    int blocks;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_of_device[device]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_trace_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                return set_error(AR_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                                                  cudaGetErrorString(e));
            }
            const size_t smem = static_cast<size_t>(kStackShared) * kTraceBlock * 4;
            int b0 = 1, b1 = 1;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_trace_rays_static<false, false>, kTraceBlock, smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_trace_rays_static<true, false>, kTraceBlock, smem);
            cudaGetLastError();
            g_blocks_of_device[device] = std::max(1, std::min(std::min(b0, b1) * sms, kStaticMaxBlocks));
            g_scratch_of_device[device] = static_cast<unsigned char*>(p);
        }
        scratch = g_scratch_of_device[device];
        blocks = g_blocks_of_device[device];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t smem = static_cast<size_t>(kStackShared) * kTraceBlock * 4;
    // The work counter is a 32-bit int that the last fetches of every warp can
    // carry past the ray count by up to 32 x 4 warps x blocks: chunks of 2^30
    // rays keep it far below INT_MAX.  The header (counter and error word) is
    // cleared before each chunk, so with several chunks each chunk's error
    // word is read back before the next clear.
    const size_t chunk = size_t(1) << 30;
    cudaError_t e = cudaSuccess;
    int err_any = 0;
    for (size_t first = 0; first < n && e == cudaSuccess && err_any == 0; first += chunk) {
        const int cnt = static_cast<int>(std::min(chunk, n - first));
        const float4* r4 = reinterpret_cast<const float4*>(rays) + 2 * first;
        int32_t* obj = hit_object + first;
        float* tt = hit_t ? hit_t + first : nullptr;
        e = cudaMemsetAsync(scratch, 0, kStaticHeaderBytes, st);  // work counter and error word
        if (e == cudaSuccess) {
            if (view.num_sdf > 0) {
                StaticRaysIO<true> io;
                io.rays = r4;
                io.out_obj = obj;
                io.out_t = tt;
                io.any = any_hit ? 1 : 0;
                if (any_hit) k_trace_rays_static<true, true><<<blocks, kTraceBlock, smem, st>>>(view, io, cnt, scratch);
                else k_trace_rays_static<false, true><<<blocks, kTraceBlock, smem, st>>>(view, io, cnt, scratch);
            } else {
                StaticRaysIO<false> io;
                io.rays = r4;
                io.out_obj = obj;
                io.out_t = tt;
                io.any = any_hit ? 1 : 0;
                if (any_hit) k_trace_rays_static<true, false><<<blocks, kTraceBlock, smem, st>>>(view, io, cnt, scratch);
                else k_trace_rays_static<false, false><<<blocks, kTraceBlock, smem, st>>>(view, io, cnt, scratch);
            }
            e = cudaGetLastError();
        }
        if (n > chunk) {  // several chunks: read this chunk's error word before the next clear
            int w = 0;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&w, scratch + 4, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            err_any |= w;
        }
    }
    int err_word = err_any;
    if (e == cudaSuccess && n <= chunk)
        e = cudaMemcpyAsync(&err_word, scratch + 4, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(AR_ERR_CUDA, std::string("ar_trace_rays_static: ") + cudaGetErrorString(e));
    }
    if (err_word != 0) return set_error(AR_ERR_DEVICE_FAULT, "traversal stack overflow reported by a kernel");
    return AR_OK;
}
