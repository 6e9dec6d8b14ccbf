// Top-K peak search that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the moment they need peaks: callers
// inside a host framework that owns the device's memory through its own pool
// and forbids outside allocations (a MATLAB MEX running next to gpuArray
// data, a serving process with a fixed memory budget), and real-time loops
// that must not risk an allocation failure mid-run.  For them this variant of
// tomgpu_topk_dev keeps its scratch — a working copy of the volume that the
// peak rounds zero in place, and the 64-bit arg-max key — in file-scope
// __device__ arrays, so every call uses memory that already exists.
//
// Limits and sharing: the working copy holds at most 2^24 voxels (64 MiB); the
// arrays exist on every GPU where this code is loaded, until the process
// exits.  All calls share them, so calls that overlap on the GPU (different
// streams or host threads without ordering) race and corrupt each other.  The
// first call on a device looks up the arrays' device addresses and should come
// before any stream capture on that device.  The addresses are kept for the
// life of the process: after cudaDeviceReset (which ends the context that held
// the arrays) this entry point must not be called again in that process.
#include <cmath>
#include <mutex>
#include <string>

#include "ctx.h"
#include "peak.h"

namespace tg {

namespace {
constexpr long long kNoAllocMaxVoxels = 1ll << 24;

__device__ __align__(256) float g_topk_work[kNoAllocMaxVoxels];
__device__ __align__(256) unsigned long long g_topk_key[4];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float* g_work[kMaxDevices] = {};
unsigned long long* g_key[kMaxDevices] = {};

// Device addresses of the scratch arrays for the current device (looked up
// once per device: in host code the array names are host-side stand-ins).
int scratch_for_device(int dev, float** work, unsigned long long** key) {
    if (dev < 0 || dev >= kMaxDevices) return fail(nullptr, TOMGPU_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_work[dev]) {
        void* w = nullptr;
        void* k = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&w, g_topk_work);
        if (e == cudaSuccess) e = cudaGetSymbolAddress(&k, g_topk_key);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(nullptr, TOMGPU_ERR_CUDA,
                        std::string("allocation-free top-K set-up (cudaGetSymbolAddress): ") + cudaGetErrorString(e));
        }
        g_work[dev] = static_cast<float*>(w);
        g_key[dev] = static_cast<unsigned long long*>(k);
    }
    *work = g_work[dev];
    *key = g_key[dev];
    return TOMGPU_OK;
}
}  // namespace

}  // namespace tg

extern "C" int tomgpu_topk_noalloc_dev(void* stream, const float* v_dev, const int dims[3], int K, double radius,
                                       float* vals_dev, int* pos1_dev) {
    using namespace tg;
    if (!v_dev || !dims || !vals_dev || !pos1_dev || K < 0 || !(radius >= 0) || std::isinf(radius))
        return fail(nullptr, TOMGPU_ERR_ARG, "null pointer, negative K or bad radius (negative, NaN or infinite)");
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0) return fail(nullptr, TOMGPU_ERR_ARG, "bad dims");
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    if (n > kNoAllocMaxVoxels)
        return fail(nullptr, TOMGPU_ERR_UNSUPPORTED,
                    "volume of " + std::to_string(n) + " voxels exceeds the allocation-free top-K limit of " +
                        std::to_string(kNoAllocMaxVoxels) + " voxels; use tomgpu_topk_dev");
    if (K == 0) return TOMGPU_OK;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, TOMGPU_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    }
    float* work = nullptr;
    unsigned long long* key = nullptr;
    TG_TRY(scratch_for_device(dev, &work, &key));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t launches = 0;
    e = cudaMemcpyAsync(work, v_dev, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = topk_rounds(work, dims, K, radius, key, vals_dev, pos1_dev, st, &launches);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(nullptr, TOMGPU_ERR_CUDA, std::string("allocation-free top-K: ") + cudaGetErrorString(e));
    }
    return TOMGPU_OK;
}
