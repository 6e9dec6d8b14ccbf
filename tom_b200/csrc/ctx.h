// Internal context shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/tomgpu.h"

struct tomgpu_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int64_t launches = 0;
    int* d_err = nullptr;  // device error word (kernels write, host reads)
    // small scratch for reductions (peak keys, partial sums)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // tomgpu_match's plan and device buffers, kept for the next call with the
    // same sizes and parameters (released by tomgpu_ctx_trim and at destroy)
    void* match_cache = nullptr;
    // tomgpu_av3_align's grow-only device workspace, kept for the next call
    // (released by tomgpu_ctx_trim and at destroy)
    void* align_scratch = nullptr;
    // kernel-class timers (tomgpu_ctx_profile)
    bool prof = false;
    struct Pending { int kind; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    double prof_ms[TOMGPU_K_COUNT] = {0};
    int64_t prof_n[TOMGPU_K_COUNT] = {0};
};

namespace tg {

// Device error word codes (mirrors TgDeviceError in common.cuh).
enum { TG_DEV_OK_CODE = 0, TG_DEV_BAD_INDEX_CODE = 1, TG_DEV_TIMEOUT_CODE = 2 };

// Record an error message on the context and return the status.
int fail(tomgpu_ctx* ctx, int status, const std::string& msg);
int cuda_fail(tomgpu_ctx* ctx, cudaError_t e, const char* where);

// Make the context's device current for this host thread.
int use_device(tomgpu_ctx* ctx);

// Grow the context scratch buffer to at least `bytes`.
int ensure_scratch(tomgpu_ctx* ctx, size_t bytes);

// Read and clear the device error word (synchronises the stream).
int check_device_error(tomgpu_ctx* ctx);

// Records a CUDA event pair around the launches issued in its scope when the
// context's profiling is on.
struct ProfScope {
    tomgpu_ctx* ctx;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(tomgpu_ctx* c, int k);
    ~ProfScope();
};
// Drain recorded event pairs into the per-class totals (synchronises).
int profile_drain(tomgpu_ctx* ctx);

// Host-side ZXZ matrix of rot3d (bit-exact float arithmetic).
void euler_matrix_host(const float euler_deg[3], float m9[9]);

}  // namespace tg

#define TG_TRY_CUDA(ctx, expr)                                        \
    do {                                                              \
        cudaError_t _e = (expr);                                      \
        if (_e != cudaSuccess) return tg::cuda_fail((ctx), _e, #expr); \
    } while (0)

#define TG_TRY(expr)              \
    do {                          \
        int _s = (expr);          \
        if (_s != TOMGPU_OK) return _s; \
    } while (0)
