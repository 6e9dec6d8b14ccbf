// C ABI of libtomgpu (include/tomgpu.h).  Argument checking, context and
// buffer management; the arithmetic runs in the CUDA translation units.
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "analysis.h"
#include "ctx.h"
#include "fft3d.h"
#include "match.h"
#include "misc.h"
#include "peak.h"
#include "rotate.h"
#include "twiddles.h"

// tomgpu_match's state kept in the context between calls
struct MatchCache {
    tomgpu_match_plan* plan = nullptr;
    int vol[3] = {0, 0, 0}, tm[3] = {0, 0, 0};
    tomgpu_match_params prm{};
    bool psf = false;
    float *d_vol = nullptr, *d_t = nullptr, *d_m = nullptr, *d_p = nullptr, *d_cc = nullptr;
    int* d_i = nullptr;

    bool same(const int v[3], const int t[3], const tomgpu_match_params& p, bool has_psf) const {
        for (int d = 0; d < 3; ++d)
            if (vol[d] != v[d] || tm[d] != t[d]) return false;
        return has_psf == psf && std::memcmp(&prm, &p, sizeof(p)) == 0;
    }
    ~MatchCache() {
        void* ptrs[] = {d_vol, d_t, d_m, d_p, d_cc, d_i};
        for (void* q : ptrs)
            if (q) cudaFree(q);
        tomgpu_match_plan_destroy(plan);
    }
};

static void drop_match_cache(tomgpu_ctx* ctx) {
    delete static_cast<MatchCache*>(ctx->match_cache);
    ctx->match_cache = nullptr;
}

static void drop_align_scratch(tomgpu_ctx* ctx) {
    tg::align_scratch_free(static_cast<tg::AlignScratch*>(ctx->align_scratch));
    ctx->align_scratch = nullptr;
}

namespace tg {

static thread_local std::string g_create_error;

int fail(tomgpu_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    else g_create_error = msg;
    return status;
}

int cuda_fail(tomgpu_ctx* ctx, cudaError_t e, const char* where) {
    if (e == cudaSuccess) e = cudaErrorUnknown;
    const int status = (e == cudaErrorMemoryAllocation) ? TOMGPU_ERR_OOM : TOMGPU_ERR_CUDA;
    cudaGetLastError();  // clear a non-sticky error
    return fail(ctx, status, std::string(where) + ": " + cudaGetErrorString(e));
}

int use_device(tomgpu_ctx* ctx) {
    if (!ctx) return TOMGPU_ERR_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e) return cuda_fail(ctx, e, "cudaSetDevice");
    return TOMGPU_OK;
}

int ensure_scratch(tomgpu_ctx* ctx, size_t bytes) {
    if (ctx->scratch_bytes >= bytes) return TOMGPU_OK;
    if (ctx->scratch) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratch_bytes = 0;
    }
    size_t want = bytes < 4096 ? 4096 : bytes;
    cudaError_t e = cudaMalloc(&ctx->scratch, want);
    if (e) return cuda_fail(ctx, e, "scratch allocation");
    ctx->scratch_bytes = want;
    return TOMGPU_OK;
}

int check_device_error(tomgpu_ctx* ctx) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
    if (!e) e = cudaStreamSynchronize(ctx->stream);
    if (e) return cuda_fail(ctx, e, "device error readback");
    if (h) {
        cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream);
        return fail(ctx, h == TG_DEV_TIMEOUT_CODE ? TOMGPU_ERR_TIMEOUT : TOMGPU_ERR_DEVICE,
                    "kernel reported device error code " + std::to_string(h));
    }
    return TOMGPU_OK;
}

static cudaEvent_t take_event(tomgpu_ctx* ctx) {
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

ProfScope::ProfScope(tomgpu_ctx* c, int k) : ctx(c), kind(k) {
    if (!ctx || !ctx->prof) return;
    a = take_event(ctx);
    if (a) cudaEventRecord(a, ctx->stream);
}

ProfScope::~ProfScope() {
    if (!a) return;
    cudaEvent_t b = take_event(ctx);
    if (!b) return;
    cudaEventRecord(b, ctx->stream);
    ctx->pending.push_back({kind, a, b});
}

int profile_drain(tomgpu_ctx* ctx) {
    if (ctx->pending.empty()) return TOMGPU_OK;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e) return cuda_fail(ctx, e, "profile sync");
    for (auto& p : ctx->pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            ctx->prof_ms[p.kind] += ms;
            ctx->prof_n[p.kind] += 1;
        } else {
            cudaGetLastError();
        }
        ctx->event_pool.push_back(p.a);
        ctx->event_pool.push_back(p.b);
    }
    ctx->pending.clear();
    return TOMGPU_OK;
}

}  // namespace tg

using namespace tg;

static bool dims_ok(const int d[3]) { return d && d[0] > 0 && d[1] > 0 && d[2] > 0; }
static long long numel(const int d[3]) { return (long long)d[0] * d[1] * d[2]; }

extern "C" {

const char* tomgpu_version(void) { return "tomgpu 0.1 sm_100a"; }

const char* tomgpu_status_string(int s) {
    switch (s) {
        case TOMGPU_OK: return "ok";
        case TOMGPU_ERR_ARG: return "invalid argument";
        case TOMGPU_ERR_UNSUPPORTED: return "unsupported size";
        case TOMGPU_ERR_OOM: return "out of device memory";
        case TOMGPU_ERR_CUDA: return "CUDA error";
        case TOMGPU_ERR_STATE: return "invalid call order";
        case TOMGPU_ERR_DEVICE: return "device-side error flag";
        case TOMGPU_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

const char* tomgpu_last_error(const tomgpu_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

int tomgpu_ctx_create(int device, tomgpu_ctx** out) {
    if (!out) return fail(nullptr, TOMGPU_ERR_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e || device < 0 || device >= n) {
        cudaGetLastError();
        return fail(nullptr, TOMGPU_ERR_CUDA, "no CUDA device " + std::to_string(device));
    }
    tomgpu_ctx* c = new tomgpu_ctx();
    c->device = device;
    if ((e = cudaSetDevice(device)) || (e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) ||
        (e = cudaMalloc(&c->d_err, sizeof(int))) || (e = cudaMemset(c->d_err, 0, sizeof(int)))) {
        std::string m = std::string("context creation: ") + cudaGetErrorString(e);
        cudaGetLastError();
        if (c->own_stream) cudaStreamDestroy(c->own_stream);
        delete c;
        return fail(nullptr, TOMGPU_ERR_CUDA, m);
    }
    c->stream = c->own_stream;
    *out = c;
    return TOMGPU_OK;
}

int tomgpu_ctx_destroy(tomgpu_ctx* ctx) {
    if (!ctx) return TOMGPU_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_match_cache(ctx);
    drop_align_scratch(ctx);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->d_err) cudaFree(ctx->d_err);
    for (auto& p : ctx->pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (auto e : ctx->event_pool) cudaEventDestroy(e);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return TOMGPU_OK;
}

int tomgpu_ctx_set_stream(tomgpu_ctx* ctx, void* s) {
    if (!ctx) return TOMGPU_ERR_ARG;
    cudaStream_t ns = static_cast<cudaStream_t>(s);
    if (ns == ctx->stream) return TOMGPU_OK;
    TG_TRY(use_device(ctx));
    // work already queued on the previous stream completes before any work
    // issued on the new one: an event wait on the device, the host does not block
    cudaEvent_t ev = nullptr;
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (!e) e = cudaEventRecord(ev, ctx->stream);
    if (!e) e = cudaStreamWaitEvent(ns, ev, 0);
    if (ev) cudaEventDestroy(ev);
    if (e) return cuda_fail(ctx, e, "stream switch");
    ctx->stream = ns;
    return TOMGPU_OK;
}

int tomgpu_ctx_synchronize(tomgpu_ctx* ctx) {
    TG_TRY(use_device(ctx));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return check_device_error(ctx);
}

int64_t tomgpu_ctx_launch_count(const tomgpu_ctx* ctx) { return ctx ? ctx->launches : 0; }

int tomgpu_ctx_profile(tomgpu_ctx* ctx, int enable) {
    if (!ctx) return TOMGPU_ERR_ARG;
    TG_TRY(use_device(ctx));
    TG_TRY(profile_drain(ctx));
    if (enable) {
        for (int k = 0; k < TOMGPU_K_COUNT; ++k) { ctx->prof_ms[k] = 0; ctx->prof_n[k] = 0; }
    }
    ctx->prof = enable != 0;
    return TOMGPU_OK;
}

int tomgpu_ctx_profile_read(tomgpu_ctx* ctx, int kernel, double* total_ms, int64_t* launches) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (kernel < 0 || kernel >= TOMGPU_K_COUNT || !total_ms || !launches)
        return fail(ctx, TOMGPU_ERR_ARG, "bad kernel class or null output");
    TG_TRY(use_device(ctx));
    TG_TRY(profile_drain(ctx));
    *total_ms = ctx->prof_ms[kernel];
    *launches = ctx->prof_n[kernel];
    return TOMGPU_OK;
}

// ------------------------------------------------------------- rotation
int tomgpu_euler_matrix(const float euler[3], float m9[9]) {
    if (!euler || !m9) return TOMGPU_ERR_ARG;
    euler_matrix_host(euler, m9);
    return TOMGPU_OK;
}

static int rotate_dev(tomgpu_ctx* ctx, const float* in, float* out, const int dims[3], const float* mats_host,
                      int R, const float center[3], const float* mask) {
    TG_TRY(ensure_scratch(ctx, sizeof(float) * 9 * (size_t)R));
    float* d_m = static_cast<float*>(ctx->scratch);
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_m, mats_host, sizeof(float) * 9 * R, cudaMemcpyHostToDevice, ctx->stream));
    TG_TRY_CUDA(ctx, rotate3d_batch(in, out, dims, d_m, R, center, mask, ctx->stream));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // mats_host may go out of scope
    return TOMGPU_OK;
}

int tomgpu_rotate3d(tomgpu_ctx* ctx, const float* in, float* out, const int dims[3], const float* eom, int mode,
                    const float center[3]) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !out || !eom || !center || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    if (mode != TOMGPU_EULER_DEG && mode != TOMGPU_MATRIX) return fail(ctx, TOMGPU_ERR_ARG, "mode must be 1 or 3");
    TG_TRY(use_device(ctx));
    float m[9];
    if (mode == TOMGPU_EULER_DEG) euler_matrix_host(eom, m);
    else memcpy(m, eom, sizeof m);
    const size_t bytes = sizeof(float) * numel(dims);
    float *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, bytes) || cudaMalloc(&d_out, bytes)) {
        if (d_in) cudaFree(d_in);
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "rotate buffers");
    }
    int rc = TOMGPU_OK;
    cudaError_t e = cudaMemcpyAsync(d_in, in, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e) rc = cuda_fail(ctx, e, "upload");
    if (!rc) rc = rotate_dev(ctx, d_in, d_out, dims, m, 1, center, nullptr);
    if (!rc && (e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost))) rc = cuda_fail(ctx, e, "download");
    cudaFree(d_in);
    cudaFree(d_out);
    return rc;
}

int tomgpu_rotate3d_batch_dev(tomgpu_ctx* ctx, const float* in_dev, float* out_dev, const int dims[3],
                              const float* eulers, int R, const float center[3], const float* mask_dev) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in_dev || !out_dev || !eulers || !center || !dims_ok(dims) || R < 0)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    if (R == 0) return TOMGPU_OK;
    TG_TRY(use_device(ctx));
    std::vector<float> m(9 * (size_t)R);
    for (int r = 0; r < R; ++r) euler_matrix_host(eulers + 3 * r, m.data() + 9 * r);
    return rotate_dev(ctx, in_dev, out_dev, dims, m.data(), R, center, mask_dev);
}

// ---------------------------------------------------------------- peaks
int tomgpu_peak_dev(tomgpu_ctx* ctx, const float* v, const int dims[3], float* val, int pos1[3]) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!v || !val || !pos1 || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    const long long n = numel(dims);
    if (n > 0xFFFFFFFFll) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "more than 2^32 voxels");
    TG_TRY(use_device(ctx));
    TG_TRY(ensure_scratch(ctx, 64));
    unsigned long long* d_key = static_cast<unsigned long long*>(ctx->scratch);
    TG_TRY_CUDA(ctx, argmax_key(v, n, d_key, ctx->stream));
    ctx->launches += 1;
    unsigned long long key = 0;
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(&key, d_key, sizeof key, cudaMemcpyDeviceToHost, ctx->stream));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (key == 0) {  // nothing above the scan's start value: the reference leaves pos untouched
        *val = -99999.0f;
        return TOMGPU_OK;
    }
    const unsigned long long idx = 0xFFFFFFFFull - (key & 0xFFFFFFFFull);
    *val = peak_key_to_value(key);
    pos1[0] = (int)(idx % dims[0]) + 1;
    pos1[1] = (int)((idx / dims[0]) % dims[1]) + 1;
    pos1[2] = (int)(idx / ((unsigned long long)dims[0] * dims[1])) + 1;
    return TOMGPU_OK;
}

int tomgpu_peak(tomgpu_ctx* ctx, const float* v, const int dims[3], float* val, int pos1[3]) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!v || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    const size_t bytes = sizeof(float) * numel(dims);
    float* d = nullptr;
    if (cudaMalloc(&d, bytes)) return cuda_fail(ctx, cudaErrorMemoryAllocation, "peak buffer");
    int rc = TOMGPU_OK;
    cudaError_t e = cudaMemcpy(d, v, bytes, cudaMemcpyHostToDevice);
    if (e) rc = cuda_fail(ctx, e, "upload");
    if (!rc) rc = tomgpu_peak_dev(ctx, d, dims, val, pos1);
    cudaFree(d);
    return rc;
}

int tomgpu_topk_dev(tomgpu_ctx* ctx, const float* v, const int dims[3], int K, double radius, float* vals,
                    int* pos1) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!v || !vals || !pos1 || !dims_ok(dims) || K < 0 || !(radius >= 0) || std::isinf(radius))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims, K or radius (negative, NaN or infinite)");
    const long long n = numel(dims);
    if (n > 0xFFFFFFFFll) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "more than 2^32 voxels");
    if (K == 0) return TOMGPU_OK;
    TG_TRY(use_device(ctx));
    float* work = nullptr;
    float* d_vals = nullptr;
    int* d_pos = nullptr;
    if (cudaMalloc(&work, sizeof(float) * n) || cudaMalloc(&d_vals, sizeof(float) * K) ||
        cudaMalloc(&d_pos, sizeof(int) * 3 * K)) {
        if (work) cudaFree(work);
        if (d_vals) cudaFree(d_vals);
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "topk buffers");
    }
    int rc = TOMGPU_OK;
    do {
        if (ensure_scratch(ctx, 64)) { rc = TOMGPU_ERR_OOM; break; }
        cudaError_t e = cudaMemcpyAsync(work, v, sizeof(float) * n, cudaMemcpyDeviceToDevice, ctx->stream);
        if (!e) e = topk_rounds(work, dims, K, radius, static_cast<unsigned long long*>(ctx->scratch), d_vals,
                                d_pos, ctx->stream, &ctx->launches);
        if (!e) e = cudaMemcpyAsync(vals, d_vals, sizeof(float) * K, cudaMemcpyDeviceToHost, ctx->stream);
        if (!e) e = cudaMemcpyAsync(pos1, d_pos, sizeof(int) * 3 * K, cudaMemcpyDeviceToHost, ctx->stream);
        if (!e) e = cudaStreamSynchronize(ctx->stream);
        if (e) rc = cuda_fail(ctx, e, "topk");
    } while (0);
    cudaFree(work);
    cudaFree(d_vals);
    cudaFree(d_pos);
    return rc;
}

int tomgpu_peak_radius_dev(tomgpu_ctx* ctx, float* v, const int dims[3], double radius, float* val, int pos1[3]) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!v || !val || !pos1 || !dims_ok(dims) || !(radius >= 0) || std::isinf(radius))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims or radius (negative, NaN or infinite)");
    if (numel(dims) > 0xFFFFFFFFll) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "more than 2^32 voxels");
    TG_TRY(use_device(ctx));
    TG_TRY(ensure_scratch(ctx, 64 + 4 * sizeof(int)));
    unsigned long long* d_key = static_cast<unsigned long long*>(ctx->scratch);
    float* d_val = reinterpret_cast<float*>(static_cast<char*>(ctx->scratch) + 16);
    int* d_pos = reinterpret_cast<int*>(static_cast<char*>(ctx->scratch) + 32);
    TG_TRY_CUDA(ctx, topk_rounds(v, dims, 1, radius, d_key, d_val, d_pos, ctx->stream, &ctx->launches));
    int h[3];
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(val, d_val, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d_pos, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (h[0] > 0) { pos1[0] = h[0]; pos1[1] = h[1]; pos1[2] = h[2]; }
    return TOMGPU_OK;
}

int tomgpu_peak_spline_dev(tomgpu_ctx* ctx, const float* v, const int dims[3], const int pos1[3], double coord[3],
                           double* val) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!v || !pos1 || !coord || !val || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    for (int d = 0; d < 3; ++d)
        if (pos1[d] < 1 || pos1[d] > dims[d]) return fail(ctx, TOMGPU_ERR_ARG, "peak position outside the volume");
    TG_TRY(use_device(ctx));
    TG_TRY(ensure_scratch(ctx, 6 * sizeof(double)));
    double* d_out = static_cast<double*>(ctx->scratch);
    const int p0[3] = {pos1[0] - 1, pos1[1] - 1, pos1[2] - 1};
    TG_TRY_CUDA(ctx, spline_peak(v, dims, p0, d_out, ctx->stream));
    ctx->launches += 1;
    double h[6];
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d_out, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int d = 0; d < 3; ++d) coord[d] = h[d];
    *val = std::fmax(h[3], std::fmax(h[4], h[5]));
    return TOMGPU_OK;
}

// -------------------------------------------------------- weights, masks
int tomgpu_weight3d(tomgpu_ctx* ctx, const int dims[3], const double* angles, int n_tilt, double thickness,
                    float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(dims) || !out || n_tilt < 0 || (n_tilt > 0 && !angles))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    // frequency coordinate sequences exactly as the reference accumulates them
    std::vector<float> f[3];
    for (int d = 0; d < 3; ++d) {
        f[d].resize(dims[d]);
        float c = 0;
        for (int i = 1; i <= dims[d]; ++i) {
            f[d][i - 1] = c;
            c = c + (float)1.0 / dims[d];
            if (i == dims[d] / 2) c = -c;
        }
    }
    // tilt normals (Filtrans/tom_calc_weight_functioninc.c:181-190)
    const float pi_c = 3.1416f;
    const int thick = (int)thickness;
    std::vector<float> nrm(3 * (size_t)(n_tilt > 0 ? n_tilt : 1));
    for (int t = 0; t < n_tilt; ++t) {
        const float phi = (float)angles[2 * t] * pi_c / 180;
        const float th = (float)angles[2 * t + 1] * pi_c / 180;
        const float zw = (float)std::sin(th) * pi_c * thick;
        nrm[3 * t] = (float)zw * (float)std::cos(phi);
        nrm[3 * t + 1] = (float)zw * (float)std::sin(phi);
        nrm[3 * t + 2] = (float)std::cos(th) * pi_c * thick;
    }
    const long long n = numel(dims);
    float *d_w = nullptr, *d_f = nullptr, *d_n = nullptr;
    const size_t fl = (size_t)dims[0] + dims[1] + dims[2];
    if (cudaMalloc(&d_w, sizeof(float) * n) || cudaMalloc(&d_f, sizeof(float) * fl) ||
        cudaMalloc(&d_n, sizeof(float) * nrm.size())) {
        if (d_w) cudaFree(d_w);
        if (d_f) cudaFree(d_f);
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "weight buffers");
    }
    int rc = TOMGPU_OK;
    cudaError_t e = cudaMemcpy(d_f, f[0].data(), sizeof(float) * dims[0], cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_f + dims[0], f[1].data(), sizeof(float) * dims[1], cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_f + dims[0] + dims[1], f[2].data(), sizeof(float) * dims[2], cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(d_n, nrm.data(), sizeof(float) * nrm.size(), cudaMemcpyHostToDevice);
    if (!e) e = weight3d(d_w, dims, d_f, d_f + dims[0], d_f + dims[0] + dims[1], d_n, n_tilt, ctx->stream);
    if (!e) e = cudaStreamSynchronize(ctx->stream);
    if (!e) e = cudaMemcpy(out, d_w, sizeof(float) * n, cudaMemcpyDeviceToHost);
    if (e) rc = cuda_fail(ctx, e, "weight3d");
    ctx->launches += 1;
    cudaFree(d_w);
    cudaFree(d_f);
    cudaFree(d_n);
    return rc;
}

int tomgpu_wedge_dev(tomgpu_ctx* ctx, const int dims[3], double a, double b, int av3, float* out_dev) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(dims) || !out_dev) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    const double deg = 3.14159265358979323846 / 180.0;
    double t1, t2 = 0;
    if (!av3) t1 = std::tan(a * deg);
    else {
        t1 = std::tan(3.14159265358979323846 / 2 - b * deg);
        t2 = std::tan(-3.14159265358979323846 / 2 - a * deg);
    }
    TG_TRY_CUDA(ctx, wedge(out_dev, dims, t1, t2, av3, ctx->stream));
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_av3_average_add_dev(tomgpu_ctx* ctx, const int n[3], const tomgpu_avg_item* items, int K, double* avg,
                               double* wei) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(n) || K < 0 || (K > 0 && !items) || !avg || !wei)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims or negative count");
    for (int d = 0; d < 3; ++d)
        if (!fft_length_supported(n[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "box size not an FFT length");
    for (int k = 0; k < K; ++k)
        if (!items[k].particle || !items[k].wedge) return fail(ctx, TOMGPU_ERR_ARG, "item without particle or wedge");
    if (K == 0) return TOMGPU_OK;
    TG_TRY(use_device(ctx));
    return av3_average_add(ctx, n, items, K, avg, wei);
}

int tomgpu_av3_average_final_dev(tomgpu_ctx* ctx, const int n[3], const double* avg, const double* wei, double* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(n) || !avg || !wei || !out) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    for (int d = 0; d < 3; ++d)
        if (!fft_length_supported(n[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "box size not an FFT length");
    TG_TRY(use_device(ctx));
    return av3_average_final(ctx, n, avg, wei, out);
}

int tomgpu_corr3d_peaks_dev(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt,
                            const float* const* particles, int np, const double* angles_deg, int nang, const float* mask,
                            const tomgpu_wedge_spec* wedge_t, const tomgpu_wedge_spec* wedge_p, const float* mask_cc,
                            double* peak, double* val, int32_t* angle_idx) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(n) || nt < 1 || np < 1 || nang < 1 || !templates || !particles || !angles_deg || !peak || !val ||
        !angle_idx)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims or empty input");
    for (int d = 0; d < 3; ++d)
        if (!fft_length_supported(n[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "box size not an FFT length");
    for (int t = 0; t < nt; ++t) {
        if (!templates[t]) return fail(ctx, TOMGPU_ERR_ARG, "null template");
        if (wedge_t && (wedge_t[t].kind < 0 || wedge_t[t].kind > 2 ||
                        (wedge_t[t].kind == TOMGPU_WEDGE_VOLUME && !wedge_t[t].volume)))
            return fail(ctx, TOMGPU_ERR_ARG, "bad template wedge");
    }
    for (int p = 0; p < np; ++p) {
        if (!particles[p]) return fail(ctx, TOMGPU_ERR_ARG, "null particle");
        if (wedge_p && (wedge_p[p].kind < 0 || wedge_p[p].kind > 2 ||
                        (wedge_p[p].kind == TOMGPU_WEDGE_VOLUME && !wedge_p[p].volume)))
            return fail(ctx, TOMGPU_ERR_ARG, "bad particle wedge");
    }
    TG_TRY(use_device(ctx));
    return corr3d_peaks(ctx, n, templates, nt, particles, np, angles_deg, nang, mask, wedge_t, wedge_p, mask_cc, peak,
                        val, angle_idx);
}

int tomgpu_corr3d_peaks(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt,
                        const float* const* particles, int np, const double* angles_deg, int nang, const float* mask,
                        const tomgpu_wedge_spec* wedge_t, const tomgpu_wedge_spec* wedge_p, const float* mask_cc,
                        double* peak, double* val, int32_t* angle_idx) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!dims_ok(n) || nt < 1 || np < 1 || nang < 1 || !templates || !particles || !angles_deg || !peak || !val ||
        !angle_idx)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims or empty input");
    for (int t = 0; t < nt; ++t)
        if (!templates[t]) return fail(ctx, TOMGPU_ERR_ARG, "null template");
    for (int p = 0; p < np; ++p)
        if (!particles[p]) return fail(ctx, TOMGPU_ERR_ARG, "null particle");
    TG_TRY(use_device(ctx));
    // every host volume (templates, particles, masks, wedge volumes) goes into
    // one device buffer; the device entry point then gets pointers into it
    const long long nv = numel(n);
    std::vector<const float*> src;
    for (int t = 0; t < nt; ++t) src.push_back(templates[t]);
    for (int p = 0; p < np; ++p) src.push_back(particles[p]);
    const int i_mask = mask ? (int)src.size() : -1;
    if (mask) src.push_back(mask);
    const int i_mcc = mask_cc ? (int)src.size() : -1;
    if (mask_cc) src.push_back(mask_cc);
    std::vector<tomgpu_wedge_spec> wt, wp;
    std::vector<int> wt_i, wp_i;
    auto wedges = [&](const tomgpu_wedge_spec* w, int cnt, std::vector<tomgpu_wedge_spec>& out,
                      std::vector<int>& at) -> bool {
        if (!w) return true;
        for (int i = 0; i < cnt; ++i) {
            if (w[i].kind < 0 || w[i].kind > 2 || (w[i].kind == TOMGPU_WEDGE_VOLUME && !w[i].volume)) return false;
            out.push_back(w[i]);
            at.push_back(w[i].kind == TOMGPU_WEDGE_VOLUME ? (int)src.size() : -1);
            if (w[i].kind == TOMGPU_WEDGE_VOLUME) src.push_back(w[i].volume);
        }
        return true;
    };
    if (!wedges(wedge_t, nt, wt, wt_i)) return fail(ctx, TOMGPU_ERR_ARG, "bad template wedge");
    if (!wedges(wedge_p, np, wp, wp_i)) return fail(ctx, TOMGPU_ERR_ARG, "bad particle wedge");
    float* d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * nv * src.size()) != cudaSuccess)
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "corr3d input buffer");
    int rc = TOMGPU_OK;
    for (size_t i = 0; i < src.size() && !rc; ++i) {
        cudaError_t e = cudaMemcpyAsync(d + nv * i, src[i], sizeof(float) * nv, cudaMemcpyHostToDevice, ctx->stream);
        if (e) rc = cuda_fail(ctx, e, "corr3d upload");
    }
    if (!rc) {
        std::vector<const float*> tp(nt), pp(np);
        for (int t = 0; t < nt; ++t) tp[t] = d + nv * t;
        for (int p = 0; p < np; ++p) pp[p] = d + nv * (nt + p);
        for (size_t i = 0; i < wt.size(); ++i)
            if (wt_i[i] >= 0) wt[i].volume = d + nv * wt_i[i];
        for (size_t i = 0; i < wp.size(); ++i)
            if (wp_i[i] >= 0) wp[i].volume = d + nv * wp_i[i];
        rc = tomgpu_corr3d_peaks_dev(ctx, n, tp.data(), nt, pp.data(), np, angles_deg, nang,
                                     i_mask >= 0 ? d + nv * i_mask : nullptr, wedge_t ? wt.data() : nullptr,
                                     wedge_p ? wp.data() : nullptr, i_mcc >= 0 ? d + nv * i_mcc : nullptr, peak, val,
                                     angle_idx);
    }
    cudaStreamSynchronize(ctx->stream);
    cudaFree(d);
    return rc;
}

int tomgpu_analyze_psr_dev(tomgpu_ctx* ctx, const float* peak, const int map_dims[3], const int tmpl_dims[3],
                           float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!peak || !out || !dims_ok(map_dims) || !dims_ok(tmpl_dims))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    PeakAnalysis an;
    TG_TRY(an.create(ctx, map_dims, tmpl_dims, nullptr));
    TG_TRY(an.spectra(peak));
    TG_TRY(an.psr(peak, out));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_template_autocorr_dev(tomgpu_ctx* ctx, const float* t, const int tmpl_dims[3], float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!t || !out || !dims_ok(tmpl_dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    // the map-sized part is not used: size it at the template
    int nd[3] = {tmpl_dims[0], tmpl_dims[1], tmpl_dims[2]};
    PeakAnalysis an;
    TG_TRY(an.create(ctx, nd, tmpl_dims, nullptr));
    TG_TRY(an.autocorr(t, out));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_analyze_autocorr_dev(tomgpu_ctx* ctx, const float* peak, const int map_dims[3], const float* t,
                                const int tmpl_dims[3], const float* mask, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!peak || !t || !out || !dims_ok(map_dims) || !dims_ok(tmpl_dims))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    PeakAnalysis an;
    TG_TRY(an.create(ctx, map_dims, tmpl_dims, mask));
    TG_TRY(an.autocorr(t, an.tmp_t));
    TG_TRY(an.spectra(peak));
    TG_TRY(an.soc(peak, an.tmp_t, out));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_apply_weight_dev(tomgpu_ctx* ctx, const float* in, const float* w, const int dims[3], float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !w || !out || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    for (int d = 0; d < 3; ++d)
        if (dims[d] > 1 && !fft_length_supported(dims[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "size not an FFT length");
    TG_TRY(use_device(ctx));
    const long long n = numel(dims);
    double2* c = nullptr;
    double* r = nullptr;
    float* ws = nullptr;
    if (cudaMalloc(&c, sizeof(double2) * n) || cudaMalloc(&r, sizeof(double) * n) || cudaMalloc(&ws, sizeof(float) * n)) {
        if (c) cudaFree(c);
        if (r) cudaFree(r);
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "weight buffers");
    }
    cudaStream_t st = ctx->stream;
    cudaError_t e = ifftshift_real(w, ws, dims, st);
    if (!e) e = real_to_c64(in, c, n, st);
    if (!e) e = c2c3d<double2>(c, dims, -1, 1.0, st);
    if (!e) e = mul_weight_c64(c, ws, n, st);
    if (!e) e = c2c3d<double2>(c, dims, +1, 1.0 / (double)n, st);
    if (!e) e = re_c64(c, r, n, 1.0, st);
    if (!e) e = double_to_float(r, out, n, st);
    if (!e) e = cudaStreamSynchronize(st);
    ctx->launches += 10;
    cudaFree(c);
    cudaFree(r);
    cudaFree(ws);
    if (e) return cuda_fail(ctx, e, "apply_weight");
    return TOMGPU_OK;
}

// ----------------------------------------------------------------- FFTs
static int fft_dims_ok(tomgpu_ctx* ctx, const int dims[3]) {
    if (!dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "bad dims");
    for (int d = 0; d < 3; ++d)
        if (dims[d] > 1 && !fft_length_supported(dims[d]))
            return fail(ctx, TOMGPU_ERR_UNSUPPORTED,
                        "FFT length " + std::to_string(dims[d]) +
                            " beyond the line limits (every length up to 3528; {2,3,5,7,11,13}-smooth up to 7150)");
    return TOMGPU_OK;
}

int tomgpu_fft3d_c2c_dev(tomgpu_ctx* ctx, void* data, const int dims[3], int dir, int precision) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!data || (dir != -1 && dir != 1) || (precision != 32 && precision != 64))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, dir or precision");
    TG_TRY(fft_dims_ok(ctx, dims));
    TG_TRY(use_device(ctx));
    const double sc = dir > 0 ? 1.0 / (double)numel(dims) : 1.0;
    cudaError_t e = precision == 32 ? c2c3d<float2>((float2*)data, dims, dir, sc, ctx->stream)
                                    : c2c3d<double2>((double2*)data, dims, dir, sc, ctx->stream);
    ctx->launches += 3;
    if (e) return cuda_fail(ctx, e, "fft3d_c2c");
    return TOMGPU_OK;
}

int tomgpu_fft3d_r2c_dev(tomgpu_ctx* ctx, const void* real, void* half, const int dims[3], int precision) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!real || !half || (precision != 32 && precision != 64)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or precision");
    TG_TRY(fft_dims_ok(ctx, dims));
    TG_TRY(use_device(ctx));
    cudaError_t e = precision == 32 ? r2c3d<float2>(real, (float2*)half, dims, ctx->stream)
                                    : r2c3d<double2>(real, (double2*)half, dims, ctx->stream);
    ctx->launches += 3;
    if (e) return cuda_fail(ctx, e, "fft3d_r2c");
    return TOMGPU_OK;
}

int tomgpu_fft3d_c2r_dev(tomgpu_ctx* ctx, void* half, void* real, const int dims[3], int precision) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!real || !half || (precision != 32 && precision != 64)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or precision");
    TG_TRY(fft_dims_ok(ctx, dims));
    TG_TRY(use_device(ctx));
    const double sc = 1.0 / (double)numel(dims);
    cudaError_t e = precision == 32 ? c2r3d<float2>((float2*)half, real, dims, sc, ctx->stream)
                                    : c2r3d<double2>((double2*)half, real, dims, sc, ctx->stream);
    ctx->launches += 3;
    if (e) return cuda_fail(ctx, e, "fft3d_c2r");
    return TOMGPU_OK;
}

// ------------------------------------------------------------- matching
int tomgpu_match_plan_create(tomgpu_ctx* ctx, const int vol[3], const int tm[3], const tomgpu_match_params* params,
                             tomgpu_match_plan** out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!out || !dims_ok(vol) || !dims_ok(tm)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    *out = nullptr;
    if (params && params->batch < 0) return fail(ctx, TOMGPU_ERR_ARG, "negative batch");
    if (params && (params->path < 0 || params->path > 3)) return fail(ctx, TOMGPU_ERR_ARG, "path is 0, 1, 2 or 3");
    TG_TRY(use_device(ctx));
    tomgpu_match_plan* p = new tomgpu_match_plan();
    int rc = p->p.create(ctx, vol, tm, params ? params->batch : 0, params ? params->path == 1 : false);
    p->p.no_tma = params && params->path == 2;
    p->p.tc_inv_z = params && params->path == 3;
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return TOMGPU_OK;
}

int tomgpu_match_plan_destroy(tomgpu_match_plan* plan) {
    if (!plan) return TOMGPU_OK;
    if (plan->p.ctx) {
        cudaSetDevice(plan->p.ctx->device);
        cudaStreamSynchronize(plan->p.ctx->stream);
    }
    delete plan;
    return TOMGPU_OK;
}

int64_t tomgpu_match_plan_bytes(const tomgpu_match_plan* plan) { return plan ? plan->p.bytes_held : 0; }

int tomgpu_match_set_template_dev(tomgpu_match_plan* plan, const float* t, const float* mask, const float* psf) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!t || !mask) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "template and mask are required");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.set_template(t, mask, psf);
}

int tomgpu_match_set_volume_dev(tomgpu_match_plan* plan, const float* vol) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!vol) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "volume is NULL");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.set_volume(vol);
}

int tomgpu_match_init_results_dev(tomgpu_match_plan* plan, float* maxcc, int32_t* angidx) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!maxcc || !angidx) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null result buffer");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.init_results(maxcc, angidx);
}

int tomgpu_match_run_dev(tomgpu_match_plan* plan, const float* eulers, int R, int index_offset, float* maxcc,
                         int32_t* angidx) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (R < 0 || (R > 0 && (!eulers || !maxcc || !angidx)) || index_offset < 0)
        return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null pointer, negative count or offset");
    // the result update moves voxel pairs as 8-byte words
    if ((reinterpret_cast<uintptr_t>(maxcc) | reinterpret_cast<uintptr_t>(angidx)) & 7u)
        return fail(plan->p.ctx, TOMGPU_ERR_ARG, "result buffers must be 8-byte aligned");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.run(eulers, R, index_offset, maxcc, angidx);
}

int tomgpu_match_autotune(tomgpu_match_plan* plan, const float* eulers, int R, const int* cands, int n_cand,
                          int* best, float* ms_per_rot) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!eulers || !cands || R <= 0 || n_cand <= 0) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "bad autotune arguments");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.autotune(eulers, R, cands, n_cand, best, ms_per_rot);
}

int tomgpu_match_set_template_raw_dev(tomgpu_match_plan* plan, const float* t, const float* mask) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!t || !mask) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "template and mask are required");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.set_template(t, mask, nullptr, true);
}

int tomgpu_match_init_analysis_dev(tomgpu_match_plan* plan, float* maxcc, int32_t* angidx, float* psr, float* soc) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!maxcc || !angidx || !psr || !soc) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null result buffer");
    TG_TRY(use_device(plan->p.ctx));
    return analysis_init(plan->p.ctx, plan->p.nvox, maxcc, angidx, psr, soc);
}

int tomgpu_match_run_analysis_dev(tomgpu_match_plan* plan, const float* eulers, int R, int index_offset, int flags,
                                  float* maxcc, int32_t* angidx, float* psr, float* soc) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (R < 0 || (R > 0 && (!eulers || !maxcc || !angidx || !psr || !soc)) || index_offset < 0)
        return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null pointer, negative count or offset");
    if ((flags & 7) == 0 || (flags & ~7))
        return fail(plan->p.ctx, TOMGPU_ERR_ARG, "flags must select ccc, psr and/or autocorr");
    TG_TRY(use_device(plan->p.ctx));
    TG_TRY(plan->p.run_analysis(eulers, R, index_offset, flags, maxcc, angidx, psr, soc));
    TG_TRY_CUDA(plan->p.ctx, cudaStreamSynchronize(plan->p.ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_match_corr_dev(tomgpu_match_plan* plan, const float* t, float* cc) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!t || !cc) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null pointer");
    if (reinterpret_cast<uintptr_t>(cc) & 3u) return fail(plan->p.ctx, TOMGPU_ERR_ARG, "cc must be 4-byte aligned");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.corr(t, cc);
}

int tomgpu_match_rescore_fp64_dev(tomgpu_match_plan* plan, const float* vol, const float* eulers, const int* pos1,
                                  int K, double* cc) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (K < 0 || (K > 0 && (!vol || !eulers || !pos1 || !cc)))
        return fail(plan->p.ctx, TOMGPU_ERR_ARG, "null pointer or negative count");
    TG_TRY(use_device(plan->p.ctx));
    return plan->p.rescore(vol, eulers, pos1, K, cc);
}

int tomgpu_match_stats_dev(tomgpu_match_plan* plan, float* mean, float* std) {
    if (!plan) return TOMGPU_ERR_ARG;
    if (!plan->p.has_volume) return fail(plan->p.ctx, TOMGPU_ERR_STATE, "no volume set");
    TG_TRY(use_device(plan->p.ctx));
    tomgpu_ctx* ctx = plan->p.ctx;
    const size_t bytes = sizeof(float) * plan->p.nvox;
    if (mean) {
        // local mean of I = local mean of I - c, plus c
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(mean, plan->p.d_mu0, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        TG_TRY_CUDA(ctx, normalize_f32(mean, mean, plan->p.nvox, 1.0, plan->p.vmean, 0.0, 1.0, ctx->stream));
        ctx->launches += 1;
    }
    if (std) TG_TRY_CUDA(ctx, cudaMemcpyAsync(std, plan->p.d_sig, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_corr_dev(tomgpu_ctx* ctx, const float* a, const float* b, const int dims[3], const float* mask,
                    const float* psf1, const float* psf2, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!a || !b || !out || !dims_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    return corr_norm(ctx, a, b, dims, mask, psf1, psf2, out);
}

int tomgpu_av3_align_ex_dev(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs,
                            const tomgpu_align_params* params, float* angles, float* shifts, float* ccf_peak) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (n_jobs < 0 || (n_jobs > 0 && (!jobs || !angles || !shifts || !ccf_peak)))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or negative job count");
    tomgpu_align_params prm{};
    if (params) prm = *params;
    if (prm.path < 0 || prm.path > 2) return fail(ctx, TOMGPU_ERR_ARG, "path must be 0, 1 or 2");
    TG_TRY(use_device(ctx));
    for (int j = 0; j < n_jobs; ++j) {
        const tomgpu_align_job& jb = jobs[j];
        if (!dims_ok(jb.n)) return fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(j) + ": bad box size");
        for (int a = 0; a < 3; ++a) {
            const float* r = a == 0 ? jb.phi : (a == 1 ? jb.psi : jb.theta);
            if (r[1] < 0 || (r[1] == 0 && r[2] != r[0]) || r[2] < r[0])
                return fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(j) + ": bad angle range");
        }
        if (!jb.ref || !jb.part || !jb.mask)
            return fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(j) + ": job needs ref, part and mask");
    }
    // jobs of a compiled cubic edge run batched, per (edge, wedge form); the rest one by one
    std::map<std::pair<int, int>, std::vector<int>> buckets;
    std::vector<int> rest;
    for (int j = 0; j < n_jobs; ++j) {
        if (prm.path != 1 && align_fused_supported(jobs[j]))
            buckets[{jobs[j].n[0], jobs[j].wedge_ref ? 1 : 0}].push_back(j);
        else
            rest.push_back(j);
    }
    if (!ctx->align_scratch) ctx->align_scratch = align_scratch_new();
    AlignScratch* scratch = static_cast<AlignScratch*>(ctx->align_scratch);
    int rc = TOMGPU_OK;
    for (auto& kv : buckets) {
        if (rc) break;
        rc = align_fused(ctx, jobs, kv.second.data(), (int)kv.second.size(), angles, shifts, ccf_peak,
                         prm.batch_bytes, prm.path != 2, scratch);
    }
    for (int j : rest) {
        if (rc) break;
        rc = align_job(ctx, jobs[j], angles + 3 * j, shifts + 3 * j, ccf_peak + j, (size_t)1 << 24, scratch);
    }
    cudaStreamSynchronize(ctx->stream);
    return rc;
}

int tomgpu_av3_align_dev(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs, float* angles, float* shifts,
                         float* ccf_peak) {
    return tomgpu_av3_align_ex_dev(ctx, jobs, n_jobs, nullptr, angles, shifts, ccf_peak);
}

int tomgpu_av3_align(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, int n_jobs, const tomgpu_align_params* params,
                     float* angles, float* shifts, float* ccf_peak) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (n_jobs < 0 || (n_jobs > 0 && (!jobs || !angles || !shifts || !ccf_peak)))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or negative job count");
    TG_TRY(use_device(ctx));
    // the distinct host arrays, each with its voxel count
    std::map<const float*, long long> vols;
    for (int j = 0; j < n_jobs; ++j) {
        const tomgpu_align_job& jb = jobs[j];
        if (!dims_ok(jb.n)) return fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(j) + ": bad box size");
        const long long nn = numel(jb.n);
        const float* p[6] = {jb.ref, jb.part, jb.mask, jb.mask_ccf, jb.wedge_ref, jb.wedge_part};
        for (const float* q : p) {
            if (!q) continue;
            auto it = vols.find(q);
            if (it == vols.end()) vols.emplace(q, nn);
            else if (it->second != nn)
                return fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(j) + ": an array shared by jobs of "
                                                 "different box sizes");
        }
    }
    long long total = 0;
    for (auto& kv : vols) total += kv.second;
    float* dev = nullptr;
    if (total > 0 && cudaMalloc(&dev, sizeof(float) * total) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, TOMGPU_ERR_OOM, "av3_align: device copies of the volumes");
    }
    std::map<const float*, const float*> where;
    long long off = 0;
    int rc = TOMGPU_OK;
    for (auto& kv : vols) {
        if (cudaError_t e = cudaMemcpyAsync(dev + off, kv.first, sizeof(float) * kv.second, cudaMemcpyHostToDevice,
                                            ctx->stream)) {
            rc = cuda_fail(ctx, e, "av3_align: upload");
            break;
        }
        where[kv.first] = dev + off;
        off += kv.second;
    }
    if (!rc) {
        std::vector<tomgpu_align_job> dj(jobs, jobs + n_jobs);
        auto map = [&](const float* q) { return q ? where[q] : nullptr; };
        for (auto& jb : dj) {
            jb.ref = map(jb.ref);
            jb.part = map(jb.part);
            jb.mask = map(jb.mask);
            jb.mask_ccf = map(jb.mask_ccf);
            jb.wedge_ref = map(jb.wedge_ref);
            jb.wedge_part = map(jb.wedge_part);
        }
        rc = tomgpu_av3_align_ex_dev(ctx, dj.data(), n_jobs, params, angles, shifts, ccf_peak);
    }
    cudaStreamSynchronize(ctx->stream);
    if (dev) cudaFree(dev);
    return rc;
}

int tomgpu_ctx_trim(tomgpu_ctx* ctx) {
    if (!ctx) return TOMGPU_ERR_ARG;
    TG_TRY(use_device(ctx));
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_match_cache(ctx);
    drop_align_scratch(ctx);
    return TOMGPU_OK;
}

int tomgpu_match(tomgpu_ctx* ctx, const float* tomo, const int vol[3], const float* tmpl, const int tm[3],
                 const float* mask, const float* psf, const float* eulers, int R, const tomgpu_match_params* params,
                 float* maxcc, int32_t* angidx) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!tomo || !tmpl || !mask || !maxcc || !angidx || (R > 0 && !eulers) || R < 0 || !dims_ok(vol) || !dims_ok(tm))
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer or bad dims");
    TG_TRY(use_device(ctx));
    tomgpu_match_params prm{};
    if (params) prm = *params;
    MatchCache* mc = static_cast<MatchCache*>(ctx->match_cache);
    if (mc && !mc->same(vol, tm, prm, psf != nullptr)) {
        cudaStreamSynchronize(ctx->stream);
        drop_match_cache(ctx);
        mc = nullptr;
    }
    const long long nv = numel(vol), nt = numel(tm);
    if (!mc) {
        mc = new MatchCache();
        for (int d = 0; d < 3; ++d) { mc->vol[d] = vol[d]; mc->tm[d] = tm[d]; }
        mc->prm = prm;
        mc->psf = psf != nullptr;
        int rc = tomgpu_match_plan_create(ctx, vol, tm, params, &mc->plan);
        if (!rc && (cudaMalloc(&mc->d_vol, sizeof(float) * nv) || cudaMalloc(&mc->d_t, sizeof(float) * nt) ||
                    cudaMalloc(&mc->d_m, sizeof(float) * nt) || (psf && cudaMalloc(&mc->d_p, sizeof(float) * nt)) ||
                    cudaMalloc(&mc->d_cc, sizeof(float) * nv) || cudaMalloc(&mc->d_i, sizeof(int) * nv))) {
            cudaGetLastError();
            rc = cuda_fail(ctx, cudaErrorMemoryAllocation, "match buffers");
        }
        if (rc) {
            delete mc;
            return rc;
        }
        ctx->match_cache = mc;
    }
    tomgpu_match_plan* plan = mc->plan;
    int rc = TOMGPU_OK;
    cudaStream_t st = ctx->stream;
    do {
        cudaError_t e = cudaMemcpyAsync(mc->d_vol, tomo, sizeof(float) * nv, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(mc->d_t, tmpl, sizeof(float) * nt, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(mc->d_m, mask, sizeof(float) * nt, cudaMemcpyHostToDevice, st);
        if (!e && psf) e = cudaMemcpyAsync(mc->d_p, psf, sizeof(float) * nt, cudaMemcpyHostToDevice, st);
        if (e) { rc = cuda_fail(ctx, e, "upload"); break; }
        if ((rc = tomgpu_match_set_template_dev(plan, mc->d_t, mc->d_m, mc->d_p))) break;
        if ((rc = tomgpu_match_set_volume_dev(plan, mc->d_vol))) break;
        if ((rc = tomgpu_match_init_results_dev(plan, mc->d_cc, mc->d_i))) break;
        if ((rc = tomgpu_match_run_dev(plan, eulers, R, 0, mc->d_cc, mc->d_i))) break;
        e = cudaMemcpyAsync(maxcc, mc->d_cc, sizeof(float) * nv, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaMemcpyAsync(angidx, mc->d_i, sizeof(int) * nv, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) { rc = cuda_fail(ctx, e, "download"); break; }
    } while (0);
    if (rc) {  // leave nothing half-set for the next call
        cudaStreamSynchronize(st);
        drop_match_cache(ctx);
    }
    return rc;
}

}  // extern "C"

// ---------------------------------------------------------------- learned proposer
namespace tg {
cudaError_t cnn_conv_fwd(const float* in, int ci, const int d[3], const float* w, const float* b, int co, int dil,
                         int relu, float* out, cudaStream_t st);
cudaError_t cnn_conv_wgrad(const float* in, int ci, const int d[3], const float* gout, int co, int dil, float* gw,
                           float* gb, cudaStream_t st);
cudaError_t cnn_flip_weights(const float* w, int co, int ci, float* wt, cudaStream_t st);
cudaError_t cnn_relu_bwd(float* g, const float* act, long long n, cudaStream_t st);
cudaError_t cnn_bce(const float* logit, const float* target, long long n, float pw, float* grad, double* loss,
                    cudaStream_t st);
cudaError_t cnn_softmax_ce(const float* logits, const int* labels, int K, int P, float* grad, double* loss,
                           cudaStream_t st);
cudaError_t cnn_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                     int step, cudaStream_t st);
cudaError_t cnn_dense_fwd(const float* W, const float* b, const float* F, int K, int C, long long P, int relu,
                          float* out, cudaStream_t st);
cudaError_t cnn_dense_bwd(const float* W, const float* F, const float* g, int K, int C, long long P, float* gF,
                          float* gW, float* gb, cudaStream_t st);
cudaError_t cnn_gather(const float* f, int C, long long nv, const long long* idx, int P, float* out, cudaStream_t st);
cudaError_t cnn_scatter_add(const float* g, int C, long long nv, const long long* idx, int P, float* gf,
                            cudaStream_t st);
}  // namespace tg

static bool cnn_ch_ok(int c) { return c == 1 || c == 8 || c == 16 || c == 32 || c == 64; }

int tomgpu_cnn_conv3d_fwd_dev(tomgpu_ctx* ctx, const float* in, int ci, const int dims[3], const float* w,
                              const float* b, int co, int dil, int relu, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !w || !out || !dims_ok(dims) || ci < 1 || dil < 1 || dil > 16)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims, channels or dilation");
    if (!cnn_ch_ok(co)) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "output channels must be 1, 8, 16, 32 or 64");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_conv_fwd(in, ci, dims, w, b, co, dil, relu, out, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_conv3d_bwd_data_dev(tomgpu_ctx* ctx, const float* gout, int co, const int dims[3], const float* w,
                                   int ci, int dil, float* gin) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!gout || !w || !gin || !dims_ok(dims) || co < 1 || dil < 1 || dil > 16)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims, channels or dilation");
    if (!cnn_ch_ok(ci)) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "input channels must be 1, 8, 16, 32 or 64");
    TG_TRY(use_device(ctx));
    TG_TRY(ensure_scratch(ctx, sizeof(float) * (size_t)co * ci * 27));
    float* wt = static_cast<float*>(ctx->scratch);
    TG_TRY_CUDA(ctx, cnn_flip_weights(w, co, ci, wt, ctx->stream));
    TG_TRY_CUDA(ctx, cnn_conv_fwd(gout, co, dims, wt, nullptr, ci, dil, 0, gin, ctx->stream));
    ctx->launches += 2;
    return TOMGPU_OK;
}

int tomgpu_cnn_conv3d_bwd_weight_dev(tomgpu_ctx* ctx, const float* in, int ci, const int dims[3], const float* gout,
                                     int co, int dil, float* gw, float* gb) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !gout || !gw || !dims_ok(dims) || ci < 1 || co < 1 || dil < 1 || dil > 16)
        return fail(ctx, TOMGPU_ERR_ARG, "null pointer, bad dims, channels or dilation");
    TG_TRY(use_device(ctx));
    ctx->launches += gb ? 2 : 1;
    TG_TRY_CUDA(ctx, cnn_conv_wgrad(in, ci, dims, gout, co, dil, gw, gb, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_dense_fwd_dev(tomgpu_ctx* ctx, const float* W, const float* b, const float* F, int K, int C, int64_t P,
                             int relu, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!W || !F || !out || K < 1 || C < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad dense layer arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_dense_fwd(W, b, F, K, C, P, relu, out, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_dense_bwd_dev(tomgpu_ctx* ctx, const float* W, const float* F, const float* g, int K, int C, int64_t P,
                             float* gF, float* gW, float* gb) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!W || !F || !g || K < 1 || C < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad dense layer arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 3;
    TG_TRY_CUDA(ctx, cnn_dense_bwd(W, F, g, K, C, P, gF, gW, gb, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_relu_bwd_dev(tomgpu_ctx* ctx, float* g, const float* act, int64_t n) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!g || !act || n < 0) return fail(ctx, TOMGPU_ERR_ARG, "null pointer");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_relu_bwd(g, act, n, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_bce_dev(tomgpu_ctx* ctx, const float* logit, const float* target, int64_t n, float pos_weight,
                       float* grad, double* loss_dev) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!logit || !target || !grad || !loss_dev || n < 1) return fail(ctx, TOMGPU_ERR_ARG, "null pointer");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_bce(logit, target, n, pos_weight, grad, loss_dev, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_softmax_ce_dev(tomgpu_ctx* ctx, const float* logits, const int32_t* labels, int K, int P, float* grad,
                              double* loss_dev) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!logits || !labels || !grad || !loss_dev || K < 2 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_softmax_ce(logits, labels, K, P, grad, loss_dev, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_adam_dev(tomgpu_ctx* ctx, float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1,
                        float b2, float eps, int step) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!p || !g || !m || !v || n < 1 || step < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_adam(p, g, m, v, n, lr, b1, b2, eps, step, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_gather_dev(tomgpu_ctx* ctx, const float* f, int C, int64_t nv, const int64_t* idx, int P, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!f || !idx || !out || C < 1 || nv < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_gather(f, C, nv, reinterpret_cast<const long long*>(idx), P, out, ctx->stream));
    return TOMGPU_OK;
}

int tomgpu_cnn_scatter_add_dev(tomgpu_ctx* ctx, const float* g, int C, int64_t nv, const int64_t* idx, int P,
                               float* gf) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!g || !idx || !gf || C < 1 || nv < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cnn_scatter_add(g, C, nv, reinterpret_cast<const long long*>(idx), P, gf, ctx->stream));
    return TOMGPU_OK;
}
