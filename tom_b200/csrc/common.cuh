// Shared device helpers for the tomgpu CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define TG_HD __host__ __device__ __forceinline__
#define TG_D __device__ __forceinline__

// ---------------------------------------------------------------- complex
TG_HD float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
TG_HD float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
TG_HD float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
TG_HD float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
TG_HD float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
TG_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

TG_HD double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
TG_HD double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
TG_HD double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
TG_HD double2 cmulc(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
TG_HD double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
TG_HD double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

template <typename C> struct CTraits;
template <> struct CTraits<float2> {
    typedef float R;
    static TG_HD float2 make(float a, float b) { return make_float2(a, b); }
};
template <> struct CTraits<double2> {
    typedef double R;
    static TG_HD double2 make(double a, double b) { return make_double2(a, b); }
};

// multiply by +i (s = +1) or -i (s = -1)
template <int S, typename C> TG_HD C cmul_i(C a) {
    return S > 0 ? CTraits<C>::make(-a.y, a.x) : CTraits<C>::make(a.y, -a.x);
}

// ------------------------------------------------------- error reporting
// Kernels never trap: a kernel that meets an impossible state writes a code
// into a device error word and returns; the host reads it after the stream
// synchronises and turns it into a status code.
enum TgDeviceError : int {
    TG_DEV_OK = 0,
    TG_DEV_BAD_INDEX = 1,
    TG_DEV_TIMEOUT = 2,
};

TG_D void tg_flag_error(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

// floor division / positive modulo for signed offsets
TG_HD int pmod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }
