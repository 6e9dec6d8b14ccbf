// 29-point DFT for the 928 / 464 edges (928 = 29 x 32, 464 = 29 x 16).
//
// Direct evaluation with the real/imaginary symmetry of the kernel: for
// k = 1..14, X[k] and X[29-k] share x0 + sum_n (x_n + x_{29-n}) cos(2 pi nk/29)
// and differ in the sign of i sum_n (x_n - x_{29-n}) sin(2 pi nk/29), so a
// transform costs 14 x 28 complex-by-real multiply-adds.  The cosines and
// sines (the host's double values rounded to float) come in a kernel
// parameter, so every use is a constant-bank operand of the multiply-add.
#pragma once
#include "common.cuh"

namespace tgpq {

struct Cos29 {
    float c[29];  // cos(2 pi j / 29)
    float s[29];  // sin(2 pi j / 29)
};

// In place, v[0..28]; DIR -1: X[k] = sum x[n] exp(-2 pi i nk/29), DIR +1: exp(+...).
template <int DIR>
TG_D void dft29(float2* v, const Cos29& t) {
    float2 p[14], m[14];
#pragma unroll
    for (int n = 1; n <= 14; ++n) {
        p[n - 1] = cadd(v[n], v[29 - n]);
        m[n - 1] = csub(v[n], v[29 - n]);
    }
    const float2 x0 = v[0];
    float2 s0 = x0;
#pragma unroll
    for (int n = 0; n < 14; ++n) s0 = cadd(s0, p[n]);
    v[0] = s0;
#pragma unroll
    for (int k = 1; k <= 14; ++k) {
        float2 re = x0, im = make_float2(0.f, 0.f);
#pragma unroll
        for (int n = 1; n <= 14; ++n) {
            const int j = (n * k) % 29;
            const float c = t.c[j], s = t.s[j];
            re.x = fmaf(c, p[n - 1].x, re.x);
            re.y = fmaf(c, p[n - 1].y, re.y);
            im.x = fmaf(s, m[n - 1].x, im.x);
            im.y = fmaf(s, m[n - 1].y, im.y);
        }
        // DIR i im
        const float2 d = DIR > 0 ? make_float2(-im.y, im.x) : make_float2(im.y, -im.x);
        v[k] = cadd(re, d);
        v[29 - k] = csub(re, d);
    }
}

// The same transform without an output array: the inputs are folded in place
// into x0, the 14 sums and the 14 differences, and each output is handed to
// emit(k, X[k]) as soon as it is formed (k a compile-time index after
// unrolling), so the caller stores or consumes it without holding all 29.
template <int DIR, typename Emit>
TG_D void dft29_emit(float2* v, const Cos29& t, Emit&& emit) {
#pragma unroll
    for (int n = 1; n <= 14; ++n) {
        const float2 a = v[n], b = v[29 - n];
        v[n] = cadd(a, b);       // p_n
        v[29 - n] = csub(a, b);  // m_n
    }
    const float2 x0 = v[0];
    float2 s0 = x0;
#pragma unroll
    for (int n = 1; n <= 14; ++n) s0 = cadd(s0, v[n]);
    emit(0, s0);
#pragma unroll
    for (int k = 1; k <= 14; ++k) {
        float2 re = x0, im = make_float2(0.f, 0.f);
#pragma unroll
        for (int n = 1; n <= 14; ++n) {
            const int j = (n * k) % 29;
            const float c = t.c[j], s = t.s[j];
            re.x = fmaf(c, v[n].x, re.x);
            re.y = fmaf(c, v[n].y, re.y);
            im.x = fmaf(s, v[29 - n].x, im.x);
            im.y = fmaf(s, v[29 - n].y, im.y);
        }
        const float2 d = DIR > 0 ? make_float2(-im.y, im.x) : make_float2(im.y, -im.x);
        emit(k, cadd(re, d));
        emit(29 - k, csub(re, d));
    }
}

}  // namespace tgpq
