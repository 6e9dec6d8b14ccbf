// Generic batched line FFTs and 3-D transforms (see fft3d.cu).
#pragma once
#include <cuda_runtime.h>

#include "twiddles.h"
#include "fft_plan.h"

namespace tg {

enum { FFT_C2C = 0, FFT_R2C = 1, FFT_C2R = 2 };

// Lines of a 3-D array: element e of line l sits at
//   (l % cnt0) * s0 + (l / cnt0) * s1 + e * es      (in array elements).
struct LineGeom {
    long es;
    int cnt0;
    long s0;
    int cnt1;
    long s1;
};

// Any line length the library transforms (compile-time or run-time plan).
bool fft_length_supported(int L);

// One batched FFT of length L along lines (in and out may alias: each block
// reads all of its lines before writing).  R2C reads reals and writes the
// L/2+1 non-negative frequencies; C2R reads L/2+1 frequencies (Hermitian
// extension) and writes reals.  scale multiplies the output.
template <typename C>
cudaError_t fft_lines(int L, int dir, int mode, const void* in, void* out, const LineGeom& gi,
                      const LineGeom& go, long nlines, double scale, cudaStream_t st);

template <typename C> cudaError_t r2c3d(const void* real_in, C* half_out, const int n[3], cudaStream_t st);
template <typename C>
cudaError_t c2r3d(C* half_inout, void* real_out, const int n[3], double scale, cudaStream_t st);
template <typename C> cudaError_t c2c3d(C* data, const int n[3], int dir, double scale, cudaStream_t st);
// E volumes stored one after another (FP32)
template <typename C>
cudaError_t r2c3d_batch(const void* real_in, C* half_out, const int n[3], int E, cudaStream_t st);
template <typename C>
cudaError_t c2r3d_batch(C* half_inout, void* real_out, const int n[3], int E, double scale, cudaStream_t st);

}  // namespace tg
