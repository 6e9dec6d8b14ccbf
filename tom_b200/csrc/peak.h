#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
namespace tg {
// 64-bit key of the first strict maximum (0 when no value exceeds -99999).
cudaError_t argmax_key(const float* v, long long n, unsigned long long* d_key, cudaStream_t st);
// K rounds of (arg-max, zero the ball of `radius`), in place on `work`.
cudaError_t topk_rounds(float* work, const int dims[3], int K, double radius, unsigned long long* d_key,
                        float* d_vals, int* d_pos, cudaStream_t st, int64_t* launches);
// tom_intpeak at the 0-based integer peak pos0: d_out = 3 coords (1-based) + 3 values.
cudaError_t spline_peak(const float* v, const int dims[3], const int pos0[3], double* d_out, cudaStream_t st);
float peak_key_to_value(unsigned long long key);
}  // namespace tg
