#pragma once
#include <cuda_runtime.h>
namespace tg {
// K candidates (0-based positions pos0_dev, K x 3) of templates t3 (K x T^3 doubles,
// already rotated, masked, filtered) rescored in FP64 by direct sums.
cudaError_t rescore_fp64(const float* vol, const int N[3], const double* t3, const float* mask, const int T[3],
                         const int* pos0_dev, int K, double msize, double tmean, double tstd, double* out_dev,
                         cudaStream_t st);
cudaError_t f32_to_f64(const float* a, double* b, long long n, cudaStream_t st);
}  // namespace tg
