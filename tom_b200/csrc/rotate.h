#pragma once
#include <cuda_runtime.h>
namespace tg {
// R rotations of `in` (dims[0] x dims[1] x dims[2], x fastest) with the R x 9
// matrices at mats_dev; out holds R volumes; optional mask multiplies.
cudaError_t rotate3d_batch(const float* in, float* out, const int dims[3], const float* mats_dev, int R,
                           const float center[3], const float* mask, cudaStream_t st);
}  // namespace tg
