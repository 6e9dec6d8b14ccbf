// Trilinear ZXZ rotation (replaces rot3d, Sptrans/tom_rotatec.c:291-399).
//
// One thread per output voxel, blockIdx.y selects the rotation of a batch.
// The arithmetic follows rot3d operation by operation with explicit
// round-to-nearest intrinsics (no FMA contraction), so the output equals the
// reference bit for bit given the same 9 matrix floats: source coordinate
// r = c + M (x - c) with the integer-truncated offsets rot3d uses, rejection
// outside [0, n-1] per axis, and rot3d's trilinear form in which the first
// x-interpolation is written a + (b - a) w and the other three a u + b w, with
// neighbours beyond the last index read as 0.
#include "rotate.h"
#include "rotate_sample.cuh"

namespace tg {

struct Mat9 { float m[9]; };

__global__ void __launch_bounds__(256) k_rotate3d(const float* __restrict__ in, float* __restrict__ out,
                                                  int sx, int sy, int sz, const float* __restrict__ mats,
                                                  float px, float py, float pz,
                                                  const float* __restrict__ mask) {
    const long long n = (long long)sx * sy * sz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (v >= n) return;
    float m[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = __ldg(mats + 9 * r + q);
    const int i = (int)(v % sx);
    const int j = (int)((v / sx) % sy);
    const int k = (int)(v / ((long long)sx * sy));
    float val = rot_sample(in, sx, sy, sz, m, px, py, pz, i, j, k);
    if (mask) val = __fmul_rn(val, __ldg(mask + v));
    out[(long long)r * n + v] = val;
}

cudaError_t rotate3d_batch(const float* in, float* out, const int dims[3], const float* mats_dev, int R,
                           const float center[3], const float* mask, cudaStream_t st) {
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    if (n <= 0 || R <= 0) return cudaSuccess;
    dim3 grid((unsigned)((n + 255) / 256), (unsigned)R);
    k_rotate3d<<<grid, 256, 0, st>>>(in, out, dims[0], dims[1], dims[2], mats_dev, center[0],
                                     center[1], center[2], mask);
    return cudaGetLastError();
}

}  // namespace tg
