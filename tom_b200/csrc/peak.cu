// Peak search (replaces find_max, Analysis/tom_peakinc.c:23-52, and the
// tom_peak variants of Analysis/tom_peak.m).
//
// The arg-max is a single pass: every candidate becomes a 64-bit key whose
// high word is the value mapped to an order-preserving unsigned integer and
// whose low word is the complement of the linear (x-fastest) index, so the
// largest key is the largest value and, among equal values, the first one -
// the reference's strict '>' scan from -99999.  Warp shuffles and one 64-bit
// atomicMax per block reduce the keys.
#include "peak.h"

#include <algorithm>
#include <cmath>

namespace tg {

__device__ __forceinline__ unsigned long long peak_key(float v, unsigned idx) {
    if (!(v > -99999.0f)) return 0ull;  // the scan's start value; NaN never wins
    unsigned u = __float_as_uint(v == 0.f ? 0.f : v);
    const unsigned ord = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)ord << 32) | (unsigned long long)(0xFFFFFFFFu - idx);
}

__host__ __device__ inline float key_value(unsigned long long key) {
    const unsigned ord = (unsigned)(key >> 32);
    const unsigned u = (ord & 0x80000000u) ? (ord & 0x7FFFFFFFu) : ~ord;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}

__global__ void __launch_bounds__(256) k_argmax(const float* __restrict__ v, long long n,
                                                unsigned long long* __restrict__ out) {
    unsigned long long best = 0ull;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned long long k = peak_key(__ldg(v + i), (unsigned)i);
        best = k > best ? k : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
        best = t > best ? t : best;
    }
    __shared__ unsigned long long warp_best[8];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) warp_best[w] = best;
    __syncthreads();
    if (w == 0) {
        best = lane < (int)(blockDim.x >> 5) ? warp_best[lane] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
            best = t > best ? t : best;
        }
        if (lane == 0 && best) atomicMax(out, best);
    }
}

// Zero the ball of radius R around the peak recorded in *key and append the
// peak (value, 1-based position) to the output lists.  The ball's bounding box
// [p - r, p + r] (r = floor(R)) is clamped on each axis to the volume, as the
// reference clamps its sub-block (Analysis/tom_peak.m:218-270); the launch
// covers w = min(2r + 1, n) positions per axis, which always hold the clamped
// range, and the distance test uses R^2 in double.  One thread per position.
__global__ void k_zero_ball(float* __restrict__ v, int sx, int sy, int sz, const unsigned long long* key,
                            int r, double r2, int wx, int wy, int wz, float* __restrict__ vals,
                            int* __restrict__ pos, int k) {
    const unsigned long long kk = *key;
    if (kk == 0ull) {  // nothing above the start value left
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            vals[k] = -99999.0f;
            pos[3 * k] = pos[3 * k + 1] = pos[3 * k + 2] = 0;
        }
        return;
    }
    const unsigned idx = 0xFFFFFFFFu - (unsigned)(kk & 0xFFFFFFFFull);
    const int px = (int)(idx % (unsigned)sx);
    const int py = (int)((idx / (unsigned)sx) % (unsigned)sy);
    const int pz = (int)(idx / ((unsigned)sx * (unsigned)sy));
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        vals[k] = key_value(kk);
        pos[3 * k] = px + 1;
        pos[3 * k + 1] = py + 1;
        pos[3 * k + 2] = pz + 1;
    }
    if (t >= (long long)wx * wy * wz) return;
    // r <= max(n) keeps p +- r inside the int range
    const int x = max(px - r, 0) + (int)(t % wx);
    const int y = max(py - r, 0) + (int)((t / wx) % wy);
    const int z = max(pz - r, 0) + (int)(t / ((long long)wx * wy));
    if (x > min(px + r, sx - 1) || y > min(py + r, sy - 1) || z > min(pz + r, sz - 1)) return;
    const double dx = x - px, dy = y - py, dz = z - pz;
    if (dx * dx + dy * dy + dz * dz <= r2) v[x + (long long)sx * (y + (long long)sy * z)] = 0.f;
}

// tom_intpeak per axis: parabola through the 3 neighbours (a 3-point
// not-a-knot spline), maximised on the grid 1:0.001:3 (first maximum).
__global__ void k_spline(const float* __restrict__ v, int sx, int sy, int sz, int px, int py, int pz,
                         double* __restrict__ out /* 3 coords + 3 values */) {
    const int d = threadIdx.x;
    if (d >= 3) return;
    const int p[3] = {px, py, pz};
    const int n[3] = {sx, sy, sz};
    const long long center = px + (long long)sx * (py + (long long)sy * pz);
    const double vc = v[center];
    if (p[d] == 0 || p[d] == n[d] - 1) {
        out[d] = p[d] + 1;
        out[3 + d] = vc;
        return;
    }
    const long long step = d == 0 ? 1 : (d == 1 ? sx : (long long)sx * sy);
    const double y0 = v[center - step], y1 = vc, y2 = v[center + step];
    const double A = (y0 - 2 * y1 + y2) / 2, B = (y1 - y0) - 3 * A, C = y0 - A - B;
    double best = -1e300;
    int bj = 0;
    for (int j = 0; j <= 2000; ++j) {
        const double x = 1.0 + j * 0.001;
        const double yv = (A * x + B) * x + C;
        if (yv > best) { best = yv; bj = j; }
    }
    out[d] = p[d] + bj * 0.001;  // (s - 1) + 1 + j*0.001 with s 1-based
    out[3 + d] = best;
}

cudaError_t argmax_key(const float* v, long long n, unsigned long long* d_key, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(d_key, 0, sizeof(unsigned long long), st);
    if (e) return e;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    k_argmax<<<(unsigned)blocks, 256, 0, st>>>(v, n, d_key);
    return cudaGetLastError();
}

cudaError_t topk_rounds(float* work, const int dims[3], int K, double radius, unsigned long long* d_key,
                        float* d_vals, int* d_pos, cudaStream_t st, int64_t* launches) {
    if (!(radius >= 0) || std::isinf(radius)) return cudaErrorInvalidValue;  // callers reject these first
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    const int nmax = std::max(dims[0], std::max(dims[1], dims[2]));
    // beyond the largest edge the clamped box is the whole volume on every axis
    const int r = radius > (double)nmax ? nmax : (int)radius;
    const int wx = std::min(2 * r + 1, dims[0]), wy = std::min(2 * r + 1, dims[1]), wz = std::min(2 * r + 1, dims[2]);
    const long long box = (long long)wx * wy * wz;  // at most n <= 2^32 voxels
    const unsigned blocks = (unsigned)((box + 255) / 256);
    for (int k = 0; k < K; ++k) {
        cudaError_t e = argmax_key(work, n, d_key, st);
        if (e) return e;
        k_zero_ball<<<blocks, 256, 0, st>>>(work, dims[0], dims[1], dims[2], d_key, r, radius * radius, wx, wy, wz,
                                            d_vals, d_pos, k);
        if ((e = cudaGetLastError())) return e;
        *launches += 2;
    }
    return cudaSuccess;
}

cudaError_t spline_peak(const float* v, const int dims[3], const int pos0[3], double* d_out, cudaStream_t st) {
    k_spline<<<1, 32, 0, st>>>(v, dims[0], dims[1], dims[2], pos0[0], pos0[1], pos0[2], d_out);
    return cudaGetLastError();
}

float peak_key_to_value(unsigned long long key) { return key_value(key); }

}  // namespace tg
