// FP64 rescoring of candidate peaks: the FLCF of tom_os3_corr at one voxel
// (search/tom_os3_corr.m:151-176) evaluated by direct summation over the
// template box in double precision — no FFT, so no FP32 rounding of the
// spectral path.  One block per candidate:
//   S  = sum_j t3(j) I(x + j + d0)          correlation sum (template offset d0)
//   m1 = sum_j M(j) I(x + c - j),  m2 = sum_j M(j) I(x + c - j)^2   (tom_os3_mean/std)
//   cc = (S/M - mu mu_T) / (sigma_T sigma),  mu = m1/M,  sigma = sqrt(max(m2/M - mu^2, 0))
// with t3 = mask * filter(mask * rot(template)) supplied per candidate.
#include <cfloat>

#include "common.cuh"
#include "rescore.h"

namespace tg {

__global__ void __launch_bounds__(256) k_rescore(const float* __restrict__ vol, int nx, int ny, int nz,
                                                 const double* __restrict__ t3, const float* __restrict__ mask,
                                                 int tx, int ty, int tz, const int* __restrict__ pos0, double msize,
                                                 double tmean, double tstd, double* __restrict__ out) {
    const int k = blockIdx.x;
    const long long tn = (long long)tx * ty * tz;
    const double* t = t3 + (long long)k * tn;
    const int px = pos0[3 * k], py = pos0[3 * k + 1], pz = pos0[3 * k + 2];
    const int cx = tx / 2, cy = ty / 2, cz = tz / 2;
    const int dx = pmod(2 * (nx / 2) - cx, nx), dy = pmod(2 * (ny / 2) - cy, ny), dz = pmod(2 * (nz / 2) - cz, nz);
    double s = 0, m1 = 0, m2 = 0;
    for (long long j = threadIdx.x; j < tn; j += blockDim.x) {
        const int jx = (int)(j % tx), jy = (int)((j / tx) % ty), jz = (int)(j / ((long long)tx * ty));
        const double m = mask[j];
        const double tv = t[j] * m;
        if (tv != 0.0) {
            const int ix = pmod(px + jx + dx, nx), iy = pmod(py + jy + dy, ny), iz = pmod(pz + jz + dz, nz);
            s += tv * (double)vol[ix + (long long)nx * (iy + (long long)ny * iz)];
        }
        if (m != 0.0) {
            const int ix = pmod(px + cx - jx, nx), iy = pmod(py + cy - jy, ny), iz = pmod(pz + cz - jz, nz);
            const double v = vol[ix + (long long)nx * (iy + (long long)ny * iz)];
            m1 += m * v;
            m2 += m * v * v;
        }
    }
    __shared__ double red[3][8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m1 += __shfl_xor_sync(0xffffffffu, m1, o);
        m2 += __shfl_xor_sync(0xffffffffu, m2, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { red[0][w] = s; red[1][w] = m1; red[2][w] = m2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0, A = 0, B = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) { S += red[0][i]; A += red[1][i]; B += red[2][i]; }
        const double mu = A / msize;
        const double var = B / msize - mu * mu;
        const double sig = sqrt(var > 0 ? var : 0.0);
        const double den = (double)(float)(tstd * sig * 10000.0);
        out[k] = fabs(den - DBL_EPSILON) > DBL_EPSILON ? (S / msize - mu * tmean) / (tstd * sig) : 0.0;
    }
}

__global__ void k_f32_to_f64_masked(const float* __restrict__ a, double* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}

cudaError_t rescore_fp64(const float* vol, const int N[3], const double* t3, const float* mask, const int T[3],
                         const int* pos0_dev, int K, double msize, double tmean, double tstd, double* out_dev,
                         cudaStream_t st) {
    if (K <= 0) return cudaSuccess;
    k_rescore<<<K, 256, 0, st>>>(vol, N[0], N[1], N[2], t3, mask, T[0], T[1], T[2], pos0_dev, msize, tmean, tstd,
                                 out_dev);
    return cudaGetLastError();
}

cudaError_t f32_to_f64(const float* a, double* b, long long n, cudaStream_t st) {
    long long g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_f32_to_f64_masked<<<(unsigned)(g < 1 ? 1 : g), 256, 0, st>>>(a, b, n);
    return cudaGetLastError();
}

}  // namespace tg
