// Averaging step after alignment (av3/alignment/av3_tomomatch.m:239-249 and
// :263-265):
//
//   average += tom_rotate(tom_shift(particle, -tshift), [-psi -phi -theta])
//   wei     += 2*tom_limit(tom_limit(tom_rotate(wedge, [-psi -phi -theta]), 0.5, 1, 'z'), 0, 0.5)
//   ...
//   wei = 1./wei; wei(wei > 100000) = 0;
//   average = real(tom_ifourier(ifftshift(tom_spheremask(fftshift(tom_fourier(average)).*wei, lowp))))
//
// tom_shift (Filtrans/tom_shift.m) multiplies the FP64 spectrum by
// exp(-2 pi i sum_d delta_d f_d / n_d) with f the signed frequency (Nyquist
// negative) and keeps the real part; tom_rotate rotates the single-precision
// copy (rot3d, bit-exact here); the sums are double.  The nested tom_limit is
// 1 where the rotated wedge is >= 0.5 and 0 elsewhere.  Particles are added
// in the given order, one thread per voxel looping over the particles of a
// chunk, so the double sums are reproducible.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "fft3d.h"
#include "match.h"
#include "misc.h"
#include "rotate_sample.cuh"

namespace tg {

namespace {

struct AvgParam {
    const float* part;
    const float* wedge;
    double delta[3];  // -tshift / n per axis
    float m[9];       // rot3d matrix of [-psi -phi -theta]
};

#define TG_GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

unsigned grid_n(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

__global__ void k_avg_load(const AvgParam* __restrict__ p, double2* __restrict__ z, long long nn, int K) {
    TG_GRID_STRIDE(i, nn * K) {
        const int k = (int)(i / nn);
        const long long v = i - (long long)k * nn;
        z[i] = make_double2((double)p[k].part[v], 0.0);
    }
}

__device__ __forceinline__ int signed_freq(int j, int n) { return j < n - n / 2 ? j : j - n; }

__global__ void k_avg_phase(const AvgParam* __restrict__ p, double2* __restrict__ z, int nx, int ny, int nz, int K) {
    const long long nn = (long long)nx * ny * nz;
    TG_GRID_STRIDE(i, nn * K) {
        const int k = (int)(i / nn);
        const long long v = i - (long long)k * nn;
        const int a = (int)(v % nx), b = (int)((v / nx) % ny), c = (int)(v / ((long long)nx * ny));
        const double x = p[k].delta[0] * signed_freq(a, nx) + p[k].delta[1] * signed_freq(b, ny) +
                         p[k].delta[2] * signed_freq(c, nz);
        double s, co;
        sincos(-2.0 * M_PI * x, &s, &co);
        z[i] = cmul(z[i], make_double2(co, s));
    }
}

__global__ void k_avg_real_f32(const double2* __restrict__ z, float* __restrict__ s, long long n) {
    TG_GRID_STRIDE(i, n) s[i] = (float)z[i].x;
}

// one thread per voxel: add the K rotated particles and wedge indicators in order
__global__ void k_avg_accumulate(const AvgParam* __restrict__ p, const float* __restrict__ shifted, int nx, int ny,
                                 int nz, int K, float cx, float cy, float cz, double* __restrict__ avg,
                                 double* __restrict__ wei) {
    const long long nn = (long long)nx * ny * nz;
    TG_GRID_STRIDE(v, nn) {
        const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((long long)nx * ny));
        double a = avg[v], w = wei[v];
        for (int q = 0; q < K; ++q) {
            float m[9];
#pragma unroll
            for (int e = 0; e < 9; ++e) m[e] = p[q].m[e];
            a += (double)rot_sample(shifted + (long long)q * nn, nx, ny, nz, m, cx, cy, cz, i, j, k);
            const float rw = rot_sample(p[q].wedge, nx, ny, nz, m, cx, cy, cz, i, j, k);
            w += rw >= 0.5f ? 1.0 : 0.0;
        }
        avg[v] = a;
        wei[v] = w;
    }
}

__global__ void k_avg_to_c(const double* __restrict__ a, double2* __restrict__ z, long long n) {
    TG_GRID_STRIDE(i, n) z[i] = make_double2(a[i], 0.0);
}

// F(j) *= M((j + floor(n/2)) mod n), M = (1/wei with values above 1e5 set to 0)
// times tom_spheremask(., lowp) (zero where the distance from floor(n/2)+1 is >= lowp)
__global__ void k_avg_weight(double2* __restrict__ z, const double* __restrict__ wei, int nx, int ny, int nz,
                             double lowp) {
    const long long nn = (long long)nx * ny * nz;
    TG_GRID_STRIDE(v, nn) {
        const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((long long)nx * ny));
        const int ci = (i + nx / 2) % nx, cj = (j + ny / 2) % ny, ck = (k + nz / 2) % nz;
        const long long c = ci + (long long)nx * (cj + (long long)ny * ck);
        const double dx = ci - nx / 2, dy = cj - ny / 2, dz = ck - nz / 2;
        const double dist = sqrt(dx * dx + dy * dy + dz * dz);
        double w = 1.0 / wei[c];
        if (w > 100000.0) w = 0.0;
        if (dist >= lowp) w = 0.0;
        z[v] = cscale(z[v], w);
    }
}

__global__ void k_avg_out(const double2* __restrict__ z, double* __restrict__ out, long long n) {
    TG_GRID_STRIDE(i, n) out[i] = z[i].x;
}

}  // namespace

int av3_average_add(tomgpu_ctx* ctx, const int n[3], const tomgpu_avg_item* items, int K, double* avg,
                    double* wei) {
    cudaStream_t st = ctx->stream;
    const long long nn = (long long)n[0] * n[1] * n[2];
    // chunk: at most 2^24 voxels of complex doubles (256 MiB)
    const int chunk = (int)std::max<long long>(1, std::min<long long>(K, (1LL << 24) / nn));
    double2* z = nullptr;
    float* s = nullptr;
    AvgParam* dp = nullptr;
    if (cudaMalloc(&z, sizeof(double2) * nn * chunk) || cudaMalloc(&s, sizeof(float) * nn * chunk) ||
        cudaMalloc(&dp, sizeof(AvgParam) * chunk)) {
        if (z) cudaFree(z);
        if (s) cudaFree(s);
        return cuda_fail(ctx, cudaErrorMemoryAllocation, "averaging buffers");
    }
    const float center[3] = {(float)((n[0] + 1) / 2), (float)((n[1] + 1) / 2), (float)((n[2] + 1) / 2)};
    std::vector<AvgParam> hp(chunk);
    cudaError_t e = cudaSuccess;
    for (int k0 = 0; k0 < K && !e; k0 += chunk) {
        const int kb = std::min(chunk, K - k0);
        for (int q = 0; q < kb; ++q) {
            const tomgpu_avg_item& it = items[k0 + q];
            AvgParam& a = hp[q];
            a.part = it.particle;
            a.wedge = it.wedge;
            for (int d = 0; d < 3; ++d) a.delta[d] = -(double)it.shift[d] / (double)n[d];
            const float inv[3] = {-it.angles[1], -it.angles[0], -it.angles[2]};  // [-psi -phi -theta]
            euler_matrix_host(inv, a.m);
        }
        e = cudaMemcpyAsync(dp, hp.data(), sizeof(AvgParam) * kb, cudaMemcpyHostToDevice, st);
        if (e) break;
        k_avg_load<<<grid_n(nn * kb), 256, 0, st>>>(dp, z, nn, kb);
        if ((e = c2c3d_batch64(z, n, kb, -1, 1.0, st))) break;
        k_avg_phase<<<grid_n(nn * kb), 256, 0, st>>>(dp, z, n[0], n[1], n[2], kb);
        if ((e = c2c3d_batch64(z, n, kb, +1, 1.0 / (double)nn, st))) break;
        k_avg_real_f32<<<grid_n(nn * kb), 256, 0, st>>>(z, s, nn * kb);
        k_avg_accumulate<<<grid_n(nn), 256, 0, st>>>(dp, s, n[0], n[1], n[2], kb, center[0], center[1], center[2],
                                                      avg, wei);
        e = cudaGetLastError();
        if (!e) e = cudaStreamSynchronize(st);  // hp is rewritten by the next chunk
        ctx->launches += 4 + 6;
    }
    cudaFree(z);
    cudaFree(s);
    cudaFree(dp);
    if (e) return cuda_fail(ctx, e, "av3 average accumulate");
    return TOMGPU_OK;
}

int av3_average_final(tomgpu_ctx* ctx, const int n[3], const double* avg, const double* wei, double* out) {
    cudaStream_t st = ctx->stream;
    const long long nn = (long long)n[0] * n[1] * n[2];
    double2* z = nullptr;
    if (cudaMalloc(&z, sizeof(double2) * nn)) return cuda_fail(ctx, cudaErrorMemoryAllocation, "averaging buffer");
    const double lowp = (double)(n[0] / 2 - 3);
    cudaError_t e = cudaSuccess;
    k_avg_to_c<<<grid_n(nn), 256, 0, st>>>(avg, z, nn);
    if (!(e = c2c3d<double2>(z, n, -1, 1.0, st))) {
        k_avg_weight<<<grid_n(nn), 256, 0, st>>>(z, wei, n[0], n[1], n[2], lowp);
        if (!(e = c2c3d<double2>(z, n, +1, 1.0 / (double)nn, st))) {
            k_avg_out<<<grid_n(nn), 256, 0, st>>>(z, out, nn);
            e = cudaGetLastError();
        }
    }
    if (!e) e = cudaStreamSynchronize(st);
    ctx->launches += 9;
    cudaFree(z);
    if (e) return cuda_fail(ctx, e, "av3 average weighting");
    return TOMGPU_OK;
}

}  // namespace tg
