// Register-resident kernels for the 128 edges (the 128^3 tomogram): z edge
// 128 and x edge 128 (complex half length 64); the y edge 128 runs the warp
// kernel corr_y_w<128> of match_fast.cu.  Same arithmetic contract as the
// generic kernels in match.cu.  At this size a rotation batch of spectra fits
// in L2, so the kernels are built for many lines per block and short lines:
//
//   inv_z_b128  32 y lines x 8 threads per block: 16 8-point DFTs per line
//               from global memory (32 consecutive y per request), one block
//               exchange, 8 16-point DFTs per line back to global memory.
//   c2r_b8      32 x lines per block, 8 threads per line (x edge 128: 8 x 8;
//               x edge 256: 16 x 8): the half-spectrum unpack and 8-point
//               DFTs, a warp-local exchange, 8- or 16-point DFTs; the running
//               maximum over the batch in registers and the FLCF at the
//               read-modify-write.
//   c2r_h256    x edge 512: a half-warp per line, 16 lines per block, 16 x 16.
//
// Running maximum without per-voxel coefficients: with gamma >= 0 and
// mu0 mu_T fixed per voxel, cc_b = (u_b - mu0 mu_T) gamma is a non-decreasing
// function of u_b = out_b/(N M) + kappa_b, so the batch keeps the best u and
// its rotation (16-bit batch indices, two voxels per word) and applies the
// FLCF formula once, at the read-modify-write.  (Rotations whose cc round to
// the same float but whose u differ may pick a later index than the strict
// first-wins scan; such voxels have no CC separation between those angles.
// gamma = 0 voxels keep the reference's value 0 with the batch's first
// rotation.)
//
// Index map (inverse): with n = q + Q m and k = k1 + P k2,
// y(n) = sum_k1 WP^(m k1) WL^(q k1) sum_k2 Y(k) WQ^(q k2).
#include "ctx.h"
#include "match.h"
#include "tile_copy.cuh"
#include "twiddles.h"
#include "warp_fft.cuh"

namespace tg {

namespace {

constexpr int IZ1_LS = 129;

// NZ = 128 = 16 (P) x 8 (Q)
__global__ void __launch_bounds__(256) k_inv_z_b128(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                                    int nh1, const float2* __restrict__ tw_g) {
    constexpr int NZ = 128, P = 16, QN = 8, LS = IZ1_LS;
    __shared__ __align__(16) float2 s[32 * LS];
    __shared__ __align__(16) float2 T[P * QN];  // W128^(+q k1) at [k1][q]
    for (int i = threadIdx.x; i < P * QN; i += blockDim.x) {
        const int k1 = i >> 3, q = i & 7;
        T[i] = cconj(__ldg(tw_g + (q * k1) % NZ));
    }
    const int tid = threadIdx.x, l = tid & 31, j = tid >> 5;
    const int y = blockIdx.x * 32 + l, kx = blockIdx.y, b = blockIdx.z;
    const bool ok = y < Ny;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k1 = j + 8 * h;
        float2 u[QN];
#pragma unroll
        for (int k2 = 0; k2 < QN; ++k2)
            u[k2] = ok ? Q[base + (long long)(k1 + P * k2) * Ny + y] : make_float2(0.f, 0.f);
        tgfft::dft8<+1>(u);
#pragma unroll
        for (int q = 0; q < QN; ++q) s[l * LS + k1 * QN + q] = cmul(u[q], T[k1 * QN + q]);
    }
    __syncthreads();
    float2 v[P];
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) v[k1] = s[l * LS + k1 * QN + j];
    tgfft::dft16<+1>(v);
    if (ok) {
#pragma unroll
        for (int m = 0; m < P; ++m) H[base + (long long)(j + QN * m) * Ny + y] = v[m];
    }
}

constexpr int C1_YT = 32, C1_XR = 9;

// Short x lines, 8 threads per line, 32 lines per block: NH = P x 8 with
// P = 8 (NH 64) or 16 (NH 128, two first-stage tasks per thread).
template <int NH, int P>
__global__ void __launch_bounds__(256) k_c2r_b8(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                const float* __restrict__ gam, const double* __restrict__ tsum,
                                                int Ny, int Nz, int nb, float inv_nm, double c_mean, double inv_m,
                                                double mu_t, int index0, float* __restrict__ maxcc,
                                                int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                const float2* __restrict__ tw_x) {
    constexpr int NH1 = NH + 1, NX = 2 * NH, QN = 8, YT = C1_YT, TS = NH + 1, XR = C1_XR;
    static_assert(NH == P * QN, "NH = P x 8");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);  // [2][YT][TS]
    float2* xb = tile + 2 * YT * TS;                      // [YT][P][XR] exchange
    float2* T = xb + YT * P * XR;                         // [QN][P]: W_NH^(+q k1) at [q][k1]
    float2* twx = T + P * QN;                             // [NH]: W_NX^(+k)
    float* kaps = reinterpret_cast<float*>(twx + NH);     // [nb]
    const int tid = threadIdx.x, line = tid >> 3, j = tid & 7;
    const int y0 = blockIdx.x * YT, z = blockIdx.y, y = y0 + line;
    for (int i = tid; i < P * QN; i += blockDim.x) {
        const int k1 = i / QN, q = i - k1 * QN;
        T[q * P + k1] = cconj(__ldg(tw_h + (q * k1) % NH));
    }
    for (int i = tid; i < NH; i += blockDim.x) twx[i] = cconj(__ldg(tw_x + i));
    for (int b = tid; b < nb; b += blockDim.x) kaps[b] = (float)(c_mean * (tsum[b] * inv_m - mu_t));
    float bu[P][2];
    unsigned bb[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        bu[m][0] = bu[m][1] = -INFINITY;
        bb[m] = 0u;
    }
    const tgtile::TileCopy<YT, NH1, 256> copy(tile, TS, H, tid, y0, z, Ny, Nz);
    auto issue = [&](int b, int which) { copy.issue(b, which * (unsigned)(YT * TS * sizeof(float2))); };
    issue(0, 0);
    float2* xl = xb + line * P * XR;
    for (int b = 0; b < nb; ++b) {
        if (b + 1 < nb) issue(b + 1, (b + 1) & 1);
        else tgtile::commit();
        tgtile::wait<1>();
        __syncthreads();
        const float2* X = tile + (b & 1) * YT * TS + line * TS;
#pragma unroll
        for (int h = 0; h < P / 8; ++h) {
            const int k1 = j + 8 * h;
            float2 u[QN];
#pragma unroll
            for (int k2 = 0; k2 < QN; ++k2) {
                const int k = k1 + P * k2;
                const float2 xa = X[k], xc = cconj(X[NH - k]);
                const float2 d = cmul(twx[k], csub(xa, xc));
                u[k2] = cadd(cadd(xa, xc), make_float2(-d.y, d.x));
            }
            tgfft::dft8<+1>(u);
#pragma unroll
            for (int q = 0; q < QN; ++q) xl[k1 * XR + q] = cmul(u[q], T[q * P + k1]);
        }
        __syncwarp();
        float2 v[P];
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[k1] = xl[k1 * XR + j];
        if constexpr (P == 8) tgfft::dft8<+1>(v);
        else tgfft::dft16<+1>(v);
        const float kap = kaps[b];
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float u0 = fmaf(v[m].x, inv_nm, kap);
            const float u1 = fmaf(v[m].y, inv_nm, kap);
            if (u0 > bu[m][0]) { bu[m][0] = u0; bb[m] = (bb[m] & 0xFFFF0000u) | (unsigned)b; }
            if (u1 > bu[m][1]) { bu[m][1] = u1; bb[m] = (bb[m] & 0x0000FFFFu) | ((unsigned)b << 16); }
        }
        __syncthreads();  // the tile and the exchange are rewritten next
    }
    if (y >= Ny) return;
    const float mt = (float)mu_t;
    const long long row = ((long long)z * Ny + y) * NX;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const long long v = row + 2 * (j + QN * m);
        const float2 a = __ldg(reinterpret_cast<const float2*>(mu0 + v));
        const float2 g = __ldg(reinterpret_cast<const float2*>(gam + v));
        float2 cur = *reinterpret_cast<const float2*>(maxcc + v);
        int2 ci = *reinterpret_cast<const int2*>(angidx + v);
        bool ch = false;
        const float c0 = g.x != 0.f ? (bu[m][0] - a.x * mt) * g.x : 0.f;
        const float c1 = g.y != 0.f ? (bu[m][1] - a.y * mt) * g.y : 0.f;
        const int b0 = g.x != 0.f ? (int)(bb[m] & 0xFFFFu) : 0, b1 = g.y != 0.f ? (int)(bb[m] >> 16) : 0;
        if (c0 > cur.x) { cur.x = c0; ci.x = index0 + b0; ch = true; }
        if (c1 > cur.y) { cur.y = c1; ci.y = index0 + b1; ch = true; }
        if (ch) {
            *reinterpret_cast<float2*>(maxcc + v) = cur;
            *reinterpret_cast<int2*>(angidx + v) = ci;
        }
    }
}

constexpr int CH_YT = 16, CH_TS = 273, CH_XR = 17, CH_STG = 3;
static_assert(15 * CH_XR + 15 < CH_TS, "the exchange fits in a tile row");

// NH = 256 = 16 (P) x 16 (Q); a half-warp per x line, 16 lines per block
// (128-byte rows of y per request), two radix-16 stages with one exchange.
// Three tiles in flight (the next two rotations load while one is
// transformed); the exchange reuses the row of the tile being transformed
// (row stride 273: both the tile and the exchange accesses are conflict-free),
// so two blocks still fit an SM.
__global__ void __launch_bounds__(256, 2) k_c2r_h256(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                     const float* __restrict__ gam, const double* __restrict__ tsum,
                                                     int Ny, int Nz, int nb, float inv_nm, double c_mean, double inv_m,
                                                     double mu_t, int index0, float* __restrict__ maxcc,
                                                     int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                     const float2* __restrict__ tw_x) {
    constexpr int NH = 256, NH1 = NH + 1, NX = 2 * NH, P = 16, QN = 16, YT = CH_YT, TS = CH_TS, XR = CH_XR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);  // [3][YT][TS]: a row is a line, then its exchange [P][XR]
    float2* T = tile + CH_STG * YT * TS;                  // [QN][P]: W256^(+q k1) at [q][k1]
    float2* twx = T + P * QN;                             // [NH]: W512^(+k)
    float* kaps = reinterpret_cast<float*>(twx + NH);     // [nb]
    const int tid = threadIdx.x, line = tid >> 4, j = tid & 15;
    const int y0 = blockIdx.x * YT, z = blockIdx.y, y = y0 + line;
    for (int i = tid; i < P * QN; i += blockDim.x) {
        const int k1 = i >> 4, q = i & 15;
        T[q * P + k1] = cconj(__ldg(tw_h + (q * k1) % NH));
    }
    for (int i = tid; i < NH; i += blockDim.x) twx[i] = cconj(__ldg(tw_x + i));
    for (int b = tid; b < nb; b += blockDim.x) kaps[b] = (float)(c_mean * (tsum[b] * inv_m - mu_t));
    float bu[P][2];
    unsigned bb[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        bu[m][0] = bu[m][1] = -INFINITY;
        bb[m] = 0u;
    }
    const tgtile::TileCopy<YT, NH1, 256> copy(tile, TS, H, tid, y0, z, Ny, Nz);
    auto issue = [&](int b, int which) { copy.issue(b, which * (unsigned)(YT * TS * sizeof(float2))); };
    issue(0, 0);
    if (1 < nb) issue(1, 1);
    else tgtile::commit();
    int cur = 0;  // stage of rotation b
    for (int b = 0; b < nb; ++b) {
        const int nxt = cur == 0 ? 2 : cur - 1;  // stage of rotation b + 2
        if (b + 2 < nb) issue(b + 2, nxt);
        else tgtile::commit();
        tgtile::wait<2>();
        __syncthreads();
        float2* X = tile + cur * YT * TS + line * TS;
        float2* xl = X;  // the exchange overwrites the row once the half-warp has read it
        {
            float2 u[QN];
#pragma unroll
            for (int k2 = 0; k2 < QN; ++k2) {
                const int k = j + P * k2;
                const float2 xa = X[k], xc = cconj(X[NH - k]);
                const float2 d = cmul(twx[k], csub(xa, xc));
                u[k2] = cadd(cadd(xa, xc), make_float2(-d.y, d.x));
            }
            __syncwarp();  // every lane of the line has read the row
            tgfft::dft16<+1>(u);
#pragma unroll
            for (int q = 0; q < QN; ++q) xl[j * XR + q] = cmul(u[q], T[q * P + j]);
        }
        __syncwarp();
        float2 v[P];
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[k1] = xl[k1 * XR + j];
        tgfft::dft16<+1>(v);
        const float kap = kaps[b];
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float u0 = fmaf(v[m].x, inv_nm, kap);
            const float u1 = fmaf(v[m].y, inv_nm, kap);
            if (u0 > bu[m][0]) { bu[m][0] = u0; bb[m] = (bb[m] & 0xFFFF0000u) | (unsigned)b; }
            if (u1 > bu[m][1]) { bu[m][1] = u1; bb[m] = (bb[m] & 0x0000FFFFu) | ((unsigned)b << 16); }
        }
        cur = cur == 2 ? 0 : cur + 1;
        __syncthreads();  // this stage is loaded again next
    }
    if (y >= Ny) return;
    const float mt = (float)mu_t;
    const long long row = ((long long)z * Ny + y) * NX;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const long long v = row + 2 * (j + QN * m);
        const float2 a = __ldg(reinterpret_cast<const float2*>(mu0 + v));
        const float2 g = __ldg(reinterpret_cast<const float2*>(gam + v));
        float2 cur = *reinterpret_cast<const float2*>(maxcc + v);
        int2 ci = *reinterpret_cast<const int2*>(angidx + v);
        bool ch = false;
        const float c0 = g.x != 0.f ? (bu[m][0] - a.x * mt) * g.x : 0.f;
        const float c1 = g.y != 0.f ? (bu[m][1] - a.y * mt) * g.y : 0.f;
        const int b0 = g.x != 0.f ? (int)(bb[m] & 0xFFFFu) : 0, b1 = g.y != 0.f ? (int)(bb[m] >> 16) : 0;
        if (c0 > cur.x) { cur.x = c0; ci.x = index0 + b0; ch = true; }
        if (c1 > cur.y) { cur.y = c1; ci.y = index0 + b1; ch = true; }
        if (ch) {
            *reinterpret_cast<float2*>(maxcc + v) = cur;
            *reinterpret_cast<int2*>(angidx + v) = ci;
        }
    }
}

}  // namespace

cudaError_t launch_c2r_h256(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st) {
    const size_t smem =
        sizeof(float2) * (CH_STG * CH_YT * CH_TS + 16 * 16 + 256) + sizeof(float) * nb;
    cudaFuncSetAttribute(k_c2r_h256, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 g((Ny + CH_YT - 1) / CH_YT, Nz);
    k_c2r_h256<<<g, 256, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx,
                                     twiddle_table<float2>(256), twiddle_table<float2>(512));
    return cudaGetLastError();
}

cudaError_t launch_inv_z_b128(const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st) {
    dim3 g((Ny + 31) / 32, nh1, nb);
    k_inv_z_b128<<<g, 256, 0, st>>>(Q, H, Ny, nh1, twiddle_table<float2>(128));
    return cudaGetLastError();
}

template <int NH, int P>
static cudaError_t launch_c2r_b8(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                                 int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                                 float* maxcc, int* angidx, cudaStream_t st) {
    const size_t smem = sizeof(float2) * (2 * C1_YT * (NH + 1) + C1_YT * P * C1_XR + P * 8 + NH) + sizeof(float) * nb;
    cudaFuncSetAttribute(k_c2r_b8<NH, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 g((Ny + C1_YT - 1) / C1_YT, Nz);
    k_c2r_b8<NH, P><<<g, 256, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc,
                                          angidx, twiddle_table<float2>(NH), twiddle_table<float2>(2 * NH));
    return cudaGetLastError();
}

cudaError_t launch_c2r_b64(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                           int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                           int* angidx, cudaStream_t st) {
    return launch_c2r_b8<64, 8>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
}

cudaError_t launch_c2r_b128(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st) {
    return launch_c2r_b8<128, 16>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
}

}  // namespace tg
