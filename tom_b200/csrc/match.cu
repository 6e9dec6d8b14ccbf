// FLCF template matching: the hot loop of tom_os3_findTemplate
// (Oscar3/matlabPicker/search/tom_os3_findTemplate.m:255-307) on sm_100a.
//
// Per rotation r the reference computes
//   cc_r(x) = (sum_j t_r(j) I(x + j - c) / M - mu_I(x) mu_T) / (sigma_T sigma_I(x))
// with t_r = mask * filter(mask * rot_r(template)) and keeps the strict running
// maximum and its angle index (search/tom_os3_corr.m:151-176,
// search/tom_os3_bestPeak.m:42-47).  Here the correlation runs through the
// tomogram's half spectrum F_I (once per volume) and a pruned spectrum of the
// small template:
//
//   spec_x  (per rotation)  x-DFT of the T^3 template lines        -> A[kx][jz][jy]
//   spec_z  (per rotation)  z-DFT of A (T samples -> Nz)           -> Z[kx][kz][jy]
//   corr_y  (hot)  y-DFT of Z (T samples -> Ny), times F_I^*, inverse y-DFT -> Q[kx][kz][y]
//   inv_z   (hot)  inverse z-DFT                                   -> H[kx][z][y]
//   c2r_x   (hot)  half-length complex inverse + real unpacking along x,
//                  FLCF normalisation, running max / arg-max over a rotation batch
//
// Every stage keeps its lines in shared memory (fft_engine.cuh); the
// intermediate layouts are chosen so that every global load and store moves
// whole 64-128 byte rows.  The FLCF is evaluated against the tomogram with its
// global mean c removed (F_I is the spectrum of I - c, mu0 the local mean of
// I - c); the constant restores the reference's value exactly:
//   cc = (out / (N M) - mu0 mu_T + c (S_r / M - mu_T)) * gamma,
// S_r = sum_j t_r(j) in FP64, gamma = 1 / (sigma_T sigma_I) (0 where the
// reference skips the division).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "fft3d.h"
#include "fft_engine.cuh"
#include "analysis.h"
#include "match.h"
#include "misc.h"
#include "rescore.h"
#include "rotate.h"
#include "twiddles.h"

namespace tg {

// ------------------------------------------------------------- kernels
template <int L> struct HotCfg {
    static constexpr int NT = 256;
    static constexpr int LS = L + 1;
};

// x-stage of the template spectrum.  Lines (jy, jz, b) of the rotated,
// filtered template t2 (times the mask once more, tom_os3_corr.m:151) are
// placed at (jx + d0x) mod Nx and transformed; kx in [0, Nx/2] is kept.
// Also accumulates S_b = sum t2*mask in FP64.
template <int NX>
__global__ void __launch_bounds__(256) k_spec_x(const float* __restrict__ t2, const float* __restrict__ mask,
                                                float2* __restrict__ A, int Tx, int Ty, int Tz, int d0x,
                                                const float2* __restrict__ tw, double* __restrict__ tsum) {
    constexpr int NL = (4096 / NX) < 1 ? 1 : ((4096 / NX) > 16 ? 16 : (4096 / NX));
    constexpr int NT = 256, LS = NX + 1, NH1 = NX / 2 + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const int line0 = blockIdx.x * NL, b = blockIdx.y;
    const int nlines = Ty * Tz;  // lines of rotation b: rem = jz * Ty + jy
    double acc = 0.0;
    for (int i = tid; i < NL * NX; i += NT) {
        const int li = i / NX, e = i - li * NX;
        const int rem = line0 + li;
        const int jx = pmod(e - d0x, NX);
        float v = 0.f;
        if (rem < nlines && jx < Tx) {
            v = t2[((long long)b * nlines + rem) * Tx + jx] * mask[(long long)rem * Tx + jx];
            acc += (double)v;
        }
        s[li * LS + e] = make_float2(v, 0.f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((tid & 31) == 0) red[tid >> 5] = acc;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) t += red[w];
        atomicAdd(tsum + b, t);
    }
    tgfft::smem_fft<NX, -1, NL, NT, LS, float2>(s, tw, tid);
    for (int i = tid; i < NL * NH1; i += NT) {
        const int kx = i / NL, li = i - kx * NL;
        const int rem = line0 + li;
        if (rem >= nlines) continue;
        const int jz = rem / Ty, jy = rem - jz * Ty;
        A[(((long long)b * NH1 + kx) * Tz + jz) * Ty + jy] = s[li * LS + kx];
    }
}

// z-stage: Z[b][kx][kz][jy] = sum_jz A[b][kx][jz][jy] exp(-2 pi i kz (jz + d0z) / Nz)
template <int NZ>
__global__ void __launch_bounds__(256) k_spec_z(const float2* __restrict__ A, float2* __restrict__ Z, int Ty,
                                                int Tz, int d0z, int nh1, const float2* __restrict__ tw) {
    constexpr int NL = 8, NT = 256, LS = NZ + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const int jy0 = blockIdx.x * NL, kx = blockIdx.y, b = blockIdx.z;
    const long long abase = ((long long)b * nh1 + kx) * Tz * Ty;
    for (int i = tid; i < NL * NZ; i += NT) {
        const int e = i / NL, li = i - e * NL;
        const int jy = jy0 + li;
        const int jz = pmod(e - d0z, NZ);
        float2 v = make_float2(0.f, 0.f);
        if (jy < Ty && jz < Tz) v = A[abase + (long long)jz * Ty + jy];
        s[li * LS + e] = v;
    }
    __syncthreads();
    tgfft::smem_fft<NZ, -1, NL, NT, LS, float2>(s, tw, tid);
    const long long zbase = ((long long)b * nh1 + kx) * NZ * Ty;
    for (int i = tid; i < NL * NZ; i += NT) {
        const int kz = i / NL, li = i - kz * NL;
        const int jy = jy0 + li;
        if (jy < Ty) Z[zbase + (long long)kz * Ty + jy] = s[li * LS + kz];
    }
}

// Hot stage 1: per column (kx, kz) and rotation b, the y-DFT of the template
// (Ty samples placed at (jy + d0y) mod Ny), the product F_I * conj(G) and the
// inverse y-DFT.  F_I stays in registers across the rotation batch.
template <int NY>
__global__ void __launch_bounds__(256) k_corr_y(const float2* __restrict__ fimg, const float2* __restrict__ Z,
                                                float2* __restrict__ Q, int Ty, int d0y, long long ncols,
                                                int nb, const float2* __restrict__ tw) {
    constexpr int NL = (2048 / NY) < 1 ? 1 : ((2048 / NY) > 16 ? 16 : (2048 / NY));
    constexpr int NT = 256, LS = NY + 1;
    constexpr int EPT = (NL * NY + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const long long col0 = (long long)blockIdx.x * NL;
    float2 f[EPT];
    int jyq[EPT];
#pragma unroll
    for (int q = 0; q < EPT; ++q) {
        const int idx = tid + q * NT;
        const int li = idx / NY, e = idx - li * NY;
        const bool ok = idx < NL * NY && col0 + li < ncols;
        f[q] = ok ? fimg[(col0 + li) * NY + e] : make_float2(0.f, 0.f);
        const int jy = pmod(e - d0y, NY);
        jyq[q] = (ok && jy < Ty) ? jy : -1;
    }
    for (int b = 0; b < nb; ++b) {
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = tid + q * NT;
            if (idx < NL * NY) {
                const int li = idx / NY, e = idx - li * NY;
                float2 v = make_float2(0.f, 0.f);
                if (jyq[q] >= 0) v = Z[((long long)b * ncols + col0 + li) * Ty + jyq[q]];
                s[li * LS + e] = v;
            }
        }
        __syncthreads();
        tgfft::smem_fft<NY, -1, NL, NT, LS, float2>(s, tw, tid);
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = tid + q * NT;
            if (idx < NL * NY) {
                const int li = idx / NY, e = idx - li * NY;
                s[li * LS + e] = cmulc(f[q], s[li * LS + e]);
            }
        }
        __syncthreads();
        tgfft::smem_fft<NY, +1, NL, NT, LS, float2>(s, tw, tid);
#pragma unroll
        for (int q = 0; q < EPT; ++q) {
            const int idx = tid + q * NT;
            if (idx < NL * NY) {
                const int li = idx / NY, e = idx - li * NY;
                if (col0 + li < ncols) Q[((long long)b * ncols + col0 + li) * NY + e] = s[li * LS + e];
            }
        }
    }
}

// Hot stage 2: inverse z-DFT, Q[b][kx][kz][y] -> H[b][kx][z][y] for a tile of
// YT consecutive y.
template <int NZ>
__global__ void __launch_bounds__(256) k_inv_z(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                               int nh1, const float2* __restrict__ tw) {
    constexpr int YT = 16, NT = 256, LS = NZ + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * YT, kx = blockIdx.y, b = blockIdx.z;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    for (int i = tid; i < YT * NZ; i += NT) {
        const int kz = i / YT, yl = i - kz * YT;
        const int y = y0 + yl;
        s[yl * LS + kz] = y < Ny ? Q[base + (long long)kz * Ny + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    tgfft::smem_fft<NZ, +1, YT, NT, LS, float2>(s, tw, tid);
    for (int i = tid; i < YT * NZ; i += NT) {
        const int z = i / YT, yl = i - z * YT;
        const int y = y0 + yl;
        if (y < Ny) H[base + (long long)z * Ny + y] = s[yl * LS + z];
    }
}

// Hot stage 3: complex-to-real inverse along x (half-length complex FFT plus
// the even/odd unpacking), FLCF normalisation, and the strict running maximum
// over the rotation batch; one read-modify-write of the result per batch.
template <int NH>
__global__ void __launch_bounds__(256) k_c2r_x_flcf(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                    const float* __restrict__ gam,
                                                    const double* __restrict__ tsum, int Ny, int Nz, int nb,
                                                    float inv_nm, double c_mean, double inv_m, double mu_t,
                                                    int index0, float* __restrict__ maxcc,
                                                    int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                    const float2* __restrict__ tw_x) {
    constexpr int YT = 8, NT = 256, NH1 = NH + 1, LS = NH + 1, NX = 2 * NH;
    constexpr int PPT = (YT * NH + NT - 1) / NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * YT, z = blockIdx.y;
    const long long nh1l = NH1;
    float bm[PPT][2];
    int bi[PPT][2];
    float m0[PPT][2], g0[PPT][2];
    const float mt = (float)mu_t;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        const int p = tid + q * NT;
        const int yl = p / NH, m = p - yl * NH;
        const int y = y0 + yl;
        bm[q][0] = bm[q][1] = -INFINITY;
        bi[q][0] = bi[q][1] = -1;
        m0[q][0] = m0[q][1] = g0[q][0] = g0[q][1] = 0.f;
        if (p < YT * NH && y < Ny) {
            const long long v = ((long long)z * Ny + y) * NX + 2 * m;
            const float2 a = *reinterpret_cast<const float2*>(mu0 + v);
            const float2 g = *reinterpret_cast<const float2*>(gam + v);
            m0[q][0] = a.x; m0[q][1] = a.y;
            g0[q][0] = g.x; g0[q][1] = g.y;
        }
    }
    for (int b = 0; b < nb; ++b) {
        const long long hb = (long long)b * nh1l * Nz * Ny;
        for (int i = tid; i < YT * NH1; i += NT) {
            const int kx = i / YT, yl = i - kx * YT;
            const int y = y0 + yl;
            s[yl * LS + kx] = y < Ny ? H[hb + ((long long)kx * Nz + z) * Ny + y] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        // unpack: Z[k] = (X[k] + X*[NH-k]) + i w^k (X[k] - X*[NH-k]), w = exp(+2 pi i / NX)
        for (int i = tid; i < YT * (NH / 2 + 1); i += NT) {
            const int yl = i / (NH / 2 + 1), k = i - yl * (NH / 2 + 1);
            float2* row = s + yl * LS;
            const float2 xa = row[k], xb = row[NH - k];
            {
                const float2 bc = cconj(xb);
                const float2 w = cconj(__ldg(tw_x + k));
                const float2 d = cmul(w, csub(xa, bc));
                row[k] = cadd(cadd(xa, bc), make_float2(-d.y, d.x));
            }
            if (k > 0 && k < NH - k) {
                const float2 ac = cconj(xa);
                const float2 w = cconj(__ldg(tw_x + (NH - k)));
                const float2 d = cmul(w, csub(xb, ac));
                row[NH - k] = cadd(cadd(xb, ac), make_float2(-d.y, d.x));
            }
        }
        __syncthreads();
        tgfft::smem_fft<NH, +1, YT, NT, LS, float2>(s, tw_h, tid);
        const float kap = (float)(c_mean * (tsum[b] * inv_m - mu_t));
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            const int p = tid + q * NT;
            if (p < YT * NH) {
                const int yl = p / NH, m = p - yl * NH;
                const float2 o = s[yl * LS + m];
                const float c0 = (fmaf(o.x, inv_nm, -m0[q][0] * mt) + kap) * g0[q][0];
                const float c1 = (fmaf(o.y, inv_nm, -m0[q][1] * mt) + kap) * g0[q][1];
                if (c0 > bm[q][0]) { bm[q][0] = c0; bi[q][0] = index0 + b; }
                if (c1 > bm[q][1]) { bm[q][1] = c1; bi[q][1] = index0 + b; }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        const int p = tid + q * NT;
        const int yl = p / NH, m = p - yl * NH;
        const int y = y0 + yl;
        if (p < YT * NH && y < Ny) {
            const long long v = ((long long)z * Ny + y) * NX + 2 * m;
            float2 cur = *reinterpret_cast<float2*>(maxcc + v);
            int2 ci = *reinterpret_cast<int2*>(angidx + v);
            bool ch = false;
            if (bm[q][0] > cur.x) { cur.x = bm[q][0]; ci.x = bi[q][0]; ch = true; }
            if (bm[q][1] > cur.y) { cur.y = bm[q][1]; ci.y = bi[q][1]; ch = true; }
            if (ch) {
                *reinterpret_cast<float2*>(maxcc + v) = cur;
                *reinterpret_cast<int2*>(angidx + v) = ci;
            }
        }
    }
}

// Single-map variant of stage 3 (tom_os3_corr output for one rotation).
template <int NH>
__global__ void __launch_bounds__(256) k_c2r_x_map(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                   const float* __restrict__ gam, const double* __restrict__ tsum,
                                                   int Ny, int Nz, float inv_nm, double c_mean, double inv_m,
                                                   double mu_t, float* __restrict__ cc,
                                                   const float2* __restrict__ tw_h,
                                                   const float2* __restrict__ tw_x) {
    constexpr int YT = 8, NT = 256, NH1 = NH + 1, LS = NH + 1, NX = 2 * NH;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * YT, z = blockIdx.y;
    for (int i = tid; i < YT * NH1; i += NT) {
        const int kx = i / YT, yl = i - kx * YT;
        const int y = y0 + yl;
        s[yl * LS + kx] = y < Ny ? H[((long long)kx * Nz + z) * Ny + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int i = tid; i < YT * (NH / 2 + 1); i += NT) {
        const int yl = i / (NH / 2 + 1), k = i - yl * (NH / 2 + 1);
        float2* row = s + yl * LS;
        const float2 xa = row[k], xb = row[NH - k];
        {
            const float2 bc = cconj(xb);
            const float2 w = cconj(__ldg(tw_x + k));
            const float2 d = cmul(w, csub(xa, bc));
            row[k] = cadd(cadd(xa, bc), make_float2(-d.y, d.x));
        }
        if (k > 0 && k < NH - k) {
            const float2 ac = cconj(xa);
            const float2 w = cconj(__ldg(tw_x + (NH - k)));
            const float2 d = cmul(w, csub(xb, ac));
            row[NH - k] = cadd(cadd(xb, ac), make_float2(-d.y, d.x));
        }
    }
    __syncthreads();
    tgfft::smem_fft<NH, +1, YT, NT, LS, float2>(s, tw_h, tid);
    const float kap = (float)(c_mean * (tsum[0] * inv_m - mu_t));
    const float mt = (float)mu_t;
    for (int p = tid; p < YT * NH; p += NT) {
        const int yl = p / NH, m = p - yl * NH;
        const int y = y0 + yl;
        if (y >= Ny) continue;
        const long long v = ((long long)z * Ny + y) * NX + 2 * m;
        const float2 o = s[yl * LS + m];
        cc[v] = (fmaf(o.x, inv_nm, -mu0[v] * mt) + kap) * gam[v];
        cc[v + 1] = (fmaf(o.y, inv_nm, -mu0[v + 1] * mt) + kap) * gam[v + 1];
    }
}

// F_I in FP64 [z][y][kx] -> FP32 [kx][kz][ky]
__global__ void k_pack_fimg(const double2* __restrict__ in, float2* __restrict__ out, int nh1, int ny, int nz) {
    const long long n = (long long)nh1 * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        // i indexes the output: ky fastest, then kz, then kx
        const int ky = (int)(i % ny);
        const int kz = (int)((i / ny) % nz);
        const int kx = (int)(i / ((long long)ny * nz));
        const double2 v = in[((long long)kz * ny + ky) * nh1 + kx];
        out[i] = make_float2((float)v.x, (float)v.y);
    }
}

__global__ void k_fill_results(float* __restrict__ maxcc, int* __restrict__ idx, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        maxcc[i] = -1000.f;
        idx[i] = -1;
    }
}

// per-batch filter helpers (FP32): real -> complex, multiply weight, complex -> real
__global__ void k_r2c_f32(const float* __restrict__ a, float2* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = make_float2(a[i], 0.f);
}
__global__ void k_mulw_f32(float2* __restrict__ a, const float* __restrict__ w, long long n, long long tn) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = cscale(a[i], w[i % tn]);
}
__global__ void k_c2r_f32(const float2* __restrict__ a, float* __restrict__ b, long long n, float s) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i].x * s;
}

static unsigned grid_n(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

// ------------------------------------------------------- dispatch tables
template <typename K> static void raise_smem(K kern, size_t smem) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

#define TG_HOT_LENGTHS(X) X(16) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(256) X(464) X(512) X(928) X(1024)
#define TG_HALF_LENGTHS(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(232) X(256) X(464) X(512)

static bool hot_len(int L) {
    switch (L) {
#define C_(N) case N:
        TG_HOT_LENGTHS(C_)
#undef C_
        return true;
        default: return false;
    }
}

static bool half_len(int L) {
    switch (L) {
#define C_(N) case N:
        TG_HALF_LENGTHS(C_)
#undef C_
        return true;
        default: return false;
    }
}

// Any volume and template edge MATLAB's fftn takes, within the line-length
// limits of the FFT engines (fft_length_supported; lengths without a
// compile-time kernel run on match_rt.cu's kernels); the template no larger
// than the volume.
bool match_sizes_supported(const int N[3], const int T[3]) {
    for (int d = 0; d < 3; ++d) {
        if (T[d] < 1 || T[d] > N[d]) return false;
        if (!fft_length_supported(N[d]) || !fft_length_supported(T[d])) return false;
        if (!hot_len(N[d]) && !match_rt_length_ok(N[d])) return false;
    }
    if (!(N[0] % 2 == 0 && half_len(N[0] / 2)) && !match_rt_length_ok(N[0])) return false;
    return true;
}

// the x edges the compile-time c2r kernels (half-length packing) cover
static bool c2r_compiled(int NX) { return NX % 2 == 0 && half_len(NX / 2); }

static cudaError_t launch_spec_x(int NX, const float* t2, const float* mask, float2* A, const int T[3], int d0x,
                                 int nb, double* tsum, cudaStream_t st) {
    switch (NX) {
#define C_(N)                                                                                        \
    case N: {                                                                                        \
        constexpr int NL = (4096 / N) < 1 ? 1 : ((4096 / N) > 16 ? 16 : (4096 / N));                 \
        const size_t smem = (size_t)NL * (N + 1) * sizeof(float2);                                   \
        raise_smem(k_spec_x<N>, smem);                                                               \
        dim3 g((T[1] * T[2] + NL - 1) / NL, nb);                                                     \
        k_spec_x<N><<<g, 256, smem, st>>>(t2, mask, A, T[0], T[1], T[2], d0x,                        \
                                          twiddle_table<float2>(N), tsum);                           \
        return cudaGetLastError();                                                                   \
    }
        TG_HOT_LENGTHS(C_)
#undef C_
        default: return launch_spec_x_rt(NX, t2, mask, A, T, d0x, nb, tsum, st);
    }
}

static cudaError_t launch_spec_z(int NZ, const float2* A, float2* Z, const int T[3], int d0z, int nh1, int nb,
                                 cudaStream_t st) {
    switch (NZ) {
#define C_(N)                                                                                     \
    case N: {                                                                                     \
        const size_t smem = (size_t)8 * (N + 1) * sizeof(float2);                                 \
        raise_smem(k_spec_z<N>, smem);                                                            \
        dim3 g((T[1] + 7) / 8, nh1, nb);                                                          \
        k_spec_z<N><<<g, 256, smem, st>>>(A, Z, T[1], T[2], d0z, nh1, twiddle_table<float2>(N));   \
        return cudaGetLastError();                                                                \
    }
        TG_HOT_LENGTHS(C_)
#undef C_
        default: return launch_spec_z_rt(NZ, A, Z, T, d0z, nh1, nb, st);
    }
}

static cudaError_t launch_corr_y(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                                 long long ncols, int nb, cudaStream_t st) {
    switch (NY) {
#define C_(N)                                                                                          \
    case N: {                                                                                          \
        constexpr int NL = (2048 / N) < 1 ? 1 : ((2048 / N) > 16 ? 16 : (2048 / N));                   \
        const size_t smem = (size_t)NL * (N + 1) * sizeof(float2);                                     \
        raise_smem(k_corr_y<N>, smem);                                                                 \
        k_corr_y<N><<<(unsigned)((ncols + NL - 1) / NL), 256, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols,  \
                                                                          nb, twiddle_table<float2>(N)); \
        return cudaGetLastError();                                                                     \
    }
        TG_HOT_LENGTHS(C_)
#undef C_
        default: return launch_corr_y_rt(NY, fimg, Z, Q, Ty, d0y, ncols, nb, st);
    }
}

static cudaError_t launch_inv_z(int NZ, const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st) {
    switch (NZ) {
#define C_(N)                                                                              \
    case N: {                                                                              \
        const size_t smem = (size_t)16 * (N + 1) * sizeof(float2);                         \
        raise_smem(k_inv_z<N>, smem);                                                      \
        dim3 g((Ny + 15) / 16, nh1, nb);                                                   \
        k_inv_z<N><<<g, 256, smem, st>>>(Q, H, Ny, nh1, twiddle_table<float2>(N));          \
        return cudaGetLastError();                                                         \
    }
        TG_HOT_LENGTHS(C_)
#undef C_
        default: return launch_inv_z_rt(NZ, Q, H, Ny, nh1, nb, st);
    }
}

static cudaError_t launch_c2r_flcf(int NH, const float2* H, const float* mu0, const float* gam, const double* tsum,
                                   int Ny, int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t,
                                   int index0, float* maxcc, int* angidx, cudaStream_t st) {
    switch (NH) {
#define C_(N)                                                                                             \
    case N: {                                                                                             \
        const size_t smem = (size_t)8 * (N + 1) * sizeof(float2);                                         \
        raise_smem(k_c2r_x_flcf<N>, smem);                                                                \
        dim3 g((Ny + 7) / 8, Nz);                                                                         \
        k_c2r_x_flcf<N><<<g, 256, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t,      \
                                              index0, maxcc, angidx, twiddle_table<float2>(N),            \
                                              twiddle_table<float2>(2 * N));                              \
        return cudaGetLastError();                                                                        \
    }
        TG_HALF_LENGTHS(C_)
#undef C_
        default: return cudaErrorInvalidValue;
    }
}

static cudaError_t launch_c2r_map(int NH, const float2* H, const float* mu0, const float* gam, const double* tsum,
                                  int Ny, int Nz, float inv_nm, double c, double inv_m, double mu_t, float* cc,
                                  cudaStream_t st) {
    switch (NH) {
#define C_(N)                                                                                         \
    case N: {                                                                                         \
        const size_t smem = (size_t)8 * (N + 1) * sizeof(float2);                                     \
        raise_smem(k_c2r_x_map<N>, smem);                                                             \
        dim3 g((Ny + 7) / 8, Nz);                                                                     \
        k_c2r_x_map<N><<<g, 256, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, inv_nm, c, inv_m, mu_t, cc,    \
                                             twiddle_table<float2>(N), twiddle_table<float2>(2 * N)); \
        return cudaGetLastError();                                                                    \
    }
        TG_HALF_LENGTHS(C_)
#undef C_
        default: return cudaErrorInvalidValue;
    }
}

// ------------------------------------------------------------ the plan
static int d0_corr(int N, int T) { return pmod(2 * (N / 2) - T / 2, N); }

MatchPlan::~MatchPlan() { release(); }

void MatchPlan::release() {
    delete an;
    an = nullptr;
    void* ptrs[] = {d_tmpl, d_mask, d_wu, d_fimg, d_mu0, d_sig, d_gam, d_mats, d_t1, d_tc, d_tsum,
                    d_A, d_Z, d_Q, d_H, d_tmp64, d_cc, d_psr, d_soc, d_auto};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    d_tmpl = d_mask = d_wu = nullptr;
    d_fimg = nullptr;
    d_mu0 = d_sig = d_gam = nullptr;
    d_mats = d_t1 = nullptr;
    d_tc = nullptr;
    d_tsum = nullptr;
    d_A = d_Z = d_Q = d_H = nullptr;
    d_tmp64 = nullptr;
    d_cc = d_psr = d_soc = d_auto = nullptr;
    if (h_mats) cudaFreeHost(h_mats);
    h_mats = nullptr;
    if (ev_mats) cudaEventDestroy(ev_mats);
    ev_mats = nullptr;
}

int MatchPlan::alloc(void** p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(ctx, TOMGPU_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed");
    }
    bytes_held += (int64_t)bytes;
    return TOMGPU_OK;
}

int MatchPlan::create(tomgpu_ctx* c, const int vol[3], const int tm[3], int batch, bool generic) {
    ctx = c;
    generic_only = generic;
    for (int d = 0; d < 3; ++d) { N[d] = vol[d]; T[d] = tm[d]; }
    if (!match_sizes_supported(N, T))
        return fail(ctx, TOMGPU_ERR_UNSUPPORTED,
                    "volume/template sizes not supported by the FFT kernels");
    if (batch > 4096) return fail(ctx, TOMGPU_ERR_ARG, "rotation batch above 4096");
    nvox = (long long)N[0] * N[1] * N[2];
    nh1 = N[0] / 2 + 1;
    tn = (long long)T[0] * T[1] * T[2];
    const long long hs = nh1 * (long long)N[1] * N[2];
    TG_TRY(alloc((void**)&d_tmpl, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_mask, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_wu, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_fimg, sizeof(float2) * hs));
    TG_TRY(alloc((void**)&d_mu0, sizeof(float) * nvox));
    TG_TRY(alloc((void**)&d_sig, sizeof(float) * nvox));
    TG_TRY(alloc((void**)&d_gam, sizeof(float) * nvox));
    TG_TRY(alloc_batch(batch > 0 ? batch : default_batch()));
    TG_TRY_CUDA(ctx, cudaEventCreateWithFlags(&ev_mats, cudaEventDisableTiming));
    // twiddle tables are built now so that later calls allocate nothing
    const int lens[] = {N[0], N[1], N[2], N[0] / 2, T[0], T[1], T[2]};
    for (int L : lens) {
        if (L < 1) continue;
        tgrt::Plan p32, p64;
        tgrt::Tabs<float2> t32;
        tgrt::Tabs<double2> t64;
        if (!twiddle_table<float2>(L) || !twiddle_table<double2>(L) ||
            (rt_plan(L, (int)sizeof(float2), &p32) && !rt_tabs<float2>(p32, &t32)) ||
            (rt_plan(L, (int)sizeof(double2), &p64) && !rt_tabs<double2>(p64, &t64)))
            return fail(ctx, TOMGPU_ERR_CUDA, "twiddle table allocation failed");
    }
    return TOMGPU_OK;
}

// The per-batch work buffers (rotated templates, their spectra, Q and H).
void MatchPlan::free_batch() {
    void* ptrs[] = {d_t1, d_tc, d_tsum, d_A, d_Z, d_Q, d_H};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    d_t1 = nullptr;
    d_tc = nullptr;
    d_tsum = nullptr;
    d_A = d_Z = d_Q = d_H = nullptr;
    bytes_held -= batch_bytes;
    batch_bytes = 0;
}

// Without a requested batch: the largest of 64, 32 and 16 rotations whose
// buffers take at most half of the device memory free at this point (the
// rest is left to the caller), else 8.
int MatchPlan::default_batch() const {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 8;
    }
    for (int nb : {64, 32, 16})
        if (batch_need(nb) <= (int64_t)(fr / 2)) return nb;
    return 8;
}

int64_t MatchPlan::batch_need(int nb) const {
    const long long hs = nh1 * (long long)N[1] * N[2];
    return (int64_t)nb * ((int64_t)sizeof(float) * tn + (int64_t)sizeof(float2) * tn + (int64_t)sizeof(double) +
                          (int64_t)sizeof(float2) * nh1 * T[1] * T[2] + (int64_t)sizeof(float2) * nh1 * N[2] * T[1] +
                          2 * (int64_t)sizeof(float2) * hs);
}

int MatchPlan::alloc_batch(int nb) {
    const long long hs = nh1 * (long long)N[1] * N[2];
    const int64_t before = bytes_held;
    int rc = TOMGPU_OK;
    if (!rc) rc = alloc((void**)&d_t1, sizeof(float) * tn * nb);
    if (!rc) rc = alloc((void**)&d_tc, sizeof(float2) * tn * nb);
    if (!rc) rc = alloc((void**)&d_tsum, sizeof(double) * nb);
    if (!rc) rc = alloc((void**)&d_A, sizeof(float2) * nh1 * T[1] * T[2] * nb);
    if (!rc) rc = alloc((void**)&d_Z, sizeof(float2) * nh1 * N[2] * T[1] * nb);
    if (!rc) rc = alloc((void**)&d_Q, sizeof(float2) * hs * nb);
    if (!rc) rc = alloc((void**)&d_H, sizeof(float2) * hs * nb);
    batch_bytes = bytes_held - before;
    if (rc) {
        free_batch();
        return rc;
    }
    B = nb;
    return TOMGPU_OK;
}

// Rotation-batch autotuner: for each candidate batch size the per-batch
// buffers are re-allocated (a candidate whose buffers would leave less than
// 2 GiB of the device free, or whose allocation fails, is skipped) and R
// rotations are timed with CUDA events on the context's stream after one
// untimed batch; the fastest per rotation is kept.  Results go to scratch
// buffers, so the caller's maxima are untouched.
int MatchPlan::autotune(const float* eulers, int R, const int* cands, int nc, int* best_out, float* ms_out) {
    if (!has_template || !has_volume) return fail(ctx, TOMGPU_ERR_STATE, "template and volume must be set");
    if (R <= 0 || nc <= 0) return fail(ctx, TOMGPU_ERR_ARG, "no rotations or no candidates");
    cudaStream_t st = ctx->stream;
    float* cc = nullptr;
    int* idx = nullptr;
    if (cudaMalloc(&cc, sizeof(float) * nvox) || cudaMalloc(&idx, sizeof(int) * nvox)) {
        if (cc) cudaFree(cc);
        cudaGetLastError();
        return fail(ctx, TOMGPU_ERR_OOM, "autotune scratch");
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int orig = B;
    int best = -1;
    float best_ms = 0.f;
    int rc = TOMGPU_OK;
    for (int c = 0; c < nc && !rc; ++c) {
        const int nb = cands[c];
        if (nb <= 0 || nb > 4096) continue;
        size_t fr = 0, tot = 0;
        if (cudaError_t e_ = cudaMemGetInfo(&fr, &tot)) {
            rc = cuda_fail(ctx, e_, "autotune memory query");
            break;
        }
        // the current batch buffers come back with free_batch
        if (batch_need(nb) + (int64_t(2) << 30) > (int64_t)fr + batch_bytes) continue;
        free_batch();
        if (alloc_batch(nb)) {  // does not fit: skip
            ctx->last_error.clear();
            continue;
        }
        if ((rc = init_results(cc, idx))) break;
        if ((rc = run(eulers, std::min(R, nb), 0, cc, idx))) break;
        cudaEventRecord(e0, st);
        if ((rc = run(eulers, R, 0, cc, idx))) break;
        cudaEventRecord(e1, st);
        if (cudaError_t e_ = cudaEventSynchronize(e1)) { rc = cuda_fail(ctx, e_, "autotune"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= (float)R;
        if (ms_out) ms_out[c] = ms;
        if (best < 0 || ms < best_ms) {
            best = nb;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(cc);
    cudaFree(idx);
    free_batch();
    // the batch buffers come back after an error too, so the plan stays usable;
    // the first error's status and message are the ones reported
    const int keep = best > 0 ? best : orig;
    const std::string first = ctx->last_error;
    const int rc2 = alloc_batch(keep);
    if (!rc) rc = rc2;
    else if (rc2) ctx->last_error = first;
    if (best_out) *best_out = best > 0 ? best : 0;
    return rc;
}

// Template, volume and the rotation-batch buffers (which a failed
// re-allocation in the autotuner can leave absent) before any batch work.
int MatchPlan::check_ready() {
    if (!has_template || !has_volume) return fail(ctx, TOMGPU_ERR_STATE, "template and volume must be set");
    if (!d_t1 || !d_A || !d_Z || !d_Q || !d_H)
        return fail(ctx, TOMGPU_ERR_STATE,
                    "the plan has no rotation-batch buffers (their re-allocation failed): destroy and re-create it");
    return TOMGPU_OK;
}

int MatchPlan::ensure_mats(int R) {
    if (R <= mats_cap) return TOMGPU_OK;
    if (d_mats) { cudaFree(d_mats); bytes_held -= sizeof(float) * 9 * mats_cap; d_mats = nullptr; }
    if (h_mats) { cudaEventSynchronize(ev_mats); cudaFreeHost(h_mats); h_mats = nullptr; }
    TG_TRY(alloc((void**)&d_mats, sizeof(float) * 9 * R));
    if (cudaMallocHost((void**)&h_mats, sizeof(float) * 9 * R) != cudaSuccess)
        return fail(ctx, TOMGPU_ERR_OOM, "pinned host allocation failed");
    mats_cap = R;
    return TOMGPU_OK;
}

int MatchPlan::upload_mats(const float* eulers, int R) {
    TG_TRY(ensure_mats(R));
    TG_TRY_CUDA(ctx, cudaEventSynchronize(ev_mats));  // previous copy out of h_mats finished
    for (int r = 0; r < R; ++r) euler_matrix_host(eulers + 3 * r, h_mats + 9 * r);
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_mats, h_mats, sizeof(float) * 9 * R, cudaMemcpyHostToDevice, ctx->stream));
    TG_TRY_CUDA(ctx, cudaEventRecord(ev_mats, ctx->stream));
    return TOMGPU_OK;
}

int MatchPlan::set_template(const float* tmpl, const float* mask, const float* psf, bool raw) {
    cudaStream_t st = ctx->stream;
    // The volume's local mean and std are made with the mask, its FLCF
    // denominators (gamma) with the template's std: with the same mask the
    // volume stays set and gamma is recomputed at the end; a new mask unsets
    // the volume.  A template that fails half-way leaves the plan unset.
    std::vector<float> m((size_t)tn);
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(m.data(), mask, sizeof(float) * tn, cudaMemcpyDeviceToHost, st));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    const bool keep_volume =
        has_volume && h_mask.size() == m.size() && std::memcmp(h_mask.data(), m.data(), sizeof(float) * tn) == 0;
    has_template = false;
    has_volume = false;
    if (an) {  // the peak analysis holds the old mask's spectrum
        delete an;
        an = nullptr;
    }
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_mask, mask, sizeof(float) * tn, cudaMemcpyDeviceToDevice, st));
    double* d_red = nullptr;
    TG_TRY(ensure_scratch(ctx, 64));
    d_red = static_cast<double*>(ctx->scratch);
    double h[2];
    // mask size (nonzeros)
    TG_TRY_CUDA(ctx, count_nonzero(d_mask, tn, d_red, st));
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    msize = h[0];
    if (msize <= 0) return fail(ctx, TOMGPU_ERR_ARG, "mask has no nonzero voxel");
    if (raw) {
        // tom_os3_corr without cached statistics: normUnderMask of the given template
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_tmpl, tmpl, sizeof(float) * tn, cudaMemcpyDeviceToDevice, st));
        psf = nullptr;
    } else {
        // tom_norm(1e5*(t+1),'mean0+1std'): a = 2e5 t + 2e5 + 100, (a - mean)/std
        const double s = 2e5, o = 2e5 + 100;
        TG_TRY_CUDA(ctx, sum_affine_f32(tmpl, tn, s, o, d_red, st));
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st));
        TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
        const double amean = h[0] / (double)tn;
        TG_TRY_CUDA(ctx, sum_sqdev_f32(tmpl, tn, s, o, amean, d_red, st));
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st));
        TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
        const double astd = std::sqrt(h[0] / (double)tn);
        TG_TRY_CUDA(ctx, normalize_f32(tmpl, d_tmpl, tn, s, o, amean, astd != 0 ? 1.0 / astd : 1.0, st));
        ctx->launches += 4;
    }
    // statistics of the unrotated, filtered template in FP64
    double2* tc64 = nullptr;
    double* tv64 = nullptr;
    if (cudaMalloc(&tc64, sizeof(double2) * tn) != cudaSuccess ||
        cudaMalloc(&tv64, sizeof(double) * tn) != cudaSuccess) {
        if (tc64) cudaFree(tc64);
        return fail(ctx, TOMGPU_ERR_OOM, "template workspace allocation failed");
    }
    int rc = TOMGPU_OK;
    has_psf = psf != nullptr;
    do {
        if (has_psf) {
            if (cudaError_t e_ = ifftshift_real(psf, d_wu, T, st)) { rc = cuda_fail(ctx, e_, "ifftshift"); break; }
            real_to_c64(d_tmpl, tc64, tn, st);
            if (cudaError_t e_ = c2c3d<double2>(tc64, T, -1, 1.0, st)) { rc = cuda_fail(ctx, e_, "fft"); break; }
            mul_weight_c64(tc64, d_wu, tn, st);
            if (cudaError_t e_ = c2c3d<double2>(tc64, T, +1, 1.0 / (double)tn, st)) { rc = cuda_fail(ctx, e_, "ifft"); break; }
            re_c64(tc64, tv64, tn, 1.0, st);
            ctx->launches += 10;
        } else {
            affine_f32_to_f64(d_tmpl, tv64, tn, 1.0, 0.0, st);
            ctx->launches += 1;
        }
        if (cudaError_t e_ = norm_under_mask_sums(tv64, d_mask, tn, d_red, nullptr, 0, 0, st)) { rc = cuda_fail(ctx, e_, "sum"); break; }
        cudaMemcpyAsync(h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        tmean = h[0] / msize;
        if (cudaError_t e_ = norm_under_mask_sums(tv64, d_mask, tn, nullptr, d_red, tmean, 1, st)) { rc = cuda_fail(ctx, e_, "sum"); break; }
        cudaMemcpyAsync(h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (cudaError_t e_ = cudaStreamSynchronize(st)) { rc = cuda_fail(ctx, e_, "sync"); break; }
        tstd = std::sqrt(h[0] / msize);
        ctx->launches += 2;
    } while (0);
    cudaFree(tc64);
    cudaFree(tv64);
    if (rc) return rc;
    h_mask.swap(m);
    has_template = true;
    if (keep_volume) {
        TG_TRY_CUDA(ctx, gamma_from_sigma(d_sig, d_gam, nvox, tstd, st));
        ctx->launches += 1;
        has_volume = true;
    }
    return TOMGPU_OK;
}

int MatchPlan::set_volume(const float* vol) {
    if (!has_template) return fail(ctx, TOMGPU_ERR_STATE, "set the template and mask before the volume");
    cudaStream_t st = ctx->stream;
    TG_TRY(ensure_scratch(ctx, 64));
    double* d_red = static_cast<double*>(ctx->scratch);
    double h = 0;
    TG_TRY_CUDA(ctx, sum_affine_f32(vol, nvox, 1.0, 0.0, d_red, st));
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(&h, d_red, sizeof(double), cudaMemcpyDeviceToHost, st));
    TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    vmean = h / (double)nvox;
    const long long hs = nh1 * (long long)N[1] * N[2];
    double* v64 = nullptr;
    double2 *f1 = nullptr, *f2 = nullptr, *fm = nullptr;
    double* m2 = nullptr;
    bool owns_ws = true;  // false while the workspace is borrowed from Q and H
    auto cleanup = [&]() {
        if (!owns_ws) return;
        if (v64) cudaFree(v64);
        if (f1) cudaFree(f1);
        if (f2) cudaFree(f2);
        if (fm) cudaFree(fm);
        if (m2) cudaFree(m2);
    };
    // The FP64 workspace (about 40 bytes per voxel) lives in the rotation-batch
    // buffers Q and H when they are large enough: they are idle between batch
    // calls, and a search over many tomograms then allocates nothing per volume.
    // Otherwise it is allocated for this call.
    {
        struct Piece { void** p; size_t bytes; };
        const Piece pieces[] = {{(void**)&v64, sizeof(double) * nvox}, {(void**)&m2, sizeof(double) * nvox},
                                {(void**)&f1, sizeof(double2) * hs}, {(void**)&f2, sizeof(double2) * hs},
                                {(void**)&fm, sizeof(double2) * hs}};
        const size_t cap = d_Q && d_H ? sizeof(float2) * hs * (size_t)B : 0;
        char* bufs[2] = {reinterpret_cast<char*>(d_Q), reinterpret_cast<char*>(d_H)};
        size_t used[2] = {0, 0};
        bool borrowed = cap > 0;
        for (const Piece& pc : pieces) {
            const size_t b = (pc.bytes + 255) & ~size_t(255);
            int k = used[0] + b <= cap ? 0 : (used[1] + b <= cap ? 1 : -1);
            if (k < 0) { borrowed = false; break; }
            *pc.p = bufs[k] + used[k];
            used[k] += b;
        }
        if (!borrowed) {
            v64 = m2 = nullptr;
            f1 = f2 = fm = nullptr;
            if (cudaMalloc(&v64, sizeof(double) * nvox) || cudaMalloc(&f1, sizeof(double2) * hs) ||
                cudaMalloc(&f2, sizeof(double2) * hs) || cudaMalloc(&fm, sizeof(double2) * hs) ||
                cudaMalloc(&m2, sizeof(double) * nvox)) {
                cudaGetLastError();
                cleanup();
                return fail(ctx, TOMGPU_ERR_OOM, "set_volume FP64 workspace allocation failed");
            }
        } else {
            owns_ws = false;
        }
    }
    int rc = TOMGPU_OK;
    do {
        const int T0[3] = {T[0], T[1], T[2]};
        // I0 = I - c and its spectrum
        if (cudaError_t e_ = affine_f32_to_f64(vol, v64, nvox, 1.0, -vmean, st)) { rc = cuda_fail(ctx, e_, "affine"); break; }
        if (cudaError_t e_ = r2c3d<double2>(v64, f1, N, st)) { rc = cuda_fail(ctx, e_, "r2c"); break; }
        {
            long long n = hs;
            k_pack_fimg<<<grid_n(n), 256, 0, st>>>(f1, d_fimg, (int)nh1, N[1], N[2]);
        }
        // spectrum of I0^2
        if (cudaError_t e_ = square_f64(v64, nvox, st)) { rc = cuda_fail(ctx, e_, "square"); break; }
        if (cudaError_t e_ = r2c3d<double2>(v64, f2, N, st)) { rc = cuda_fail(ctx, e_, "r2c"); break; }
        // mask placed at (j - floor(T/2)) mod N: convolution kernel of tom_os3_mean / tom_os3_std
        if (cudaError_t e_ = cudaMemsetAsync(v64, 0, sizeof(double) * nvox, st)) { rc = cuda_fail(ctx, e_, "memset"); break; }
        const int off[3] = {-(T[0] / 2), -(T[1] / 2), -(T[2] / 2)};
        if (cudaError_t e_ = place_f64(d_mask, T0, v64, N, off, st)) { rc = cuda_fail(ctx, e_, "place"); break; }
        if (cudaError_t e_ = r2c3d<double2>(v64, fm, N, st)) { rc = cuda_fail(ctx, e_, "r2c"); break; }
        const double sc = 1.0 / ((double)nvox * msize);
        mul_c64(f1, fm, hs, st);
        if (cudaError_t e_ = c2r3d<double2>(f1, v64, N, sc, st)) { rc = cuda_fail(ctx, e_, "c2r"); break; }
        mul_c64(f2, fm, hs, st);
        if (cudaError_t e_ = c2r3d<double2>(f2, m2, N, sc, st)) { rc = cuda_fail(ctx, e_, "c2r"); break; }
        if (cudaError_t e_ = stats_final(v64, m2, d_mu0, d_sig, nvox, st)) { rc = cuda_fail(ctx, e_, "stats"); break; }
        if (cudaError_t e_ = gamma_from_sigma(d_sig, d_gam, nvox, tstd, st)) { rc = cuda_fail(ctx, e_, "gamma"); break; }
        if (cudaError_t e_ = cudaStreamSynchronize(st)) { rc = cuda_fail(ctx, e_, "sync"); break; }
        ctx->launches += 4 * 3 + 3 * 2 + 8;
    } while (0);
    cleanup();
    if (rc) return rc;
    has_volume = true;
    return TOMGPU_OK;
}

int MatchPlan::prepare_batch(int off, int nb) {
    cudaStream_t st = ctx->stream;
    const float center[3] = {(float)((T[0] + 1) / 2), (float)((T[1] + 1) / 2), (float)((T[2] + 1) / 2)};
    {
        ProfScope ps(ctx, TOMGPU_K_ROTATE);
        TG_TRY_CUDA(ctx, rotate3d_batch(d_tmpl, d_t1, T, d_mats + 9 * (long long)off, nb, center, d_mask, st));
    }
    ctx->launches += 1;
    if (has_psf) {
        ProfScope ps(ctx, TOMGPU_K_FILTER);
        const long long n = tn * nb;
        k_r2c_f32<<<grid_n(n), 256, 0, st>>>(d_t1, d_tc, n);
        TG_TRY_CUDA(ctx, c2c3d_batch(d_tc, T, nb, -1, 1.0, st));
        k_mulw_f32<<<grid_n(n), 256, 0, st>>>(d_tc, d_wu, n, tn);
        TG_TRY_CUDA(ctx, c2c3d_batch(d_tc, T, nb, +1, 1.0, st));
        k_c2r_f32<<<grid_n(n), 256, 0, st>>>(d_tc, d_t1, n, 1.0f / (float)tn);
        TG_TRY_CUDA(ctx, cudaGetLastError());
        ctx->launches += 3 + 6;
    }
    TG_TRY_CUDA(ctx, cudaMemsetAsync(d_tsum, 0, sizeof(double) * nb, st));
    {
        ProfScope ps(ctx, TOMGPU_K_SPEC_X);
        TG_TRY_CUDA(ctx, launch_spec_x(N[0], d_t1, d_mask, d_A, T, d0_corr(N[0], T[0]), nb, d_tsum, st));
    }
    {
        ProfScope ps(ctx, TOMGPU_K_SPEC_Z);
        if (!generic_only && fast_spec_z(N[2], T[2]))
            TG_TRY_CUDA(ctx, launch_spec_z_fast(N[2], d_A, d_Z, T[1], T[2], d0_corr(N[2], T[2]), (int)nh1, nb, st));
        else
            TG_TRY_CUDA(ctx, launch_spec_z(N[2], d_A, d_Z, T, d0_corr(N[2], T[2]), (int)nh1, nb, st));
    }
    ctx->launches += 2;
    return TOMGPU_OK;
}

int MatchPlan::run(const float* eulers, int R, int index_offset, float* maxcc, int* angidx) {
    if (int rc = check_ready()) return rc;
    if (R <= 0) return TOMGPU_OK;
    cudaStream_t st = ctx->stream;
    TG_TRY(upload_mats(eulers, R));
    const long long ncols = nh1 * (long long)N[2];
    const float inv_nm = (float)(1.0 / ((double)nvox * msize));
    for (int off = 0; off < R; off += B) {
        const int nb = std::min(B, R - off);
        TG_TRY(prepare_batch(off, nb));
        const int d0y = d0_corr(N[1], T[1]);
        {
            ProfScope ps(ctx, TOMGPU_K_CORR_Y);
            if (!generic_only && fast_corr_y(N[1], T[1]))
                TG_TRY_CUDA(ctx, launch_corr_y_fast(N[1], d_fimg, d_Z, d_Q, T[1], d0y, ncols, nb, st, !no_tma));
            else
                TG_TRY_CUDA(ctx, launch_corr_y(N[1], d_fimg, d_Z, d_Q, T[1], d0y, ncols, nb, st));
        }
        {
            ProfScope ps(ctx, TOMGPU_K_INV_Z);
            if (!generic_only && tc_inv_z && N[2] == 256)
                TG_TRY_CUDA(ctx, launch_inv_z_tc256(d_Q, d_H, N[1], (int)nh1, nb, ctx->d_err, st));
            else if (!generic_only && fast_inv_z(N[2]))
                TG_TRY_CUDA(ctx, launch_inv_z_fast(N[2], d_Q, d_H, N[1], (int)nh1, nb, st));
            else
                TG_TRY_CUDA(ctx, launch_inv_z(N[2], d_Q, d_H, N[1], (int)nh1, nb, st));
        }
        {
            ProfScope ps(ctx, TOMGPU_K_C2R_FLCF);
            if (!generic_only && !no_tma && N[0] == 512 && N[1] % 2 == 0 && tma_c2r_available())
                TG_TRY_CUDA(ctx, launch_c2r_t256(d_H, d_mu0, d_gam, d_tsum, N[1], N[2], nb, inv_nm, vmean, 1.0 / msize,
                                                 tmean, index_offset + off, maxcc, angidx, ctx->d_err, st));
            else if (!generic_only && !no_tma && N[0] == 928 && N[1] % 2 == 0 && tma_c2r_available())
                TG_TRY_CUDA(ctx, launch_c2r_t464(d_H, d_mu0, d_gam, d_tsum, N[1], N[2], nb, inv_nm, vmean, 1.0 / msize,
                                                 tmean, index_offset + off, maxcc, angidx, ctx->d_err, st));
            else if (!generic_only && N[0] % 2 == 0 && fast_c2r(N[0] / 2))
                TG_TRY_CUDA(ctx, launch_c2r_fast(N[0] / 2, d_H, d_mu0, d_gam, d_tsum, N[1], N[2], nb, inv_nm, vmean,
                                                 1.0 / msize, tmean, index_offset + off, maxcc, angidx, st));
            else if (c2r_compiled(N[0]))
                TG_TRY_CUDA(ctx, launch_c2r_flcf(N[0] / 2, d_H, d_mu0, d_gam, d_tsum, N[1], N[2], nb, inv_nm, vmean,
                                                 1.0 / msize, tmean, index_offset + off, maxcc, angidx, st));
            else
                TG_TRY_CUDA(ctx, launch_c2r_flcf_rt(N[0], d_H, d_mu0, d_gam, d_tsum, N[1], N[2], nb, inv_nm, vmean,
                                                    1.0 / msize, tmean, index_offset + off, maxcc, angidx, st));
        }
        ctx->launches += 3;
    }
    return TOMGPU_OK;
}

int MatchPlan::corr(const float* t, float* cc) {
    if (int rc = check_ready()) return rc;
    cudaStream_t st = ctx->stream;
    // the given template is already rotated, masked and filtered: S and the
    // spectrum come from t * mask (tom_os3_corr.m:151)
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_t1, t, sizeof(float) * tn, cudaMemcpyDeviceToDevice, st));
    TG_TRY_CUDA(ctx, cudaMemsetAsync(d_tsum, 0, sizeof(double), st));
    TG_TRY_CUDA(ctx, launch_spec_x(N[0], d_t1, d_mask, d_A, T, d0_corr(N[0], T[0]), 1, d_tsum, st));
    TG_TRY_CUDA(ctx, launch_spec_z(N[2], d_A, d_Z, T, d0_corr(N[2], T[2]), (int)nh1, 1, st));
    ctx->launches += 2;
    return cc_map_tail(cc);
}

int MatchPlan::cc_map_tail(float* cc) {
    cudaStream_t st = ctx->stream;
    const long long ncols = nh1 * (long long)N[2];
    TG_TRY_CUDA(ctx, launch_corr_y(N[1], d_fimg, d_Z, d_Q, T[1], d0_corr(N[1], T[1]), ncols, 1, st));
    TG_TRY_CUDA(ctx, launch_inv_z(N[2], d_Q, d_H, N[1], (int)nh1, 1, st));
    const float inv_nm = (float)(1.0 / ((double)nvox * msize));
    if (c2r_compiled(N[0]))
        TG_TRY_CUDA(ctx, launch_c2r_map(N[0] / 2, d_H, d_mu0, d_gam, d_tsum, N[1], N[2], inv_nm, vmean, 1.0 / msize,
                                        tmean, cc, st));
    else
        TG_TRY_CUDA(ctx, launch_c2r_map_rt(N[0], d_H, d_mu0, d_gam, d_tsum, N[1], N[2], inv_nm, vmean, 1.0 / msize,
                                           tmean, cc, st));
    ctx->launches += 3;
    return TOMGPU_OK;
}

// tom_os3_findTemplate.m:255-307 with the PSR and autocorrelation maps of every
// rotation (tom_os3_analyzePeak) and tom_os3_bestPeak's update for the
// selected criteria: one rotation at a time, each rotation's maps in FP64.
int MatchPlan::run_analysis(const float* eulers, int R, int index_offset, int flags, float* maxcc, int* angidx,
                            float* psr, float* soc) {
    if (int rc = check_ready()) return rc;
    if (R <= 0) return TOMGPU_OK;
    if (!an) {
        an = new (std::nothrow) PeakAnalysis();
        if (!an) return fail(ctx, TOMGPU_ERR_OOM, "peak-analysis state");
        int rc = an->create(ctx, N, T, d_mask);
        if (!rc) rc = alloc((void**)&d_cc, sizeof(float) * nvox);
        if (!rc) rc = alloc((void**)&d_psr, sizeof(float) * nvox);
        if (!rc) rc = alloc((void**)&d_soc, sizeof(float) * nvox);
        if (!rc) rc = alloc((void**)&d_auto, sizeof(float) * tn);
        if (rc) {
            delete an;
            an = nullptr;
            return rc;
        }
    }
    TG_TRY(upload_mats(eulers, R));
    for (int r = 0; r < R; ++r) {
        TG_TRY(prepare_batch(r, 1));          // d_t1: the rotated, masked, filtered template
        TG_TRY(cc_map_tail(d_cc));
        TG_TRY(an->autocorr(d_t1, d_auto));
        TG_TRY(an->spectra(d_cc));
        TG_TRY(an->psr(d_cc, d_psr));
        TG_TRY(an->soc(d_cc, d_auto, d_soc));
        TG_TRY(analysis_update(ctx, d_cc, d_psr, d_soc, nvox, flags, index_offset + r, maxcc, angidx, psr, soc));
    }
    return TOMGPU_OK;
}

int MatchPlan::init_results(float* maxcc, int* angidx) {
    k_fill_results<<<grid_n(nvox), 256, 0, ctx->stream>>>(maxcc, angidx, nvox);
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cudaGetLastError());
    return TOMGPU_OK;
}

// batched full complex 3-D transform of nb volumes [nb][tz][ty][tx]
template <typename C>
static cudaError_t c2c3d_batch_t(C* data, const int t[3], int nb, int dir, double scale, cudaStream_t st) {
    const long tx = t[0], ty = t[1], tz = t[2];
    cudaError_t e;
    LineGeom gx{1, (int)ty, tx, (int)(tz * nb), tx * ty};
    if ((e = fft_lines<C>((int)tx, dir, FFT_C2C, data, data, gx, gx, ty * tz * nb, 1.0, st))) return e;
    LineGeom gy{tx, (int)tx, 1, (int)(tz * nb), tx * ty};
    if ((e = fft_lines<C>((int)ty, dir, FFT_C2C, data, data, gy, gy, tx * tz * nb, 1.0, st))) return e;
    LineGeom gz{tx * ty, (int)(tx * ty), 1, nb, tx * ty * tz};
    return fft_lines<C>((int)tz, dir, FFT_C2C, data, data, gz, gz, tx * ty * nb, scale, st);
}
cudaError_t c2c3d_batch(float2* data, const int t[3], int nb, int dir, double scale, cudaStream_t st) {
    return c2c3d_batch_t<float2>(data, t, nb, dir, scale, st);
}
cudaError_t c2c3d_batch64(double2* data, const int t[3], int nb, int dir, double scale, cudaStream_t st) {
    return c2c3d_batch_t<double2>(data, t, nb, dir, scale, st);
}

__global__ void k_mulw_c64_batch(double2* __restrict__ a, const float* __restrict__ w, long long n, long long tn) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = cscale(a[i], (double)w[i % tn]);
}

int MatchPlan::rescore(const float* vol, const float* eulers, const int* pos1, int K, double* out) {
    if (!has_template) return fail(ctx, TOMGPU_ERR_STATE, "set the template first");
    if (K <= 0) return TOMGPU_OK;
    for (int k = 0; k < K; ++k)
        for (int d = 0; d < 3; ++d)
            if (pos1[3 * k + d] < 1 || pos1[3 * k + d] > N[d])
                return fail(ctx, TOMGPU_ERR_ARG, "candidate position outside the volume");
    cudaStream_t st = ctx->stream;
    std::vector<float> mats(9 * (size_t)K);
    for (int k = 0; k < K; ++k) euler_matrix_host(eulers + 3 * k, mats.data() + 9 * k);
    std::vector<int> p0(3 * (size_t)K);
    for (int i = 0; i < 3 * K; ++i) p0[i] = pos1[i] - 1;
    float *d_m = nullptr, *d_t = nullptr;
    double *d_t64 = nullptr, *d_out = nullptr;
    double2* d_c = nullptr;
    int* d_p = nullptr;
    const long long n = tn * K;
    auto cleanup = [&]() {
        if (d_m) cudaFree(d_m);
        if (d_t) cudaFree(d_t);
        if (d_t64) cudaFree(d_t64);
        if (d_out) cudaFree(d_out);
        if (d_c) cudaFree(d_c);
        if (d_p) cudaFree(d_p);
    };
    if (cudaMalloc(&d_m, sizeof(float) * 9 * K) || cudaMalloc(&d_t, sizeof(float) * n) ||
        cudaMalloc(&d_t64, sizeof(double) * n) || cudaMalloc(&d_out, sizeof(double) * K) ||
        cudaMalloc(&d_p, sizeof(int) * 3 * K) || (has_psf && cudaMalloc(&d_c, sizeof(double2) * n))) {
        cudaGetLastError();
        cleanup();
        return fail(ctx, TOMGPU_ERR_OOM, "rescoring workspace allocation failed");
    }
    int rc = TOMGPU_OK;
    do {
        cudaError_t e = cudaMemcpyAsync(d_m, mats.data(), sizeof(float) * 9 * K, cudaMemcpyHostToDevice, st);
        if (!e) e = cudaMemcpyAsync(d_p, p0.data(), sizeof(int) * 3 * K, cudaMemcpyHostToDevice, st);
        const float center[3] = {(float)((T[0] + 1) / 2), (float)((T[1] + 1) / 2), (float)((T[2] + 1) / 2)};
        if (!e) e = rotate3d_batch(d_tmpl, d_t, T, d_m, K, center, d_mask, st);
        if (!e && !has_psf) e = f32_to_f64(d_t, d_t64, n, st);
        if (!e && has_psf) {
            e = real_to_c64(d_t, d_c, n, st);
            if (!e) e = c2c3d_batch64(d_c, T, K, -1, 1.0, st);
            if (!e) {
                k_mulw_c64_batch<<<grid_n(n), 256, 0, st>>>(d_c, d_wu, n, tn);
                e = cudaGetLastError();
            }
            if (!e) e = c2c3d_batch64(d_c, T, K, +1, 1.0 / (double)tn, st);
            if (!e) e = re_c64(d_c, d_t64, n, 1.0, st);
        }
        if (!e) e = rescore_fp64(vol, N, d_t64, d_mask, T, d_p, K, msize, tmean, tstd, d_out, st);
        if (!e) e = cudaMemcpyAsync(out, d_out, sizeof(double) * K, cudaMemcpyDeviceToHost, st);
        if (!e) e = cudaStreamSynchronize(st);
        if (e) rc = cuda_fail(ctx, e, "rescore_fp64");
        ctx->launches += has_psf ? 11 : 3;
    } while (0);
    cleanup();
    return rc;
}

}  // namespace tg
