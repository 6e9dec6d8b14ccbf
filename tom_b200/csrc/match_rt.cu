// FLCF matching kernels for any tomogram edge (the stages of match.cu on the
// run-time line engine, fft_rt.cuh).
//
// match.cu's kernels are compiled per line length and cover the lengths the
// library builds fast paths for; MATLAB's fftn (search/tom_os3_corr.m:151-153,
// search/tom_os3_findTemplate.m:245) takes any size, so every other edge runs
// here: the same five stages over the same buffers and layouts (A[b][kx][jz][jy],
// Z[b][kx][kz][jy], Q[b][kx][kz][y], H[b][kx][z][y], results [z][y][x]) with
// the line length a kernel argument.  The x edge may be odd: the last stage is
// a full-length complex inverse of the Hermitian-extended half spectrum (its
// real part is the real inverse) rather than the half-length packing the
// even-edge kernels use.  Same arithmetic otherwise: FLCF
//   cc = (out / (N M) - mu0 mu_T + c (S_r / M - mu_T)) * gamma
// and the strict running maximum over the rotations, first angle kept on ties
// (search/tom_os3_bestPeak.m:42-47), per rotation.
#include <algorithm>

#include "fft_rt.cuh"
#include "match.h"
#include "twiddles.h"

namespace tg {

namespace {

constexpr int NT = 256;

struct RtLines {
    tgrt::Plan p;
    tgrt::Tabs<float2> t;
    int LS;
};

// plan and tables of an FP32 line length on the current device
bool rt_lines(int L, RtLines* out) {
    if (!rt_plan(L, (int)sizeof(float2), &out->p)) return false;
    if (!rt_tabs<float2>(out->p, &out->t)) return false;
    out->LS = tgrt::pitch(out->p);
    return true;
}

// lines per block: as many two-buffer lines (plus extra bytes per line) as fit
// `budget`, at least 1 and at most cap; 0 when one line does not fit a block
int lines_per_block(int LS, size_t extra_per_line, size_t budget, int cap) {
    const size_t per = 2 * (size_t)LS * sizeof(float2) + extra_per_line;
    if (per > (size_t)tgrt::kMaxBlockSmem) return 0;
    int nl = (int)std::max<size_t>(1, budget / per);
    return std::min(nl, cap);
}

// above 40 KB of dynamic shared memory a kernel's static arrays could take
// the block past the 48 KB a launch gets without opting in
template <typename K> cudaError_t allow_smem(K kern, size_t smem) {
    if (smem <= 40 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace

// x-stage of the template spectrum: lines (jy, jz) of rotation b, placed at
// (jx + d0x) mod Nx, times the mask; kx in [0, Nx/2] kept.  S_b in FP64.
__global__ void __launch_bounds__(NT) k_spec_x_rt(const float* __restrict__ t2, const float* __restrict__ mask,
                                                  float2* __restrict__ A, int Tx, int Ty, int Tz, int d0x,
                                                  tgrt::Plan p, tgrt::Tabs<float2> tabs, int NL, int LS,
                                                  double* __restrict__ tsum) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[NT / 32];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    const int NX = p.L, NH1 = NX / 2 + 1;
    const int tid = threadIdx.x;
    const int line0 = blockIdx.x * NL, b = blockIdx.y;
    const int nlines = Ty * Tz;
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
    const float2* res = tgrt::fft<-1>(s, s2, p, tabs, NL, LS, tid, NT);
    for (int i = tid; i < NL * NH1; i += NT) {
        const int kx = i / NL, li = i - kx * NL;
        const int rem = line0 + li;
        if (rem >= nlines) continue;
        const int jz = rem / Ty, jy = rem - jz * Ty;
        A[(((long long)b * NH1 + kx) * Tz + jz) * Ty + jy] = res[li * LS + kx];
    }
}

// z-stage: Z[b][kx][kz][jy] = sum_jz A[b][kx][jz][jy] exp(-2 pi i kz (jz + d0z) / Nz)
__global__ void __launch_bounds__(NT) k_spec_z_rt(const float2* __restrict__ A, float2* __restrict__ Z, int Ty,
                                                  int Tz, int d0z, int nh1, tgrt::Plan p, tgrt::Tabs<float2> tabs,
                                                  int NL, int LS) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    const int NZ = p.L;
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
    const float2* res = tgrt::fft<-1>(s, s2, p, tabs, NL, LS, tid, NT);
    const long long zbase = ((long long)b * nh1 + kx) * NZ * Ty;
    for (int i = tid; i < NL * NZ; i += NT) {
        const int kz = i / NL, li = i - kz * NL;
        const int jy = jy0 + li;
        if (jy < Ty) Z[zbase + (long long)kz * Ty + jy] = res[li * LS + kz];
    }
}

// Per spectrum column (kx, kz) and rotation b: the y-DFT of the template
// column (Ty samples at (jy + d0y) mod Ny), the product F_I conj(G), the
// inverse y-DFT.  The block's F_I columns are staged once in shared memory.
__global__ void __launch_bounds__(NT) k_corr_y_rt(const float2* __restrict__ fimg, const float2* __restrict__ Z,
                                                  float2* __restrict__ Q, int Ty, int d0y, long long ncols, int nb,
                                                  tgrt::Plan p, tgrt::Tabs<float2> tabs, int NL, int LS) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    float2* sf = s2 + (size_t)NL * LS;  // NL x NY
    const int NY = p.L;
    const int tid = threadIdx.x;
    const long long col0 = (long long)blockIdx.x * NL;
    for (int i = tid; i < NL * NY; i += NT) {
        const int li = i / NY, e = i - li * NY;
        sf[i] = col0 + li < ncols ? fimg[(col0 + li) * NY + e] : make_float2(0.f, 0.f);
    }
    for (int b = 0; b < nb; ++b) {
        for (int i = tid; i < NL * NY; i += NT) {
            const int li = i / NY, e = i - li * NY;
            const int jy = pmod(e - d0y, NY);
            float2 v = make_float2(0.f, 0.f);
            if (jy < Ty && col0 + li < ncols) v = Z[((long long)b * ncols + col0 + li) * Ty + jy];
            s[li * LS + e] = v;
        }
        __syncthreads();
        float2* X = tgrt::fft<-1>(s, s2, p, tabs, NL, LS, tid, NT);
        float2* Y = X == s ? s2 : s;
        for (int i = tid; i < NL * NY; i += NT) {
            const int li = i / NY, e = i - li * NY;
            X[li * LS + e] = cmulc(sf[i], X[li * LS + e]);
        }
        __syncthreads();
        const float2* res = tgrt::fft<+1>(X, Y, p, tabs, NL, LS, tid, NT);
        for (int i = tid; i < NL * NY; i += NT) {
            const int li = i / NY, e = i - li * NY;
            if (col0 + li < ncols) Q[((long long)b * ncols + col0 + li) * NY + e] = res[li * LS + e];
        }
        __syncthreads();
    }
}

// Inverse z-DFT, Q[b][kx][kz][y] -> H[b][kx][z][y], for NL consecutive y.
__global__ void __launch_bounds__(NT) k_inv_z_rt(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                                 int nh1, tgrt::Plan p, tgrt::Tabs<float2> tabs, int NL, int LS) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    const int NZ = p.L;
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * NL, kx = blockIdx.y, b = blockIdx.z;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    for (int i = tid; i < NL * NZ; i += NT) {
        const int kz = i / NL, yl = i - kz * NL;
        const int y = y0 + yl;
        s[yl * LS + kz] = y < Ny ? Q[base + (long long)kz * Ny + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* res = tgrt::fft<+1>(s, s2, p, tabs, NL, LS, tid, NT);
    for (int i = tid; i < NL * NZ; i += NT) {
        const int z = i / NL, yl = i - z * NL;
        const int y = y0 + yl;
        if (y < Ny) H[base + (long long)z * Ny + y] = res[yl * LS + z];
    }
}

// Load the x lines (y0 + l, z) of rotation b's half spectrum, Hermitian-extended
// to the full length NX.
__device__ __forceinline__ void load_x_lines(const float2* __restrict__ H, long long hb, float2* s, int NL, int LS,
                                             int NX, int y0, int z, int Ny, int Nz, int tid) {
    for (int i = tid; i < NL * NX; i += NT) {
        const int e = i / NL, yl = i - e * NL;
        const int y = y0 + yl;
        float2 v = make_float2(0.f, 0.f);
        if (y < Ny) {
            const int kx = e <= NX / 2 ? e : NX - e;
            v = H[hb + ((long long)kx * Nz + z) * Ny + y];
            if (e > NX / 2) v = cconj(v);
        }
        s[yl * LS + e] = v;
    }
}

// Inverse x-DFT to reals, FLCF, strict running maximum over the batch kept in
// shared memory, one read-modify-write of the results per batch.
__global__ void __launch_bounds__(NT) k_c2r_flcf_rt(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                    const float* __restrict__ gam, const double* __restrict__ tsum,
                                                    int Ny, int Nz, int nb, float inv_nm, double c_mean,
                                                    double inv_m, double mu_t, int index0,
                                                    float* __restrict__ maxcc, int* __restrict__ angidx,
                                                    tgrt::Plan p, tgrt::Tabs<float2> tabs, int NL, int LS) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    const int NX = p.L;
    float* bm = reinterpret_cast<float*>(s2 + (size_t)NL * LS);  // NL x NX
    int* bi = reinterpret_cast<int*>(bm + (size_t)NL * NX);       // NL x NX
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * NL, z = blockIdx.y;
    const long long nh1 = NX / 2 + 1;
    const float mt = (float)mu_t;
    for (int i = tid; i < NL * NX; i += NT) {
        bm[i] = -INFINITY;
        bi[i] = -1;
    }
    for (int b = 0; b < nb; ++b) {
        load_x_lines(H, (long long)b * nh1 * Nz * Ny, s, NL, LS, NX, y0, z, Ny, Nz, tid);
        __syncthreads();
        const float2* res = tgrt::fft<+1>(s, s2, p, tabs, NL, LS, tid, NT);
        const float kap = (float)(c_mean * (tsum[b] * inv_m - mu_t));
        for (int i = tid; i < NL * NX; i += NT) {
            const int yl = i / NX, x = i - yl * NX;
            const int y = y0 + yl;
            if (y >= Ny) continue;
            const long long v = ((long long)z * Ny + y) * NX + x;
            const float cc = (fmaf(res[yl * LS + x].x, inv_nm, -__ldg(mu0 + v) * mt) + kap) * __ldg(gam + v);
            if (cc > bm[i]) {
                bm[i] = cc;
                bi[i] = index0 + b;
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < NL * NX; i += NT) {
        const int yl = i / NX, x = i - yl * NX;
        const int y = y0 + yl;
        if (y >= Ny) continue;
        const long long v = ((long long)z * Ny + y) * NX + x;
        if (bm[i] > maxcc[v]) {
            maxcc[v] = bm[i];
            angidx[v] = bi[i];
        }
    }
}

// Single-map variant (tom_os3_corr's output for one rotation).
__global__ void __launch_bounds__(NT) k_c2r_map_rt(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                   const float* __restrict__ gam, const double* __restrict__ tsum,
                                                   int Ny, int Nz, float inv_nm, double c_mean, double inv_m,
                                                   double mu_t, float* __restrict__ cc, tgrt::Plan p,
                                                   tgrt::Tabs<float2> tabs, int NL, int LS) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* s2 = s + (size_t)NL * LS;
    const int NX = p.L;
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * NL, z = blockIdx.y;
    load_x_lines(H, 0, s, NL, LS, NX, y0, z, Ny, Nz, tid);
    __syncthreads();
    const float2* res = tgrt::fft<+1>(s, s2, p, tabs, NL, LS, tid, NT);
    const float kap = (float)(c_mean * (tsum[0] * inv_m - mu_t));
    const float mt = (float)mu_t;
    for (int i = tid; i < NL * NX; i += NT) {
        const int yl = i / NX, x = i - yl * NX;
        const int y = y0 + yl;
        if (y >= Ny) continue;
        const long long v = ((long long)z * Ny + y) * NX + x;
        cc[v] = (fmaf(res[yl * LS + x].x, inv_nm, -mu0[v] * mt) + kap) * gam[v];
    }
}

// ------------------------------------------------------------ launchers
bool match_rt_length_ok(int L) {
    tgrt::Plan p;
    if (!rt_plan(L, (int)sizeof(float2), &p)) return false;
    const int LS = tgrt::pitch(p);
    // the heaviest per-line use: corr_y's F_I column, c2r's running maximum
    return lines_per_block(LS, (size_t)L * sizeof(float2), tgrt::kMaxBlockSmem, 1) > 0;
}

cudaError_t launch_spec_x_rt(int NX, const float* t2, const float* mask, float2* A, const int T[3], int d0x, int nb,
                             double* tsum, cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NX, &r)) return cudaErrorInvalidValue;
    const int nlines = T[1] * T[2];
    const int NL = std::min(lines_per_block(r.LS, 0, 48 * 1024, 16), std::max(nlines, 1));
    if (NL <= 0) return cudaErrorInvalidValue;
    const size_t smem = 2 * (size_t)NL * r.LS * sizeof(float2);
    if (cudaError_t e = allow_smem(k_spec_x_rt, smem)) return e;
    dim3 g((nlines + NL - 1) / NL, nb);
    k_spec_x_rt<<<g, NT, smem, st>>>(t2, mask, A, T[0], T[1], T[2], d0x, r.p, r.t, NL, r.LS, tsum);
    return cudaGetLastError();
}

cudaError_t launch_spec_z_rt(int NZ, const float2* A, float2* Z, const int T[3], int d0z, int nh1, int nb,
                             cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NZ, &r)) return cudaErrorInvalidValue;
    const int NL = std::min(lines_per_block(r.LS, 0, 48 * 1024, 8), std::max(T[1], 1));
    if (NL <= 0) return cudaErrorInvalidValue;
    const size_t smem = 2 * (size_t)NL * r.LS * sizeof(float2);
    if (cudaError_t e = allow_smem(k_spec_z_rt, smem)) return e;
    dim3 g((T[1] + NL - 1) / NL, nh1, nb);
    k_spec_z_rt<<<g, NT, smem, st>>>(A, Z, T[1], T[2], d0z, nh1, r.p, r.t, NL, r.LS);
    return cudaGetLastError();
}

cudaError_t launch_corr_y_rt(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                             long long ncols, int nb, cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NY, &r)) return cudaErrorInvalidValue;
    const size_t extra = (size_t)NY * sizeof(float2);
    int NL = lines_per_block(r.LS, extra, 48 * 1024, 16);
    if (NL <= 0) return cudaErrorInvalidValue;
    NL = (int)std::min<long long>(NL, std::max<long long>(ncols, 1));
    const size_t smem = (2 * (size_t)r.LS * sizeof(float2) + extra) * NL;
    if (cudaError_t e = allow_smem(k_corr_y_rt, smem)) return e;
    k_corr_y_rt<<<(unsigned)((ncols + NL - 1) / NL), NT, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, r.p, r.t, NL,
                                                                       r.LS);
    return cudaGetLastError();
}

cudaError_t launch_inv_z_rt(int NZ, const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NZ, &r)) return cudaErrorInvalidValue;
    const int NL = std::min(lines_per_block(r.LS, 0, 64 * 1024, 16), std::max(Ny, 1));
    if (NL <= 0) return cudaErrorInvalidValue;
    const size_t smem = 2 * (size_t)NL * r.LS * sizeof(float2);
    if (cudaError_t e = allow_smem(k_inv_z_rt, smem)) return e;
    dim3 g((Ny + NL - 1) / NL, nh1, nb);
    k_inv_z_rt<<<g, NT, smem, st>>>(Q, H, Ny, nh1, r.p, r.t, NL, r.LS);
    return cudaGetLastError();
}

cudaError_t launch_c2r_flcf_rt(int NX, const float2* H, const float* mu0, const float* gam, const double* tsum,
                               int Ny, int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                               float* maxcc, int* angidx, cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NX, &r)) return cudaErrorInvalidValue;
    const size_t extra = (size_t)NX * (sizeof(float) + sizeof(int));
    const int NL = std::min(lines_per_block(r.LS, extra, 64 * 1024, 8), std::max(Ny, 1));
    if (NL <= 0) return cudaErrorInvalidValue;
    const size_t smem = (2 * (size_t)r.LS * sizeof(float2) + extra) * NL;
    if (cudaError_t e = allow_smem(k_c2r_flcf_rt, smem)) return e;
    dim3 g((Ny + NL - 1) / NL, Nz);
    k_c2r_flcf_rt<<<g, NT, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx,
                                       r.p, r.t, NL, r.LS);
    return cudaGetLastError();
}

cudaError_t launch_c2r_map_rt(int NX, const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                              int Nz, float inv_nm, double c, double inv_m, double mu_t, float* cc, cudaStream_t st) {
    RtLines r;
    if (!rt_lines(NX, &r)) return cudaErrorInvalidValue;
    const int NL = std::min(lines_per_block(r.LS, 0, 48 * 1024, 8), std::max(Ny, 1));
    if (NL <= 0) return cudaErrorInvalidValue;
    const size_t smem = 2 * (size_t)NL * r.LS * sizeof(float2);
    if (cudaError_t e = allow_smem(k_c2r_map_rt, smem)) return e;
    dim3 g((Ny + NL - 1) / NL, Nz);
    k_c2r_map_rt<<<g, NT, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, inv_nm, c, inv_m, mu_t, cc, r.p, r.t, NL, r.LS);
    return cudaGetLastError();
}

}  // namespace tg
