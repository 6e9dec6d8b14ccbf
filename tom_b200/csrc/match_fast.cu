// Register-resident variants of the three hot FLCF kernels for the common
// power-of-two sizes (y edge 256/512, z edge 256, x edge 256/512).  Same
// arithmetic contract as the generic kernels in match.cu; faster data flow:
//
//   corr_y_w  one warp per spectrum column; the y-DFT of the template, the
//             product with F_I (staged once in shared memory) and the inverse
//             y-DFT all stay in registers with two warp-private exchanges per
//             transform (warp_fft.cuh); the next rotation's template values
//             are fetched while the current one is transformed.
//   inv_z_b   16 consecutive y lines per block, 16 threads per line holding
//             16 values: radix 16 straight from global memory, one block-wide
//             exchange, radix 16 straight back to global memory.
//   c2r_w     one warp per x line, the next three rotations' tiles in flight
//             (cp.async) while the current one is transformed; running max and
//             the FLCF coefficients of the lane's voxels stay in registers.
#include "ctx.h"
#include "match.h"
#include "twiddles.h"
#include "warp_fft.cuh"

namespace tg {

template <int NY>
__global__ void __launch_bounds__(256, 2) k_corr_y_w(const float2* __restrict__ fimg, const float2* __restrict__ Z,
                                                     float2* __restrict__ Q, int Ty, int d0y, long long ncols, int nb,
                                                     const float2* __restrict__ tw_g) {
    constexpr int EPT = NY / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tw = reinterpret_cast<float2*>(smem_raw);  // [NY] stage tables
    float2* xb = tw + NY + 64;                          // [8][NY] exchange
    float2* fs = xb + 8 * NY;                           // [8][NY] F_I columns
    float2* zs = fs + 8 * NY;                           // [8][2][64] template column, double buffered
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long col = (long long)blockIdx.x * 8 + warp;
    static_assert(tgwfft::WTab<NY>::size <= NY + 64, "stage tables exceed their slot");
    tgwfft::build_stage_tables<NY>(tw, tw_g);
    float2* buf = xb + warp * NY;
    float2* fw = fs + warp * NY;
    float2* zw = zs + warp * 128;
    if (col < ncols) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int p = tgwfft::out_pos<NY>(i, lane);
            fw[p] = fimg[col * NY + p];  // each lane later reads only its own entries
        }
        const float2* zc = Z + col * Ty;  // rotation 0
        if (lane < Ty) zw[lane] = zc[lane];
        if (lane + 32 < Ty) zw[lane + 32] = zc[lane + 32];
    }
    __syncthreads();  // the table; the only block-wide barrier
    if (col >= ncols) return;
    for (int b = 0; b < nb; ++b) {
        // next rotation's column: two loads per lane, parked in registers
        float2 n0 = make_float2(0.f, 0.f), n1 = make_float2(0.f, 0.f);
        if (b + 1 < nb) {
            const float2* zc = Z + ((long long)(b + 1) * ncols + col) * Ty;
            if (lane < Ty) n0 = zc[lane];
            if (lane + 32 < Ty) n1 = zc[lane + 32];
        }
        const float2* cur = zw + (b & 1) * 64;
        float2 v[EPT];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int jy = (tgwfft::in_pos<NY>(i, lane) - d0y) & (NY - 1);
            v[i] = jy < Ty ? cur[jy] : make_float2(0.f, 0.f);
        }
        tgwfft::warp_fft<NY, -1>(v, buf, tw, lane);
#pragma unroll
        for (int i = 0; i < EPT; ++i) v[i] = cmulc(fw[tgwfft::out_pos<NY>(i, lane)], v[i]);
        tgwfft::warp_fft<NY, +1>(v, buf, tw, lane);
        float2* qc = Q + ((long long)b * ncols + col) * NY;
#pragma unroll
        for (int i = 0; i < EPT; ++i) qc[tgwfft::out_pos<NY>(i, lane)] = v[i];
        float2* nx = zw + ((b + 1) & 1) * 64;
        if (lane < Ty) nx[lane] = n0;
        if (lane + 32 < Ty) nx[lane + 32] = n1;
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) k_inv_z_b256(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                                    int nh1, const float2* __restrict__ tw_g) {
    constexpr int NZ = 256, LS = NZ + 1;
    __shared__ __align__(16) float2 s[16 * LS];
    __shared__ __align__(16) float2 tw[NZ];
    tgwfft::stage_table(tw, tw_g, NZ);
    const int tid = threadIdx.x, l = tid & 15, j = tid >> 4;
    const int y = blockIdx.x * 16 + l, kx = blockIdx.y, b = blockIdx.z;
    const bool ok = y < Ny;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = ok ? Q[base + (long long)(j + 16 * r) * Ny + y] : make_float2(0.f, 0.f);
    tgfft::dft16<+1>(v);
#pragma unroll
    for (int r = 0; r < 16; ++r) s[l * LS + 16 * j + r] = v[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = s[l * LS + j + 16 * r];
    float2 w[16];
    tgwfft::twiddle_powers<16, +1>(tw, j, w);
#pragma unroll
    for (int r = 1; r < 16; ++r) v[r] = cmul(v[r], w[r]);
    tgfft::dft16<+1>(v);
    if (ok) {
#pragma unroll
        for (int r = 0; r < 16; ++r) H[base + (long long)(j + 16 * r) * Ny + y] = v[r];
    }
}

constexpr int C2R_STAGES = 2;

TG_D void cp_async8(void* smem_dst, const void* gsrc, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
TG_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> TG_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Running maximum without per-voxel coefficients: with gamma >= 0 and
// mu0 mu_T fixed per voxel, cc_b = (u_b - mu0 mu_T) gamma is a non-decreasing
// function of u_b = out_b/(N M) + kappa_b, so the batch keeps the best u and
// its rotation and applies the FLCF formula once, at the read-modify-write.
// (Rotations whose cc round to the same float but whose u differ may pick a
// later index than the strict first-wins scan; such voxels have no CC
// separation between those angles.  gamma = 0 voxels keep the reference's
// value 0 with the batch's first rotation.)
template <int NH>
__global__ void __launch_bounds__(256, 4) k_c2r_w(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                  const float* __restrict__ gam, const double* __restrict__ tsum,
                                                  int Ny, int Nz, int nb, float inv_nm, double c_mean, double inv_m,
                                                  double mu_t, int index0, float* __restrict__ maxcc,
                                                  int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                  const float2* __restrict__ tw_x) {
    constexpr int YT = 8, NH1 = NH + 1, TS = NH + 2, EPT = NH / 32, NX = 2 * NH, NSTG = C2R_STAGES;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);  // [NSTG][YT][TS]
    float2* xbuf = tile + NSTG * YT * TS;                 // [8][NH]
    float2* twh = xbuf + 8 * NH;                          // [NH + 64] stage tables
    float2* twx = twh + NH + 64;                          // [NX]
    float* kaps = reinterpret_cast<float*>(twx + NX);    // [nb]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = blockIdx.x * YT, z = blockIdx.y, y = y0 + warp;
    const bool yok = y < Ny;
    const long long nh1l = NH1;
    float bu[EPT][2];
    unsigned bb[EPT];  // best rotation of the voxel pair, 16 bits each (nb <= 65535)
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
        bu[i][0] = bu[i][1] = -INFINITY;
        bb[i] = 0u;
    }
    static_assert(tgwfft::WTab<NH>::size <= NH + 64, "stage tables exceed their slot");
    tgwfft::build_stage_tables<NH>(twh, tw_h);
    tgwfft::stage_table(twx, tw_x, NX);
    for (int b = threadIdx.x; b < nb; b += blockDim.x) kaps[b] = (float)(c_mean * (tsum[b] * inv_m - mu_t));
    auto issue = [&](int b, int which) {
        float2* t = tile + which * YT * TS;
        const long long hb = (long long)b * nh1l * Nz * Ny;
        for (int e = tid; e < YT * NH1; e += 256) {
            const int kx = e / YT, yl = e - kx * YT;
            const bool ok = y0 + yl < Ny;
            const float2* src = H + hb + ((long long)kx * Nz + z) * Ny + (ok ? y0 + yl : 0);
            cp_async8(t + yl * TS + kx, src, ok ? 8 : 0);
        }
        cp_async_commit();
    };
    // NSTG-deep pipeline: tiles b+1 .. b+NSTG-1 are in flight while b is
    // transformed; every iteration commits one group (possibly empty) so that
    // "all but the newest NSTG-1 groups complete" means tile b has landed.
#pragma unroll
    for (int s = 0; s < NSTG - 1; ++s) {
        if (s < nb) issue(s, s);
        else cp_async_commit();
    }
    for (int b = 0; b < nb; ++b) {
        if (b + NSTG - 1 < nb) issue(b + NSTG - 1, (b + NSTG - 1) % NSTG);
        else cp_async_commit();
        cp_async_wait<NSTG - 1>();
        __syncthreads();
        const float2* X = tile + (b % NSTG) * YT * TS + warp * TS;
        float2 v[EPT];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            // unpack: Z[k] = (X[k] + X*[NH-k]) + i w^k (X[k] - X*[NH-k]), w = exp(+2 pi i / NX)
            const int k = tgwfft::in_pos<NH>(i, lane);
            const float2 xa = X[k], xb = cconj(X[NH - k]);
            const float2 w = cconj(twx[k]);
            const float2 d = cmul(w, csub(xa, xb));
            v[i] = cadd(cadd(xa, xb), make_float2(-d.y, d.x));
        }
        tgwfft::warp_fft<NH, +1>(v, xbuf + warp * NH, twh, lane);
        const float kap = kaps[b];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const float u0 = fmaf(v[i].x, inv_nm, kap);
            const float u1 = fmaf(v[i].y, inv_nm, kap);
            if (u0 > bu[i][0]) { bu[i][0] = u0; bb[i] = (bb[i] & 0xFFFF0000u) | (unsigned)b; }
            if (u1 > bu[i][1]) { bu[i][1] = u1; bb[i] = (bb[i] & 0x0000FFFFu) | ((unsigned)b << 16); }
        }
        __syncthreads();
    }
    if (!yok) return;
    const float mt = (float)mu_t;
    // every load of the read-modify-write first, then the stores (the loads
    // would otherwise wait behind stores the compiler cannot disambiguate)
    float2 av[EPT], gv[EPT], cv[EPT];
    int2 iv[EPT];
    const long long row = ((long long)z * Ny + y) * NX;
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
        const long long v = row + 2 * tgwfft::out_pos<NH>(i, lane);
        av[i] = __ldg(reinterpret_cast<const float2*>(mu0 + v));
        gv[i] = __ldg(reinterpret_cast<const float2*>(gam + v));
        cv[i] = *reinterpret_cast<const float2*>(maxcc + v);
        iv[i] = *reinterpret_cast<const int2*>(angidx + v);
    }
#pragma unroll
    for (int i = 0; i < EPT; ++i) {
        const long long v = row + 2 * tgwfft::out_pos<NH>(i, lane);
        const float2 a = av[i], g = gv[i];
        float2 cur = cv[i];
        int2 ci = iv[i];
        bool ch = false;
        const float c0 = g.x != 0.f ? (bu[i][0] - a.x * mt) * g.x : 0.f;
        const float c1 = g.y != 0.f ? (bu[i][1] - a.y * mt) * g.y : 0.f;
        const int b0 = g.x != 0.f ? (int)(bb[i] & 0xFFFFu) : 0, b1 = g.y != 0.f ? (int)(bb[i] >> 16) : 0;
        if (c0 > cur.x) { cur.x = c0; ci.x = index0 + b0; ch = true; }
        if (c1 > cur.y) { cur.y = c1; ci.y = index0 + b1; ch = true; }
        if (ch) {
            *reinterpret_cast<float2*>(maxcc + v) = cur;
            *reinterpret_cast<int2*>(angidx + v) = ci;
        }
    }
}

// ------------------------------------------------------------- dispatch

bool fast_corr_y(int NY, int Ty) { return (NY == 128 || NY == 256 || NY == 512 || NY == 928) && Ty <= 64; }
bool fast_inv_z(int NZ) { return NZ == 128 || NZ == 256 || NZ == 464; }
bool fast_c2r(int NH) { return NH == 64 || NH == 128 || NH == 256 || NH == 464; }

cudaError_t launch_corr_y_fast(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                               long long ncols, int nb, cudaStream_t st) {
    if (NY == 928) return launch_corr_y_p928(fimg, Z, Q, Ty, d0y, ncols, nb, st);
    const unsigned g = (unsigned)((ncols + 7) / 8);
    const size_t smem = sizeof(float2) * (NY * 17 + 64 + 8 * 128);
    if (NY == 512) {
        cudaFuncSetAttribute(k_corr_y_w<512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_corr_y_w<512><<<g, 256, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, twiddle_table<float2>(512));
    } else if (NY == 256) {
        cudaFuncSetAttribute(k_corr_y_w<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_corr_y_w<256><<<g, 256, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, twiddle_table<float2>(256));
    } else if (NY == 128) {
        cudaFuncSetAttribute(k_corr_y_w<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_corr_y_w<128><<<g, 256, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, twiddle_table<float2>(128));
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_inv_z_fast(int NZ, const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st) {
    if (NZ == 464) return launch_inv_z_p464(Q, H, Ny, nh1, nb, st);
    if (NZ == 128) return launch_inv_z_b128(Q, H, Ny, nh1, nb, st);
    if (NZ != 256) return cudaErrorInvalidValue;
    dim3 g((Ny + 15) / 16, nh1, nb);
    k_inv_z_b256<<<g, 256, 0, st>>>(Q, H, Ny, nh1, twiddle_table<float2>(256));
    return cudaGetLastError();
}

template <int NH>
static cudaError_t launch_c2r_t(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                                int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                                float* maxcc, int* angidx, cudaStream_t st) {
    constexpr int YT = 8, TS = NH + 2;
    const size_t smem = sizeof(float2) * (C2R_STAGES * YT * TS + 8 * NH + 3 * NH + 64) + sizeof(float) * nb;
    cudaFuncSetAttribute(k_c2r_w<NH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 g((Ny + YT - 1) / YT, Nz);
    k_c2r_w<NH><<<g, 256, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx,
                                      twiddle_table<float2>(NH), twiddle_table<float2>(2 * NH));
    return cudaGetLastError();
}

cudaError_t launch_c2r_fast(int NH, const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                            int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                            float* maxcc, int* angidx, cudaStream_t st) {
    // x edge 512: the half-warp kernel (k_c2r_h256 measured 20 % faster than the
    // warp-per-line k_c2r_w<256> on the 512x512x256 search)
    if (NH == 256)
        return launch_c2r_h256(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
    if (NH == 128)
        return launch_c2r_b128(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
    if (NH == 64)
        return launch_c2r_b64(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
    if (NH == 464)
        return launch_c2r_p464(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc, angidx, st);
    return cudaErrorInvalidValue;
}

}  // namespace tg
