// Register-resident FLCF kernels for the 928 / 464 edges (the 928x928x464
// tomogram): y edge 928 = 29 x 32, z edge 464 = 29 x 16, x edge 928 (complex
// half length 464).  Same arithmetic contract as the generic kernels in
// match.cu, two-factor Cooley-Tukey instead of the generic engine's three
// shared-memory passes:
//
//   corr_y_p928  one warp per spectrum column: each lane a 29-point DFT of
//                the samples q + 32 m (in registers), the 928-point twiddle,
//                one warp-private exchange, 29 lanes a 32-point DFT; the
//                product with F_I (staged once per column); the inverse the
//                same way back.  The y samples and the output stay in natural
//                order, so the global accesses of a lane group are contiguous.
//   inv_z_p464   16 y lines x 16 threads per block: 29 16-point DFTs per line
//                straight from global memory, one block exchange, 16 29-point
//                DFTs per line straight back to global memory.
//   c2r_p464     8 x lines per block, 16 threads per line: the half-spectrum
//                unpack, 29 16-point DFTs, a half-warp exchange, 16 29-point
//                DFTs, the running maximum over the batch in registers and the
//                FLCF at the read-modify-write (as c2r_b8).
//
// Index map (inverse; the forward is the conjugate): with n = q + Q m and
// k = k1 + 29 k2,  y(n) = sum_k1 W29^(m k1) WL^(q k1) sum_k2 Y(k) WQ^(q k2).
#include "ctx.h"
#include "match.h"
#include "pq29.cuh"
#include "tile_copy.cuh"
#include "tma_util.cuh"
#include "tmem_util.cuh"
#include "twiddles.h"
#include "warp_fft.cuh"

namespace tg {

namespace {

tgpq::Cos29 cos29_table() {
    tgpq::Cos29 t;
    for (int j = 0; j < 29; ++j) {
        const double a = 2.0 * M_PI * (double)j / 29.0;
        t.c[j] = (float)std::cos(a);
        t.s[j] = (float)std::sin(a);
    }
    return t;
}

constexpr int CY_WARPS = 4, CY_RS = 33;

__global__ void __launch_bounds__(32 * CY_WARPS) k_corr_y_p928(const float2* __restrict__ fimg,
                                                               const float2* __restrict__ Z, float2* __restrict__ Q,
                                                               int Ty, int d0y, long long ncols, int nb,
                                                               const float2* __restrict__ tw_g, tgpq::Cos29 cs) {
    constexpr int NY = 928, P = 29, RS = CY_RS, WS = 2 * P * RS + 128;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* T = reinterpret_cast<float2*>(smem_raw);  // [29][RS]: W928^(-q k1)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2* xb = T + P * RS + warp * WS;  // [29][RS] exchange
    float2* fs = xb + P * RS;         // [29][RS] F_I at k1 + 29 k2
    float2* zs = fs + P * RS;         // [2][64] template column
    float2* w29 = T + P * RS + CY_WARPS * WS;  // [29]: exp(-2 pi i j / 29)
    for (int i = threadIdx.x; i < NY; i += blockDim.x) {
        const int k1 = i >> 5, q = i & 31;
        T[k1 * RS + q] = __ldg(tw_g + (q * k1) % NY);
    }
    if (threadIdx.x < P) w29[threadIdx.x] = make_float2(cs.c[threadIdx.x], -cs.s[threadIdx.x]);
    const long long col = (long long)blockIdx.x * CY_WARPS + warp;
    if (col < ncols) {
        for (int e = lane; e < NY; e += 32) {
            const int k2 = e / P, k1 = e - k2 * P;
            fs[k1 * RS + k2] = fimg[col * NY + e];
        }
        const float2* zc = Z + col * Ty;
        if (lane < Ty) zs[lane] = zc[lane];
        if (lane + 32 < Ty) zs[lane + 32] = zc[lane + 32];
    }
    __syncthreads();
    if (col >= ncols) return;
    for (int b = 0; b < nb; ++b) {
        float2 n0 = make_float2(0.f, 0.f), n1 = make_float2(0.f, 0.f);
        if (b + 1 < nb) {
            const float2* zc = Z + ((long long)(b + 1) * ncols + col) * Ty;
            if (lane < Ty) n0 = zc[lane];
            if (lane + 32 < Ty) n1 = zc[lane + 32];
        }
        const float2* cur = zs + (b & 1) * 64;
        {
            // the template column covers Ty <= 64 consecutive y (from d0y, cyclic), so a
            // lane's samples q + 32 m hold at most two nonzeros: the 29-point DFT of the
            // lane is two scaled columns of the DFT matrix
            const int o = (lane - d0y) & 31;  // first window offset with y = lane (mod 32)
            const float2 a0 = o < Ty ? cur[o] : make_float2(0.f, 0.f);
            const float2 a1 = o + 32 < Ty ? cur[o + 32] : make_float2(0.f, 0.f);
            const int m0 = ((d0y + o) % NY - lane) >> 5;
            const int m1 = m0 == P - 1 ? 0 : m0 + 1;
            int j0 = 0, j1 = 0;
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) {
                const float2 x = cadd(cmul(a0, w29[j0]), cmul(a1, w29[j1]));
                xb[k1 * RS + lane] = cmul(x, T[k1 * RS + lane]);
                j0 += m0;
                j0 -= j0 >= P ? P : 0;
                j1 += m1;
                j1 -= j1 >= P ? P : 0;
            }
        }
        __syncwarp();
        if (lane < P) {
            float2 u[32];
#pragma unroll
            for (int q = 0; q < 32; ++q) u[q] = xb[lane * RS + q];
            tgfft::dft32<-1>(u);
#pragma unroll
            for (int k2 = 0; k2 < 32; ++k2) u[k2] = cmulc(fs[lane * RS + k2], u[k2]);
            tgfft::dft32<+1>(u);
#pragma unroll
            for (int q = 0; q < 32; ++q) xb[lane * RS + q] = cmulc(u[q], T[lane * RS + q]);
        }
        __syncwarp();
        {
            float2 v[P];
#pragma unroll
            for (int k1 = 0; k1 < P; ++k1) v[k1] = xb[k1 * RS + lane];
            float2* qc = Q + ((long long)b * ncols + col) * NY;
            tgpq::dft29_emit<+1>(v, cs, [&](int m, float2 x) { qc[lane + 32 * m] = x; });
        }
        float2* nx = zs + ((b + 1) & 1) * 64;
        if (lane < Ty) nx[lane] = n0;
        if (lane + 32 < Ty) nx[lane + 32] = n1;
        __syncwarp();
    }
}

constexpr int IZ_LS = 465;

__global__ void __launch_bounds__(256, 3) k_inv_z_p464(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                                    int nh1, const float2* __restrict__ tw_g, tgpq::Cos29 cs) {
    constexpr int NZ = 464, P = 29, LS = IZ_LS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);  // [16][LS]
    float2* T = s + 16 * LS;                           // [29][16]: W464^(+q k1)
    for (int i = threadIdx.x; i < P * 16; i += blockDim.x) {
        const int k1 = i >> 4, q = i & 15;
        T[i] = cconj(__ldg(tw_g + (q * k1) % NZ));
    }
    const int tid = threadIdx.x, l = tid & 15, j = tid >> 4;
    const int y = blockIdx.x * 16 + l, kx = blockIdx.y, b = blockIdx.z;
    const bool ok = y < Ny;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    __syncthreads();
#pragma unroll 1
    for (int k1 = j; k1 < P; k1 += 16) {
        float2 u[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2)
            u[k2] = ok ? Q[base + (long long)(k1 + P * k2) * Ny + y] : make_float2(0.f, 0.f);
        tgfft::dft16<+1>(u);
#pragma unroll
        for (int q = 0; q < 16; ++q) s[l * LS + k1 * 16 + q] = cmul(u[q], T[k1 * 16 + q]);
    }
    __syncthreads();
    float2 v[P];
#pragma unroll
    for (int k1 = 0; k1 < P; ++k1) v[k1] = s[l * LS + k1 * 16 + j];
    float2* hl = H + base + (long long)j * Ny + y;
    tgpq::dft29_emit<+1>(v, cs, [&](int m, float2 x) {
        if (ok) hl[(long long)(16 * m) * Ny] = x;
    });
}

constexpr int C2_YT = 8, C2_TS = 466, C2_XR = 17, C2_XL = 29 * C2_XR;

// The running maximum keeps u = out/(N M) + kappa_b and the batch index of
// the best rotation per voxel (as k_c2r_b8); the FLCF is applied at the
// read-modify-write.
__global__ void __launch_bounds__(16 * C2_YT, 3) k_c2r_p464(const float2* __restrict__ H, const float* __restrict__ mu0,
                                                             const float* __restrict__ gam,
                                                             const double* __restrict__ tsum, int Ny, int Nz, int nb,
                                                             float inv_nm, double c_mean, double inv_m, double mu_t,
                                                             int index0, float* __restrict__ maxcc,
                                                             int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                             const float2* __restrict__ tw_x, tgpq::Cos29 cs) {
    constexpr int NH = 464, NH1 = NH + 1, NX = 2 * NH, P = 29, YT = C2_YT, TS = C2_TS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);  // [2][YT][TS]
    float2* xb = tile + 2 * YT * TS;                      // [YT][29][17] exchange
    float2* T = xb + YT * C2_XL;                          // [16][32]: W464^(+q k1) at [q][k1]
    float2* twx = T + 16 * 32;                            // [NH]: W928^(+k)
    float* kaps = reinterpret_cast<float*>(twx + NH);     // [nb]
    const int tid = threadIdx.x, line = tid >> 4, q = tid & 15;
    const int y0 = blockIdx.x * YT, z = blockIdx.y, y = y0 + line;
    for (int i = tid; i < P * 16; i += blockDim.x) {
        const int k1 = i >> 4, qq = i & 15;
        T[qq * 32 + k1] = cconj(__ldg(tw_h + (qq * k1) % NH));
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
    auto issue = [&](int b, int which) {
        float2* t = tile + which * YT * TS;
        const long long hb = (long long)b * NH1 * Nz * Ny;
        for (int e = tid; e < YT * NH1; e += blockDim.x) {
            const int kx = e / YT, yl = e - kx * YT;
            const bool okl = y0 + yl < Ny;
            const float2* src = H + hb + ((long long)kx * Nz + z) * Ny + (okl ? y0 + yl : 0);
            tgtile::cp_async8((unsigned)__cvta_generic_to_shared(t + yl * TS + kx), src, okl ? 8 : 0);
        }
        tgtile::commit();
    };
    issue(0, 0);
    float2* xl = xb + line * C2_XL;
    for (int b = 0; b < nb; ++b) {
        if (b + 1 < nb) issue(b + 1, (b + 1) & 1);
        else tgtile::commit();
        tgtile::wait<1>();
        __syncthreads();
        const float2* X = tile + (b & 1) * YT * TS + line * TS;
        // unpack and the inner 16-point DFTs: k = k1 + 29 k2
#pragma unroll 1
        for (int k1 = q; k1 < P; k1 += 16) {
            float2 u[16];
#pragma unroll
            for (int k2 = 0; k2 < 16; ++k2) {
                const int k = k1 + P * k2;
                const float2 xa = X[k], xc = cconj(X[NH - k]);
                const float2 d = cmul(twx[k], csub(xa, xc));
                u[k2] = cadd(cadd(xa, xc), make_float2(-d.y, d.x));
            }
            tgfft::dft16<+1>(u);
#pragma unroll
            for (int qq = 0; qq < 16; ++qq) xl[k1 * C2_XR + qq] = cmul(u[qq], T[qq * 32 + k1]);
        }
        __syncwarp();
        float2 v[P];
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[k1] = xl[k1 * C2_XR + q];
        const float kap = kaps[b];
        tgpq::dft29_emit<+1>(v, cs, [&](int m, float2 x) {
            const float u0 = fmaf(x.x, inv_nm, kap);
            const float u1 = fmaf(x.y, inv_nm, kap);
            if (u0 > bu[m][0]) { bu[m][0] = u0; bb[m] = (bb[m] & 0xFFFF0000u) | (unsigned)b; }
            if (u1 > bu[m][1]) { bu[m][1] = u1; bb[m] = (bb[m] & 0x0000FFFFu) | ((unsigned)b << 16); }
        });
        __syncthreads();  // the tile and the exchange are rewritten next
    }
    if (y >= Ny) return;
    const float mt = (float)mu_t;
    const long long row = ((long long)z * Ny + y) * NX;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const long long v = row + 2 * (q + 16 * m);
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

// k_c2r_p464 with its tiles loaded by the Tensor Memory Accelerator: one
// thread issues two tiled loads per rotation (boxes 8 y x 1 z x 256 kx and
// 8 y x 1 z x 209 kx over H viewed as floats, 64-byte rows with the 64-byte
// swizzle: chunk c of row k at chunk c ^ ((k >> 1) mod 4)) completing on a
// per-stage mbarrier, instead of ~29 eight-byte cp.async per thread.  Two
// stages; waits bounded (a stage that never fills sets the device error word
// and the block returns without touching the results).  1-GPU code: the maps
// cover this GPU's own H, no load multicasts.  A thread's unpack twiddles and
// exchange twiddles (for its k1 = q and q + 16) sit in its TMEM lane and are
// read with tcgen05.ld instead of from shared memory.
constexpr int T4_STAGE = 30720;              // 465 rows x 64 bytes, rounded up to 1 KB
constexpr unsigned T4_TX = 465u * 64u;
constexpr long long T4_WAIT_LIMIT = 1ll << 20;

__global__ void __launch_bounds__(16 * C2_YT, 2) k_c2r_t464(const __grid_constant__ CUtensorMap tm_a,
                                                            const __grid_constant__ CUtensorMap tm_b,
                                                            const float* __restrict__ mu0,
                                                            const float* __restrict__ gam,
                                                            const double* __restrict__ tsum, int Ny, int Nz, int nb,
                                                            float inv_nm, double c_mean, double inv_m, double mu_t,
                                                            int index0, float* __restrict__ maxcc,
                                                            int* __restrict__ angidx, const float2* __restrict__ tw_h,
                                                            const float2* __restrict__ tw_x, tgpq::Cos29 cs,
                                                            int* __restrict__ err) {
    constexpr int NH = 464, NX = 2 * NH, P = 29, YT = C2_YT;
    // once a block of this launch has timed out, the rest return at once (one
    // read, shared, so the whole block decides alike)
    __shared__ int skip_block;
    if (threadIdx.x == 0) skip_block = err && *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (skip_block) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((1024u - (tgtma::smem_u32(smem_raw) & 1023u)) & 1023u);
    float2* xb = reinterpret_cast<float2*>(base + 2 * T4_STAGE);  // [YT][29][17] exchange
    float2* T = xb + YT * C2_XL;                                     // [16][32]: W464^(+q k1) at [q][k1]
    float2* twx = T + 16 * 32;                                       // [NH]: W928^(+k)
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(twx + NH);
    int* flag = reinterpret_cast<int*>(bars + 2);
    float* kaps = reinterpret_cast<float*>(flag + 2);  // [nb]
    const int tid = threadIdx.x, line = tid >> 4, q = tid & 15;
    const int y0 = blockIdx.x * YT, z = blockIdx.y, y = y0 + line;
    for (int i = tid; i < P * 16; i += blockDim.x) {
        const int k1 = i >> 4, qq = i & 15;
        T[qq * 32 + k1] = cconj(__ldg(tw_h + (qq * k1) % NH));
    }
    for (int i = tid; i < NH; i += blockDim.x) twx[i] = cconj(__ldg(tw_x + i));
    for (int b = tid; b < nb; b += blockDim.x) kaps[b] = (float)(c_mean * (tsum[b] * inv_m - mu_t));
    unsigned* tmem_slot = reinterpret_cast<unsigned*>(flag + 1);
    const int warp = tid >> 5;
    if (warp == 0) tgtm::alloc<128>(tmem_slot);
    if (tid == 0) {
        tgtma::mbar_init(tgtma::smem_u32(bars), 1);
        tgtma::mbar_init(tgtma::smem_u32(bars + 1), 1);
        *flag = 0;
        tgtma::fence_barrier_init();
        tgtma::prefetch_map(&tm_a);
        tgtma::prefetch_map(&tm_b);
    }
    tgtm::fence_before();
    __syncthreads();
    tgtm::fence_after();
    // this thread's constants into its TMEM lane (warp w: lanes 32 w): for
    // it = 0, 1 (k1 = q + 16 it) columns 64 it + [0, 32) the unpack twiddles
    // of k = k1 + 29 k2 and 64 it + [32, 64) the exchange twiddles T[qq][k1]
    // (zeros where k1 >= 29)
    const unsigned taddr = tgtm::lane_addr(*tmem_slot, warp, 0u);
    {
        float t[16];
#pragma unroll
        for (int it = 0; it < 2; ++it) {
            const int k1 = q + 16 * it;
#pragma unroll
            for (int h = 0; h < 4; ++h) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int c = 8 * (h & 1) + i;
                    float2 w = make_float2(0.f, 0.f);
                    if (k1 < P) w = h < 2 ? twx[k1 + P * c] : T[c * 32 + k1];
                    t[2 * i] = w.x;
                    t[2 * i + 1] = w.y;
                }
                tgtm::st16(taddr + 64u * (unsigned)it + 16u * (unsigned)h, t);
            }
        }
        tgtm::wait_st();
    }
    const unsigned sbase = tgtma::smem_u32(base);
    auto issue = [&](int b, int s) {
        if (tid == 0) {
            const unsigned bar = tgtma::smem_u32(bars + s), dst = sbase + (unsigned)(s * T4_STAGE);
            tgtma::mbar_expect_tx(bar, T4_TX);
            tgtma::load_4d(dst, &tm_a, 2 * y0, z, 0, b, bar);
            tgtma::load_4d(dst + 256u * 64u, &tm_b, 2 * y0, z, 256, b, bar);
        }
    };
    float bu[P][2];
    unsigned bb[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        bu[m][0] = bu[m][1] = -INFINITY;
        bb[m] = 0u;
    }
    issue(0, 0);
    float2* xl = xb + line * C2_XL;
    const int cy = line >> 1, hy = (line & 1) << 3;  // chunk and half of this line's y in a 64-byte row
    for (int b = 0; b < nb; ++b) {
        if (b + 1 < nb) issue(b + 1, (b + 1) & 1);
        const int cur = b & 1;
        const unsigned bar = tgtma::smem_u32(bars + cur), parity = (unsigned)((b >> 1) & 1);
        if (tid == 0 && !tgtma::mbar_wait_bounded(bar, parity, T4_WAIT_LIMIT)) *flag = 1;
        __syncthreads();
        if (*flag) {
            if (tid == 0) {
                tg_flag_error(err, TG_DEV_TIMEOUT);
                if (b + 1 < nb) tgtma::mbar_wait_bounded(tgtma::smem_u32(bars + ((b + 1) & 1)),
                                                         (unsigned)(((b + 1) >> 1) & 1), T4_WAIT_LIMIT);
            }
            break;
        }
        (void)tgtma::mbar_test_wait(bar, parity);
        const unsigned char* st = base + cur * T4_STAGE;
        // unpack and the inner 16-point DFTs: k = k1 + 29 k2, k1 = q + 16 it;
        // every lane takes part in the TMEM loads (warp-collective), the
        // lanes with k1 >= 29 skip the arithmetic
#pragma unroll 1
        for (int it = 0; it < 2; ++it) {
            const int k1 = q + 16 * it;
            const bool ok = k1 < P;
            float2 u[16];
            float tk[16];
#pragma unroll
            for (int k2 = 0; k2 < 16; ++k2) {
                if ((k2 & 7) == 0) {
                    __syncwarp();
                    tgtm::ld16(taddr + 64u * (unsigned)it + 2u * (unsigned)k2, tk);
                }
                const int k = ok ? k1 + P * k2 : 0, kr = NH - k;
                const float2 xa = *reinterpret_cast<const float2*>(st + k * 64 + ((cy ^ ((k >> 1) & 3)) << 4) + hy);
                const float2 xc =
                    cconj(*reinterpret_cast<const float2*>(st + kr * 64 + ((cy ^ ((kr >> 1) & 3)) << 4) + hy));
                const float2 d = cmul(make_float2(tk[2 * (k2 & 7)], tk[2 * (k2 & 7) + 1]), csub(xa, xc));
                u[k2] = cadd(cadd(xa, xc), make_float2(-d.y, d.x));
            }
            tgfft::dft16<+1>(u);
#pragma unroll
            for (int qq = 0; qq < 16; ++qq) {
                if ((qq & 7) == 0) {
                    __syncwarp();
                    tgtm::ld16(taddr + 64u * (unsigned)it + 32u + 2u * (unsigned)qq, tk);
                }
                if (ok) xl[k1 * C2_XR + qq] = cmul(u[qq], make_float2(tk[2 * (qq & 7)], tk[2 * (qq & 7) + 1]));
            }
        }
        __syncwarp();
        float2 v[P];
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[k1] = xl[k1 * C2_XR + q];
        const float kap = kaps[b];
        tgpq::dft29_emit<+1>(v, cs, [&](int m, float2 x) {
            const float u0 = fmaf(x.x, inv_nm, kap);
            const float u1 = fmaf(x.y, inv_nm, kap);
            if (u0 > bu[m][0]) { bu[m][0] = u0; bb[m] = (bb[m] & 0xFFFF0000u) | (unsigned)b; }
            if (u1 > bu[m][1]) { bu[m][1] = u1; bb[m] = (bb[m] & 0x0000FFFFu) | ((unsigned)b << 16); }
        });
        tgtma::fence_proxy_async();
        __syncthreads();  // the stage is refilled and the exchange rewritten next
    }
    const bool failed = *flag != 0;
    tgtm::fence_before();
    __syncthreads();
    if (warp == 0) {
        tgtm::fence_after();
        tgtm::dealloc<128>(*tmem_slot);
    }
    if (failed || y >= Ny) return;
    const float mt = (float)mu_t;
    const long long row = ((long long)z * Ny + y) * NX;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const long long v = row + 2 * (q + 16 * m);
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

cudaError_t launch_corr_y_p928(const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y, long long ncols,
                               int nb, cudaStream_t st) {
    const size_t smem = sizeof(float2) * (29 * CY_RS + CY_WARPS * (2 * 29 * CY_RS + 128) + 32);
    cudaFuncSetAttribute(k_corr_y_p928, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const unsigned g = (unsigned)((ncols + CY_WARPS - 1) / CY_WARPS);
    k_corr_y_p928<<<g, 32 * CY_WARPS, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, twiddle_table<float2>(928),
                                                  cos29_table());
    return cudaGetLastError();
}

cudaError_t launch_inv_z_p464(const float2* Q, float2* H, int Ny, int nh1, int nb, cudaStream_t st) {
    const size_t smem = sizeof(float2) * (16 * IZ_LS + 29 * 16);
    cudaFuncSetAttribute(k_inv_z_p464, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 g((Ny + 15) / 16, nh1, nb);
    k_inv_z_p464<<<g, 256, smem, st>>>(Q, H, Ny, nh1, twiddle_table<float2>(464), cos29_table());
    return cudaGetLastError();
}

cudaError_t launch_c2r_p464(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, cudaStream_t st) {
    const size_t smem = sizeof(float2) * (2 * C2_YT * C2_TS + C2_YT * C2_XL + 16 * 32 + 464) + sizeof(float) * nb;
    cudaFuncSetAttribute(k_c2r_p464, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 g((Ny + C2_YT - 1) / C2_YT, Nz);
    k_c2r_p464<<<g, 16 * C2_YT, smem, st>>>(H, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0, maxcc,
                                            angidx, twiddle_table<float2>(464), twiddle_table<float2>(928),
                                            cos29_table());
    return cudaGetLastError();
}

}  // namespace tg

namespace tg {

cudaError_t launch_c2r_t464(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, int* err, cudaStream_t st) {
    // the TMA coordinate along y (floats) is 16 blockIdx.x: 64 bytes
    if (Ny % 2 || nb < 1 || nb > 65535) return cudaErrorInvalidValue;
    CUtensorMap tm_a, tm_b;
    if (!encode_h_map(&tm_a, H, Ny, Nz, 465, nb, C2_YT, 256, CU_TENSOR_MAP_SWIZZLE_64B) ||
        !encode_h_map(&tm_b, H, Ny, Nz, 465, nb, C2_YT, 209, CU_TENSOR_MAP_SWIZZLE_64B))
        return cudaErrorInvalidValue;
    const size_t smem = 1024 + 2 * (size_t)T4_STAGE + sizeof(float2) * (C2_YT * C2_XL + 16 * 32 + 464) +
                        sizeof(unsigned long long) * 2 + 2 * sizeof(int) + sizeof(float) * nb;
    cudaError_t e = cudaFuncSetAttribute(k_c2r_t464, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return e;
    dim3 g((Ny + C2_YT - 1) / C2_YT, Nz);
    k_c2r_t464<<<g, 16 * C2_YT, smem, st>>>(tm_a, tm_b, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0,
                                            maxcc, angidx, twiddle_table<float2>(464), twiddle_table<float2>(928),
                                            cos29_table(), err);
    return cudaGetLastError();
}

}  // namespace tg
