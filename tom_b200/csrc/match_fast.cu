// Register-resident variants of the three hot FLCF kernels for the common
// power-of-two sizes (y edge 256/512, z edge 256).  Same
// arithmetic contract as the generic kernels in match.cu; faster data flow:
//
//   corr_y_w  one warp per spectrum column; the y-DFT of the template, the
//             product with F_I (staged once in shared memory) and the inverse
//             y-DFT all stay in registers with two warp-private exchanges per
//             transform (warp_fft.cuh); the next rotation's template values
//             are fetched while the current one is transformed.  y edge 128.
//   corr_y_s  y edges 256 and 512: as corr_y_w, but the forward y-DFT is
//             summed straight from the template column's nonzeros into the
//             inverse transform's register pattern (no exchange).
//   inv_z_b   16 consecutive y lines per block, 16 threads per line holding
//             16 values: radix 16 straight from global memory, one block-wide
//             exchange, radix 16 straight back to global memory.
//
// The x-line kernels (c2r with the FLCF and the running maximum) are in
// match_fast128.cu (x edge 128/256/512) and match_fast29.cu (x edge 928).
#include "ctx.h"
#include "match.h"
#include "twiddles.h"
#include "tmem_util.cuh"
#include "warp_fft.cuh"

namespace tg {

namespace {

// The 512-point inverse warp transform (plan 8, 8, 8) with the twiddles of
// stages 2 and 3 read from this thread's TMEM lane: columns c2 + 16 q and
// c3 + 16 q hold w_r (r = 1..7, conjugated) of the lane's butterfly q.
__device__ __forceinline__ void warp_ifft512_tm(float2* v, float2* buf, unsigned c2, unsigned c3, int lane) {
    tgwfft::wstage<512, 8, 1, +1>(v, nullptr, lane);
    tgwfft::wstore<512, 8, 1>(v, buf, lane);
    __syncwarp();
    tgwfft::wload<512, 8>(v, buf, lane);
    __syncwarp();
#pragma unroll
    for (int stage = 0; stage < 2; ++stage) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            float t[16];
            tgtm::ld16((stage == 0 ? c2 : c3) + 16u * q, t);
#pragma unroll
            for (int r = 1; r < 8; ++r) v[q * 8 + r] = cmul(v[q * 8 + r], make_float2(t[2 * r - 2], t[2 * r - 1]));
            tgfft::dft8<+1>(v + q * 8);
        }
        if (stage == 0) {
            tgwfft::wstore<512, 8, 8>(v, buf, lane);
            __syncwarp();
            tgwfft::wload<512, 8>(v, buf, lane);
            __syncwarp();
        }
    }
}

}  // namespace

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

// y edges 256 and 512: the forward y-DFT of the template column straight
// from its Ty <= 64 nonzeros, with no exchange.  The column holds z[t] at
// y = (d0y + t) mod NY.  With W_L = exp(-2 pi i / L), t = d + 8 i and
// k = m + (NY/8) k2:
//   X(k) = W_NY^(d0y k) sum_d W_8^(d k2) [ W_NY^(d m) sum_i z[d + 8 i] W_(NY/8)^(i m) ].
// Lane l owns m = l + 32 q (q < NY/256): the bracket is a short sum per
// residue d, the outer sum one 8-point DFT per m in registers, and the result
// lands as v[8 q + k2] = X(l + 32 q + (NY/8) k2), the pattern the inverse
// warp transform starts from.  The phase W_NY^(d0y k) is folded into the
// staged F_I column (the product is F_I conj(X)).  For NY = 512 the two m of
// a lane differ by 32, W_64^(32 i) = (-1)^i: even and odd terms are summed
// once for both.  NI = ceil(Ty / 8) terms per residue.
//
// TM (y edge 512): the lane's F_I values and the twiddles of the inverse
// transform's two twiddled stages live in tensor memory (TMEM, 256 columns
// per block: warp w uses lanes 32 (w mod 4) + lane, columns 128 (w / 4) +
// [0, 96)) and are read with tcgen05.ld, which takes those reads (74 of the
// 317 shared-memory wavefronts per column and rotation) off the
// shared-memory path that bounds this kernel.
template <int NY, int NI, bool TM>
__global__ void __launch_bounds__(256, 2) k_corr_y_s(const float2* __restrict__ fimg, const float2* __restrict__ Z,
                                                     float2* __restrict__ Q, int Ty, int d0y, long long ncols, int nb,
                                                     const float2* __restrict__ tw_g) {
    constexpr int EPT = NY / 32, NB = EPT / 8;
    static_assert(!TM || NY == 512, "the TMEM variant is built for the 512-point columns");
    __shared__ unsigned tmem_slot;
    static_assert(tgwfft::WPlan<NY>::RL == 8 && (NB == 1 || NB == 2) && NI >= 1 && NI <= 8, "plan");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tw = reinterpret_cast<float2*>(smem_raw);  // [NY + 64] stage tables
    float2* xb = tw + NY + 64;                          // [8][NY] exchange
    float2* fs = xb + 8 * NY;                           // [8][NY] F_I columns times W_NY^(-d0y k)
    float2* zs = fs + 8 * NY;                           // [8][2][64] template column, z[t] at (t % 8) * 8 + t / 8
    float2* lt = zs + 8 * 128;                          // [NI-1][32] W_L8^(i l), then [NB][7][32] W_NY^(d (l + 32 q))
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long col = (long long)blockIdx.x * 8 + warp;
    static_assert(tgwfft::WTab<NY>::size <= NY + 64, "stage tables exceed their slot");
    tgwfft::build_stage_tables<NY>(tw, tw_g);
    constexpr int NW = (NI - 1) * 32, NT = NW + NB * 7 * 32;
    for (int e = threadIdx.x; e < NT; e += blockDim.x) {
        int idx;
        if (e < NW) {
            idx = 8 * (e / 32 + 1) * (e % 32);
        } else {
            const int r = e - NW, q = r / 224, d = (r % 224) / 32 + 1, l = r % 32;
            idx = d * (l + 32 * q);
        }
        lt[e] = __ldg(tw_g + idx % NY);
    }
    float2* buf = xb + warp * NY;
    float2* fw = fs + warp * NY;
    float2* zw = zs + warp * 128;
    const int zslot0 = (lane & 7) * 8 + (lane >> 3), zslot1 = zslot0 + 4;  // t = lane, lane + 32
    const bool active = col < ncols;
    if constexpr (TM) {
        if (warp == 0) tgtm::alloc<256>(&tmem_slot);
    }
    if (active) {
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int p = tgwfft::out_pos<NY>(i, lane);
            const float2 f = cmulc(fimg[col * NY + p], __ldg(tw_g + (d0y * p) % NY));  // each lane its own
            if constexpr (!TM) fw[p] = f;
            else fw[i * 32 + lane] = f;  // staged until the TMEM copy below
        }
        const float2* zc = Z + col * Ty;  // rotation 0
        zw[zslot0] = lane < Ty ? zc[lane] : make_float2(0.f, 0.f);
        zw[zslot1] = lane + 32 < Ty ? zc[lane + 32] : make_float2(0.f, 0.f);
    }
    if constexpr (TM) tgtm::fence_before();
    __syncthreads();  // the tables (and the TMEM allocation)
    unsigned tw_base = 0;
    if constexpr (TM) {
        tgtm::fence_after();
        tw_base = tgtm::lane_addr(tmem_slot, warp, 128u * (unsigned)(warp >> 2));
        if (active) {
            // columns [0, 32): the lane's 16 F_I values; [32, 64) and [64, 96): the
            // conjugated twiddles of stage 2 (stride 8) and stage 3 (stride 64)
            float t[16];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float2 f = fw[(8 * h + i) * 32 + lane];
                    t[2 * i] = f.x;
                    t[2 * i + 1] = f.y;
                }
                tgtm::st16(tw_base + 16u * h, t);
            }
#pragma unroll
            for (int stage = 0; stage < 2; ++stage) {
                const int NS = stage == 0 ? 8 : 64;
                const float2* tab = tw + (stage == 0 ? 0 : 64);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int k = (lane + 32 * q) % NS;
#pragma unroll
                    for (int r = 1; r < 8; ++r) {
                        const float2 w = cconj(tab[r * NS + k]);
                        t[2 * r - 2] = w.x;
                        t[2 * r - 1] = w.y;
                    }
                    t[14] = t[15] = 0.f;
                    tgtm::st16(tw_base + 32u + 32u * stage + 16u * q, t);
                }
            }
            tgtm::wait_st();
        }
    }
    for (int b = 0; b < (active ? nb : 0); ++b) {
        // next rotation's column: two loads per lane, parked in registers
        float2 n0 = make_float2(0.f, 0.f), n1 = make_float2(0.f, 0.f);
        if (b + 1 < nb) {
            const float2* zc = Z + ((long long)(b + 1) * ncols + col) * Ty;
            if (lane < Ty) n0 = zc[lane];
            if (lane + 32 < Ty) n1 = zc[lane + 32];
        }
        const float2* cur = zw + (b & 1) * 64;
        float2 wi[NI];
#pragma unroll
        for (int i = 1; i < NI; ++i) wi[i] = lt[(i - 1) * 32 + lane];
        float2 v[EPT];
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            float2 zz[NI + 1];
#pragma unroll
            for (int p = 0; p < (NI + 1) / 2; ++p) {
                const float4 t = reinterpret_cast<const float4*>(cur + d * 8)[p];  // same address in every lane
                zz[2 * p] = make_float2(t.x, t.y);
                zz[2 * p + 1] = make_float2(t.z, t.w);
            }
            float2 ev = zz[0], od = make_float2(0.f, 0.f);
#pragma unroll
            for (int i = 1; i < NI; ++i) {
                const float2 a = wi[i], c = zz[i];
                if (NB == 2 && (i & 1)) {
                    od.x = fmaf(c.x, a.x, fmaf(-c.y, a.y, od.x));
                    od.y = fmaf(c.x, a.y, fmaf(c.y, a.x, od.y));
                } else {
                    ev.x = fmaf(c.x, a.x, fmaf(-c.y, a.y, ev.x));
                    ev.y = fmaf(c.x, a.y, fmaf(c.y, a.x, ev.y));
                }
            }
            float2 s0 = cadd(ev, od);
            if (d > 0) s0 = cmul(s0, lt[NW + (d - 1) * 32 + lane]);
            v[d] = s0;
            if constexpr (NB == 2) {
                float2 s1 = csub(ev, od);
                if (d > 0) s1 = cmul(s1, lt[NW + 224 + (d - 1) * 32 + lane]);
                v[8 + d] = s1;
            }
        }
        tgfft::dft8<-1>(v);
        if constexpr (NB == 2) tgfft::dft8<-1>(v + 8);
        if constexpr (TM) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float t[16];
                tgtm::ld16(tw_base + 16u * h, t);
#pragma unroll
                for (int i = 0; i < 8; ++i) v[8 * h + i] = cmulc(make_float2(t[2 * i], t[2 * i + 1]), v[8 * h + i]);
            }
            warp_ifft512_tm(v, buf, tw_base + 32u, tw_base + 64u, lane);
        } else {
#pragma unroll
            for (int i = 0; i < EPT; ++i) v[i] = cmulc(fw[tgwfft::out_pos<NY>(i, lane)], v[i]);
            tgwfft::warp_fft<NY, +1>(v, buf, tw, lane);
        }
        float2* qc = Q + ((long long)b * ncols + col) * NY;
#pragma unroll
        for (int i = 0; i < EPT; ++i) qc[tgwfft::out_pos<NY>(i, lane)] = v[i];
        float2* nx = zw + ((b + 1) & 1) * 64;
        nx[zslot0] = n0;
        nx[zslot1] = n1;
        __syncwarp();
    }
    if constexpr (TM) {
        tgtm::fence_before();
        __syncthreads();
        if (warp == 0) {
            tgtm::fence_after();
            tgtm::dealloc<256>(tmem_slot);
        }
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

// z edge 256: the z-DFT of the template's x-spectrum lines (A[kx][z][y] ->
// Z[kx][kz][y]) from their Tz <= 64 nonzeros, one warp per line, with the
// factorisation of k_corr_y_s (t = d + 8 i, kz = m + 32 k2, lane l owns
// m = l): NI terms per residue, one 8-point DFT per lane, the phase
// W_256^(d0z kz) per output.  Eight y lines per block; the block's lines are
// loaded and stored through shared memory in 64-byte runs of y.
template <int NI>
__global__ void __launch_bounds__(256) k_spec_z_s256(const float2* __restrict__ A, float2* __restrict__ Z, int Ty,
                                                     int Tz, int d0z, int nh1, const float2* __restrict__ tw_g) {
    constexpr int NZ = 256, NW = (NI - 1) * 32, NT = NW + 7 * 32, OS = 9;
    __shared__ __align__(16) float2 lt[14 * 32];  // [NI-1][32] W_32^(i l), then [7][32] W_256^(d l)
    __shared__ __align__(16) float2 zs[8 * 64];   // [line][slot]: z[t] at (t % 8) * 8 + t / 8
    __shared__ __align__(16) float2 ob[NZ * OS];  // [kz][line]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int jy0 = blockIdx.x * 8, kx = blockIdx.y, b = blockIdx.z;
    for (int e = tid; e < NT; e += 256) {
        const int idx = e < NW ? 8 * (e / 32 + 1) * (e % 32) : ((e - NW) / 32 + 1) * (e % 32);
        lt[e] = __ldg(tw_g + idx % NZ);
    }
    const long long abase = ((long long)b * nh1 + kx) * Tz * Ty;
    for (int i = tid; i < 64 * 8; i += 256) {
        const int t = i >> 3, li = i & 7;
        float2 v = make_float2(0.f, 0.f);
        if (t < Tz && jy0 + li < Ty) v = A[abase + (long long)t * Ty + jy0 + li];
        zs[li * 64 + (t & 7) * 8 + (t >> 3)] = v;
    }
    __syncthreads();
    const float2* zw = zs + w * 64;
    float2 wi[NI];
#pragma unroll
    for (int i = 1; i < NI; ++i) wi[i] = lt[(i - 1) * 32 + lane];
    float2 v[8];
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        float2 zz[NI + 1];
#pragma unroll
        for (int p = 0; p < (NI + 1) / 2; ++p) {
            const float4 t = reinterpret_cast<const float4*>(zw + d * 8)[p];  // same address in every lane
            zz[2 * p] = make_float2(t.x, t.y);
            zz[2 * p + 1] = make_float2(t.z, t.w);
        }
        float2 acc = zz[0];
#pragma unroll
        for (int i = 1; i < NI; ++i) {
            const float2 a = wi[i], c = zz[i];
            acc.x = fmaf(c.x, a.x, fmaf(-c.y, a.y, acc.x));
            acc.y = fmaf(c.x, a.y, fmaf(c.y, a.x, acc.y));
        }
        if (d > 0) acc = cmul(acc, lt[NW + (d - 1) * 32 + lane]);
        v[d] = acc;
    }
    tgfft::dft8<-1>(v);
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        const int kz = lane + 32 * k2;
        ob[kz * OS + w] = cmul(v[k2], __ldg(tw_g + (d0z * kz) % NZ));
    }
    __syncthreads();
    const long long zbase = ((long long)b * nh1 + kx) * NZ * Ty;
    for (int i = tid; i < NZ * 8; i += 256) {
        const int kz = i >> 3, li = i & 7;
        if (jy0 + li < Ty) Z[zbase + (long long)kz * Ty + jy0 + li] = ob[kz * OS + li];
    }
}

// z edge 464 (NZ = 8 x 58): as k_spec_z_s256 with two m per lane.  With
// L8 = NZ / 8, t = d + 8 i and kz = m + L8 k2:
//   X(kz) = W_NZ^(d0z kz) sum_d W_8^(d k2) [ W_NZ^(d m) sum_i z[d + 8 i] W_L8^(i m) ],
// lane l owns m = l + 32 q (q < ceil(L8 / 32), m < L8): NI terms per
// residue, one 8-point DFT per m, the phase W_NZ^(d0z kz) per output.  Eight
// y lines per block; the block's lines are loaded and stored through shared
// memory in 64-byte runs of y.
template <int NZ, int NI>
__global__ void __launch_bounds__(256, 3) k_spec_z_s(const float2* __restrict__ A, float2* __restrict__ Z, int Ty,
                                                  int Tz, int d0z, int nh1, const float2* __restrict__ tw_g) {
    constexpr int L8 = NZ / 8, MB = (L8 + 31) / 32, OS = 9, PER = NI - 1 + 7;
    static_assert(NZ % 8 == 0 && MB <= 2 && NI >= 1 && NI <= 8, "plan");
    __shared__ __align__(16) float2 lt[2 * 14 * 32];  // [q][NI-1][32] W_L8^(i m), then [q][7][32] W_NZ^(d m)
    __shared__ __align__(16) float2 zs[8 * 64];       // [line][slot]: z[t] at (t % 8) * 8 + t / 8
    __shared__ __align__(16) float2 ob[NZ * OS];      // [kz][line]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int jy0 = blockIdx.x * 8, kx = blockIdx.y, b = blockIdx.z;
    for (int e = tid; e < MB * PER * 32; e += 256) {
        const int q = e / (PER * 32), r = (e / 32) % PER, m = (e % 32) + 32 * q;
        const int idx = r < NI - 1 ? 8 * (r + 1) * m : (r - (NI - 1) + 1) * m;
        lt[e] = __ldg(tw_g + idx % NZ);
    }
    const long long abase = ((long long)b * nh1 + kx) * Tz * Ty;
    for (int i = tid; i < 64 * 8; i += 256) {
        const int t = i >> 3, li = i & 7;
        float2 v = make_float2(0.f, 0.f);
        if (t < Tz && jy0 + li < Ty) v = A[abase + (long long)t * Ty + jy0 + li];
        zs[li * 64 + (t & 7) * 8 + (t >> 3)] = v;
    }
    __syncthreads();
    const float2* zw = zs + w * 64;
    auto line_sums = [&](int q) {
        const int m = lane + 32 * q;
        const float2* lq = lt + q * PER * 32;
        float2 wi[NI];
#pragma unroll
        for (int i = 1; i < NI; ++i) wi[i] = lq[(i - 1) * 32 + lane];
        float2 v[8];
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            float2 zz[NI + 1];
#pragma unroll
            for (int p = 0; p < (NI + 1) / 2; ++p) {
                const float4 t = reinterpret_cast<const float4*>(zw + d * 8)[p];  // same address in every lane
                zz[2 * p] = make_float2(t.x, t.y);
                zz[2 * p + 1] = make_float2(t.z, t.w);
            }
            float2 acc = zz[0];
#pragma unroll
            for (int i = 1; i < NI; ++i) {
                const float2 a = wi[i], c = zz[i];
                acc.x = fmaf(c.x, a.x, fmaf(-c.y, a.y, acc.x));
                acc.y = fmaf(c.x, a.y, fmaf(c.y, a.x, acc.y));
            }
            if (d > 0) acc = cmul(acc, lq[(NI - 1 + d - 1) * 32 + lane]);
            v[d] = acc;
        }
        tgfft::dft8<-1>(v);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) {
            const int kz = m + L8 * k2;
            ob[kz * OS + w] = cmul(v[k2], __ldg(tw_g + (d0z * kz) % NZ));
        }
    };
    line_sums(0);
    if constexpr (MB == 2) {
        if (lane + 32 < L8) line_sums(1);
    }
    __syncthreads();
    const long long zbase = ((long long)b * nh1 + kx) * NZ * Ty;
    for (int i = tid; i < NZ * 8; i += 256) {
        const int kz = i >> 3, li = i & 7;
        if (jy0 + li < Ty) Z[zbase + (long long)kz * Ty + jy0 + li] = ob[kz * OS + li];
    }
}

// ------------------------------------------------------------- dispatch

bool fast_corr_y(int NY, int Ty) { return (NY == 128 || NY == 256 || NY == 512 || NY == 928) && Ty <= 64; }
bool fast_inv_z(int NZ) { return NZ == 128 || NZ == 256 || NZ == 464; }
bool fast_c2r(int NH) { return NH == 64 || NH == 128 || NH == 256 || NH == 464; }
bool fast_spec_z(int NZ, int Tz) { return (NZ == 256 || NZ == 464) && Tz >= 1 && Tz <= 64; }

template <int NZ>
static cudaError_t launch_spec_z_nz(const float2* A, float2* Z, int Ty, int Tz, int d0z, int nh1, int nb,
                                    cudaStream_t st) {
    const dim3 g((Ty + 7) / 8, nh1, nb);
    const float2* tw = twiddle_table<float2>(NZ);
    switch ((Tz + 7) / 8) {
#define C_(n) \
    case n: k_spec_z_s<NZ, n><<<g, 256, 0, st>>>(A, Z, Ty, Tz, d0z, nh1, tw); break;
        C_(1) C_(2) C_(3) C_(4) C_(5) C_(6) C_(7) C_(8)
#undef C_
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_spec_z_fast(int NZ, const float2* A, float2* Z, int Ty, int Tz, int d0z, int nh1, int nb,
                               cudaStream_t st) {
    if (!fast_spec_z(NZ, Tz)) return cudaErrorInvalidValue;
    if (NZ == 464) return launch_spec_z_nz<464>(A, Z, Ty, Tz, d0z, nh1, nb, st);
    const dim3 g((Ty + 7) / 8, nh1, nb);
    const float2* tw = twiddle_table<float2>(256);
    switch ((Tz + 7) / 8) {
#define C_(n) \
    case n: k_spec_z_s256<n><<<g, 256, 0, st>>>(A, Z, Ty, Tz, d0z, nh1, tw); break;
        C_(1) C_(2) C_(3) C_(4) C_(5) C_(6) C_(7) C_(8)
#undef C_
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int NY, int NI, bool TM>
static cudaError_t launch_corr_y_s_ni(const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                                      long long ncols, int nb, cudaStream_t st) {
    const unsigned g = (unsigned)((ncols + 7) / 8);
    const size_t smem = sizeof(float2) * (NY * 17 + 64 + 8 * 128 + 3 * 7 * 32);
    cudaFuncSetAttribute(k_corr_y_s<NY, NI, TM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_corr_y_s<NY, NI, TM><<<g, 256, smem, st>>>(fimg, Z, Q, Ty, d0y, ncols, nb, twiddle_table<float2>(NY));
    return cudaGetLastError();
}

template <int NY, bool TM>
static cudaError_t launch_corr_y_s(const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y, long long ncols,
                                   int nb, cudaStream_t st) {
    switch ((Ty + 7) / 8) {
        case 1: return launch_corr_y_s_ni<NY, 1, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 2: return launch_corr_y_s_ni<NY, 2, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 3: return launch_corr_y_s_ni<NY, 3, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 4: return launch_corr_y_s_ni<NY, 4, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 5: return launch_corr_y_s_ni<NY, 5, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 6: return launch_corr_y_s_ni<NY, 6, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 7: return launch_corr_y_s_ni<NY, 7, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        case 8: return launch_corr_y_s_ni<NY, 8, TM>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_corr_y_fast(int NY, const float2* fimg, const float2* Z, float2* Q, int Ty, int d0y,
                               long long ncols, int nb, cudaStream_t st, bool tmem) {
    if (NY == 928) return launch_corr_y_p928(fimg, Z, Q, Ty, d0y, ncols, nb, st);
    const unsigned g = (unsigned)((ncols + 7) / 8);
    const size_t smem = sizeof(float2) * (NY * 17 + 64 + 8 * 128);
    if (NY == 512 || NY == 256) {
        if (Ty < 1 || Ty > 64) return cudaErrorInvalidValue;
        if (NY == 256) return launch_corr_y_s<256, false>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
        return tmem ? launch_corr_y_s<512, true>(fimg, Z, Q, Ty, d0y, ncols, nb, st)
                    : launch_corr_y_s<512, false>(fimg, Z, Q, Ty, d0y, ncols, nb, st);
    }
    if (NY == 128) {
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

cudaError_t launch_c2r_fast(int NH, const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny,
                            int Nz, int nb, float inv_nm, double c, double inv_m, double mu_t, int index0,
                            float* maxcc, int* angidx, cudaStream_t st) {
    // x edge 512: a half-warp per line (20 % faster on the 512x512x256 search
    // than a warp per line); x edge 256 and 128: 8 threads per line
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
