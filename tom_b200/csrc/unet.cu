// Kernels of the U-Net candidate proposer (tom_b200/unet.py): 3x3x3
// convolutions in BF16 on the tcgen05 tensor cores with FP32 accumulation in
// tensor memory, and the small kernels around them.
//
// Activations are channels-last BF16, act[z][y][x][c] with a channel stride
// cs >= C (a layer may read or write a channel slice [off, off + C) of a wider
// buffer, which is how the decoder's concatenations are formed without a
// copy).  Convolutions are cross-correlations with zero padding ("same"):
//   out[v][co] = b[co] + sum_t sum_ci W[co][ci][t] in[v + off(t)][ci],
//   off(t) = (t % 3 - 1, t / 3 % 3 - 1, t / 9 - 1),
// with the FP32 master weights W[co][ci][27] (taps x fastest).
//
// Forward / input-gradient convolution (k_uconv_tc): one 128-thread block per
// output tile of 8 (x) x 16 (y) voxels of one z plane, i.e. M = 128 rows of
// one MMA.  Per step (one input plane dz, 16 input channels) the block loads
// the tile's input with its one-voxel halo in x and y as two TMA boxes of
// 8 channels x 10 x 18 voxels (zero-filled outside the volume), which is
// exactly the no-swizzle K-major operand layout (rows of 16 bytes = 8
// channels): the operand of tap (dx, dy) starts dy * 10 + dx rows into the box
// and steps 160 bytes per 8-row group (one y row of the tile), so the nine
// taps of a plane are nine MMAs (M = 128, N = Cout, K = 16) on the same
// staged data.  The step's packed weights ([9 taps][2 halves][Cout][8]) come
// in by one bulk copy.  One thread issues the copies and the MMAs through a
// ring of stages; the accumulator (128 lanes x Cout FP32 columns) is read
// back by the four warps (thread t = voxel t), which add the bias, apply the
// ReLU or the mask of a ReLU's derivative, round to BF16 and store.
//
// Weight gradient (k_uconv_wgrad_tc): dW[co][ci][t] = sum_v dY[v][co]
// in[v + off(t)][ci], a contraction over voxels: per tile (the same 8 x 16
// voxel tiles) and tap, one MMA chain D[co][ci] += dY^T . in_t with both
// operands MN-major straight from the channels-last boxes (8 channels
// contiguous, 8-voxel K groups 128 bytes (dY) or 160 bytes (halo box) apart).
// M = 128 rows of co, of which the first Cout are real; the others read
// staged bytes that are never used.  A block holds the accumulators of a tap
// group (the 9 taps of one plane, or the 3 of one row when Cin > 48) for a
// strided set of tiles and adds them into the FP32 gradient at the end.
//
// Every wait on an mbarrier is bounded; on a timeout a block records
// TG_DEV_TIMEOUT in the device error word, waits (bounded) for its copies and
// MMAs in flight, frees its tensor memory and returns.  Tensor maps cover this
// GPU's own buffers; no load multicasts.
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdint>

#include "common.cuh"
#include "ctx.h"
#include "tma_util.cuh"
#include "tmem_util.cuh"

namespace tg {

namespace {

constexpr int UX = 8, UY = 16;              // output tile of one z plane (M = 128 voxels)
constexpr int HX = UX + 2, HY = UY + 2;     // input box with its halo
constexpr int HBOX = HX * HY * 16;          // bytes of one 8-channel input box (2880)
constexpr int HSLOT = 2944;                 // its slot in shared memory (128-byte multiple)
constexpr int DBOX = UX * UY * 16;          // bytes of one 8-channel output-gradient box (2048)
constexpr long long U_WAIT = 1ll << 22;

TG_D unsigned long long udesc(unsigned addr, unsigned lbo, unsigned sbo) {
    // shared-memory matrix descriptor, no swizzle (version 1: sm_100)
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor of kind::f16: D F32, A and B BF16, M = 128, N = n;
// mn = 1 makes both operands MN-major
__host__ __device__ constexpr unsigned uidesc(int n, int mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (mn ? (1u << 15) | (1u << 16) : 0u) | ((unsigned)(n >> 3) << 17) |
           (8u << 24);
}

TG_D void mma_bf16(unsigned d, unsigned long long a, unsigned long long b, unsigned idesc, unsigned acc) {
    const unsigned z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

TG_D void mma_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// untiled bulk copy global -> shared (16-byte aligned, size a multiple of 16)
TG_D void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(reinterpret_cast<unsigned long long>(src)), "r"(bytes), "r"(bar)
                 : "memory");
}

TG_D float bf2f(unsigned short h) { return __uint_as_float((unsigned)h << 16); }
TG_D unsigned short f2bf(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
TG_D unsigned pack2(float a, float b) { return (unsigned)f2bf(a) | ((unsigned)f2bf(b) << 16); }

struct ConvArgs {
    int X, Y, Z, cin;
    const unsigned char* wpk;  // packed BF16 weights, [3][cin / 16][9][2][COUT][8]
    const float* bias;         // [COUT] or null
    int relu;
    unsigned short* out;
    int out_cs, out_off;
    const unsigned short* mask;  // null, or out *= (mask[v][mask_off + co] > 0)
    int mask_cs, mask_off;
    int* err;
};

template <int COUT, int NST>
__global__ void __launch_bounds__(128) k_uconv_tc(const __grid_constant__ CUtensorMap tin, ConvArgs a) {
    constexpr int BST = 9 * 2 * COUT * 16;  // packed weight bytes of one step
    constexpr int STG = 2 * HSLOT + BST;
    constexpr int TCOLS = COUT <= 32 ? 32 : (COUT <= 64 ? 64 : 128);
    constexpr unsigned IDESC = uidesc(COUT, 0);
    static_assert(COUT % 16 == 0 && COUT <= 256, "N of an M = 128 MMA");
    extern __shared__ __align__(1024) unsigned char smu[];
    unsigned char* sm = smu + ((1024u - (tgtma::smem_u32(smu) & 1023u)) & 1023u);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + NST * STG);
    unsigned long long* freeb = full + NST;
    unsigned long long* done = freeb + NST;
    unsigned* tslot = reinterpret_cast<unsigned*>(done + 1);
    int* state = reinterpret_cast<int*>(tslot + 1);  // 0 ok, 1 failed
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tiles_x = (a.X + UX - 1) / UX;
    const int x0 = (blockIdx.x % tiles_x) * UX, y0 = (blockIdx.x / tiles_x) * UY, z = blockIdx.y;
    const int nch = a.cin >> 4, steps = 3 * nch;
    if (warp == 0) tgtm::alloc<TCOLS>(tslot);
    if (tid == 0) {
        for (int i = 0; i < NST; ++i) {
            tgtma::mbar_init(tgtma::smem_u32(full + i), 1);
            tgtma::mbar_init(tgtma::smem_u32(freeb + i), 1);
        }
        tgtma::mbar_init(tgtma::smem_u32(done), 1);
        *state = 0;
        tgtma::fence_barrier_init();
        tgtma::prefetch_map(&tin);
    }
    tgtm::fence_before();
    __syncthreads();
    tgtm::fence_after();
    const unsigned tbase = *tslot;
    if (tid == 0) {
        const unsigned s0 = tgtma::smem_u32(sm);
        auto load = [&](int s) {
            const int st = s % NST, dz = s / nch, c = s - dz * nch;
            const unsigned dst = s0 + (unsigned)(st * STG), bar = tgtma::smem_u32(full + st);
            tgtma::mbar_expect_tx(bar, (unsigned)(2 * HBOX + BST));
            tgtma::load_4d(dst, &tin, 16 * c, x0 - 1, y0 - 1, z + dz - 1, bar);
            tgtma::load_4d(dst + HSLOT, &tin, 16 * c + 8, x0 - 1, y0 - 1, z + dz - 1, bar);
            bulk_g2s(dst + 2 * HSLOT, a.wpk + (size_t)s * BST, (unsigned)BST, bar);
        };
        int issued = steps < NST ? steps : NST;
        for (int s = 0; s < issued; ++s) load(s);
        int s = 0;
        bool ok = true;
        for (; s < steps; ++s) {
            const int st = s % NST;
            const unsigned ph = (unsigned)((s / NST) & 1);
            if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(full + st), ph, U_WAIT)) {
                ok = false;
                break;
            }
            tgtm::fence_after();
            const unsigned abase = s0 + (unsigned)(st * STG), bbase = abase + 2 * HSLOT;
#pragma unroll
            for (int t = 0; t < 9; ++t) {
                const int dy = t / 3, dx = t - 3 * dy;
                const unsigned long long ad = udesc(abase + (unsigned)((dy * HX + dx) * 16), HSLOT, HX * 16);
                const unsigned long long bd = udesc(bbase + (unsigned)(t * 2 * COUT * 16), COUT * 16, 128);
                mma_bf16(tbase, ad, bd, IDESC, (s > 0 || t > 0) ? 1u : 0u);
            }
            mma_commit(tgtma::smem_u32(freeb + st));
            if (issued < steps) {
                // the stage is refilled once its MMAs have read it
                if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(freeb + st), ph, U_WAIT)) {
                    ++s;
                    ok = false;
                    break;
                }
                load(issued++);
            }
        }
        mma_commit(tgtma::smem_u32(done));
        if (!ok) {
            // copies issued but not consumed, and the MMAs committed so far
            for (int r = s; r < issued; ++r)
                tgtma::mbar_wait_bounded(tgtma::smem_u32(full + r % NST), (unsigned)((r / NST) & 1), U_WAIT);
            *state = 1;
        }
        if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(done), 0u, U_WAIT)) *state = 1;
        if (*state) tg_flag_error(a.err, TG_DEV_TIMEOUT);
    }
    __syncthreads();
    tgtm::fence_after();
    if (*state == 0) {
        const int tx = tid & 7, ty = tid >> 3;
        const int x = x0 + tx, y = y0 + ty;
        const bool in = x < a.X && y < a.Y;
        const long long v = ((long long)z * a.Y + y) * a.X + x;
        const unsigned taddr = tgtm::lane_addr(tbase, warp, 0u);
#pragma unroll
        for (int c16 = 0; c16 < COUT / 16; ++c16) {
            float r[16];
            tgtm::ld16(taddr + 16u * (unsigned)c16, r);
            if (!in) continue;
            if (a.bias) {
#pragma unroll
                for (int i = 0; i < 16; ++i) r[i] += __ldg(a.bias + 16 * c16 + i);
            }
            if (a.relu) {
#pragma unroll
                for (int i = 0; i < 16; ++i) r[i] = fmaxf(r[i], 0.f);
            }
            if (a.mask) {
                const uint4* mp = reinterpret_cast<const uint4*>(a.mask + v * a.mask_cs + a.mask_off + 16 * c16);
                const uint4 m0 = __ldg(mp), m1 = __ldg(mp + 1);
                const unsigned mw[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const unsigned short h = (unsigned short)(mw[i >> 1] >> (16 * (i & 1)));
                    if (!(bf2f(h) > 0.f)) r[i] = 0.f;
                }
            }
            uint4* op = reinterpret_cast<uint4*>(a.out + v * a.out_cs + a.out_off + 16 * c16);
            op[0] = make_uint4(pack2(r[0], r[1]), pack2(r[2], r[3]), pack2(r[4], r[5]), pack2(r[6], r[7]));
            op[1] = make_uint4(pack2(r[8], r[9]), pack2(r[10], r[11]), pack2(r[12], r[13]), pack2(r[14], r[15]));
        }
    }
    tgtm::fence_before();
    __syncthreads();
    if (warp == 0) {
        tgtm::fence_after();
        tgtm::dealloc<TCOLS>(tbase);
    }
}

struct WgArgs {
    int X, Y, Z, cin, cout, group_taps;  // group_taps: 9 (one plane) or 3 (one row)
    float* gw;                            // [cout][cin][27], accumulated
    int* err;
};

constexpr int WG_NST = 4;
constexpr int WG_A = 16 * DBOX;  // the bytes an M = 128 operand of co (16 groups of 8) spans
// A stage holds the tile's real operands only: Cout / 8 output-gradient boxes
// then Cin / 8 halo boxes.  An MMA's rows past Cout read whatever follows (the
// stage's halo boxes, the next stage); those rows of the accumulator are
// never read back.  The allocation ends WG_A bytes past the last stage's
// start at least, so every such read stays inside it.
__host__ __device__ constexpr int wg_stage(int cin, int cout) { return (cout / 8) * DBOX + (cin / 8) * HSLOT; }
__host__ __device__ constexpr int wg_span(int stg) {
    return WG_NST * stg > (WG_NST - 1) * stg + WG_A ? WG_NST * stg : (WG_NST - 1) * stg + WG_A;
}

// Weight gradient; grid (splits, groups).  Group g: taps (dz = g, all dy, dx)
// when group_taps == 9, else (dz = g / 3, dy = g % 3, dx = 0..2).
__global__ void __launch_bounds__(128) k_uconv_wgrad_tc(const __grid_constant__ CUtensorMap tin,
                                                        const __grid_constant__ CUtensorMap tdy, WgArgs a) {
    const int STG = wg_stage(a.cin, a.cout), ABYTES = (a.cout / 8) * DBOX;
    extern __shared__ __align__(1024) unsigned char smu[];
    unsigned char* sm = smu + ((1024u - (tgtma::smem_u32(smu) & 1023u)) & 1023u);
    unsigned long long* full = reinterpret_cast<unsigned long long*>(sm + wg_span(STG));
    unsigned long long* freeb = full + WG_NST;
    unsigned long long* done = freeb + WG_NST;
    unsigned* tslot = reinterpret_cast<unsigned*>(done + 1);
    int* state = reinterpret_cast<int*>(tslot + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int tiles_x = (a.X + UX - 1) / UX, tiles_y = (a.Y + UY - 1) / UY;
    const int ntiles = tiles_x * tiles_y * a.Z;
    const int g = blockIdx.y, nt = a.group_taps;
    const int dz = nt == 9 ? g : g / 3, dy0 = nt == 9 ? 0 : g % 3;
    const int my = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const unsigned idesc = uidesc(a.cin, 1);
    const int ng_out = a.cout >> 3, ng_in = a.cin >> 3;
    if (warp == 0) tgtm::alloc<512>(tslot);
    if (tid == 0) {
        for (int i = 0; i < WG_NST; ++i) {
            tgtma::mbar_init(tgtma::smem_u32(full + i), 1);
            tgtma::mbar_init(tgtma::smem_u32(freeb + i), 1);
        }
        tgtma::mbar_init(tgtma::smem_u32(done), 1);
        *state = 0;
        tgtma::fence_barrier_init();
        tgtma::prefetch_map(&tin);
        tgtma::prefetch_map(&tdy);
    }
    tgtm::fence_before();
    __syncthreads();
    tgtm::fence_after();
    const unsigned tbase = *tslot;
    if (tid == 0 && my > 0) {
        const unsigned s0 = tgtma::smem_u32(sm);
        auto load = [&](int s) {
            const int tile = (int)blockIdx.x + s * (int)gridDim.x;
            const int tz = tile / (tiles_x * tiles_y), rem = tile - tz * tiles_x * tiles_y;
            const int x0 = (rem % tiles_x) * UX, y0 = (rem / tiles_x) * UY;
            const int st = s % WG_NST;
            const unsigned dst = s0 + (unsigned)(st * STG), bar = tgtma::smem_u32(full + st);
            tgtma::mbar_expect_tx(bar, (unsigned)(ng_out * DBOX + ng_in * HBOX));
            for (int j = 0; j < ng_out; ++j) tgtma::load_4d(dst + (unsigned)(j * DBOX), &tdy, 8 * j, x0, y0, tz, bar);
            for (int j = 0; j < ng_in; ++j)
                tgtma::load_4d(dst + (unsigned)(ABYTES + j * HSLOT), &tin, 8 * j, x0 - 1, y0 - 1, tz + dz - 1, bar);
        };
        int issued = my < WG_NST ? my : WG_NST;
        for (int s = 0; s < issued; ++s) load(s);
        int s = 0;
        bool ok = true;
        for (; s < my; ++s) {
            const int st = s % WG_NST;
            const unsigned ph = (unsigned)((s / WG_NST) & 1);
            if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(full + st), ph, U_WAIT)) {
                ok = false;
                break;
            }
            tgtm::fence_after();
            const unsigned abase = s0 + (unsigned)(st * STG), bbase = abase + (unsigned)ABYTES;
            for (int i = 0; i < nt; ++i) {
                const int dy = nt == 9 ? i / 3 : dy0, dx = nt == 9 ? i % 3 : i;
                const unsigned d = tbase + (unsigned)(i * a.cin);
#pragma unroll
                for (int kk = 0; kk < UY / 2; ++kk) {
                    // K = 16 voxels: tile rows 2 kk and 2 kk + 1
                    const unsigned long long ad = udesc(abase + (unsigned)(kk * 2 * UX * 16), UX * 16, DBOX);
                    const unsigned long long bd =
                        udesc(bbase + (unsigned)((((2 * kk + dy) * HX) + dx) * 16), HX * 16, HSLOT);
                    mma_bf16(d, ad, bd, idesc, (s > 0 || kk > 0) ? 1u : 0u);
                }
            }
            mma_commit(tgtma::smem_u32(freeb + st));
            if (issued < my) {
                if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(freeb + st), ph, U_WAIT)) {
                    ++s;
                    ok = false;
                    break;
                }
                load(issued++);
            }
        }
        mma_commit(tgtma::smem_u32(done));
        if (!ok) {
            for (int r = s; r < issued; ++r)
                tgtma::mbar_wait_bounded(tgtma::smem_u32(full + r % WG_NST), (unsigned)((r / WG_NST) & 1), U_WAIT);
            *state = 1;
        }
        if (!tgtma::mbar_wait_bounded(tgtma::smem_u32(done), 0u, U_WAIT)) *state = 1;
        if (*state) tg_flag_error(a.err, TG_DEV_TIMEOUT);
    }
    __syncthreads();
    tgtm::fence_after();
    if (*state == 0 && my > 0) {
        const int co = tid;  // TMEM lane = row = output channel
        const unsigned taddr = tgtm::lane_addr(tbase, warp, 0u);
        for (int i = 0; i < nt; ++i) {
            const int dy = nt == 9 ? i / 3 : dy0, dx = nt == 9 ? i % 3 : i;
            const int tap = dz * 9 + dy * 3 + dx;
            for (int c16 = 0; c16 < a.cin / 16; ++c16) {
                float r[16];
                tgtm::ld16(taddr + (unsigned)(i * a.cin + 16 * c16), r);
                if (co < a.cout) {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        atomicAdd(a.gw + ((long long)co * a.cin + 16 * c16 + j) * 27 + tap, r[j]);
                }
            }
        }
    }
    tgtm::fence_before();
    __syncthreads();
    if (warp == 0) {
        tgtm::fence_after();
        tgtm::dealloc<512>(tbase);
    }
}

// ------------------------------------------------------------ the small kernels

// packed weights of one convolution for k_uconv_tc: [3 dz][nci / 16][9][2][nco][8]
// with, for the forward form, nco = cout, nci = cin and value W[co][ci][t];
// for the input-gradient form (flip = 1) nco = cin, nci = cout and value
// W[ci'][co'][26 - t] (taps mirrored, channel roles swapped)
__global__ void k_upack(const float* __restrict__ w, int cout, int cin, int flip, unsigned short* __restrict__ pk) {
    const int nco = flip ? cin : cout, nci = flip ? cout : cin;
    const long long n = 27ll * nco * nci;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(i & 7);
        long long r = i >> 3;
        const int co = (int)(r % nco);
        r /= nco;
        const int h = (int)(r & 1);
        r >>= 1;
        const int t9 = (int)(r % 9);
        r /= 9;
        const int c = (int)(r % (nci / 16));
        const int dz = (int)(r / (nci / 16));
        const int ci = 16 * c + 8 * h + j, tap = dz * 9 + t9;
        const float v = flip ? w[((long long)ci * cin + co) * 27 + (26 - tap)] : w[((long long)co * cin + ci) * 27 + tap];
        pk[i] = f2bf(v);
    }
}

// first layer: one input channel (FP32 volume), 16 outputs with bias and ReLU
__global__ void __launch_bounds__(256) k_uconv_first(const float* __restrict__ vol, int X, int Y, int Z,
                                                     const float* __restrict__ w, const float* __restrict__ b,
                                                     unsigned short* __restrict__ out) {
    __shared__ float ws[27][16];
    __shared__ float bs[16];
    for (int i = threadIdx.x; i < 27 * 16; i += blockDim.x) ws[i % 27][i / 27] = w[i];  // w[co][0][t]
    if (threadIdx.x < 16) bs[threadIdx.x] = b ? b[threadIdx.x] : 0.f;
    __syncthreads();
    const long long n = (long long)X * Y * Z;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
        float acc[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] = bs[c];
        for (int t = 0; t < 27; ++t) {
            const int xx = x + t % 3 - 1, yy = y + t / 3 % 3 - 1, zz = z + t / 9 - 1;
            if (xx < 0 || xx >= X || yy < 0 || yy >= Y || zz < 0 || zz >= Z) continue;
            const float u = __ldg(vol + ((long long)zz * Y + yy) * X + xx);
#pragma unroll
            for (int c = 0; c < 16; ++c) acc[c] = fmaf(ws[t][c], u, acc[c]);
        }
        uint4* op = reinterpret_cast<uint4*>(out + v * 16);
        op[0] = make_uint4(pack2(fmaxf(acc[0], 0.f), fmaxf(acc[1], 0.f)), pack2(fmaxf(acc[2], 0.f), fmaxf(acc[3], 0.f)),
                           pack2(fmaxf(acc[4], 0.f), fmaxf(acc[5], 0.f)), pack2(fmaxf(acc[6], 0.f), fmaxf(acc[7], 0.f)));
        op[1] = make_uint4(pack2(fmaxf(acc[8], 0.f), fmaxf(acc[9], 0.f)), pack2(fmaxf(acc[10], 0.f), fmaxf(acc[11], 0.f)),
                           pack2(fmaxf(acc[12], 0.f), fmaxf(acc[13], 0.f)),
                           pack2(fmaxf(acc[14], 0.f), fmaxf(acc[15], 0.f)));
    }
}

// first layer's weight and bias gradients: thread j of a 448-thread block owns
// output j (j < 432: (co = j / 27, t = j % 27); j >= 432: bias co = j - 432)
// and sums over 8 x 8 x 8 voxel tiles staged in shared memory (the input with
// its one-voxel halo, the output gradient as FP32), a strided set of tiles
// per block, then one atomic add per output
__global__ void __launch_bounds__(448) k_uconv_first_wgrad(const float* __restrict__ vol, int X, int Y, int Z,
                                                          const unsigned short* __restrict__ g,
                                                          float* __restrict__ gw, float* __restrict__ gb) {
    constexpr int E = 8, H = E + 2;
    __shared__ float xin[H * H * H];
    __shared__ float gs[E * E * E][17];
    const int j = threadIdx.x;
    const int co = j < 432 ? j / 27 : j - 432, t = j < 432 ? j % 27 : -1;
    const int ox = t >= 0 ? t % 3 : 1, oy = t >= 0 ? t / 3 % 3 : 1, oz = t >= 0 ? t / 9 : 1;  // 0..2 in the halo tile
    const int tx = (X + E - 1) / E, ty = (Y + E - 1) / E, tz = (Z + E - 1) / E;
    const int ntiles = tx * ty * tz;
    float acc = 0.f;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int bx = (tile % tx) * E, by = (tile / tx % ty) * E, bz = (tile / (tx * ty)) * E;
        __syncthreads();
        for (int i = threadIdx.x; i < H * H * H; i += blockDim.x) {
            const int x = bx - 1 + i % H, y = by - 1 + i / H % H, z = bz - 1 + i / (H * H);
            xin[i] = ((unsigned)x < (unsigned)X && (unsigned)y < (unsigned)Y && (unsigned)z < (unsigned)Z)
                         ? __ldg(vol + ((long long)z * Y + y) * X + x)
                         : 0.f;
        }
        for (int i = threadIdx.x; i < E * E * E * 16; i += blockDim.x) {
            const int c = i & 15, v = i >> 4;
            const int x = bx + v % E, y = by + v / E % E, z = bz + v / (E * E);
            gs[v][c] = (x < X && y < Y && z < Z) ? bf2f(g[(((long long)z * Y + y) * X + x) * 16 + c]) : 0.f;
        }
        __syncthreads();
        for (int vz = 0; vz < E; ++vz)
            for (int vy = 0; vy < E; ++vy) {
                const float* row = xin + ((vz + oz) * H + vy + oy) * H + ox;
                const int v0 = (vz * E + vy) * E;
#pragma unroll
                for (int vx = 0; vx < E; ++vx) acc = fmaf(gs[v0 + vx][co], t >= 0 ? row[vx] : 1.f, acc);
            }
    }
    if (t >= 0)
        atomicAdd(gw + co * 27 + t, acc);
    else if (gb)
        atomicAdd(gb + co, acc);
}

// candidate head: logit[v] = wb[16] + sum_c wb[c] f[v][c] (16 channels), or
// its logistic sigmoid when prob != 0
__global__ void k_uhead(const unsigned short* __restrict__ f, long long n, const float* __restrict__ w, int prob,
                        float* __restrict__ logit) {
    const float b = __ldg(w + 16);
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const uint4* p = reinterpret_cast<const uint4*>(f + v * 16);
        const uint4 q0 = __ldg(p), q1 = __ldg(p + 1);
        const unsigned u[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        float s = b;
#pragma unroll
        for (int c = 0; c < 16; ++c) s = fmaf(__ldg(w + c), bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1)))), s);
        logit[v] = prob ? 1.f / (1.f + expf(-s)) : s;
    }
}

// head backward: gf[v][c] = g[v] w[c] (f[v][c] > 0); gw[c] += sum_v g[v] f[v][c],
// gw[16] += sum_v g[v] (block reductions, one atomic add per block and value)
__global__ void __launch_bounds__(256) k_uhead_bwd(const unsigned short* __restrict__ f, long long n,
                                                   const float* __restrict__ w, const float* __restrict__ g,
                                                   unsigned short* __restrict__ gf, float* __restrict__ gw) {
    __shared__ float red[8][17];
    float acc[17];
#pragma unroll
    for (int c = 0; c < 17; ++c) acc[c] = 0.f;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        const uint4* p = reinterpret_cast<const uint4*>(f + v * 16);
        const uint4 q0 = __ldg(p), q1 = __ldg(p + 1);
        const unsigned u[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        const float gv = g[v];
        float r[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            const float fv = bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1))));
            acc[c] = fmaf(gv, fv, acc[c]);
            r[c] = fv > 0.f ? gv * __ldg(w + c) : 0.f;
        }
        acc[16] += gv;
        uint4* op = reinterpret_cast<uint4*>(gf + v * 16);
        op[0] = make_uint4(pack2(r[0], r[1]), pack2(r[2], r[3]), pack2(r[4], r[5]), pack2(r[6], r[7]));
        op[1] = make_uint4(pack2(r[8], r[9]), pack2(r[10], r[11]), pack2(r[12], r[13]), pack2(r[14], r[15]));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < 17; ++c) {
        float s = acc[c];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp][c] = s;
    }
    __syncthreads();
    if (threadIdx.x < 17) {
        float s = 0.f;
        for (int k = 0; k < 8; ++k) s += red[k][threadIdx.x];
        atomicAdd(gw + threadIdx.x, s);
    }
}

// 2 x 2 x 2 average pool of a channel slice into a dense [C] coarse volume;
// one thread per (coarse voxel, 8 channels)
__global__ void k_upool(const unsigned short* __restrict__ in, int cs, int off, int C, int X, int Y, int Z,
                        unsigned short* __restrict__ out) {
    const int Xc = X / 2, Yc = Y / 2, Zc = Z / 2, g8 = C / 8;
    const long long n = (long long)Xc * Yc * Zc * g8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int gq = (int)(i % g8);
        const long long vc = i / g8;
        const int x = (int)(vc % Xc), y = (int)((vc / Xc) % Yc), z = (int)(vc / ((long long)Xc * Yc));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long v = ((long long)(2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X + 2 * x + (d & 1);
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(in + v * cs + off + 8 * gq));
            const unsigned u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int c = 0; c < 8; ++c) s[c] += bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1))));
        }
        *reinterpret_cast<uint4*>(out + vc * C + 8 * gq) = make_uint4(
            pack2(0.125f * s[0], 0.125f * s[1]), pack2(0.125f * s[2], 0.125f * s[3]),
            pack2(0.125f * s[4], 0.125f * s[5]), pack2(0.125f * s[6], 0.125f * s[7]));
    }
}

// pool backward: gin[v][off + c] (+)= gout[v / 2][c] / 8, times (mask > 0) when
// a mask is given (the mask has gin's stride and offset)
__global__ void k_upool_bwd(const unsigned short* __restrict__ gout, int C, int X, int Y, int Z,
                            const unsigned short* __restrict__ mask, int cs, int off, unsigned short* __restrict__ gin,
                            int accumulate) {
    const int g8 = C / 8;
    const long long n = (long long)X * Y * Z * g8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int gq = (int)(i % g8);
        const long long v = i / g8;
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
        const long long vc = ((long long)(z / 2) * (Y / 2) + y / 2) * (X / 2) + x / 2;
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(gout + vc * C + 8 * gq));
        const unsigned u[4] = {q.x, q.y, q.z, q.w};
        float r[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) r[c] = 0.125f * bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1))));
        uint4* dp = reinterpret_cast<uint4*>(gin + v * cs + off + 8 * gq);
        if (mask) {
            const uint4 m = __ldg(reinterpret_cast<const uint4*>(mask + v * cs + off + 8 * gq));
            const unsigned mu[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
            for (int c = 0; c < 8; ++c)
                if (!(bf2f((unsigned short)(mu[c >> 1] >> (16 * (c & 1)))) > 0.f)) r[c] = 0.f;
        }
        if (accumulate) {
            const uint4 o = *dp;
            const unsigned ou[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
            for (int c = 0; c < 8; ++c) r[c] += bf2f((unsigned short)(ou[c >> 1] >> (16 * (c & 1))));
        }
        *dp = make_uint4(pack2(r[0], r[1]), pack2(r[2], r[3]), pack2(r[4], r[5]), pack2(r[6], r[7]));
    }
}

// nearest 2x upsample of a dense [C] coarse volume into a channel slice of the
// fine volume (X, Y, Z fine)
__global__ void k_uup(const unsigned short* __restrict__ in, int C, int X, int Y, int Z, unsigned short* __restrict__ out,
                      int cs, int off) {
    const int g8 = C / 8;
    const long long n = (long long)X * Y * Z * g8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int gq = (int)(i % g8);
        const long long v = i / g8;
        const int x = (int)(v % X), y = (int)((v / X) % Y), z = (int)(v / ((long long)X * Y));
        const long long vc = ((long long)(z / 2) * (Y / 2) + y / 2) * (X / 2) + x / 2;
        *reinterpret_cast<uint4*>(out + v * cs + off + 8 * gq) =
            __ldg(reinterpret_cast<const uint4*>(in + vc * C + 8 * gq));
    }
}

// upsample backward: gin[vc][c] = sum of the 8 fine gradients of a channel slice
__global__ void k_uup_bwd(const unsigned short* __restrict__ gout, int cs, int off, int C, int X, int Y, int Z,
                          unsigned short* __restrict__ gin) {
    const int Xc = X / 2, Yc = Y / 2, Zc = Z / 2, g8 = C / 8;
    const long long n = (long long)Xc * Yc * Zc * g8;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int gq = (int)(i % g8);
        const long long vc = i / g8;
        const int x = (int)(vc % Xc), y = (int)((vc / Xc) % Yc), z = (int)(vc / ((long long)Xc * Yc));
        float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int d = 0; d < 8; ++d) {
            const long long v = ((long long)(2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X + 2 * x + (d & 1);
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(gout + v * cs + off + 8 * gq));
            const unsigned u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
            for (int c = 0; c < 8; ++c) s[c] += bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1))));
        }
        *reinterpret_cast<uint4*>(gin + vc * C + 8 * gq) =
            make_uint4(pack2(s[0], s[1]), pack2(s[2], s[3]), pack2(s[4], s[5]), pack2(s[6], s[7]));
    }
}

// out[c] += sum_v g[v][off + c] (bias gradients); block = (C / 8) x 32 threads,
// thread (row, group) sums 8 channels over a strided set of voxels
__global__ void k_uchan_sum(const unsigned short* __restrict__ g, int cs, int off, int C, long long n,
                            float* __restrict__ out) {
    extern __shared__ float red[];  // [32][C]
    const int g8 = C / 8, gq = threadIdx.x % g8, row = threadIdx.x / g8;
    float s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long v = (long long)blockIdx.x * 32 + row; v < n; v += (long long)gridDim.x * 32) {
        const uint4 q = __ldg(reinterpret_cast<const uint4*>(g + v * cs + off + 8 * gq));
        const unsigned u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int c = 0; c < 8; ++c) s[c] += bf2f((unsigned short)(u[c >> 1] >> (16 * (c & 1))));
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) red[row * C + 8 * gq + c] = s[c];
    __syncthreads();
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        float t = 0.f;
        for (int r = 0; r < 32; ++r) t += red[r * C + c];
        atomicAdd(out + c, t);
    }
}

// sums of x and x^2 over n values (FP64, one atomic add per block and sum)
__global__ void __launch_bounds__(256) k_umoments(const float* __restrict__ x, long long n, double* __restrict__ s) {
    __shared__ double red[2][8];
    double a = 0.0, b = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double v = x[i];
        a += v;
        b += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double t = 0.0;
        for (int k = 0; k < 8; ++k) t += red[threadIdx.x][k];
        atomicAdd(s + threadIdx.x, t);
    }
}

// out = (x - mean) / std from the sums (std 0 -> 1)
__global__ void k_uaffine(const float* __restrict__ x, long long n, const double* __restrict__ s,
                          float* __restrict__ out) {
    const double mean = s[0] / (double)n;
    const double var = s[1] / (double)n - mean * mean;
    const float m = (float)mean, r = var > 0.0 ? (float)(1.0 / sqrt(var)) : 1.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (x[i] - m) * r;
}

// 2 x 2 x 2 mean of an FP32 volume (even edges) into the half-size volume
__global__ void k_ubin2(const float* __restrict__ in, int X, int Y, int Z, float* __restrict__ out) {
    const int Xc = X / 2, Yc = Y / 2, Zc = Z / 2;
    const long long n = (long long)Xc * Yc * Zc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Xc), y = (int)((i / Xc) % Yc), z = (int)(i / ((long long)Xc * Yc));
        float s = 0.f;
#pragma unroll
        for (int d = 0; d < 8; ++d)
            s += __ldg(in + ((long long)(2 * z + (d >> 2)) * Y + 2 * y + ((d >> 1) & 1)) * X + 2 * x + (d & 1));
        out[i] = 0.125f * s;
    }
}

// features at P voxels, as the dense layer's F[c][p] (FP32)
__global__ void k_ugather(const unsigned short* __restrict__ f, int C, const long long* __restrict__ idx, int P,
                          float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    const int p = i / C, c = i - p * C;
    out[(long long)c * P + p] = bf2f(f[idx[p] * C + c]);
}

// gf[idx[p]][c] += g[c][p] (f[idx[p]][c] > 0) (distinct voxels; f: the ReLU
// features whose derivative masks the gradient)
__global__ void k_uscatter_add(const float* __restrict__ g, int C, const long long* __restrict__ idx, int P,
                               const unsigned short* __restrict__ f, unsigned short* __restrict__ gf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * C) return;
    const int p = i / C, c = i - p * C;
    const long long o = idx[p] * C + c;
    if (!(bf2f(f[o]) > 0.f)) return;
    gf[o] = f2bf(bf2f(gf[o]) + g[(long long)c * P + p]);
}

// channels-last BF16 map of a channel slice: dims {C, X, Y, Z}, box {8, bx, by, 1}
bool encode_cl_map(CUtensorMap* map, const void* base, int C, int cs, int X, int Y, int Z, int bx, int by) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
    const cuuint64_t strides[3] = {(cuuint64_t)cs * 2, (cuuint64_t)cs * 2 * X, (cuuint64_t)cs * 2 * X * Y};
    const cuuint32_t box[4] = {8, (cuuint32_t)bx, (cuuint32_t)by, 1}, estr[4] = {1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int COUT>
cudaError_t launch_uconv(const CUtensorMap& tm, const ConvArgs& a, cudaStream_t st) {
    constexpr int NST = 4;
    constexpr int STG = 2 * HSLOT + 9 * 2 * COUT * 16;
    const size_t smem = 1024 + (size_t)NST * STG + sizeof(unsigned long long) * (2 * NST + 1) + 2 * sizeof(int);
    cudaError_t e = cudaFuncSetAttribute(k_uconv_tc<COUT, NST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return e;
    const int tiles = ((a.X + UX - 1) / UX) * ((a.Y + UY - 1) / UY);
    dim3 g(tiles, a.Z);
    k_uconv_tc<COUT, NST><<<g, 128, smem, st>>>(tm, a);
    return cudaGetLastError();
}

int grid_for(long long n, int block) {
    long long g = (n + block - 1) / block;
    return (int)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

bool ch_ok(int c) { return c > 0 && c % 16 == 0 && c <= 96; }
bool slice_ok(int cs, int off, int c) { return cs % 8 == 0 && off % 8 == 0 && off >= 0 && off + c <= cs; }
bool dims3_ok(const int d[3]) { return d && d[0] > 0 && d[1] > 0 && d[2] > 0; }

}  // namespace

}  // namespace tg

using namespace tg;

extern "C" {

int tomgpu_unet_pack_weights_dev(tomgpu_ctx* ctx, const float* w, int cout, int cin, int flip, uint16_t* packed) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!w || !packed || !ch_ok(cout) || !ch_ok(cin)) return fail(ctx, TOMGPU_ERR_ARG, "bad weight packing arguments");
    TG_TRY(use_device(ctx));
    ctx->launches += 1;
    k_upack<<<grid_for(27ll * cout * cin, 256), 256, 0, ctx->stream>>>(w, cout, cin, flip, packed);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    return TOMGPU_OK;
}

int tomgpu_unet_conv3_dev(tomgpu_ctx* ctx, const uint16_t* in, int in_cs, int in_off, int cin, const int dims[3],
                          const uint16_t* packed, int cout, const float* bias, int relu, const uint16_t* mask,
                          int mask_cs, int mask_off, uint16_t* out, int out_cs, int out_off) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !packed || !out || !dims3_ok(dims) || !ch_ok(cin) || !slice_ok(in_cs, in_off, cin) ||
        !slice_ok(out_cs, out_off, cout) || (mask && !slice_ok(mask_cs, mask_off, cout)))
        return fail(ctx, TOMGPU_ERR_ARG, "bad convolution arguments");
    if (cout != 16 && cout != 32 && cout != 48 && cout != 64 && cout != 96)
        return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "output channels must be 16, 32, 48, 64 or 96");
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(packed) |
         reinterpret_cast<uintptr_t>(mask)) & 15)
        return fail(ctx, TOMGPU_ERR_ARG, "buffers must be 16-byte aligned");
    TG_TRY(use_device(ctx));
    CUtensorMap tm;
    if (!encode_cl_map(&tm, in + in_off, cin, in_cs, dims[0], dims[1], dims[2], HX, HY))
        return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "tensor map refused for this volume");
    ConvArgs a{dims[0], dims[1], dims[2], cin, reinterpret_cast<const unsigned char*>(packed), bias, relu,
               reinterpret_cast<unsigned short*>(out), out_cs, out_off,
               reinterpret_cast<const unsigned short*>(mask), mask_cs, mask_off, ctx->d_err};
    cudaError_t e;
    switch (cout) {
        case 16: e = launch_uconv<16>(tm, a, ctx->stream); break;
        case 32: e = launch_uconv<32>(tm, a, ctx->stream); break;
        case 48: e = launch_uconv<48>(tm, a, ctx->stream); break;
        case 64: e = launch_uconv<64>(tm, a, ctx->stream); break;
        default: e = launch_uconv<96>(tm, a, ctx->stream); break;
    }
    TG_TRY_CUDA(ctx, e);
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_conv3_wgrad_dev(tomgpu_ctx* ctx, const uint16_t* in, int in_cs, int in_off, int cin,
                                const int dims[3], const uint16_t* gout, int g_cs, int g_off, int cout, float* gw) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !gout || !gw || !dims3_ok(dims) || !ch_ok(cin) || !ch_ok(cout) || cout > 64 ||
        !slice_ok(in_cs, in_off, cin) || !slice_ok(g_cs, g_off, cout))
        return fail(ctx, TOMGPU_ERR_ARG, "bad weight-gradient arguments");
    if ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(gout)) & 15)
        return fail(ctx, TOMGPU_ERR_ARG, "buffers must be 16-byte aligned");
    TG_TRY(use_device(ctx));
    CUtensorMap tin, tdy;
    if (!encode_cl_map(&tin, in + in_off, cin, in_cs, dims[0], dims[1], dims[2], HX, HY) ||
        !encode_cl_map(&tdy, gout + g_off, cout, g_cs, dims[0], dims[1], dims[2], UX, UY))
        return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "tensor map refused for this volume");
    const int group_taps = cin <= 48 ? 9 : 3, groups = 27 / group_taps;
    const int ntiles = ((dims[0] + UX - 1) / UX) * ((dims[1] + UY - 1) / UY) * dims[2];
    int splits = 148 / groups;
    if (splits < 1) splits = 1;
    if (splits > ntiles) splits = ntiles;
    // the stages, the span of the last stage's operand rows, the barriers; at
    // least 116 KB, more than half the SM's shared memory, so one block (512
    // TMEM columns) per SM
    size_t smem = 1024 + (size_t)wg_span(wg_stage(cin, cout)) + 256;
    if (smem < 116 * 1024) smem = 116 * 1024;
    TG_TRY_CUDA(ctx, cudaFuncSetAttribute(k_uconv_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    WgArgs a{dims[0], dims[1], dims[2], cin, cout, group_taps, gw, ctx->d_err};
    k_uconv_wgrad_tc<<<dim3(splits, groups), 128, smem, ctx->stream>>>(tin, tdy, a);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_conv_first_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], const float* w, const float* b,
                               uint16_t* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!vol || !w || !out || !dims3_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "bad first-layer arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    k_uconv_first<<<grid_for(n, 256), 256, 0, ctx->stream>>>(vol, dims[0], dims[1], dims[2], w, b,
                                                             reinterpret_cast<unsigned short*>(out));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_conv_first_wgrad_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], const uint16_t* gout,
                                     float* gw, float* gb) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!vol || !gout || !gw || !dims3_ok(dims)) return fail(ctx, TOMGPU_ERR_ARG, "bad first-layer arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    long long blocks = (n + 511) / 512;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_uconv_first_wgrad<<<(int)blocks, 448, 0, ctx->stream>>>(vol, dims[0], dims[1], dims[2],
                                                               reinterpret_cast<const unsigned short*>(gout), gw, gb);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_head_dev(tomgpu_ctx* ctx, const uint16_t* f, int64_t n, const float* w, int prob, float* logit) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!f || !w || !logit || n < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad head arguments");
    TG_TRY(use_device(ctx));
    k_uhead<<<grid_for(n, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(f), n, w, prob,
                                                       logit);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_head_bwd_dev(tomgpu_ctx* ctx, const uint16_t* f, int64_t n, const float* w, const float* g,
                             uint16_t* gf, float* gw) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!f || !w || !g || !gf || !gw || n < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad head arguments");
    TG_TRY(use_device(ctx));
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_uhead_bwd<<<(int)blocks, 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(f), n, w, g,
                                                       reinterpret_cast<unsigned short*>(gf), gw);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_pool_dev(tomgpu_ctx* ctx, const uint16_t* in, int cs, int off, int C, const int dims[3],
                         uint16_t* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !out || !dims3_ok(dims) || dims[0] % 2 || dims[1] % 2 || dims[2] % 2 || C % 8 || !slice_ok(cs, off, C))
        return fail(ctx, TOMGPU_ERR_ARG, "bad pooling arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2] / 8 * (C / 8);
    k_upool<<<grid_for(n, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(in), cs, off, C,
                                                       dims[0], dims[1], dims[2],
                                                       reinterpret_cast<unsigned short*>(out));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_pool_bwd_dev(tomgpu_ctx* ctx, const uint16_t* gout, int C, const int dims[3], const uint16_t* mask,
                             int cs, int off, uint16_t* gin, int accumulate) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!gout || !gin || !dims3_ok(dims) || dims[0] % 2 || dims[1] % 2 || dims[2] % 2 || C % 8 ||
        !slice_ok(cs, off, C))
        return fail(ctx, TOMGPU_ERR_ARG, "bad pooling arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2] * (C / 8);
    k_upool_bwd<<<grid_for(n, 256), 256, 0, ctx->stream>>>(
        reinterpret_cast<const unsigned short*>(gout), C, dims[0], dims[1], dims[2],
        reinterpret_cast<const unsigned short*>(mask), cs, off, reinterpret_cast<unsigned short*>(gin), accumulate);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_upsample_dev(tomgpu_ctx* ctx, const uint16_t* in, int C, const int dims[3], uint16_t* out, int cs,
                             int off) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!in || !out || !dims3_ok(dims) || dims[0] % 2 || dims[1] % 2 || dims[2] % 2 || C % 8 || !slice_ok(cs, off, C))
        return fail(ctx, TOMGPU_ERR_ARG, "bad upsampling arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2] * (C / 8);
    k_uup<<<grid_for(n, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(in), C, dims[0], dims[1],
                                                     dims[2], reinterpret_cast<unsigned short*>(out), cs, off);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_upsample_bwd_dev(tomgpu_ctx* ctx, const uint16_t* gout, int cs, int off, int C, const int dims[3],
                                 uint16_t* gin) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!gout || !gin || !dims3_ok(dims) || dims[0] % 2 || dims[1] % 2 || dims[2] % 2 || C % 8 ||
        !slice_ok(cs, off, C))
        return fail(ctx, TOMGPU_ERR_ARG, "bad upsampling arguments");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2] / 8 * (C / 8);
    k_uup_bwd<<<grid_for(n, 256), 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(gout), cs, off, C,
                                                         dims[0], dims[1], dims[2],
                                                         reinterpret_cast<unsigned short*>(gin));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_channel_sum_dev(tomgpu_ctx* ctx, const uint16_t* g, int cs, int off, int C, int64_t n, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!g || !out || n < 1 || C < 8 || C % 8 || C > 96 || !slice_ok(cs, off, C))
        return fail(ctx, TOMGPU_ERR_ARG, "bad channel-sum arguments");
    TG_TRY(use_device(ctx));
    long long blocks = (n + 31) / 32;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_uchan_sum<<<(int)blocks, (C / 8) * 32, sizeof(float) * 32 * C, ctx->stream>>>(
        reinterpret_cast<const unsigned short*>(g), cs, off, C, n, out);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_normalise_dev(tomgpu_ctx* ctx, const float* vol, int64_t n, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!vol || !out || n < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad normalisation arguments");
    TG_TRY(use_device(ctx));
    TG_TRY(ensure_scratch(ctx, 2 * sizeof(double)));
    double* s = static_cast<double*>(ctx->scratch);
    TG_TRY_CUDA(ctx, cudaMemsetAsync(s, 0, 2 * sizeof(double), ctx->stream));
    k_umoments<<<grid_for(n, 256), 256, 0, ctx->stream>>>(vol, n, s);
    k_uaffine<<<grid_for(n, 256), 256, 0, ctx->stream>>>(vol, n, s, out);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return TOMGPU_OK;
}

int tomgpu_unet_bin2_dev(tomgpu_ctx* ctx, const float* vol, const int dims[3], float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!vol || !out || !dims3_ok(dims) || dims[0] % 2 || dims[1] % 2 || dims[2] % 2)
        return fail(ctx, TOMGPU_ERR_ARG, "bad binning arguments (even edges)");
    TG_TRY(use_device(ctx));
    const long long n = (long long)dims[0] * dims[1] * dims[2] / 8;
    k_ubin2<<<grid_for(n, 256), 256, 0, ctx->stream>>>(vol, dims[0], dims[1], dims[2], out);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_gather_dev(tomgpu_ctx* ctx, const uint16_t* f, int C, const int64_t* idx, int P, float* out) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!f || !idx || !out || C < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad gather arguments");
    TG_TRY(use_device(ctx));
    k_ugather<<<(P * C + 255) / 256, 256, 0, ctx->stream>>>(reinterpret_cast<const unsigned short*>(f), C,
                                                            reinterpret_cast<const long long*>(idx), P, out);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

int tomgpu_unet_scatter_add_dev(tomgpu_ctx* ctx, const float* g, int C, const int64_t* idx, int P, const uint16_t* f,
                                uint16_t* gf) {
    if (!ctx) return TOMGPU_ERR_ARG;
    if (!g || !idx || !f || !gf || C < 1 || P < 1) return fail(ctx, TOMGPU_ERR_ARG, "bad scatter arguments");
    TG_TRY(use_device(ctx));
    k_uscatter_add<<<(P * C + 255) / 256, 256, 0, ctx->stream>>>(g, C, reinterpret_cast<const long long*>(idx), P,
                                                                 reinterpret_cast<const unsigned short*>(f),
                                                                 reinterpret_cast<unsigned short*>(gf));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    return TOMGPU_OK;
}

}  // extern "C"
