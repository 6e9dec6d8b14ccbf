// x-line kernel of the FLCF search for the x edge 512 with its tiles loaded by
// the Tensor Memory Accelerator (cp.async.bulk.tensor), 1-GPU code.
//
// Same arithmetic as k_c2r_h256 (match_fast128.cu): a half-warp per x line,
// 16 lines (16 consecutive y at one z) per block, the half-spectrum unpack,
// 256 = 16 x 16 with one exchange, the running maximum over u = out/(N M) +
// kappa and the FLCF at the read-modify-write (search/tom_os3_corr.m:151-176,
// search/tom_os3_bestPeak.m:42-47).  What changes is how a rotation's tile
// (all 257 kx rows of 16 y, 128 bytes per row) reaches shared memory: instead
// of ~17 eight-byte cp.async per thread, one thread issues two tiled TMA
// loads per rotation (boxes 16 y x 1 z x 256 kx and 16 y x 1 z x 1 kx over
// H[b][kx][z][y], viewed as floats) that complete on a per-stage mbarrier.
// Three stages are in flight.  The tensor maps cover only this GPU's own H
// buffer, and no load multicasts.
//
// Shared layout of a stage: row kx at kx * 128 bytes, the 128-byte swizzle
// of the TMA placing the 16-byte chunk c of row k at chunk c ^ (k mod 8), so
// the half-warp's reads down a column (rows j + 16 k2, j = lane) fall on
// distinct banks.  After every line has read its tile, the stage holds the
// exchange (line yl at yl * 2 KB, [j][q ^ j]), then is refilled by the TMA.
//
// Per-thread constants in tensor memory: a thread's 16 unpack twiddles
// W512^k (k = j + 16 k2) and its 16 exchange twiddles W256^(q j) depend only
// on its lane in the line, so they sit in its TMEM lane (128 columns per
// block, warp w at lanes 32 (w mod 4), columns 64 (w / 4) + [0, 64)) and are
// read with tcgen05.ld, which takes 32 of a thread's 96 shared-memory
// accesses per rotation off the shared-memory pipe.
//
// Waits are bounded: a stage that does not fill within the limit sets the
// context's device error word (TOMGPU_ERR_TIMEOUT at the next synchronise),
// the block waits (bounded) for its other loads, releases its TMEM and
// returns without touching the results.
#include "ctx.h"
#include "match.h"
#include "tma_util.cuh"
#include "tmem_util.cuh"
#include "twiddles.h"
#include "warp_fft.cuh"

namespace tg {

namespace {

constexpr int CT_YT = 16;                 // lines (y) per block
constexpr int CT_STG = 3;                 // stages in flight
constexpr int CT_ROWB = 128;              // bytes per kx row: 16 y x 8 bytes
constexpr int CT_STAGE = 33792;           // 257 rows rounded up to 1 KB (swizzle atom)
constexpr unsigned CT_TX = 257u * CT_ROWB;  // bytes one stage receives
constexpr long long CT_WAIT_LIMIT = 1ll << 20;

using tgtma::smem_u32;

// NH = 256 = 16 (P) x 16 (Q), as k_c2r_h256.
__global__ void __launch_bounds__(256, 2) k_c2r_t256(const __grid_constant__ CUtensorMap tm_rows,
                                                     const __grid_constant__ CUtensorMap tm_last,
                                                     const float* __restrict__ mu0, const float* __restrict__ gam,
                                                     const double* __restrict__ tsum, int Ny, int Nz, int nb,
                                                     float inv_nm, double c_mean, double inv_m, double mu_t, int index0,
                                                     float* __restrict__ maxcc, int* __restrict__ angidx,
                                                     const float2* __restrict__ tw_h, const float2* __restrict__ tw_x,
                                                     int* __restrict__ err) {
    constexpr int NH = 256, NX = 2 * NH, P = 16, QN = 16;
    // once a block of this launch has timed out, the rest return at once (one
    // read, shared, so the whole block decides alike)
    __shared__ int skip_block;
    if (threadIdx.x == 0) skip_block = err && *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (skip_block) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // the swizzled stages need a 1 KB aligned base (the launch adds the slack)
    unsigned char* base =
        smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    float2* T = reinterpret_cast<float2*>(base + CT_STG * CT_STAGE);  // [QN][P]: W256^(+q k1) at [q][k1]
    float2* twx = T + P * QN;                                         // [NH]: W512^(+k)
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(twx + NH);
    int* flag = reinterpret_cast<int*>(bars + CT_STG);
    float* kaps = reinterpret_cast<float*>(flag + 4);  // [nb]
    const int tid = threadIdx.x, line = tid >> 4, j = tid & 15;
    const int y0 = blockIdx.x * CT_YT, z = blockIdx.y, y = y0 + line;
    for (int i = tid; i < P * QN; i += blockDim.x) {
        const int k1 = i >> 4, q = i & 15;
        T[q * P + k1] = cconj(__ldg(tw_h + (q * k1) % NH));
    }
    for (int i = tid; i < NH; i += blockDim.x) twx[i] = cconj(__ldg(tw_x + i));
    for (int b = tid; b < nb; b += blockDim.x) kaps[b] = (float)(c_mean * (tsum[b] * inv_m - mu_t));
    unsigned* tmem_slot = reinterpret_cast<unsigned*>(flag + 1);
    const int warp = tid >> 5;
    if (warp == 0) tgtm::alloc<128>(tmem_slot);
    if (tid == 0) {
        for (int s = 0; s < CT_STG; ++s) tgtma::mbar_init(smem_u32(bars + s), 1);
        *flag = 0;
        tgtma::fence_barrier_init();
        tgtma::prefetch_map(&tm_rows);
        tgtma::prefetch_map(&tm_last);
    }
    tgtm::fence_before();
    __syncthreads();
    tgtm::fence_after();
    // this thread's constants into its TMEM lane: columns [0, 32) the unpack
    // twiddles of k = j + 16 k2, [32, 64) the exchange twiddles T[q][j]
    const unsigned taddr = tgtm::lane_addr(*tmem_slot, warp, 64u * (unsigned)(warp >> 2));
    {
        float t[16];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int c = 8 * (h & 1) + i;
                const float2 w = h < 2 ? twx[j + P * c] : T[c * P + j];
                t[2 * i] = w.x;
                t[2 * i + 1] = w.y;
            }
            tgtm::st16(taddr + 16u * h, t);
        }
        tgtm::wait_st();
    }
    const unsigned sbase = smem_u32(base);
    // rotation b into stage s: rows kx 0..255, then row 256 (box edges stop at 256)
    auto issue = [&](int b, int s) {
        if (tid == 0) {
            const unsigned bar = smem_u32(bars + s), dst = sbase + (unsigned)(s * CT_STAGE);
            tgtma::mbar_expect_tx(bar, CT_TX);
            tgtma::load_4d(dst, &tm_rows, 2 * y0, z, 0, b, bar);
            tgtma::load_4d(dst + 256u * CT_ROWB, &tm_last, 2 * y0, z, 256, b, bar);
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
    if (1 < nb) issue(1, 1);
    int cur = 0;  // stage of rotation b
    for (int b = 0; b < nb; ++b) {
        const int nxt = cur == 0 ? 2 : cur - 1;  // stage of rotation b + 2
        if (b + 2 < nb) issue(b + 2, nxt);
        const unsigned bar = smem_u32(bars + cur), parity = (unsigned)((b / CT_STG) & 1);
        if (tid == 0 && !tgtma::mbar_wait_bounded(bar, parity, CT_WAIT_LIMIT)) *flag = 1;
        __syncthreads();
        if (*flag) {
            // the stage never filled: wait (bounded) for the loads still in
            // flight, report; the block leaves the loop and the results alone
            if (tid == 0) {
                tg_flag_error(err, TG_DEV_TIMEOUT);
                for (int r = b + 1; r < nb && r <= b + 2; ++r) {
                    const int s = r % CT_STG;
                    tgtma::mbar_wait_bounded(smem_u32(bars + s), (unsigned)((r / CT_STG) & 1), CT_WAIT_LIMIT);
                }
            }
            break;
        }
        (void)tgtma::mbar_test_wait(bar, parity);  // every thread observes the completed phase
        const unsigned char* st = base + cur * CT_STAGE;
        const int cy = line >> 1, hy = (line & 1) << 3;  // chunk and half of this line's y in a row
        float2 u[QN];
        float tk[16];
#pragma unroll
        for (int k2 = 0; k2 < QN; ++k2) {
            const int k = j + P * k2, kr = NH - k;
            if ((k2 & 7) == 0) tgtm::ld16(taddr + 2u * (unsigned)k2, tk);
            const float2 xa = *reinterpret_cast<const float2*>(st + k * CT_ROWB + ((cy ^ (k & 7)) << 4) + hy);
            const float2 xc =
                cconj(*reinterpret_cast<const float2*>(st + kr * CT_ROWB + ((cy ^ (kr & 7)) << 4) + hy));
            const float2 d = cmul(make_float2(tk[2 * (k2 & 7)], tk[2 * (k2 & 7) + 1]), csub(xa, xc));
            u[k2] = cadd(cadd(xa, xc), make_float2(-d.y, d.x));
        }
        __syncthreads();  // every line has read the tile: the stage takes the exchange
        tgfft::dft16<+1>(u);
        float2* xl = reinterpret_cast<float2*>(base + cur * CT_STAGE) + line * 256;
#pragma unroll
        for (int q = 0; q < QN; ++q) {
            if ((q & 7) == 0) tgtm::ld16(taddr + 32u + 2u * (unsigned)q, tk);
            xl[j * 16 + (q ^ j)] = cmul(u[q], make_float2(tk[2 * (q & 7)], tk[2 * (q & 7) + 1]));
        }
        __syncwarp();
        float2 v[P];
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) v[k1] = xl[k1 * 16 + (j ^ k1)];
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
        // the exchange writes precede the next TMA fill of this stage
        tgtma::fence_proxy_async();
        __syncthreads();
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
        const long long v = row + 2 * (j + QN * m);
        const float2 a = __ldg(reinterpret_cast<const float2*>(mu0 + v));
        const float2 g = __ldg(reinterpret_cast<const float2*>(gam + v));
        float2 cv = *reinterpret_cast<const float2*>(maxcc + v);
        int2 ci = *reinterpret_cast<const int2*>(angidx + v);
        bool ch = false;
        const float c0 = g.x != 0.f ? (bu[m][0] - a.x * mt) * g.x : 0.f;
        const float c1 = g.y != 0.f ? (bu[m][1] - a.y * mt) * g.y : 0.f;
        const int b0 = g.x != 0.f ? (int)(bb[m] & 0xFFFFu) : 0, b1 = g.y != 0.f ? (int)(bb[m] >> 16) : 0;
        if (c0 > cv.x) { cv.x = c0; ci.x = index0 + b0; ch = true; }
        if (c1 > cv.y) { cv.y = c1; ci.y = index0 + b1; ch = true; }
        if (ch) {
            *reinterpret_cast<float2*>(maxcc + v) = cv;
            *reinterpret_cast<int2*>(angidx + v) = ci;
        }
    }
}

}  // namespace

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}

bool encode_h_map(CUtensorMap* map, const void* H, int Ny, int Nz, int nh1, int nb, int yt, int rows,
                  CUtensorMapSwizzle swizzle) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)2 * Ny, (cuuint64_t)Nz, (cuuint64_t)nh1, (cuuint64_t)nb};
    const cuuint64_t strides[3] = {(cuuint64_t)8 * Ny, (cuuint64_t)8 * Ny * Nz, (cuuint64_t)8 * Ny * Nz * nh1};
    const cuuint32_t box[4] = {(cuuint32_t)(2 * yt), 1, (cuuint32_t)rows, 1}, estr[4] = {1, 1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(H), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

bool tma_c2r_available() { return tensor_map_encoder() != nullptr; }

cudaError_t launch_c2r_t256(const float2* H, const float* mu0, const float* gam, const double* tsum, int Ny, int Nz,
                            int nb, float inv_nm, double c, double inv_m, double mu_t, int index0, float* maxcc,
                            int* angidx, int* err, cudaStream_t st) {
    // the TMA coordinate along y (floats) is 2 y0 = 32 blockIdx.x: a multiple of
    // 16 bytes; strides are multiples of 16 bytes when Ny is even
    if (Ny % 2 || nb < 1 || nb > 65535) return cudaErrorInvalidValue;
    CUtensorMap tm_rows, tm_last;
    if (!encode_h_map(&tm_rows, H, Ny, Nz, 257, nb, CT_YT, 256, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_h_map(&tm_last, H, Ny, Nz, 257, nb, CT_YT, 1, CU_TENSOR_MAP_SWIZZLE_128B))
        return cudaErrorInvalidValue;
    const size_t smem = 1024 + (size_t)CT_STG * CT_STAGE + sizeof(float2) * (16 * 16 + 256) +
                        sizeof(unsigned long long) * CT_STG + 4 * sizeof(int) + sizeof(float) * nb;
    cudaError_t e = cudaFuncSetAttribute(k_c2r_t256, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return e;
    dim3 grid((Ny + CT_YT - 1) / CT_YT, Nz);
    k_c2r_t256<<<grid, 256, smem, st>>>(tm_rows, tm_last, mu0, gam, tsum, Ny, Nz, nb, inv_nm, c, inv_m, mu_t, index0,
                                        maxcc, angidx, twiddle_table<float2>(256), twiddle_table<float2>(512), err);
    return cudaGetLastError();
}

}  // namespace tg
