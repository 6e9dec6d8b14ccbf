// Inverse z-DFT of the FLCF search (z edge 256) with its two radix-16 stages
// as tcgen05 tensor-core contractions (sm_100a).
//
// The pass turns Q[b][kx][kz][y] into H[b][kx][z][y] for every (b, kx, y):
// the inverse 256-point DFT along kz of the spectrum product
// (search/tom_os3_corr.m:153, the z part of ifftn).  With kz = k1 + 16 k2 and
// z = q + 16 m,
//   Y[k1][q] = sum_k2 X[k1 + 16 k2] W16^(-q k2)         (stage A)
//   x[q + 16 m] = sum_k1 (Y[k1][q] W256^(-q k1)) W16^(-m k1)   (stage B)
// and each stage is, for a block of 16 consecutive y, one real matrix product
//   D[256 rows x 32] = A[256 x 32] . F[32 x 32]
// with the 16-point inverse DFT matrix F expanded to real 2 x 2 blocks
// (interleaved re / im along K and N), rows (k1, y) in stage A and (q, y) in
// stage B, issued as kind::tf32 MMAs of M = 128, N = 32, K = 8 from shared
// memory descriptors into a 64-column TMEM accumulator.
//
// Precision: each FP32 operand is split into TF32 hi + lo (x = hi + lo
// exactly, lo rounded to TF32 again) and the product summed as
// hi.Fhi + hi.Flo + lo.Fhi with FP32 accumulation, which keeps the stage
// within a few FP32 ulps of the exact DFT (the lo.lo term is below 2^-21 of
// the product).  The twiddle multiply between the stages runs in FP32 on the
// CUDA cores while the data moves from TMEM back into the stage-B operand.
//
// Block: 256 threads; thread t owns row t of both stages (its loads, its
// TMEM lane for tcgen05.ld and its stores), so every global access moves
// 128-byte rows of y and every shared-memory store of an operand row is
// conflict-free.  Operands use the no-swizzle K-major canonical layout: core
// matrices of 8 rows x 16 bytes, rows 16 bytes apart, 8-row groups 128 bytes
// apart (SBO), 16-byte K chunks 4096 bytes apart (LBO; 256 rows).
//
// Waits on the MMA-completion mbarrier are bounded; on a timeout the block
// sets the context's device error word, releases its TMEM and returns.
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "match.h"
#include "twiddles.h"

namespace tg {

namespace {

constexpr int TZ_ROWS = 256;                 // operand rows (two M = 128 groups)
constexpr int TZ_OPB = TZ_ROWS * 32 * 4;     // bytes of one TF32 operand (256 x 32)
constexpr int TZ_FB = 32 * 32 * 4;           // bytes of one DFT-matrix operand (32 x 32)
constexpr long long TZ_WAIT_LIMIT = 1ll << 20;
// instruction descriptor: D F32, A and B TF32, both K-major, N = 32, M = 128
constexpr unsigned TZ_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle, K-major (version 1: sm_100)
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
    return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
           ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(unsigned d_tmem, unsigned long long a, unsigned long long b, unsigned acc) {
    const unsigned z = 0;
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(TZ_IDESC), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ float tf32_round(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// 32 consecutive FP32 TMEM columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// write element pair (k-chunk half h of chunk kb, row r) of a K-major operand: 8 bytes
__device__ __forceinline__ void put2(unsigned char* op, int kb, int r, int h, float a, float b) {
    *reinterpret_cast<float2*>(op + ((kb * TZ_ROWS + r) << 4) + (h << 3)) = make_float2(a, b);
}

// One stage: D[256 x 32] = A . F with A = Ahi + Alo, F = Fhi + Flo (three
// products per K step), rows 0-127 into TMEM columns 0-31, rows 128-255 into
// columns 32-63.  Issued by one thread; completion arrives on bar.
__device__ __forceinline__ void issue_stage(unsigned tmem, unsigned a_hi, unsigned a_lo, unsigned f_hi, unsigned f_lo,
                                            unsigned bar) {
#pragma unroll
    for (int g = 0; g < 2; ++g) {
        const unsigned d = tmem + 32u * g;
#pragma unroll
        for (int ks = 0; ks < 4; ++ks) {
            // K step of 8 TF32 = two 16-byte chunks: chunk 2 ks at 4096-byte (A) / 512-byte (F) spacing
            const unsigned ao = (unsigned)(2 * ks * TZ_ROWS * 16 + g * 128 * 16), fo = (unsigned)(2 * ks * 32 * 16);
            const unsigned long long ah = smem_desc(a_hi + ao, TZ_ROWS * 16, 128);
            const unsigned long long al = smem_desc(a_lo + ao, TZ_ROWS * 16, 128);
            const unsigned long long fh = smem_desc(f_hi + fo, 32 * 16, 128);
            const unsigned long long fl = smem_desc(f_lo + fo, 32 * 16, 128);
            mma_tf32(d, ah, fh, ks > 0 ? 1u : 0u);
            mma_tf32(d, ah, fl, 1u);
            mma_tf32(d, al, fh, 1u);
        }
    }
    mma_commit(bar);
}

__global__ void __launch_bounds__(256) k_inv_z_tc256(const float2* __restrict__ Q, float2* __restrict__ H, int Ny,
                                                     int nh1, const float* __restrict__ fmat,
                                                     const float2* __restrict__ tw_g, int* __restrict__ err) {
    constexpr int NZ = 256;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* a_hi = smem_raw;                  // [8 chunks][256 rows][16 B]
    unsigned char* a_lo = a_hi + TZ_OPB;
    unsigned char* f_hi = a_lo + TZ_OPB;             // [8 chunks][32 rows][16 B]
    unsigned char* f_lo = f_hi + TZ_FB;
    float2* tw = reinterpret_cast<float2*>(f_lo + TZ_FB);  // [k1][q]: W256^(+q k1)
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(tw + 256);
    unsigned* tmem_slot = reinterpret_cast<unsigned*>(bar + 1);
    int* flag = reinterpret_cast<int*>(tmem_slot + 1);
    const int tid = threadIdx.x, warp = tid >> 5;
    // once a block of this launch has timed out, the rest return at once (one
    // read, shared, so the whole block decides alike)
    __shared__ int skip_block;
    if (threadIdx.x == 0) skip_block = err && *reinterpret_cast<volatile int*>(err);
    __syncthreads();
    if (skip_block) return;
    const int k1 = tid >> 4, yl = tid & 15;  // stage A row (k1, y); stage B row (q = k1, y)
    const int y = blockIdx.x * 16 + yl, kx = blockIdx.y, b = blockIdx.z;
    const bool ok = y < Ny;
    const long long base = ((long long)b * nh1 + kx) * NZ * Ny;
    // this thread's 16 inputs X[k1 + 16 k2][y]: loads first, the set-up overlaps them
    float2 x[16];
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) x[k2] = ok ? Q[base + (long long)(k1 + 16 * k2) * Ny + y] : make_float2(0.f, 0.f);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(smem_u32(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        *flag = 0;
    }
    // the DFT matrix operands (hi and lo, built on the host) and the twiddles
    for (int i = tid; i < 2 * TZ_FB / 16; i += 256)
        reinterpret_cast<float4*>(f_hi)[i] = __ldg(reinterpret_cast<const float4*>(fmat) + i);
    for (int i = tid; i < 256; i += 256) {
        const int a = i >> 4, q = i & 15;
        tw[i] = cconj(__ldg(tw_g + a * q));
    }
    // stage A operand: row tid, K = (k2, re / im)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float h[4], l[4];
        const float in[4] = {x[2 * c].x, x[2 * c].y, x[2 * c + 1].x, x[2 * c + 1].y};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            h[e] = tf32_round(in[e]);
            l[e] = tf32_round(in[e] - h[e]);
        }
        *reinterpret_cast<float4*>(a_hi + ((c * TZ_ROWS + tid) << 4)) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(a_lo + ((c * TZ_ROWS + tid) << 4)) = make_float4(l[0], l[1], l[2], l[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tmem_slot;
    const unsigned sbar = smem_u32(bar);
    // this thread's TMEM lane and column block
    const unsigned taddr = tmem + ((unsigned)(32 * (warp & 3)) << 16) + 32u * (unsigned)(warp >> 2);
    float d[32];
    for (int stage = 0; stage < 2; ++stage) {
        if (tid == 0) {
            issue_stage(tmem, smem_u32(a_hi), smem_u32(a_lo), smem_u32(f_hi), smem_u32(f_lo), sbar);
            bool done = false;
            for (long long i = 0; i < TZ_WAIT_LIMIT && !done; ++i) done = mbar_try_wait(sbar, (unsigned)stage);
            if (!done) *flag = 1;
        }
        __syncthreads();
        if (*flag) break;
        (void)mbar_try_wait(sbar, (unsigned)stage);  // every thread observes the completed phase
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tmem_ld32(taddr, d);
        if (stage == 1) break;
        // twiddle W256^(+q k1) and the stage B operand: row (q, y), K = (k1, re / im)
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float2 v = cmul(make_float2(d[2 * q], d[2 * q + 1]), tw[k1 * 16 + q]);
            const float hr = tf32_round(v.x), hi = tf32_round(v.y);
            const int r = q * 16 + yl;
            put2(a_hi, k1 >> 1, r, k1 & 1, hr, hi);
            put2(a_lo, k1 >> 1, r, k1 & 1, tf32_round(v.x - hr), tf32_round(v.y - hi));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    const bool failed = *flag != 0;
    if (!failed && ok) {
        // row (q = k1, y): x[q + 16 m] for m = 0..15
#pragma unroll
        for (int m = 0; m < 16; ++m) H[base + (long long)(k1 + 16 * m) * Ny + y] = make_float2(d[2 * m], d[2 * m + 1]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem));
    }
    if (failed && tid == 0) tg_flag_error(err, TG_DEV_TIMEOUT);
}

// The real 32 x 32 operand F of the 16-point inverse DFT, K-major core-matrix
// layout [chunk (4 K values)][n][4], hi then lo: F[k][n] with k = (k2, re/im),
// n = (q, re/im): W = exp(+2 pi i q k2 / 16).
const float* dft16_operand() {
    static const float* dev[64] = {};
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= 64) return nullptr;
    if (dev[d]) return dev[d];
    float F[32][32];  // [k][n]
    for (int k2 = 0; k2 < 16; ++k2)
        for (int q = 0; q < 16; ++q) {
            const int e = (q * k2) % 16;
            const double a = 6.283185307179586476925286766559 * e / 16.0;
            const double c = e == 4 || e == 12 ? 0.0 : std::cos(a), s = e == 0 || e == 8 ? 0.0 : std::sin(a);
            F[2 * k2][2 * q] = (float)c;
            F[2 * k2 + 1][2 * q] = (float)-s;
            F[2 * k2][2 * q + 1] = (float)s;
            F[2 * k2 + 1][2 * q + 1] = (float)c;
        }
    // TF32 split on the host: keep the top 10 mantissa bits (round to nearest, ties away)
    auto tf32 = [](float v) {
        unsigned u;
        std::memcpy(&u, &v, 4);
        u = (u + 0x1000u) & 0xFFFFE000u;
        float r;
        std::memcpy(&r, &u, 4);
        return r;
    };
    std::vector<float> host(2 * 32 * 32);
    for (int k = 0; k < 32; ++k)
        for (int n = 0; n < 32; ++n) {
            const int idx = ((k >> 2) * 32 + n) * 4 + (k & 3);
            const float h = tf32(F[k][n]);
            host[idx] = h;
            host[32 * 32 + idx] = tf32(F[k][n] - h);
        }
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(float) * host.size()) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (cudaMemcpy(p, host.data(), sizeof(float) * host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(p);
        return nullptr;
    }
    dev[d] = static_cast<const float*>(p);
    return dev[d];
}

}  // namespace

cudaError_t launch_inv_z_tc256(const float2* Q, float2* H, int Ny, int nh1, int nb, int* err, cudaStream_t st) {
    const float* f = dft16_operand();
    if (!f) return cudaErrorMemoryAllocation;
    const size_t smem = 2 * TZ_OPB + 2 * TZ_FB + 256 * sizeof(float2) + 64;
    cudaError_t e = cudaFuncSetAttribute(k_inv_z_tc256, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e) return e;
    dim3 g((Ny + 15) / 16, nh1, nb);
    k_inv_z_tc256<<<g, 256, smem, st>>>(Q, H, Ny, nh1, f, twiddle_table<float2>(256), err);
    return cudaGetLastError();
}

}  // namespace tg
