// Batched subtomogram alignment as one fused pipeline per box edge
// (tom_av3_align, av3_new/tom_av3_align.m:97-189, with tom_corr 'norm' of
// Analysis/tom_corr.m:51-121 in the scan).
//
// The jobs of a call that share a cubic box edge N and the wedge form make one
// stream of entries, an entry being one (particle, Euler triplet) pair of a
// particle's scan in the reference's loop order (phi outer, psi, theta inner).
// Batches of entries run through seven kernels, each one pass over the batch's
// half spectra, held as [entry][kx][z][y] (kx <= N/2, y fastest):
//
//   x1  rot(ref) * mask (rot3d's trilinear arithmetic), forward x-DFT    -> A
//   pa  per (entry, kx) plane: forward y and z DFTs, times the Hermitian
//       part of the particle's wedge (the spectrum of psf_part), inverse
//       z and y DFTs                                                   A -> A
//   x2  inverse x-DFT (complex-to-real), the sums of the result inside the
//       mask, times the mask indicator, forward x-DFT                  A -> A
//   pb  per plane: F(part * mask) times the Hermitian part of the rotated
//       reference wedge, inverse z and y DFTs                            -> B
//   x2  the same on B                                                  B -> B
//   pc  per plane: forward y and z DFTs of A and of B, each normalised in
//       Fourier space, (F(x i) - mean F(i)) / std = F(norm_inside_mask(x))
//       with i the mask indicator; C = F(b) conj F(a); inverse z, y    -> B
//   x3  inverse x-DFT of C, / the mask size, fftshift, running maximum and
//       angle index over a group of consecutive entries          B -> partial
//
// and a merge of the groups' partial maxima, in scan order, into the
// particle's running maximum and angle index volumes.  Without wedges the
// a-side is rot(ref) normalised inside the mask and the b-side the particle
// normalised once (tom_corr 'norm' without psfs): x1 keeps the sums and pc
// multiplies by the particle's normalised spectrum.
//
// Every line DFT runs in shared memory on a tile of N lines of pitch N + 1
// (odd) with the threads of a warp on consecutive lines, so the strided
// z-lines of a plane and the contiguous lines alike touch 16 distinct bank
// pairs per 64-bit wavefront; each Stockham stage loads all of a thread's
// butterflies, waits at a barrier and stores them, so the tile is
// transformed in place.  The reference and its wedge are read through brick
// volumes (the eight trilinear corners of a voxel in two float4).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "fft_engine.cuh"
#include "match.h"
#include "rotate_sample.cuh"
#include "twiddles.h"
#include "wedge_pair.cuh"

namespace tg {

namespace {

template <int NT_, int MINB_, int NTX_, int MINBX_, typename R_> struct CfgOf {
    static constexpr int NT = NT_, MINB = MINB_, NTX = NTX_, MINBX = MINBX_;
    typedef R_ R;
};

// Per box edge: threads per block, blocks per SM the registers are sized for
// (every butterfly of a stage lives in registers, N * N / NT elements per
// thread), and the radices of the line DFTs.
template <int N> struct Cfg;
// NT / MINB: the (y, z)-plane kernels and the full x3 (N lines per tile);
// NTX / MINBX: the x-line kernels, which pack two real lines into one complex
// line (N / 2 lines per tile).
template <> struct Cfg<24> : CfgOf<192, 4, 96, 8, tgfft::seq<8, 3>> {};
template <> struct Cfg<32> : CfgOf<256, 4, 128, 8, tgfft::seq<8, 4>> {};
template <> struct Cfg<40> : CfgOf<320, 3, 160, 6, tgfft::seq<8, 5>> {};
template <> struct Cfg<48> : CfgOf<160, 6, 192, 6, tgfft::seq<16, 3>> {};
template <> struct Cfg<64> : CfgOf<256, 4, 256, 4, tgfft::seq<8, 8>> {};
template <> struct Cfg<72> : CfgOf<384, 2, 352, 3, tgfft::seq<8, 3, 3>> {};
template <> struct Cfg<80> : CfgOf<256, 3, 224, 5, tgfft::seq<16, 5>> {};
template <> struct Cfg<96> : CfgOf<384, 2, 288, 4, tgfft::seq<16, 6>> {};
template <> struct Cfg<56> : CfgOf<448, 2, 224, 5, tgfft::seq<8, 7>> {};
template <> struct Cfg<100> : CfgOf<512, 1, 320, 3, tgfft::seq<4, 5, 5>> {};
template <> struct Cfg<112> : CfgOf<800, 1, 416, 2, tgfft::seq<16, 7>> {};
template <> struct Cfg<120> : CfgOf<960, 1, 480, 2, tgfft::seq<8, 3, 5>> {};
template <> struct Cfg<128> : CfgOf<1024, 1, 512, 2, tgfft::seq<16, 8>> {};

constexpr int kEdges[] = {24, 32, 40, 48, 56, 64, 72, 80, 96, 100, 112, 120, 128};

// whole warps only: the kernels' warp shuffles name all 32 lanes
template <int N> constexpr bool whole_warps() { return Cfg<N>::NT % 32 == 0 && Cfg<N>::NTX % 32 == 0; }
static_assert(whole_warps<24>() && whole_warps<32>() && whole_warps<40>() && whole_warps<48>() &&
                  whole_warps<56>() && whole_warps<64>() && whole_warps<72>() && whole_warps<80>() &&
                  whole_warps<96>() && whole_warps<100>() && whole_warps<112>() && whole_warps<120>() &&
                  whole_warps<128>(),
              "block sizes must be multiples of 32");

// Particles whose data is resident at once: a batch holds at most
// kBatchParticles of them, and a particle's slot (its index mod kMaxSlots) is
// reused only after the batch that follows its last one, which is when its
// deferred final step has run.
constexpr int kMaxSlots = 16;
constexpr int kBatchParticles = 7;
constexpr int kMaxPrune = 32;   // coordinates per axis of a pruned final inverse
constexpr int kMaxGroups = 160;  // x3 entry groups per batch

// One particle's device data.
struct Slot {
    const float4* refb;   // bricks of the reference
    const float4* wrefb;  // bricks of the reference wedge (wedge form)
    const uint4* wrefh;   // the same as half bricks when every wedge value is exact in half precision
    const float* mask;
    const float2* mk;     // F(mask != 0), [kx][z][y]
    const float2* b0;     // wedge form: F(part * mask); without: F(norm_inside_mask(part))
    const float* wph;     // wedge form: Hermitian part of the particle wedge, [kx][z][y]
    float* cmax;          // running maximum of the scan
    float* amax;          // its angle index (tom_av3_angle2index, as float)
    double nmask;         // non-zero voxels of the mask
    // pruned final inverse: the unshifted z, y, x coordinates whose ccf is
    // needed (lists of nz, ny, nx at pl, pl + kMaxPrune, pl + 2 kMaxPrune) and
    // the inverse-DFT tables wy[ky][yi], wx[kx][xi] (Hermitian weights folded in)
    const int* pl;
    const float2* wy;
    const float2* wx;
    int nz, ny, nx;
};
struct SlotTab { Slot s[kMaxSlots]; };
// One (particle, rotation) entry: slot, angle index, rot3d matrix of the
// reference (tom_angles2rotmatrix) and Euler-mode matrix of its wedge.
struct Entry {
    int slot, aidx;
    float mref[9], mw[9];
};
struct Group { int slot, e0, e1; };
struct GroupTab { Group g[kMaxGroups]; int n; };
struct Seg { int slot, g0, g1; };
struct SegTab { Seg s[kMaxSlots + 1]; int n; };

// One in-place Stockham stage of radix R (NS = product of the earlier radices)
// over NL lines of length N of a tile, element e of line l at
// s[l * LST + e * EST].  Butterfly b: line b % NL, index j = b / NL.
template <int N, int NL, int R, int NS, int DIR, int NT, int EST, int LST>
TG_D void pstage(float2* s, const float2* __restrict__ tw, int tid) {
    constexpr int NBL = N / R, NB = NL * NBL, BPT = (NB + NT - 1) / NT;
    float2 v[BPT][R];
#pragma unroll
    for (int q = 0; q < BPT; ++q) {
        const int b = tid + q * NT;
        if (NB % NT == 0 || b < NB) {
            const int l = b % NL, j = b / NL;
            const float2* src = s + l * LST;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = src[(j + r * NBL) * EST];
            if (NS > 1) {
                // one table load per butterfly; the powers w^r by products
                // (a few ulp, far inside the line DFT's own rounding)
                const int k = j % NS;
                float2 w1 = tgfft::ldtw(tw, k * (N / (NS * R)));
                if (DIR > 0) w1 = cconj(w1);
                float2 w = w1;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    v[q][r] = cmul(v[q][r], w);
                    if (r + 1 < R) w = cmul(w, w1);
                }
            }
            tgfft::dft<R, DIR>(v[q], tw, N / R);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BPT; ++q) {
        const int b = tid + q * NT;
        if (NB % NT == 0 || b < NB) {
            const int l = b % NL, j = b / NL;
            const int k = j % NS;
            float2* dst = s + l * LST;
            const int p0 = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[(p0 + r * NS) * EST] = v[q][r];
        }
    }
    __syncthreads();
}

template <int N, int NL, int DIR, int NT, int EST, int LST, int NS, int R, int... Rest>
TG_D void pstages(float2* s, const float2* __restrict__ tw, int tid) {
    pstage<N, NL, R, NS, DIR, NT, EST, LST>(s, tw, tid);
    if constexpr (sizeof...(Rest) > 0) pstages<N, NL, DIR, NT, EST, LST, NS * R, Rest...>(s, tw, tid);
}
template <int N, int NL, int DIR, int NT, int EST, int LST, int... Rs>
TG_D void pfft_seq(float2* s, const float2* __restrict__ tw, int tid, tgfft::seq<Rs...>) {
    pstages<N, NL, DIR, NT, EST, LST, 1, Rs...>(s, tw, tid);
}
// NL lines of length N of a tile by NT threads: DIR = -1 forward, +1
// unnormalised inverse.  The caller has synchronised after filling the tile;
// ends with a barrier.
template <int N, int NL, int NT, int DIR, int EST, int LST>
TG_D void pfft_l(float2* s, const float2* __restrict__ tw, int tid) {
    pfft_seq<N, NL, DIR, NT, EST, LST>(s, tw, tid, typename Cfg<N>::R{});
}
// the N lines of a plane-sized tile by the plane kernels' NT threads
template <int N, int DIR, int EST, int LST>
TG_D void pfft(float2* s, const float2* __restrict__ tw, int tid) {
    pfft_l<N, N, Cfg<N>::NT, DIR, EST, LST>(s, tw, tid);
}

// Block sum of two doubles added to out[0], out[1] (called by every thread).
template <int NT> TG_D void block_add2(double a, double b, double* out) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    __shared__ double ws[2][NT / 32];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        ws[0][w] = a;
        ws[1][w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0, sb = 0;
        for (int k = 0; k < NT / 32; ++k) {
            sa += ws[0][k];
            sb += ws[1][k];
        }
        atomicAdd(out, sa);
        atomicAdd(out + 1, sb);
    }
}

// mean and 1/std of norm_inside_mask from the sums of x and x^2 over the
// mask's n voxels (std with n - 1)
TG_D void mean_istd(const double* st, double n, float& mu, float& is) {
    const double m = st[0] / n;
    const double var = (st[1] - st[0] * m) / (n - 1.0);
    mu = (float)m;
    is = (float)(1.0 / sqrt(var));
}

TG_D float2 norm_bin(float2 x, float2 m, float mu, float is) {
    return make_float2((x.x - mu * m.x) * is, (x.y - mu * m.y) * is);
}

// ------------------------------------------------------------- x-line passes
enum XMode {
    X_ROT_MASK = 0,   // rot(ref) * mask (wedge form)
    X_ROT_STATS = 1,  // rot(ref) with its sums inside the mask, times the indicator (no wedges)
    X_C2R_R2C = 2,    // inverse x, sums inside the mask, times the indicator, forward x
    X_IND = 3,        // set-up: the mask indicator, and its count
    X_MUL = 4,        // set-up: src * srcmask
    X_STATS = 5,      // set-up: src with its sums inside srcmask, times the indicator
};

// grid (N z-slabs, entries).  The x-lines y = 2j and 2j + 1 of the slab
// travel as one complex line Z = a + i b (tile s[j * P + x], N / 2 lines): the
// inverse DFT of H_2j + i H_2j+1 (each Hermitian-extended) is a + i b, and
// the forward DFT of a + i b gives H_2j = (Z_k + conj Z_-k) / 2 and H_2j+1 =
// (Z_k - conj Z_-k) / 2i.
template <int N, int MODE>
__global__ void __launch_bounds__(Cfg<N>::NTX, Cfg<N>::MINBX) k_ax(float2* __restrict__ H, long long hstride,
                                                   const Entry* __restrict__ ent, const __grid_constant__ SlotTab slots,
                                                   const float* __restrict__ src, const float* __restrict__ srcmask,
                                                   double* __restrict__ stats, int side,
                                                   const float2* __restrict__ tw, float inv_n3) {
    constexpr int NT = Cfg<N>::NTX, P = N + 1, NH = N / 2 + 1, NL = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int z = blockIdx.x, e = blockIdx.y, tid = threadIdx.x;
    float2* Hs = H + (long long)e * hstride;
    const long long zo = (long long)z * N * N;
    double acc0 = 0, acc1 = 0;
    if (MODE == X_C2R_R2C) {
        for (int i = tid; i < NH * NL; i += NT) {
            const int kx = i / NL, j = i - kx * NL;
            const float4 h = *reinterpret_cast<const float4*>(Hs + ((long long)kx * N + z) * N + 2 * j);
            float2 a = make_float2(h.x, h.y), b = make_float2(h.z, h.w);
            if (kx == 0 || 2 * kx == N) {  // complex-to-real reads the real parts there
                a.y = 0.f;
                b.y = 0.f;
            }
            s[j * P + kx] = make_float2(a.x - b.y, a.y + b.x);
            if (kx > 0 && 2 * kx != N) s[j * P + N - kx] = make_float2(a.x + b.y, b.x - a.y);
        }
        __syncthreads();
        pfft_l<N, NL, NT, +1, 1, P>(s, tw, tid);
        const float* mask = slots.s[ent[e].slot].mask;
        for (int i = tid; i < NL * N; i += NT) {
            const int j = i / N, x = i - j * N;
            const float2 v = s[j * P + x];
            const float r0 = v.x * inv_n3, r1 = v.y * inv_n3;
            const bool in0 = mask[zo + 2 * j * N + x] != 0.f, in1 = mask[zo + (2 * j + 1) * N + x] != 0.f;
            if (in0) {
                acc0 += (double)r0;
                acc1 += (double)r0 * (double)r0;
            }
            if (in1) {
                acc0 += (double)r1;
                acc1 += (double)r1 * (double)r1;
            }
            s[j * P + x] = make_float2(in0 ? r0 : 0.f, in1 ? r1 : 0.f);
        }
        __syncthreads();
    } else if (MODE == X_ROT_MASK || MODE == X_ROT_STATS) {
        const Entry* en = ent + e;
        const Slot& sl = slots.s[en->slot];
        float m[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) m[q] = en->mref[q];
        const float c = (float)((N + 1) / 2);
        for (int i = tid; i < NL * N; i += NT) {
            // a warp samples an 8 (x) x 8 (y) tile of the slab (two y per thread)
            // where the edge allows, else a row
            int x, j;
            if constexpr (N % 8 == 0) {
                const int lane = i & 31, t = i >> 5;
                x = (t % (N / 8)) * 8 + (lane & 7);
                j = (t / (N / 8)) * 4 + (lane >> 3);
            } else {
                j = i / N;
                x = i - j * N;
            }
            float a[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int y = 2 * j + h;
                const float mk = sl.mask[zo + y * N + x];
                // outside the mask the value is zero in both forms: no sample
                float v = mk != 0.f ? rot_sample_brick(sl.refb, N, N, N, m, c, c, c, x, y, z) : 0.f;
                if (MODE == X_ROT_MASK) {
                    v = __fmul_rn(v, mk);
                } else {
                    const bool in = mk != 0.f;
                    if (in) {
                        acc0 += (double)v;
                        acc1 += (double)v * (double)v;
                    }
                    v = in ? v : 0.f;
                }
                a[h] = v;
            }
            s[j * P + x] = make_float2(a[0], a[1]);
        }
        __syncthreads();
    } else {
        for (int i = tid; i < NL * N; i += NT) {
            const int j = i / N, x = i - j * N;
            float a[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long long vi = zo + (2 * j + h) * N + x;
                float v = src[vi];
                if (MODE == X_IND) {
                    v = v != 0.f ? 1.f : 0.f;
                    acc0 += (double)v;
                } else if (MODE == X_MUL) {
                    if (srcmask) v = v * srcmask[vi];
                } else {
                    const bool in = srcmask[vi] != 0.f;
                    if (in) {
                        acc0 += (double)v;
                        acc1 += (double)v * (double)v;
                    }
                    v = in ? v : 0.f;
                }
                a[h] = v;
            }
            s[j * P + x] = make_float2(a[0], a[1]);
        }
        __syncthreads();
    }
    pfft_l<N, NL, NT, -1, 1, P>(s, tw, tid);
    for (int i = tid; i < NH * NL; i += NT) {
        const int kx = i / NL, j = i - kx * NL;
        const float2 zk = s[j * P + kx], zm = s[j * P + (kx == 0 ? 0 : N - kx)];
        const float4 h = make_float4(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y), 0.5f * (zk.y + zm.y),
                                     0.5f * (zm.x - zk.x));
        *reinterpret_cast<float4*>(Hs + ((long long)kx * N + z) * N + 2 * j) = h;
    }
    if (MODE == X_ROT_STATS) block_add2<NT>(acc0, acc1, stats + 4 * e);
    if (MODE == X_C2R_R2C) block_add2<NT>(acc0, acc1, stats + 4 * e + 2 * side);
    if (MODE == X_IND || MODE == X_STATS) block_add2<NT>(acc0, acc1, stats);
}

// ---------------------------------------------------------- (y, z) planes
enum PMode {
    P_WEDGE_A = 0,   // A: forward y, z; times the particle wedge's Hermitian part; inverse z, y
    P_WEDGE_B = 1,   // B = F(part * mask) times the rotated wedge's Hermitian part; inverse z, y
    P_CROSS = 2,     // A, B: forward y, z, normalised; C = F(b) conj F(a) into B; inverse z, y
    P_CROSS_NW = 3,  // A: forward y, z, normalised; C = b0 conj F(a) into B; inverse z, y
    P_FWD = 4,       // set-up: forward y, z of pin into pout
    P_FWD_NORM = 5,  // set-up: forward y, z of pin, normalised with pst / pn / pmk, into pout
};

// grid (N/2 + 1 planes kx, entries); tile s[z * P + y]: y-lines at EST 1,
// LST P; z-lines at EST P, LST 1.
template <int N, int MODE>
__global__ void __launch_bounds__(Cfg<N>::NT, Cfg<N>::MINB) k_ap(float2* __restrict__ A, float2* __restrict__ B,
                                                                  long long hstride,
                                                   const Entry* __restrict__ ent, const __grid_constant__ SlotTab slots,
                                                   const double* __restrict__ stats, const float2* __restrict__ tw,
                                                   const float2* __restrict__ pin, float2* __restrict__ pout,
                                                   const float2* __restrict__ pmk, const double* __restrict__ pst,
                                                   double pn, float2* __restrict__ cp, int cpz, int cpy) {
    constexpr int NT = Cfg<N>::NT, P = N + 1, NH = N / 2 + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    const int kx = blockIdx.x, e = blockIdx.y, tid = threadIdx.x;
    const long long po = (long long)kx * N * N;
    float2* Ap = A ? A + (long long)e * hstride + po : nullptr;
    float2* Bp = B ? B + (long long)e * hstride + po : nullptr;
    if (MODE == P_WEDGE_B) {
        const Entry* en = ent + e;
        const Slot& sl = slots.s[en->slot];
        float m[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) m[q] = en->mw[q];
        const float c = (float)((N + 1) / 2);
        for (int i = tid; i < N * N; i += NT) {
            // a warp samples an 8 (y) x 4 (z) tile of the plane where the edge
            // allows (source points spanning two rotated directions), else a row
            int y, z;
            if constexpr (N % 8 == 0) {
                const int lane = i & 31, t = i >> 5;
                y = (t % (N / 8)) * 8 + (lane & 7);
                z = (t / (N / 8)) * 4 + (lane >> 3);
            } else {
                z = i / N;
                y = i - z * N;
            }
            int s1, s2;
            wedge_pair(kx + N * (y + N * z), N, N, N, s1, s2);
            float w1, w2;
            if (sl.wrefh) {
                w1 = rot_sample_brick(sl.wrefh, N, N, N, m, c, c, c, s1 % N, (s1 / N) % N, s1 / (N * N));
                w2 = rot_sample_brick(sl.wrefh, N, N, N, m, c, c, c, s2 % N, (s2 / N) % N, s2 / (N * N));
            } else {
                w1 = rot_sample_brick(sl.wrefb, N, N, N, m, c, c, c, s1 % N, (s1 / N) % N, s1 / (N * N));
                w2 = rot_sample_brick(sl.wrefb, N, N, N, m, c, c, c, s2 % N, (s2 / N) % N, s2 / (N * N));
            }
            s[z * P + y] = cscale(sl.b0[po + z * N + y], 0.5f * (w1 + w2));
        }
        __syncthreads();
    } else {
        const float2* in = (MODE == P_FWD || MODE == P_FWD_NORM) ? pin + po : Ap;
        for (int i = tid; i < N * N; i += NT) {
            const int z = i / N, y = i - z * N;
            s[z * P + y] = in[i];
        }
        __syncthreads();
        pfft<N, -1, 1, P>(s, tw, tid);
        pfft<N, -1, P, 1>(s, tw, tid);
        if (MODE == P_WEDGE_A) {
            const float* wph = slots.s[ent[e].slot].wph + po;
            for (int i = tid; i < N * N; i += NT) {
                const int z = i / N, y = i - z * N;
                s[z * P + y] = cscale(s[z * P + y], wph[i]);
            }
            __syncthreads();
        } else if (MODE == P_FWD) {
            for (int i = tid; i < N * N; i += NT) {
                const int z = i / N, y = i - z * N;
                pout[po + i] = s[z * P + y];
            }
            return;
        } else if (MODE == P_FWD_NORM) {
            float mu, is;
            mean_istd(pst, pn, mu, is);
            for (int i = tid; i < N * N; i += NT) {
                const int z = i / N, y = i - z * N;
                pout[po + i] = norm_bin(s[z * P + y], pmk[po + i], mu, is);
            }
            return;
        } else {
            // F(norm_inside_mask(a)): written to A, read back below by the same thread
            const Slot& sl = slots.s[ent[e].slot];
            float mu, is;
            mean_istd(stats + 4 * e, sl.nmask, mu, is);
            const float2* mk = sl.mk + po;
            if (MODE == P_CROSS) {
                for (int i = tid; i < N * N; i += NT) {
                    const int z = i / N, y = i - z * N;
                    Ap[i] = norm_bin(s[z * P + y], mk[i], mu, is);
                }
                __syncthreads();
                for (int i = tid; i < N * N; i += NT) {
                    const int z = i / N, y = i - z * N;
                    s[z * P + y] = Bp[i];
                }
                __syncthreads();
                pfft<N, -1, 1, P>(s, tw, tid);
                pfft<N, -1, P, 1>(s, tw, tid);
                float mub, isb;
                mean_istd(stats + 4 * e + 2, sl.nmask, mub, isb);
                for (int i = tid; i < N * N; i += NT) {
                    const int z = i / N, y = i - z * N;
                    const float2 fb = norm_bin(s[z * P + y], mk[i], mub, isb);
                    s[z * P + y] = cmulc(fb, Ap[i]);
                }
            } else {
                const float2* fb = sl.b0 + po;
                for (int i = tid; i < N * N; i += NT) {
                    const int z = i / N, y = i - z * N;
                    s[z * P + y] = cmulc(fb[i], norm_bin(s[z * P + y], mk[i], mu, is));
                }
            }
            __syncthreads();
            if (cp) {
                // pruned: inverse z-DFT, then the inverse y-DFT only at the listed
                // (z, y): four lanes per output, each a quarter of the ky sum
                pfft<N, +1, P, 1>(s, tw, tid);
                const int nzo = sl.nz, nyo = sl.ny, tot = 4 * nzo * nyo;
                const int* zl = sl.pl;
                for (int t0 = 0; t0 < tot; t0 += NT) {
                    const int t = t0 + tid, o = t >> 2, c = t & 3;
                    float2 acc = make_float2(0.f, 0.f);
                    if (t < tot) {
                        const int zi = o / nyo, yi = o - zi * nyo;
                        const float2* row = s + zl[zi] * P;
                        for (int ky = c; ky < N; ky += 4) {
                            const float2 w = __ldg(sl.wy + ky * kMaxPrune + yi);
                            const float2 v = row[ky];
                            acc.x += v.x * w.x - v.y * w.y;
                            acc.y += v.x * w.y + v.y * w.x;
                        }
                    }
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 1);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 1);
                    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, 2);
                    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, 2);
                    if (t < tot && c == 0) {
                        const int zi = o / nyo, yi = o - zi * nyo;
                        cp[(((long long)e * NH + kx) * cpz + zi) * cpy + yi] = acc;
                    }
                }
                return;
            }
        }
    }
    pfft<N, +1, P, 1>(s, tw, tid);
    pfft<N, +1, 1, P>(s, tw, tid);
    float2* out = MODE == P_WEDGE_A ? Ap : Bp;
    for (int i = tid; i < N * N; i += NT) {
        const int z = i / N, y = i - z * N;
        out[i] = s[z * P + y];
    }
}

// ------------------------------------------------ cross-correlation maxima
// grid (N z-slabs, groups): inverse x-DFT of each entry's C slab (two lines
// per complex line, as in k_ax), ccf = value / numel / nmask, running maximum
// (strict) and angle index (at >=) over the group's entries in scan order;
// written fftshifted as (max, index).
template <int N>
__global__ void __launch_bounds__(Cfg<N>::NTX, 1) k_ax3(const float2* __restrict__ Bv, long long hstride,
                                                       const Entry* __restrict__ ent,
                                                       const __grid_constant__ SlotTab slots,
                                                       const __grid_constant__ GroupTab groups,
                                                       float2* __restrict__ partial, const float2* __restrict__ tw,
                                                       float inv_n3) {
    constexpr int NT = Cfg<N>::NTX, P = N + 1, NH = N / 2 + 1, NL = N / 2, H2 = N / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* s = reinterpret_cast<float2*>(smem_raw);
    float2* mx = s + NL * P;  // [y][x] running (max, index)
    const int z = blockIdx.x, tid = threadIdx.x;
    const Group g = groups.g[blockIdx.y];
    const double inv_nm = 1.0 / slots.s[g.slot].nmask;
    for (int i = tid; i < N * N; i += NT) mx[i] = make_float2(-INFINITY, 0.f);
    for (int e = g.e0; e < g.e1; ++e) {
        const float2* Hs = Bv + (long long)e * hstride;
        for (int i = tid; i < NH * NL; i += NT) {
            const int kx = i / NL, j = i - kx * NL;
            const float4 h = *reinterpret_cast<const float4*>(Hs + ((long long)kx * N + z) * N + 2 * j);
            float2 a = make_float2(h.x, h.y), b = make_float2(h.z, h.w);
            if (kx == 0 || 2 * kx == N) {
                a.y = 0.f;
                b.y = 0.f;
            }
            s[j * P + kx] = make_float2(a.x - b.y, a.y + b.x);
            if (kx > 0 && 2 * kx != N) s[j * P + N - kx] = make_float2(a.x + b.y, b.x - a.y);
        }
        __syncthreads();
        pfft_l<N, NL, NT, +1, 1, P>(s, tw, tid);
        const float ai = (float)ent[e].aidx;
        for (int i = tid; i < NL * N; i += NT) {
            const int j = i / N, x = i - j * N;
            const float2 v = s[j * P + x];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float c = (float)((double)((h ? v.y : v.x) * inv_n3) * inv_nm);
                float2& r = mx[(2 * j + h) * N + x];
                float2 t = r;
                if (c > t.x) t.x = c;
                if (c >= t.x) t.y = ai;
                r = t;
            }
        }
        __syncthreads();
    }
    float2* out = partial + (long long)blockIdx.y * N * N * N + (long long)((z + H2) % N) * N * N;
    for (int i = tid; i < N * N; i += NT) {
        const int y = i / N, x = i - y * N;
        out[((y + H2) % N) * N + (x + H2) % N] = mx[i];
    }
}

// groups' partial maxima merged into the particle's volumes in scan order:
// a later group's (max, index) replaces the running pair where max >= it
__global__ void k_amerge(const float2* __restrict__ partial, long long nvox, const __grid_constant__ SegTab segs,
                         const __grid_constant__ SlotTab slots) {
    const Seg sg = segs.s[blockIdx.y];
    float* cm = slots.s[sg.slot].cmax;
    float* am = slots.s[sg.slot].amax;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
         v += (long long)gridDim.x * blockDim.x) {
        float m = cm[v], a = am[v];
        for (int g = sg.g0; g < sg.g1; ++g) {
            const float2 p = partial[(long long)g * nvox + v];
            if (p.x >= m) {
                m = p.x;
                a = p.y;
            }
        }
        cm[v] = m;
        am[v] = a;
    }
}

// Pruned x-DFT: grid (voxel blocks, entries); thread = one voxel of the
// entry's particle's listed (z, y, x) product: the inverse x-DFT of the
// pruned (z, y) values at x (Hermitian weights in the table), / numel /
// nmask, into V[e][voxel].
__global__ void k_ax3v(const float2* __restrict__ cp, int N, int cpz, int cpy, const Entry* __restrict__ ent,
                       const __grid_constant__ SlotTab slots, float* __restrict__ V, int vstride, float inv_n3) {
    const int e = blockIdx.y;
    const Slot& sl = slots.s[ent[e].slot];
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sl.nz * sl.ny * sl.nx) return;
    const int NH = N / 2 + 1;
    const int xi = o % sl.nx, yi = (o / sl.nx) % sl.ny, zi = o / (sl.nx * sl.ny);
    const float2* c = cp + ((long long)e * NH * cpz + zi) * cpy + yi;
    float acc = 0.f;
    for (int kx = 0; kx < NH; ++kx) {
        const float2 u = c[(long long)kx * cpz * cpy];
        const float2 w = __ldg(sl.wx + kx * kMaxPrune + xi);
        acc += u.x * w.x - u.y * w.y;
    }
    V[(long long)e * vstride + o] = (float)((double)(acc * inv_n3) * (1.0 / sl.nmask));
}

// Running maximum over the pruned values: thread = one listed voxel of a
// segment's particle; over the segment's entries in scan order the strict
// maximum and the angle index at >=, merged into the particle's volumes at
// the fftshifted voxel.
__global__ void k_ax3s(const float* __restrict__ V, int vstride, int N, const Entry* __restrict__ ent,
                       const __grid_constant__ SlotTab slots, const __grid_constant__ SegTab segs) {
    const Seg sg = segs.s[blockIdx.y];
    const Slot& sl = slots.s[sg.slot];
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sl.nz * sl.ny * sl.nx) return;
    const int H2 = N / 2;
    const int xi = o % sl.nx, yi = (o / sl.nx) % sl.ny, zi = o / (sl.nx * sl.ny);
    const int x = sl.pl[2 * kMaxPrune + xi], y = sl.pl[kMaxPrune + yi], z = sl.pl[zi];
    const long long v = (x + H2) % N + (long long)N * ((y + H2) % N) + (long long)N * N * ((z + H2) % N);
    float m = sl.cmax[v], a = sl.amax[v];
    for (int e = sg.g0; e < sg.g1; ++e) {
        const float cc = V[(long long)e * vstride + o];
        if (cc > m) m = cc;
        if (cc >= m) a = (float)ent[e].aidx;
    }
    sl.cmax[v] = m;
    sl.amax[v] = a;
}

// The coordinates the pruned inverse needs, per particle (grid: blocks,
// particles): the unshifted (z, y, x) of every voxel where mask_ccf != 0 is
// flagged; v0 receives the first voxel where mask_ccf == 0.
__global__ void k_prune_mark(const float* const* __restrict__ mccf, int N, int* __restrict__ flags,
                             unsigned long long* __restrict__ v0) {
    const float* m = mccf[blockIdx.y];
    int* f = flags + (long long)blockIdx.y * 3 * N;
    const long long nn = (long long)N * N * N;
    const int H2 = N / 2;
    unsigned long long first = ~0ull;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn;
         v += (long long)gridDim.x * blockDim.x) {
        if (m[v] != 0.f) {
            const int x = (int)(v % N), y = (int)((v / N) % N), z = (int)(v / ((long long)N * N));
            f[(z - H2 + N) % N] = 1;
            f[N + (y - H2 + N) % N] = 1;
            f[2 * N + (x - H2 + N) % N] = 1;
        } else if (first == ~0ull) {
            first = (unsigned long long)v;  // the loop runs in increasing v: the thread's first zero
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, first, o);
        first = t < first ? t : first;
    }
    if ((threadIdx.x & 31) == 0 && first != ~0ull) atomicMin(v0 + blockIdx.y, first);
}

// flags of the first zero voxel of each particle's mask_ccf
__global__ void k_prune_v0(const unsigned long long* __restrict__ v0, int N, int np, int* __restrict__ flags) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const long long nn = (long long)N * N * N;
    const unsigned long long v = v0[p];
    if (v >= (unsigned long long)nn) return;
    int* f = flags + (long long)p * 3 * N;
    const int H2 = N / 2;
    const int x = (int)(v % N), y = (int)((v / N) % N), z = (int)(v / ((long long)N * N));
    f[(z - H2 + N) % N] = 1;
    f[N + (y - H2 + N) % N] = 1;
    f[2 * N + (x - H2 + N) % N] = 1;
}

__global__ void k_abricks(const float* __restrict__ in, float4* __restrict__ out, int N) {
    const long long nn = (long long)N * N * N;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn;
         v += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(v % N), j = (int)((v / N) % N), k = (int)(v / ((long long)N * N));
        brick_corners(in, N, N, N, i, j, k, out);
    }
}

// half bricks: the eight corners of brick_corners as halves (the caller has
// checked that every value is exact in half precision)
__global__ void k_abricks_h(const float* __restrict__ in, uint4* __restrict__ out, int N) {
    const long long nn = (long long)N * N * N;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn;
         v += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(v % N), j = (int)((v / N) % N), k = (int)(v / ((long long)N * N));
        float4 lo, hi;
        brick_values(in, N, N, N, i, j, k, lo, hi);
        const __half2 h0 = __floats2half2_rn(lo.x, lo.y), h1 = __floats2half2_rn(lo.z, lo.w);
        const __half2 h2 = __floats2half2_rn(hi.x, hi.y), h3 = __floats2half2_rn(hi.z, hi.w);
        uint4 u;
        u.x = *reinterpret_cast<const unsigned*>(&h0);
        u.y = *reinterpret_cast<const unsigned*>(&h1);
        u.z = *reinterpret_cast<const unsigned*>(&h2);
        u.w = *reinterpret_cast<const unsigned*>(&h3);
        out[v] = u;
    }
}

// ok[p] = 0 when a value of volume p is not exact in half precision (grid: blocks, volumes)
__global__ void k_half_exact(const float* const* __restrict__ vols, long long nn, int* __restrict__ ok) {
    const float* w = vols[blockIdx.y];
    bool all = true;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x)
        if (__half2float(__float2half_rn(w[v])) != w[v]) all = false;
    if (!__all_sync(0xffffffffu, all) && (threadIdx.x & 31) == 0) ok[blockIdx.y] = 0;
}

// (W'(k) + W'(-k)) / 2 of a wedge on the [kx][z][y] half grid
__global__ void k_awph(const float* __restrict__ w, float* __restrict__ out, int N) {
    const int NH = N / 2 + 1;
    const long long n = (long long)NH * N * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i % N), z = (int)((i / N) % N), kx = (int)(i / ((long long)N * N));
        int s1, s2;
        wedge_pair(kx + N * (y + N * z), N, N, N, s1, s2);
        out[i] = 0.5f * (w[s1] + w[s2]);
    }
}

__global__ void k_afill(float* __restrict__ a, float* __restrict__ b, long long n, float v) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        a[t] = v;
        b[t] = v;
    }
}

// non-zero voxels of each particle's mask (grid: blocks, particles)
__global__ void k_acount(const float* const* __restrict__ masks, long long nn, double* __restrict__ out) {
    const float* m = masks[blockIdx.y];
    double acc = 0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x)
        acc += m[v] != 0.f ? 1.0 : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int k = 0; k < 8; ++k) t += ws[k];
        atomicAdd(out + blockIdx.y, t);
    }
}

unsigned blocks_for(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)std::max<long long>(1, std::min<long long>(b, 148 * 16));
}

// the scratch pool's buffers of the batched engine, by index
struct PoolBufs {
    AlignScratch* sc;
    int next = 0;
    bool ok = true;
    template <typename T> T* get(size_t count) {
        void* p = ok ? align_scratch_buffer(sc, next++, std::max<size_t>(count, 1) * sizeof(T)) : nullptr;
        if (!p) ok = false;
        return static_cast<T*>(p);
    }
};

template <typename K> cudaError_t raise_smem(K kern, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N> int run_fused(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, const int* job_idx, int np,
                               float* angles, float* shifts, float* peaks, size_t budget, bool allow_prune,
                               AlignScratch* sc) {
    constexpr int NT = Cfg<N>::NT, NTX = Cfg<N>::NTX, P = N + 1, NH = N / 2 + 1;
    const long long nn = (long long)N * N * N;
    const long long hvol = (long long)NH * N * N;  // one half spectrum
    cudaStream_t st = ctx->stream;
    const bool wedges = jobs[job_idx[0]].wedge_ref != nullptr;
    const size_t tile = sizeof(float2) * N * P;
    const size_t xtile = sizeof(float2) * (N / 2) * P;
    const float2* tw = twiddle_table<float2>(N);
    if (!tw) return fail(ctx, TOMGPU_ERR_OOM, "twiddle table");
    cudaError_t e = cudaSuccess;
    if ((e = raise_smem(k_ax<N, X_ROT_MASK>, tile)) || (e = raise_smem(k_ax<N, X_ROT_STATS>, tile)) ||
        (e = raise_smem(k_ax<N, X_C2R_R2C>, tile)) || (e = raise_smem(k_ax<N, X_IND>, tile)) ||
        (e = raise_smem(k_ax<N, X_MUL>, tile)) || (e = raise_smem(k_ax<N, X_STATS>, tile)) ||
        (e = raise_smem(k_ap<N, P_WEDGE_A>, tile)) || (e = raise_smem(k_ap<N, P_WEDGE_B>, tile)) ||
        (e = raise_smem(k_ap<N, P_CROSS>, tile)) || (e = raise_smem(k_ap<N, P_CROSS_NW>, tile)) ||
        (e = raise_smem(k_ap<N, P_FWD>, tile)) || (e = raise_smem(k_ap<N, P_FWD_NORM>, tile)) ||
        (e = raise_smem(k_ax3<N>, xtile + sizeof(float2) * N * N)))
        return cuda_fail(ctx, e, "av3_align (fused): shared memory attribute");

    // the scan of every particle, in the reference's loop order
    std::vector<Entry> ent;
    std::vector<int> first(np + 1), nph(np), nps(np);
    for (int p = 0; p < np; ++p) {
        const tomgpu_align_job& jb = jobs[job_idx[p]];
        const std::vector<double> ph = axis_values(jb.phi), ps = axis_values(jb.psi), th = axis_values(jb.theta);
        nph[p] = (int)ph.size();
        nps[p] = (int)ps.size();
        first[p] = (int)ent.size();
        for (size_t a = 0; a < ph.size(); ++a)
            for (size_t b = 0; b < ps.size(); ++b)
                for (size_t c = 0; c < th.size(); ++c) {
                    Entry en{};
                    en.slot = p % kMaxSlots;
                    en.aidx = (int)(c * nph[p] * nps[p] + b * nph[p] + a);
                    rotmatrix_as_float(ph[a], ps[b], th[c], en.mref);
                    const float eul[3] = {(float)ph[a], (float)ps[b], (float)th[c]};
                    euler_matrix_host(eul, en.mw);
                    ent.push_back(en);
                }
    }
    if (ent.size() > (size_t)INT32_MAX) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "fused alignment: too many entries");
    first[np] = (int)ent.size();
    const long long total = (long long)ent.size();

    // batch size: both half-spectrum sets of a batch within the budget
    if (!budget) budget = (size_t)1 << 30;
    const int emax = (int)std::max<long long>(1, std::min<long long>(512, (long long)(budget / (2 * sizeof(float2) * hvol))));
    const int gsz = std::max(4, (emax + kMaxGroups - kMaxSlots - 1) / (kMaxGroups - kMaxSlots));
    const int gmax = (emax + gsz - 1) / gsz + kMaxSlots;

    PoolBufs fb{sc};
    Entry* d_ent = fb.get<Entry>(total);
    float2* HA = fb.get<float2>(emax * hvol);
    float2* HB = fb.get<float2>(emax * hvol);
    float2* part = fb.get<float2>(gmax * nn);
    double* stats = fb.get<double>(4 * emax);
    double* pst = fb.get<double>(2);
    double* d_nm = fb.get<double>(np);
    const float** d_masks = fb.get<const float*>(np);
    float2* tmpH = fb.get<float2>(hvol);
    float4* refb[kMaxSlots] = {};
    float4* wrefb[kMaxSlots] = {};
    float2 *mk[kMaxSlots] = {}, *b0[kMaxSlots] = {};
    float *wph[kMaxSlots] = {}, *cmax[kMaxSlots] = {}, *amax[kMaxSlots] = {};
    const int nslots = std::min(np, kMaxSlots);
    for (int k = 0; k < nslots; ++k) {
        refb[k] = fb.get<float4>(2 * nn);
        mk[k] = fb.get<float2>(hvol);
        b0[k] = fb.get<float2>(hvol);
        cmax[k] = fb.get<float>(nn);
        amax[k] = fb.get<float>(nn);
        if (wedges) {
            wrefb[k] = fb.get<float4>(2 * nn);
            wph[k] = fb.get<float>(hvol);
        }
    }
    // the pruned final inverse needs every particle's mask_ccf
    bool prune = allow_prune;
    for (int p = 0; p < np; ++p)
        if (!jobs[job_idx[p]].mask_ccf) prune = false;
    const float** d_mccf = prune ? fb.get<const float*>(np) : nullptr;
    const float** d_wvols = wedges ? fb.get<const float*>(np) : nullptr;
    int* d_hok = wedges ? fb.get<int>(np) : nullptr;
    int* d_flags = prune ? fb.get<int>((size_t)np * 3 * N) : nullptr;
    unsigned long long* d_v0 = prune ? fb.get<unsigned long long>(np) : nullptr;
    if (!fb.ok) {
        cudaGetLastError();
        return fail(ctx, TOMGPU_ERR_OOM, "fused alignment buffers");
    }
    int* d_plist = nullptr;
    float2 *d_wy = nullptr, *d_wx = nullptr, *CP = nullptr;
    float* VP = nullptr;
    std::vector<int> pn3;  // per particle: nz, ny, nx of the pruned lists
    int nzmax = 0, nymax = 0, nxmax = 0;
    // the b-side passes (rotated-wedge plane, its x-lines) run on a second
    // stream beside the a-side ones (rotation, particle-wedge plane, x-lines)
    // stream; each particle's final step (align_finish) runs on a third one,
    // one batch later, beside the next batch's passes
    cudaStream_t st2 = nullptr, stf = nullptr;
    cudaEvent_t ev_a = nullptr, ev_b = nullptr, ev_done = nullptr;
    if ((e = cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&stf, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&ev_a, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&ev_b, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming))) {
        if (st2) cudaStreamDestroy(st2);
        if (stf) cudaStreamDestroy(stf);
        if (ev_a) cudaEventDestroy(ev_a);
        if (ev_b) cudaEventDestroy(ev_b);
        return cuda_fail(ctx, e, "av3_align (fused): stream");
    }
    std::vector<double> nmask(np);  // non-zero voxels of each particle's mask
    std::vector<int> to_finish;     // particles whose scan ended in the previous batch
    auto finish_pending = [&]() -> int {
        if (to_finish.empty()) return TOMGPU_OK;
        cudaError_t fe = cudaStreamWaitEvent(stf, ev_done, 0);
        if (fe) return cuda_fail(ctx, fe, "av3_align (fused): final step");
        for (int p : to_finish) {
            const int j = job_idx[p], k = p % kMaxSlots;
            const int frc = align_finish(ctx, stf, jobs[j], nph[p], nps[p], cmax[k], amax[k], nmask[p], sc,
                                         angles + 3 * j, shifts + 3 * j, peaks + j);
            if (frc) return frc;
        }
        to_finish.clear();
        return TOMGPU_OK;
    };
    int rc = TOMGPU_OK;
    do {
        if ((e = cudaMemcpyAsync(d_ent, ent.data(), sizeof(Entry) * total, cudaMemcpyHostToDevice, st))) break;
        // the masks' sizes, checked before the scan
        std::vector<const float*> masks(np);
        for (int p = 0; p < np; ++p) masks[p] = jobs[job_idx[p]].mask;
        if ((e = cudaMemcpyAsync(d_masks, masks.data(), sizeof(float*) * np, cudaMemcpyHostToDevice, st))) break;
        if ((e = cudaMemsetAsync(d_nm, 0, sizeof(double) * np, st))) break;
        k_acount<<<dim3(blocks_for(nn), np), 256, 0, st>>>(d_masks, nn, d_nm);
        if ((e = cudaMemcpyAsync(nmask.data(), d_nm, sizeof(double) * np, cudaMemcpyDeviceToHost, st))) break;
        std::vector<int> flags;
        if (prune) {
            std::vector<const float*> mc(np);
            for (int p = 0; p < np; ++p) mc[p] = jobs[job_idx[p]].mask_ccf;
            flags.resize((size_t)np * 3 * N);
            if ((e = cudaMemcpyAsync(d_mccf, mc.data(), sizeof(float*) * np, cudaMemcpyHostToDevice, st))) break;
            if ((e = cudaMemsetAsync(d_flags, 0, sizeof(int) * flags.size(), st))) break;
            if ((e = cudaMemsetAsync(d_v0, 0xFF, sizeof(unsigned long long) * np, st))) break;
            k_prune_mark<<<dim3(blocks_for(nn), np), 256, 0, st>>>(d_mccf, N, d_flags, d_v0);
            k_prune_v0<<<(np + 127) / 128, 128, 0, st>>>(d_v0, N, np, d_flags);
            ctx->launches += 2;
            if ((e = cudaMemcpyAsync(flags.data(), d_flags, sizeof(int) * flags.size(), cudaMemcpyDeviceToHost, st)))
                break;
        }
        // half bricks for the reference wedges when all of them are exact in half precision
        std::vector<int> hok(wedges ? np : 0, 1);
        if (wedges) {
            std::vector<const float*> wv(np);
            for (int p = 0; p < np; ++p) wv[p] = jobs[job_idx[p]].wedge_ref;
            if ((e = cudaMemcpyAsync(d_wvols, wv.data(), sizeof(float*) * np, cudaMemcpyHostToDevice, st))) break;
            if ((e = cudaMemcpyAsync(d_hok, hok.data(), sizeof(int) * np, cudaMemcpyHostToDevice, st))) break;
            k_half_exact<<<dim3(blocks_for(nn), np), 256, 0, st>>>(d_wvols, nn, d_hok);
            ctx->launches += 1;
            if ((e = cudaMemcpyAsync(hok.data(), d_hok, sizeof(int) * np, cudaMemcpyDeviceToHost, st))) break;
        }
        if ((e = cudaStreamSynchronize(st))) break;
        ctx->launches += 1;
        bool halfw = wedges;
        for (int p = 0; p < (int)hok.size(); ++p)
            if (!hok[p]) halfw = false;
        for (int p = 0; p < np && !rc; ++p)
            if (nmask[p] < 2)
                rc = fail(ctx, TOMGPU_ERR_ARG, "job " + std::to_string(job_idx[p]) + ": mask needs at least two voxels");
        if (rc) break;
        if (prune) {
            // per particle the listed coordinates (kept when every axis stays
            // within a third of the edge: beyond that the full inverse is cheaper)
            pn3.assign((size_t)3 * np, 0);
            std::vector<int> hl((size_t)np * 3 * kMaxPrune, 0);
            for (int p = 0; p < np && prune; ++p)
                for (int a = 0; a < 3; ++a) {
                    int c = 0;
                    for (int i = 0; i < N; ++i)
                        if (flags[((size_t)p * 3 + a) * N + i]) {
                            if (c < kMaxPrune) hl[((size_t)p * 3 + a) * kMaxPrune + c] = i;
                            ++c;
                        }
                    if (c > kMaxPrune || 3 * c > N) prune = false;
                    pn3[3 * p + a] = c;
                }
            if (prune) {
                for (int p = 0; p < np; ++p) {
                    nzmax = std::max(nzmax, pn3[3 * p]);
                    nymax = std::max(nymax, pn3[3 * p + 1]);
                    nxmax = std::max(nxmax, pn3[3 * p + 2]);
                }
                // inverse-DFT tables: wy[ky][yi] = exp(2 pi i ky y / N); wx[kx][xi] the
                // same times the Hermitian weight (1 at kx = 0 and N/2, else 2)
                std::vector<float2> hy((size_t)np * N * kMaxPrune), hx((size_t)np * NH * kMaxPrune);
                const double tau = 6.283185307179586476925286766559;
                for (int p = 0; p < np; ++p) {
                    for (int k = 0; k < N; ++k)
                        for (int i = 0; i < kMaxPrune; ++i) {
                            const int c = hl[((size_t)p * 3 + 1) * kMaxPrune + i];
                            const double a = tau * (double)((k * c) % N) / N;
                            hy[((size_t)p * N + k) * kMaxPrune + i] = make_float2((float)std::cos(a), (float)std::sin(a));
                        }
                    for (int k = 0; k < NH; ++k)
                        for (int i = 0; i < kMaxPrune; ++i) {
                            const int c = hl[((size_t)p * 3 + 2) * kMaxPrune + i];
                            const double a = tau * (double)((k * c) % N) / N;
                            const double w = (k == 0 || 2 * k == N) ? 1.0 : 2.0;
                            hx[((size_t)p * NH + k) * kMaxPrune + i] =
                                make_float2((float)(w * std::cos(a)), (float)(w * std::sin(a)));
                        }
                }
                d_plist = fb.get<int>(hl.size());
                d_wy = fb.get<float2>(hy.size());
                d_wx = fb.get<float2>(hx.size());
                CP = fb.get<float2>((size_t)emax * NH * nzmax * nymax);
                VP = fb.get<float>((size_t)emax * nzmax * nymax * nxmax);
                if (!fb.ok) {
                    cudaGetLastError();
                    rc = fail(ctx, TOMGPU_ERR_OOM, "fused alignment buffers");
                    break;
                }
                if ((e = cudaMemcpyAsync(d_plist, hl.data(), sizeof(int) * hl.size(), cudaMemcpyHostToDevice, st)) ||
                    (e = cudaMemcpyAsync(d_wy, hy.data(), sizeof(float2) * hy.size(), cudaMemcpyHostToDevice, st)) ||
                    (e = cudaMemcpyAsync(d_wx, hx.data(), sizeof(float2) * hx.size(), cudaMemcpyHostToDevice, st)))
                    break;
            }
        }

        SlotTab slots{};
        const float inv_n3 = (float)(1.0 / (double)nn);
        long long e0 = 0;
        int next_prep = 0;  // first particle whose slot is not yet prepared
        while (e0 < total && !rc && !e) {
            // the batch: up to emax entries of at most kBatchParticles particles
            const int p_lo = (int)(std::upper_bound(first.begin(), first.end(), (int)e0) - first.begin()) - 1;
            long long e1 = std::min<long long>(total, e0 + emax);
            const int p_cap = std::min(np, p_lo + kBatchParticles);
            e1 = std::min<long long>(e1, first[p_cap]);
            const int nb = (int)(e1 - e0);
            const int p_hi = (int)(std::upper_bound(first.begin(), first.end(), (int)(e1 - 1)) - first.begin()) - 1;
            // set-up of the batch's new particles
            for (; next_prep <= p_hi && !e; ++next_prep) {
                const int p = next_prep, k = p % kMaxSlots;
                const tomgpu_align_job& jb = jobs[job_idx[p]];
                Slot& sl = slots.s[k];
                sl.refb = refb[k];
                sl.wrefb = wrefb[k];
                sl.mask = jb.mask;
                sl.mk = mk[k];
                sl.b0 = b0[k];
                sl.wph = wph[k];
                sl.cmax = cmax[k];
                sl.amax = amax[k];
                sl.nmask = nmask[p];
                if (prune) {
                    sl.pl = d_plist + (size_t)p * 3 * kMaxPrune;
                    sl.wy = d_wy + (size_t)p * N * kMaxPrune;
                    sl.wx = d_wx + (size_t)p * NH * kMaxPrune;
                    sl.nz = pn3[3 * p];
                    sl.ny = pn3[3 * p + 1];
                    sl.nx = pn3[3 * p + 2];
                }
                k_abricks<<<blocks_for(nn), 256, 0, st>>>(jb.ref, refb[k], N);
                k_afill<<<blocks_for(nn), 256, 0, st>>>(cmax[k], amax[k], nn, -2.f);
                if ((e = cudaMemsetAsync(pst, 0, 2 * sizeof(double), st))) break;
                // F(mask != 0)
                k_ax<N, X_IND><<<dim3(N, 1), NTX, xtile, st>>>(tmpH, hvol, nullptr, slots, jb.mask, nullptr, pst, 0, tw,
                                                               inv_n3);
                k_ap<N, P_FWD><<<dim3(NH, 1), NT, tile, st>>>(nullptr, nullptr, hvol, nullptr, slots, nullptr, tw, tmpH,
                                                               mk[k], nullptr, nullptr, 0.0, nullptr, 0, 0);
                ctx->launches += 4;
                if (wedges) {
                    const float* wp = jb.wedge_part ? jb.wedge_part : jb.wedge_ref;
                    if (halfw) {
                        sl.wrefh = reinterpret_cast<const uint4*>(wrefb[k]);
                        k_abricks_h<<<blocks_for(nn), 256, 0, st>>>(jb.wedge_ref, reinterpret_cast<uint4*>(wrefb[k]),
                                                                    N);
                    } else {
                        sl.wrefh = nullptr;
                        k_abricks<<<blocks_for(nn), 256, 0, st>>>(jb.wedge_ref, wrefb[k], N);
                    }
                    k_awph<<<blocks_for(hvol), 256, 0, st>>>(wp, wph[k], N);
                    // F(part * mask)
                    k_ax<N, X_MUL><<<dim3(N, 1), NTX, xtile, st>>>(tmpH, hvol, nullptr, slots, jb.part, jb.mask, nullptr,
                                                                   0, tw, inv_n3);
                    k_ap<N, P_FWD><<<dim3(NH, 1), NT, tile, st>>>(nullptr, nullptr, hvol, nullptr, slots, nullptr, tw,
                                                                   tmpH, b0[k], nullptr, nullptr, 0.0, nullptr, 0, 0);
                    ctx->launches += 4;
                } else {
                    // F(norm_inside_mask(part))
                    if ((e = cudaMemsetAsync(pst, 0, 2 * sizeof(double), st))) break;
                    k_ax<N, X_STATS><<<dim3(N, 1), NTX, xtile, st>>>(tmpH, hvol, nullptr, slots, jb.part, jb.mask, pst,
                                                                     0, tw, inv_n3);
                    k_ap<N, P_FWD_NORM><<<dim3(NH, 1), NT, tile, st>>>(nullptr, nullptr, hvol, nullptr, slots, nullptr,
                                                                        tw, tmpH, b0[k], mk[k], pst, nmask[p], nullptr, 0, 0);
                    ctx->launches += 2;
                }
                if ((e = cudaGetLastError())) break;
            }
            if (e) break;
            // entry groups for the maxima (each within one particle) and their merge segments
            GroupTab groups{};
            SegTab segs{};
            for (int p = p_lo; p <= p_hi; ++p) {
                const int a = (int)std::max<long long>(first[p], e0) - (int)e0;
                const int b = (int)std::min<long long>(first[p + 1], e1) - (int)e0;
                Seg& sg = segs.s[segs.n++];
                sg.slot = p % kMaxSlots;
                sg.g0 = groups.n;
                for (int q = a; q < b; q += gsz) groups.g[groups.n++] = Group{p % kMaxSlots, q, std::min(b, q + gsz)};
                sg.g1 = groups.n;
            }
            const Entry* eb = d_ent + e0;
            if ((e = cudaMemsetAsync(stats, 0, sizeof(double) * 4 * nb, st))) break;
            if (wedges) {
                if ((e = cudaEventRecord(ev_a, st)) || (e = cudaStreamWaitEvent(st2, ev_a, 0))) break;
                k_ax<N, X_ROT_MASK><<<dim3(N, nb), NTX, xtile, st>>>(HA, hvol, eb, slots, nullptr, nullptr, stats, 0,
                                                                     tw, inv_n3);
                k_ap<N, P_WEDGE_B><<<dim3(NH, nb), NT, tile, st2>>>(nullptr, HB, hvol, eb, slots, stats, tw, nullptr,
                                                                     nullptr, nullptr, nullptr, 0.0, nullptr, 0, 0);
                k_ap<N, P_WEDGE_A><<<dim3(NH, nb), NT, tile, st>>>(HA, nullptr, hvol, eb, slots, stats, tw, nullptr,
                                                                    nullptr, nullptr, nullptr, 0.0, nullptr, 0, 0);
                k_ax<N, X_C2R_R2C><<<dim3(N, nb), NTX, xtile, st2>>>(HB, hvol, eb, slots, nullptr, nullptr, stats, 1,
                                                                     tw, inv_n3);
                k_ax<N, X_C2R_R2C><<<dim3(N, nb), NTX, xtile, st>>>(HA, hvol, eb, slots, nullptr, nullptr, stats, 0, tw,
                                                                    inv_n3);
                if ((e = cudaEventRecord(ev_b, st2)) || (e = cudaStreamWaitEvent(st, ev_b, 0))) break;
                k_ap<N, P_CROSS><<<dim3(NH, nb), NT, tile, st>>>(HA, HB, hvol, eb, slots, stats, tw, nullptr, nullptr,
                                                                  nullptr, nullptr, 0.0, prune ? CP : nullptr, nzmax,
                                                                  nymax);
                ctx->launches += 6;
            } else {
                k_ax<N, X_ROT_STATS><<<dim3(N, nb), NTX, xtile, st>>>(HA, hvol, eb, slots, nullptr, nullptr, stats, 0,
                                                                      tw, inv_n3);
                k_ap<N, P_CROSS_NW><<<dim3(NH, nb), NT, tile, st>>>(HA, HB, hvol, eb, slots, stats, tw, nullptr,
                                                                     nullptr, nullptr, nullptr, 0.0,
                                                                     prune ? CP : nullptr, nzmax, nymax);
                ctx->launches += 2;
            }
            if (prune) {
                // segments as entry ranges of each particle in the batch
                SegTab es{};
                for (int p = p_lo; p <= p_hi; ++p)
                    es.s[es.n++] = Seg{p % kMaxSlots, (int)(std::max<long long>(first[p], e0) - e0),
                                       (int)(std::min<long long>(first[p + 1], e1) - e0)};
                const int prod = nzmax * nymax * nxmax;
                k_ax3v<<<dim3((prod + 127) / 128, nb), 128, 0, st>>>(CP, N, nzmax, nymax, eb, slots, VP, prod, inv_n3);
                k_ax3s<<<dim3((prod + 127) / 128, es.n), 128, 0, st>>>(VP, prod, N, eb, slots, es);
                ctx->launches += 2;
            } else {
                k_ax3<N><<<dim3(N, groups.n), NTX, xtile + sizeof(float2) * N * N, st>>>(HB, hvol, eb, slots,
                                                                                         groups, part, tw, inv_n3);
                k_amerge<<<dim3(blocks_for(nn), segs.n), 256, 0, st>>>(part, nn, segs, slots);
                ctx->launches += 2;
            }
            if ((e = cudaGetLastError())) break;
            // the previous batch's finished particles, beside this batch's passes
            if ((rc = finish_pending())) break;
            if ((e = cudaEventRecord(ev_done, st))) break;
            for (int p = p_lo; p <= p_hi; ++p)
                if (first[p + 1] <= e1) to_finish.push_back(p);
            e0 = e1;
        }
        if (!rc && !e) rc = finish_pending();
    } while (0);
    if (e && !rc) rc = cuda_fail(ctx, e, "av3_align (fused)");
    cudaStreamSynchronize(st2);
    cudaStreamSynchronize(stf);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st2);
    cudaStreamDestroy(stf);
    cudaEventDestroy(ev_a);
    cudaEventDestroy(ev_b);
    cudaEventDestroy(ev_done);
    return rc;
}

}  // namespace

bool align_fused_supported(const tomgpu_align_job& job) {
    if (job.n[0] != job.n[1] || job.n[0] != job.n[2]) return false;
    for (int n : kEdges)
        if (job.n[0] == n) return true;
    return false;
}

int align_fused(tomgpu_ctx* ctx, const tomgpu_align_job* jobs, const int* job_idx, int n, float* angles,
                float* shifts, float* peaks, size_t budget_bytes, bool allow_prune, AlignScratch* sc) {
    if (n <= 0) return TOMGPU_OK;
    // the per-particle set-up kernels take the particle as their grid's y index
    constexpr int kMaxJobs = 32768;
    if (n > kMaxJobs) {
        for (int o = 0; o < n; o += kMaxJobs) {
            const int rc = align_fused(ctx, jobs, job_idx + o, std::min(kMaxJobs, n - o), angles, shifts, peaks,
                                       budget_bytes, allow_prune, sc);
            if (rc) return rc;
        }
        return TOMGPU_OK;
    }
    switch (jobs[job_idx[0]].n[0]) {
        case 24: return run_fused<24>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 32: return run_fused<32>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 40: return run_fused<40>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 48: return run_fused<48>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 64: return run_fused<64>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 72: return run_fused<72>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 80: return run_fused<80>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 96: return run_fused<96>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 56: return run_fused<56>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 100: return run_fused<100>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 112: return run_fused<112>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 120: return run_fused<120>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        case 128: return run_fused<128>(ctx, jobs, job_idx, n, angles, shifts, peaks, budget_bytes, allow_prune, sc);
        default: return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "fused alignment: box edge not compiled");
    }
}

}  // namespace tg
