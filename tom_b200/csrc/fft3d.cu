// Generic batched FFTs along one axis of a 3-D array, and 3-D r2c / c2r / c2c
// transforms built from them (FP32 and FP64).
//
// These are the library's own replacement for MATLAB fftn/ifftn and the FFTW
// plans of the C++ picker (Filtrans/tom_fourier.m:44-50,
// Oscar3/c++Picker/src/tom/core/fftw_plan.cpp).  The matching hot loop does
// not use them: it runs its own fused kernels (match.cu).  They serve the
// once-per-volume set-up (tomogram spectrum, FP64 local statistics), the small
// template-sized wedge filter, and the tom_fourier entry points.
#include "fft3d.h"
#include "fft_engine.cuh"
#include "fft_rt.cuh"
#include "twiddles.h"

#include <algorithm>
#include <cstdio>

namespace tg {

// Skew and line pitch of the shared-memory lines, per length and element
// size, chosen by counting the bank-conflict wavefronts of every load, stage
// and store of k_fft_lines (x pass and two strided passes) for each candidate
// and kept where the measured pass time agreed (96 with 8-byte elements
// measured no faster skewed and stays unskewed, with the radix order 3, 4, 8):
// {L, SK, LS for 8-byte elements, SK, LS for 16-byte elements}.
struct LineLayout { int L, sk8, ls8, sk16, ls16; };
constexpr LineLayout kLineLayouts[] = {
    {8, 0, 9, 0, 9},       {12, 0, 19, 0, 19},    {16, 0, 17, 0, 17},    {20, 0, 21, 2, 25},
    {24, 3, 27, 3, 27},    {32, 0, 35, 3, 37},    {40, 3, 45, 3, 45},    {48, 4, 51, 4, 51},
    {64, 4, 69, 3, 73},    {80, 4, 85, 4, 85},    {96, 0, 97, 3, 109},  {128, 4, 137, 3, 145},
    {160, 4, 170, 3, 181}, {192, 4, 206, 3, 217}, {256, 4, 274, 4, 273}, {512, 4, 548, 3, 578}};
constexpr LineLayout line_layout(int L) {
    for (const LineLayout& x : kLineLayouts)
        if (x.L == L) return x;
    return {L, 0, L + 1, 0, L + 1};  // the radix-29 lengths: unskewed
}

template <int L, typename C> struct LineCfg {
    static constexpr int NL = (2048 / L) < 1 ? 1 : ((2048 / L) > 64 ? 64 : (2048 / L));
    static constexpr int NT = 256;
    static constexpr bool W16 = sizeof(C) == 16;
    static constexpr int SK = W16 ? line_layout(L).sk16 : line_layout(L).sk8;
    static constexpr int LS = W16 ? line_layout(L).ls16 : line_layout(L).ls8;
    static_assert(LS >= tgfft::skew<SK>(L - 1) + 1, "line pitch holds the skewed line");
};

template <int L, int DIR, int MODE, typename C>
__global__ void __launch_bounds__(256) k_fft_lines(const void* in, void* out,
                                                   LineGeom gi, LineGeom go, const C* __restrict__ tw,
                                                   double scale, long nlines) {
    typedef typename CTraits<C>::R Rt;
    constexpr int NL = LineCfg<L, C>::NL, NT = LineCfg<L, C>::NT, LS = LineCfg<L, C>::LS, SK = LineCfg<L, C>::SK;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    // element offsets of the block's lines (one division per line, not per element)
    __shared__ long offs_i[NL], offs_o[NL];
    const int tid = threadIdx.x;
    const long line0 = (long)blockIdx.x * NL;
    for (int l = tid; l < NL; l += NT) {
        const long gl = line0 + l;
        offs_i[l] = (gl % gi.cnt0) * gi.s0 + (gl / gi.cnt0) * gi.s1;
        offs_o[l] = (gl % go.cnt0) * go.s0 + (gl / go.cnt0) * go.s1;
    }
    __syncthreads();
    const Rt* rin = reinterpret_cast<const Rt*>(in);
    const C* cin = reinterpret_cast<const C*>(in);

    for (int i = tid; i < NL * L; i += NT) {
        int l, e;
        if (gi.es == 1) { l = i / L; e = i - l * L; }
        else { e = i / NL; l = i - e * NL; }
        const long gl = line0 + l;
        C v = CTraits<C>::make(0, 0);
        if (gl < nlines) {
            const long off = offs_i[l];
            if (MODE == FFT_R2C) {
                v = CTraits<C>::make(rin[off + e * gi.es], 0);
            } else if (MODE == FFT_C2R) {
                if (e <= L / 2) v = cin[off + e * gi.es];
                else v = cconj(cin[off + (L - e) * gi.es]);
            } else {
                v = cin[off + e * gi.es];
            }
        }
        s[l * LS + tgfft::skew<SK>(e)] = v;
    }
    __syncthreads();
    tgfft::smem_fft<L, DIR, NL, NT, LS, C, SK>(s, tw, tid);

    Rt* rout = reinterpret_cast<Rt*>(out);
    C* cout = reinterpret_cast<C*>(out);
    const Rt sc = (Rt)scale;
    for (int i = tid; i < NL * L; i += NT) {
        int l, e;
        if (go.es == 1) { l = i / L; e = i - l * L; }
        else { e = i / NL; l = i - e * NL; }
        const long gl = line0 + l;
        if (gl >= nlines) continue;
        const long off = offs_o[l];
        const C v = s[l * LS + tgfft::skew<SK>(e)];
        if (MODE == FFT_R2C) {
            if (e <= L / 2) cout[off + e * go.es] = cscale(v, sc);
        } else if (MODE == FFT_C2R) {
            rout[off + e * go.es] = v.x * sc;
        } else {
            cout[off + e * go.es] = cscale(v, sc);
        }
    }
}

template <int L, int DIR, int MODE, typename C>
static cudaError_t launch_lines_t(const void* in, void* out, const LineGeom& gi, const LineGeom& go,
                                  long nlines, double scale, cudaStream_t st) {
    constexpr int NL = LineCfg<L, C>::NL, LS = LineCfg<L, C>::LS;
    constexpr int NT = LineCfg<L, C>::NT;
    const size_t smem = (size_t)NL * LS * sizeof(C);
    auto kern = k_fft_lines<L, DIR, MODE, C>;
    static unsigned attr_mask = 0;  // one bit per device: attribute already raised
    int dev = 0;
    cudaGetDevice(&dev);
    if (smem > 48 * 1024 && dev < 32 && !(attr_mask & (1u << dev))) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr_mask |= 1u << dev;
    }
    const C* tw = twiddle_table<C>(L);
    if (!tw) return cudaErrorInvalidValue;
    const long blocks = (nlines + NL - 1) / NL;
    if (blocks <= 0) return cudaSuccess;
    kern<<<(unsigned)blocks, NT, smem, st>>>(in, out, gi, go, tw, scale, nlines);
    return cudaGetLastError();
}

// Lines of any length: the run-time engine (fft_rt.cuh), NL lines per block
// in two ping-pong buffers of pitch LS.
constexpr int kRtMaxLines = 64;

template <int DIR, int MODE, typename C>
__global__ void __launch_bounds__(256) k_fft_lines_rt(const void* in, void* out, LineGeom gi, LineGeom go,
                                                      tgrt::Plan p, tgrt::Tabs<C> tabs, int NL, int LS,
                                                      double scale, long nlines) {
    typedef typename CTraits<C>::R Rt;
    constexpr int NT = 256;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s = reinterpret_cast<C*>(smem_raw);
    C* s2 = s + (size_t)NL * LS;
    __shared__ long offs_i[kRtMaxLines], offs_o[kRtMaxLines];
    const int tid = threadIdx.x;
    const int L = p.L;
    const long line0 = (long)blockIdx.x * NL;
    for (int l = tid; l < NL; l += NT) {
        const long gl = line0 + l;
        offs_i[l] = (gl % gi.cnt0) * gi.s0 + (gl / gi.cnt0) * gi.s1;
        offs_o[l] = (gl % go.cnt0) * go.s0 + (gl / go.cnt0) * go.s1;
    }
    __syncthreads();
    const Rt* rin = reinterpret_cast<const Rt*>(in);
    const C* cin = reinterpret_cast<const C*>(in);
    for (int i = tid; i < NL * L; i += NT) {
        int l, e;
        if (gi.es == 1) { l = i / L; e = i - l * L; }
        else { e = i / NL; l = i - e * NL; }
        const long gl = line0 + l;
        C v = CTraits<C>::make(0, 0);
        if (gl < nlines) {
            const long off = offs_i[l];
            if (MODE == FFT_R2C) v = CTraits<C>::make(rin[off + e * gi.es], 0);
            else if (MODE == FFT_C2R) v = e <= L / 2 ? cin[off + e * gi.es] : cconj(cin[off + (L - e) * gi.es]);
            else v = cin[off + e * gi.es];
        }
        s[l * LS + e] = v;
    }
    __syncthreads();
    const C* res = tgrt::fft<DIR>(s, s2, p, tabs, NL, LS, tid, NT);
    Rt* rout = reinterpret_cast<Rt*>(out);
    C* cout = reinterpret_cast<C*>(out);
    const Rt sc = (Rt)scale;
    for (int i = tid; i < NL * L; i += NT) {
        int l, e;
        if (go.es == 1) { l = i / L; e = i - l * L; }
        else { e = i / NL; l = i - e * NL; }
        const long gl = line0 + l;
        if (gl >= nlines) continue;
        const long off = offs_o[l];
        const C v = res[l * LS + e];
        if (MODE == FFT_R2C) {
            if (e <= L / 2) cout[off + e * go.es] = cscale(v, sc);
        } else if (MODE == FFT_C2R) {
            rout[off + e * go.es] = v.x * sc;
        } else {
            cout[off + e * go.es] = cscale(v, sc);
        }
    }
}

// Lines per block for a run-time plan: as many as fit a 48 KB budget (at
// least one, at most 64 and at most the number of lines).
static int rt_lines_per_block(int LS, size_t elem, long nlines) {
    const size_t per = 2 * (size_t)LS * elem;
    long nl = (long)std::max<size_t>(1, (48 * 1024) / per);
    nl = std::min<long>(nl, kRtMaxLines);
    nl = std::min<long>(nl, std::max<long>(nlines, 1));
    return (int)nl;
}

template <int DIR, int MODE, typename C>
static cudaError_t launch_lines_rt(int L, const void* in, void* out, const LineGeom& gi, const LineGeom& go,
                                   long nlines, double scale, cudaStream_t st) {
    tgrt::Plan p;
    if (!rt_plan(L, (int)sizeof(C), &p)) return cudaErrorInvalidValue;
    tgrt::Tabs<C> tabs;
    if (!rt_tabs<C>(p, &tabs)) return cudaErrorMemoryAllocation;
    if (nlines <= 0) return cudaSuccess;
    const int LS = tgrt::pitch(p);
    const int NL = rt_lines_per_block(LS, sizeof(C), nlines);
    const size_t smem = 2 * (size_t)NL * LS * sizeof(C);
    auto kern = k_fft_lines_rt<DIR, MODE, C>;
    // above 40 KB the kernel's static arrays could take the block past the
    // 48 KB a launch gets without opting in
    if (smem > 40 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e) return e;
    }
    const long blocks = (nlines + NL - 1) / NL;
    kern<<<(unsigned)blocks, 256, smem, st>>>(in, out, gi, go, p, tabs, NL, LS, scale, nlines);
    return cudaGetLastError();
}

template <int DIR, int MODE, typename C>
static cudaError_t dispatch_len(int L, const void* in, void* out, const LineGeom& gi, const LineGeom& go,
                                long nlines, double scale, cudaStream_t st) {
#define TG_CASE(N) \
    case N: return launch_lines_t<N, DIR, MODE, C>(in, out, gi, go, nlines, scale, st);
    switch (L) {
        TG_CASE(8) TG_CASE(12) TG_CASE(16) TG_CASE(20) TG_CASE(24) TG_CASE(32) TG_CASE(40) TG_CASE(48) TG_CASE(64)
        TG_CASE(80) TG_CASE(96) TG_CASE(128) TG_CASE(160) TG_CASE(192) TG_CASE(232)
        TG_CASE(256) TG_CASE(464) TG_CASE(512) TG_CASE(928) TG_CASE(1024)
        default: return launch_lines_rt<DIR, MODE, C>(L, in, out, gi, go, nlines, scale, st);
    }
#undef TG_CASE
}

// Every length whose run-time plan fits one block in FP64 (the set-up
// transforms run in FP64): every L up to 3528, and beyond that the lengths
// whose prime factors are all in {2, 3, 5, 7, 11, 13}, up to 7150.
bool fft_length_supported(int L) {
    tgrt::Plan p;
    return rt_plan(L, (int)sizeof(double2), &p);
}

template <typename C>
cudaError_t fft_lines(int L, int dir, int mode, const void* in, void* out, const LineGeom& gi,
                      const LineGeom& go, long nlines, double scale, cudaStream_t st) {
    if (mode == FFT_R2C) return dispatch_len<-1, FFT_R2C, C>(L, in, out, gi, go, nlines, scale, st);
    if (mode == FFT_C2R) return dispatch_len<+1, FFT_C2R, C>(L, in, out, gi, go, nlines, scale, st);
    if (dir < 0) return dispatch_len<-1, FFT_C2C, C>(L, in, out, gi, go, nlines, scale, st);
    return dispatch_len<+1, FFT_C2C, C>(L, in, out, gi, go, nlines, scale, st);
}

template cudaError_t fft_lines<float2>(int, int, int, const void*, void*, const LineGeom&,
                                       const LineGeom&, long, double, cudaStream_t);
template cudaError_t fft_lines<double2>(int, int, int, const void*, void*, const LineGeom&,
                                        const LineGeom&, long, double, cudaStream_t);

// ------------------------------------------------------------ 3-D drivers
// Real arrays are [nz][ny][nx] (x fastest); half spectra [nz][ny][nx/2+1].
template <typename C>
cudaError_t r2c3d(const void* real_in, C* half_out, const int n[3], cudaStream_t st) {
    const long nx = n[0], ny = n[1], nz = n[2], nh = nx / 2 + 1;
    cudaError_t e;
    LineGeom gi{1, (int)ny, nx, (int)nz, nx * ny};
    LineGeom go{1, (int)ny, nh, (int)nz, nh * ny};
    if ((e = fft_lines<C>((int)nx, -1, FFT_R2C, real_in, half_out, gi, go, ny * nz, 1.0, st))) return e;
    LineGeom gy{nh, (int)nh, 1, (int)nz, nh * ny};
    if (ny > 1 && (e = fft_lines<C>((int)ny, -1, FFT_C2C, half_out, half_out, gy, gy, nh * nz, 1.0, st)))
        return e;
    LineGeom gz{nh * ny, (int)(nh * ny), 1, 1, 0};
    if (nz > 1 && (e = fft_lines<C>((int)nz, -1, FFT_C2C, half_out, half_out, gz, gz, nh * ny, 1.0, st)))
        return e;
    return cudaSuccess;
}

template <typename C>
cudaError_t c2r3d(C* half_inout, void* real_out, const int n[3], double scale, cudaStream_t st) {
    const long nx = n[0], ny = n[1], nz = n[2], nh = nx / 2 + 1;
    cudaError_t e;
    LineGeom gz{nh * ny, (int)(nh * ny), 1, 1, 0};
    if (nz > 1 && (e = fft_lines<C>((int)nz, +1, FFT_C2C, half_inout, half_inout, gz, gz, nh * ny, 1.0, st)))
        return e;
    LineGeom gy{nh, (int)nh, 1, (int)nz, nh * ny};
    if (ny > 1 && (e = fft_lines<C>((int)ny, +1, FFT_C2C, half_inout, half_inout, gy, gy, nh * nz, 1.0, st)))
        return e;
    LineGeom gi{1, (int)ny, nh, (int)nz, nh * ny};
    LineGeom go{1, (int)ny, nx, (int)nz, nx * ny};
    return fft_lines<C>((int)nx, +1, FFT_C2R, half_inout, real_out, gi, go, ny * nz, scale, st);
}

// Full complex 3-D transform in place, [nz][ny][nx] complex.
template <typename C>
cudaError_t c2c3d(C* data, const int n[3], int dir, double scale, cudaStream_t st) {
    const long nx = n[0], ny = n[1], nz = n[2];
    cudaError_t e;
    const double sx = (ny > 1 || nz > 1) ? 1.0 : scale, sy = nz > 1 ? 1.0 : scale;
    LineGeom gx{1, (int)ny, nx, (int)nz, nx * ny};
    if ((e = fft_lines<C>((int)nx, dir, FFT_C2C, data, data, gx, gx, ny * nz, sx, st))) return e;
    LineGeom gy{nx, (int)nx, 1, (int)nz, nx * ny};
    if (ny > 1 && (e = fft_lines<C>((int)ny, dir, FFT_C2C, data, data, gy, gy, nx * nz, sy, st))) return e;
    LineGeom gz{nx * ny, (int)(nx * ny), 1, 1, 0};
    if (nz > 1 && (e = fft_lines<C>((int)nz, dir, FFT_C2C, data, data, gz, gz, nx * ny, scale, st))) return e;
    return cudaSuccess;
}

// E volumes one after another (real: nx ny nz each, half: (nx/2+1) ny nz
// each): the batch joins z in the line geometry of every pass.
template <typename C>
cudaError_t r2c3d_batch(const void* real_in, C* half_out, const int n[3], int E, cudaStream_t st) {
    const long nx = n[0], ny = n[1], nz = n[2], nh = nx / 2 + 1;
    cudaError_t e;
    LineGeom gi{1, (int)ny, nx, (int)(nz * E), nx * ny};
    LineGeom go{1, (int)ny, nh, (int)(nz * E), nh * ny};
    if ((e = fft_lines<C>((int)nx, -1, FFT_R2C, real_in, half_out, gi, go, ny * nz * E, 1.0, st))) return e;
    LineGeom gy{nh, (int)nh, 1, (int)(nz * E), nh * ny};
    if (ny > 1 && (e = fft_lines<C>((int)ny, -1, FFT_C2C, half_out, half_out, gy, gy, nh * nz * E, 1.0, st)))
        return e;
    LineGeom gz{nh * ny, (int)(nh * ny), 1, E, nh * ny * nz};
    if (nz > 1 && (e = fft_lines<C>((int)nz, -1, FFT_C2C, half_out, half_out, gz, gz, nh * ny * E, 1.0, st)))
        return e;
    return cudaSuccess;
}

template <typename C>
cudaError_t c2r3d_batch(C* half_inout, void* real_out, const int n[3], int E, double scale, cudaStream_t st) {
    const long nx = n[0], ny = n[1], nz = n[2], nh = nx / 2 + 1;
    cudaError_t e;
    LineGeom gz{nh * ny, (int)(nh * ny), 1, E, nh * ny * nz};
    if (nz > 1 &&
        (e = fft_lines<C>((int)nz, +1, FFT_C2C, half_inout, half_inout, gz, gz, nh * ny * E, 1.0, st)))
        return e;
    LineGeom gy{nh, (int)nh, 1, (int)(nz * E), nh * ny};
    if (ny > 1 &&
        (e = fft_lines<C>((int)ny, +1, FFT_C2C, half_inout, half_inout, gy, gy, nh * nz * E, 1.0, st)))
        return e;
    LineGeom gi{1, (int)ny, nh, (int)(nz * E), nh * ny};
    LineGeom go{1, (int)ny, nx, (int)(nz * E), nx * ny};
    return fft_lines<C>((int)nx, +1, FFT_C2R, half_inout, real_out, gi, go, ny * nz * E, scale, st);
}

template cudaError_t r2c3d_batch<float2>(const void*, float2*, const int[3], int, cudaStream_t);
template cudaError_t c2r3d_batch<float2>(float2*, void*, const int[3], int, double, cudaStream_t);
template cudaError_t r2c3d<float2>(const void*, float2*, const int[3], cudaStream_t);
template cudaError_t r2c3d<double2>(const void*, double2*, const int[3], cudaStream_t);
template cudaError_t c2r3d<float2>(float2*, void*, const int[3], double, cudaStream_t);
template cudaError_t c2r3d<double2>(double2*, void*, const int[3], double, cudaStream_t);
template cudaError_t c2c3d<float2>(float2*, const int[3], int, double, cudaStream_t);
template cudaError_t c2c3d<double2>(double2*, const int[3], int, double, cudaStream_t);

}  // namespace tg
