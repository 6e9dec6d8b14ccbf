// The C++ picker's batched aligner: tom_mex_corr3d(..., 'peak', mask_cc)
// -> tom::corr3d_batch (Oscar3/c++Picker/src/tom/corr/corr.cpp:1217-1470)
// with CorrelationHandlerPeaks (src/tom/corr/correlation_handler.cpp:96-120).
//
// For every angle, template and particle: the template (mean 0, std 1) is
// rotated with the C++ tom::rotate (double source coordinates c + R (x - c),
// c = ceil((n-1)/2), float trilinear interpolation of
// src/tom/core/_transform.c:119-262), normalised under the mask
// (tom::norm_mask, NORM_NO_NORM, which also gives the variance) and
// transformed with its DC set to 0.  The template's rotated wedge multiplies
// the particle spectrum and the particle's wedge the template spectrum, each
// product's variance recomputed; the correlation c2r(T conj(P)) is scaled by
// 1/(sqrt(var_p var_t) N^2) and its first maximum (x fastest, under the
// ifftshifted mask_cc) kept per template/particle where it beats the best of
// the earlier angles.
//
// The reference multiplies the wedges on half spectra (z halved) and its c2r
// completes them as Hermitian; here the spectra are full (c2c), so a weight W
// acts as W(k) on the stored half, W(-k) on the other and (W(k) + W(-k))/2 on
// the kz = 0 (and kz = nz/2) planes, which is what the c2r does with them.
// The variance of a c2r output is taken from its spectrum (Parseval).
// Spectra are FP32 like the reference's single-precision path; sums FP64.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "match.h"

namespace tg {

namespace {

#define TG_GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

unsigned grid_n(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

struct Dims {
    int x, y, z;
    long long n;
};

// rotation R = Rz(phi) Rx(theta) Rz(psi) (tom_transf_init_rotmat_3d order) and
// the translation c - R c
struct Pose {
    double r[9];
    double t[3];
};

void cpp_rotmat(double phi, double theta, double psi, double R[9]) {
    double P[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    const double ang[3] = {phi, theta, psi};
    const int axes[3] = {2, 0, 2};
    for (int q = 0; q < 3; ++q) {
        const double a = ang[q];
        if (a - std::floor(a / (M_PI / 2.0)) * (2.0 * M_PI) == 0.0) continue;  // the reference's skip test
        const double s = std::sin(a), c = std::cos(a);
        const int i = axes[q] == 0 ? 1 : 0, j = axes[q] == 0 ? 2 : 1;
        for (int row = 0; row < 3; ++row) {
            const double p0 = P[3 * row + i], p1 = P[3 * row + j];
            P[3 * row + i] = p0 * c - p1 * s;
            P[3 * row + j] = p0 * s + p1 * c;
        }
    }
    for (int q = 0; q < 9; ++q) R[q] = P[q];
}

Pose make_pose(const Dims& d, double phi, double psi, double theta) {
    Pose p;
    cpp_rotmat(phi, theta, psi, p.r);
    const double c[3] = {std::ceil((d.x - 1) / 2.0), std::ceil((d.y - 1) / 2.0), std::ceil((d.z - 1) / 2.0)};
    for (int r = 0; r < 3; ++r) p.t[r] = c[r] - (p.r[3 * r] * c[0] + p.r[3 * r + 1] * c[1] + p.r[3 * r + 2] * c[2]);
    return p;
}

// ------------------------------------------------------------ C++ tom::rotate
__device__ __forceinline__ float lerp_rn(float a, float b, float w) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), w)); }

__device__ float cpp_sample(const float* __restrict__ v, int sx, int sy, int sz, double x, double y, double z) {
    if (x < 0.0 || y < 0.0 || z < 0.0 || x > (double)(sx - 1) || y > (double)(sy - 1) || z > (double)(sz - 1)) return 0.f;
    const int fx = (int)x, fy = (int)y, fz = (int)z;
    const float xo = (float)__dsub_rn(x, (double)fx), yo = (float)__dsub_rn(y, (double)fy),
                zo = (float)__dsub_rn(z, (double)fz);
    const long long sy_ = sx, sz_ = (long long)sx * sy;
    const float* s = v + fx + fy * sy_ + fz * sz_;
    const int c = (xo > 0.f ? 1 : 0) | (yo > 0.f ? 2 : 0) | (zo > 0.f ? 4 : 0);
    switch (c) {
        case 7: {
            const float x00x = lerp_rn(s[0], s[1], xo);
            const float x01x = lerp_rn(s[sy_], s[sy_ + 1], xo);
            const float x11x = lerp_rn(s[sy_ + sz_], s[sy_ + sz_ + 1], xo);
            const float x10x = lerp_rn(s[sz_], s[sz_ + 1], xo);
            const float x0yx = lerp_rn(x00x, x01x, yo);
            return lerp_rn(x0yx, lerp_rn(x10x, x11x, yo), zo);
        }
        case 6: {
            const float x0y0 = lerp_rn(s[0], s[sy_], yo);
            return lerp_rn(x0y0, lerp_rn(s[sz_], s[sz_ + sy_], yo), zo);
        }
        case 5: {
            const float x00x = lerp_rn(s[0], s[1], xo);
            return lerp_rn(x00x, lerp_rn(s[sz_], s[sz_ + 1], xo), zo);
        }
        case 3: {
            const float x00x = lerp_rn(s[0], s[1], xo);
            return lerp_rn(x00x, lerp_rn(s[sy_], s[sy_ + 1], xo), yo);
        }
        case 4: return lerp_rn(s[0], s[sz_], zo);
        case 2: return lerp_rn(s[0], s[sy_], yo);
        case 1: return lerp_rn(s[0], s[1], xo);
        default: return s[0];
    }
}

// out[b] = rotate(src[b / per_src], pose[b % per_src]); blockIdx.y = b
__global__ void k_cpp_rotate(const float* const* __restrict__ src, int per_src, const Pose* __restrict__ poses,
                             float* __restrict__ out, Dims d) {
    const int b = blockIdx.y;
    const float* v = src[b / per_src];
    const Pose p = poses[b % per_src];
    float* o = out + (long long)b * d.n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.x), y = (int)((i / d.x) % d.y), z = (int)(i / ((long long)d.x * d.y));
        double c[3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
            c[r] = __dadd_rn(__dmul_rn(p.r[3 * r], (double)x),
                             __dadd_rn(__dmul_rn(p.r[3 * r + 1], (double)y),
                                       __dadd_rn(__dmul_rn(p.r[3 * r + 2], (double)z), p.t[r])));
        o[i] = cpp_sample(v, d.x, d.y, d.z, c[0], c[1], c[2]);
    }
}

// ------------------------------------------------------------ normalisation
// One block per volume, FP64 sums.  mode 0: tom::norm_mask(NORM_NO_NORM) with
// variance; 1: stat, v - mean in float (rotated templates); 2: stat, v - mean
// in double (particles); 3: stat, (v - mean)/sqrt(var) (templates once).
template <int NT>
__device__ void block_sum2(double& a, double& b) {
    __shared__ double sa[NT / 32], sb[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0, y = 0;
        for (int w = 0; w < NT / 32; ++w) {
            x += sa[w];
            y += sb[w];
        }
        sa[0] = x;
        sb[0] = y;
    }
    __syncthreads();
    a = sa[0];
    b = sb[0];
    __syncthreads();
}

constexpr int NORM_THREADS = 512;

__global__ void __launch_bounds__(NORM_THREADS) k_normalise(const float* const* __restrict__ src, float* __restrict__ out,
                                                            const float* __restrict__ mask, long long n, int mode,
                                                            double* __restrict__ var) {
    const float* v = src ? src[blockIdx.x] : out + (long long)blockIdx.x * n;
    float* o = out + (long long)blockIdx.x * n;
    double s1 = 0, s2 = 0;
    if (mode == 0) {
        double cnt = 0;
        for (long long i = threadIdx.x; i < n; i += NORM_THREADS)
            if (mask[i] != 0.f) {
                cnt += 1;
                s1 += (double)v[i];
            }
        block_sum2<NORM_THREADS>(s1, cnt);
        const double mean0 = s1 / cnt;
        double t1 = 0, t2 = 0;
        for (long long i = threadIdx.x; i < n; i += NORM_THREADS) {
            const float m = mask[i];
            if (m != 0.f) {
                const float w = (float)(((double)v[i] - mean0) * (double)m);
                o[i] = w;
                t1 += (double)w;
                t2 += (double)w * (double)w;
            } else {
                o[i] = 0.f;
            }
        }
        block_sum2<NORM_THREADS>(t1, t2);
        const double mean1 = t1 / cnt;
        if (threadIdx.x == 0) var[blockIdx.x] = (t2 - cnt * mean1 * mean1) / (double)n;
        if (mean1 != 0.0)
            for (long long i = threadIdx.x; i < n; i += NORM_THREADS)
                if (mask[i] != 0.f) o[i] = (float)((double)o[i] - mean1);
        return;
    }
    for (long long i = threadIdx.x; i < n; i += NORM_THREADS) {
        const double x = (double)v[i];
        s1 += x;
        s2 += x * x;
    }
    block_sum2<NORM_THREADS>(s1, s2);
    const double mean = s1 / (double)n;
    const double vv = (s2 - (double)n * mean * mean) / (double)n;
    if (threadIdx.x == 0) var[blockIdx.x] = vv;
    if (mode == 1) {
        const float fm = (float)(-mean);
        for (long long i = threadIdx.x; i < n; i += NORM_THREADS) o[i] = __fmul_rn(__fadd_rn(v[i], fm), 1.f);
    } else if (mode == 2) {
        for (long long i = threadIdx.x; i < n; i += NORM_THREADS) o[i] = (float)(((double)v[i] + (-mean)) * 1.0);
    } else {
        const double sc = vv != 0.0 ? 1.0 / sqrt(vv) : 0.0;
        for (long long i = threadIdx.x; i < n; i += NORM_THREADS) o[i] = (float)(((double)v[i] + (-mean)) * sc);
    }
}

__global__ void k_real_to_c(const float* __restrict__ a, float2* __restrict__ z, long long n) {
    TG_GRID_STRIDE(i, n) z[i] = make_float2(a[i], 0.f);
}
__global__ void k_dc_zero(float2* z, long long n, int nb) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb) z[(long long)b * n] = make_float2(0.f, 0.f);
}

// ------------------------------------------------------------ wedges
// SimpleWedge on the full grid (src/tom/core/wedge.cpp:107-180), float arithmetic
struct SimpleW {
    float p[12];
    float tan_a, cut;
};
__global__ void k_simple_wedge(const SimpleW* __restrict__ ws, float* __restrict__ out, Dims d) {
    const SimpleW w = ws[blockIdx.y];
    float* o = out + (long long)blockIdx.y * d.n;
    const int ox = d.x / 2 + d.x % 2, oy = d.y / 2 + d.y % 2, oz = d.z / 2 + d.z % 2;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.x), y = (int)((i / d.x) % d.y), z = (int)(i / ((long long)d.x * d.y));
        const float xs = (float)((x + ox) % d.x), ys = (float)((y + oy) % d.y), zs = (float)((z + oz) % d.z);
        const float x_ = __fadd_rn(__fmul_rn(w.p[0], xs), __fadd_rn(__fmul_rn(w.p[1], ys), __fadd_rn(__fmul_rn(w.p[2], zs), w.p[3])));
        float r;
        if (w.cut > 0.f) {
            const float y_ = __fadd_rn(__fmul_rn(w.p[4], xs), __fadd_rn(__fmul_rn(w.p[5], ys), __fadd_rn(__fmul_rn(w.p[6], zs), w.p[7])));
            const float z_ = fabsf(__fadd_rn(__fmul_rn(w.p[8], xs), __fadd_rn(__fmul_rn(w.p[9], ys), __fadd_rn(__fmul_rn(w.p[10], zs), w.p[11]))));
            const float rr = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(x_, x_), __fmul_rn(y_, y_)), __fmul_rn(z_, z_)));
            r = (rr <= w.cut) && ((z_ < 1e-4f) || (w.tan_a <= __fdiv_rn(fabsf(x_), z_))) ? 1.f : 0.f;
        } else {
            const float z_ = __fadd_rn(__fmul_rn(w.p[8], xs), __fadd_rn(__fmul_rn(w.p[9], ys), __fadd_rn(__fmul_rn(w.p[10], zs), w.p[11])));
            r = (z_ < 1e-4f) || (w.tan_a <= __fdiv_rn(fabsf(x_), fabsf(z_))) ? 1.f : 0.f;
        }
        o[i] = r;
    }
}
// ifftshift (tom::fftshift(..., true)): out[i] = in[(i + n/2) mod n] per axis
__global__ void k_ifftshift_batch(const float* __restrict__ in, float* __restrict__ out, Dims d) {
    const float* a = in + (long long)blockIdx.y * d.n;
    float* o = out + (long long)blockIdx.y * d.n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < d.n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % d.x), y = (int)((i / d.x) % d.y), z = (int)(i / ((long long)d.x * d.y));
        const int sx = (x + d.x / 2) % d.x, sy = (y + d.y / 2) % d.y, sz = (z + d.z / 2) % d.z;
        o[i] = a[sx + (long long)d.x * (sy + (long long)d.y * sz)];
    }
}

// 1 where a volume holds a value other than 1 (VolumeWedge::active), one block per volume
__global__ void k_not_all_ones(const float* const* __restrict__ v, long long n, int* __restrict__ out) {
    const float* a = v[blockIdx.x];
    int any = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) any |= a[i] != 1.f;
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) out[blockIdx.x] = any;
}

// ------------------------------------------------------------ pairs
struct PairJob {
    int t_spec;   // index into the template spectra of the chunk
    int p;        // particle
    int wt;       // template wedge volume index in the chunk, or -1
    int wp;       // particle wedge volume index, or -1
    double var_t, var_p;  // variances without the other's wedge
};

// weight of the c2r of a z-halved product: W(k) on the stored half, W(-k) on
// the other, the mean of both on the kz = 0 (and nz/2) planes
__device__ __forceinline__ float w_eff(float wk, float wm, int z, int nz) {
    if (z == 0 || (2 * z == nz)) return 0.5f * (wk + wm);
    return z <= nz / 2 ? wk : wm;
}

constexpr int PAIR_THREADS = 512;

__global__ void __launch_bounds__(PAIR_THREADS) k_pair_product(const PairJob* __restrict__ jobs,
                                                               const float2* __restrict__ tspec,
                                                               const float2* __restrict__ pspec,
                                                               const float* __restrict__ wts,
                                                               const float* __restrict__ wps, float2* __restrict__ C,
                                                               double* __restrict__ scale, Dims d) {
    const PairJob jb = jobs[blockIdx.x];
    const float2* T = tspec + (long long)jb.t_spec * d.n;
    const float2* P = pspec + (long long)jb.p * d.n;
    const float* WT = jb.wt >= 0 ? wts + (long long)jb.wt * d.n : nullptr;
    const float* WP = jb.wp >= 0 ? wps + (long long)jb.wp * d.n : nullptr;
    float2* out = C + (long long)blockIdx.x * d.n;
    double ep = 0, et = 0;
    for (long long i = threadIdx.x; i < d.n; i += PAIR_THREADS) {
        const int x = (int)(i % d.x), y = (int)((i / d.x) % d.y), z = (int)(i / ((long long)d.x * d.y));
        const long long m = (long long)((d.x - x) % d.x) + (long long)d.x * (((d.y - y) % d.y) + (long long)d.y * ((d.z - z) % d.z));
        float wt = 1.f, wp = 1.f, wtk = 1.f, wtm = 1.f, wpk = 1.f, wpm = 1.f;
        if (WT) { wtk = WT[i]; wtm = WT[m]; wt = w_eff(wtk, wtm, z, d.z); }
        if (WP) { wpk = WP[i]; wpm = WP[m]; wp = w_eff(wpk, wpm, z, d.z); }
        const float2 t = T[i], p = P[i];
        if (WT) ep += ((double)p.x * p.x + (double)p.y * p.y) * (double)wt * (double)wt;
        if (WP) et += ((double)t.x * t.x + (double)t.y * t.y) * (double)wp * (double)wp;
        const float wc = w_eff(__fmul_rn(wtk, wpk), __fmul_rn(wtm, wpm), z, d.z);
        float2 c = cmulc(t, p);
        c.x *= wc;
        c.y *= wc;
        out[i] = i == 0 ? make_float2(0.f, 0.f) : c;
    }
    block_sum2<PAIR_THREADS>(ep, et);
    if (threadIdx.x == 0) {
        const double nn = (double)d.n * (double)d.n;
        const double vp = WT ? ep / nn : jb.var_p;
        const double vt = WP ? et / nn : jb.var_t;
        scale[blockIdx.x] = 1.0 / (sqrt(vp * vt) * (double)d.n * (double)d.n);
    }
}

// first maximum (x fastest) of (float)(re * scale) under mask (ifftshifted mask_cc)
__global__ void __launch_bounds__(PAIR_THREADS) k_pair_peak(const float2* __restrict__ C, const double* __restrict__ scale,
                                                            const float* __restrict__ mask, long long n,
                                                            float* __restrict__ val, long long* __restrict__ pos) {
    const float2* c = C + (long long)blockIdx.x * n;
    const double sc = scale[blockIdx.x];
    float best = -INFINITY;
    long long bi = -1;
    for (long long i = threadIdx.x; i < n; i += PAIR_THREADS) {
        if (mask && mask[i] == 0.f) continue;
        const float v = (float)((double)c[i].x * sc);
        if (bi < 0 || v > best) {  // i grows per thread: the first of equal values stays
            best = v;
            bi = i;
        }
    }
    __shared__ float sv[PAIR_THREADS];
    __shared__ long long si[PAIR_THREADS];
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = PAIR_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            const float ov = sv[threadIdx.x + s];
            const long long oi = si[threadIdx.x + s];
            const float mv = sv[threadIdx.x];
            const long long mi = si[threadIdx.x];
            if (oi >= 0 && (mi < 0 || ov > mv || (ov == mv && oi < mi))) {
                sv[threadIdx.x] = ov;
                si[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        val[blockIdx.x] = sv[0];
        pos[blockIdx.x] = si[0];
    }
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t get(size_t bytes) { return cudaMalloc(&p, bytes < 16 ? 16 : bytes); }
};

}  // namespace

int corr3d_peaks(tomgpu_ctx* ctx, const int n[3], const float* const* templates, int nt, const float* const* particles,
                 int np, const double* angles_deg, int nang, const float* mask, const tomgpu_wedge_spec* wedge_t,
                 const tomgpu_wedge_spec* wedge_p, const float* mask_cc, double* peak, double* val, int32_t* angle_idx) {
    cudaStream_t st = ctx->stream;
    Dims d{n[0], n[1], n[2], (long long)n[0] * n[1] * n[2]};
    const long long N = d.n;
    const int cutoff = (std::min(n[0], std::min(n[1], n[2])) - 1) / 2;  // SimpleWedge radius of the MEX
    const double deg = 3.141592653589793238512808959406186204433 / 180.;
    cudaError_t e = cudaSuccess;
#define TG_CK(x)                                              \
    do {                                                      \
        if ((e = (x)) != cudaSuccess) return cuda_fail(ctx, e, #x); \
    } while (0)

    for (int k = 0; k < nt * np; ++k) {
        val[k] = NAN;
        angle_idx[k] = 0;
        peak[3 * k] = peak[3 * k + 1] = peak[3 * k + 2] = 0;
    }
    // device pointer tables
    DevBuf d_tptr, d_pptr, d_tn, d_tvar, d_pn, d_pvar, d_pspec, d_mcc;
    TG_CK(d_tptr.get(sizeof(float*) * nt));
    TG_CK(d_pptr.get(sizeof(float*) * np));
    TG_CK(cudaMemcpyAsync(d_tptr.p, templates, sizeof(float*) * nt, cudaMemcpyHostToDevice, st));
    TG_CK(cudaMemcpyAsync(d_pptr.p, particles, sizeof(float*) * np, cudaMemcpyHostToDevice, st));
    // templates: mean 0, std 1
    TG_CK(d_tn.get(sizeof(float) * N * nt));
    TG_CK(d_tvar.get(sizeof(double) * nt));
    k_normalise<<<nt, NORM_THREADS, 0, st>>>((const float* const*)d_tptr.p, (float*)d_tn.p, nullptr, N, 3,
                                             (double*)d_tvar.p);
    // particles: normalised, spectrum with DC 0
    TG_CK(d_pn.get(sizeof(float) * N * np));
    TG_CK(d_pvar.get(sizeof(double) * np));
    k_normalise<<<np, NORM_THREADS, 0, st>>>((const float* const*)d_pptr.p, (float*)d_pn.p, mask, N, mask ? 0 : 2,
                                             (double*)d_pvar.p);
    TG_CK(d_pspec.get(sizeof(float2) * N * np));
    k_real_to_c<<<grid_n(N * np), 256, 0, st>>>((const float*)d_pn.p, (float2*)d_pspec.p, N * np);
    TG_CK(c2c3d_batch((float2*)d_pspec.p, n, np, -1, 1.0, st));
    k_dc_zero<<<(np + 127) / 128, 128, 0, st>>>((float2*)d_pspec.p, N, np);
    TG_CK(cudaGetLastError());
    std::vector<double> tvar(nt), pvar(np);
    TG_CK(cudaMemcpyAsync(tvar.data(), d_tvar.p, sizeof(double) * nt, cudaMemcpyDeviceToHost, st));
    TG_CK(cudaMemcpyAsync(pvar.data(), d_pvar.p, sizeof(double) * np, cudaMemcpyDeviceToHost, st));
    TG_CK(cudaStreamSynchronize(st));
    if (mask_cc) {  // CorrelationHandlerPeaks keeps the ifftshifted mask
        TG_CK(d_mcc.get(sizeof(float) * N));
        k_ifftshift_batch<<<dim3(grid_n(N), 1), 256, 0, st>>>(mask_cc, (float*)d_mcc.p, d);
    }

    // particle wedges (unrotated), full grid
    auto wedge_active = [&](const tomgpu_wedge_spec* w) {
        if (!w || w->kind == TOMGPU_WEDGE_NONE) return false;
        if (w->kind == TOMGPU_WEDGE_SIMPLE) return w->angle_deg * deg > 0 || cutoff > 0;
        return true;
    };
    // VolumeWedge::active: a weight volume of all ones is no wedge
    std::vector<int> t_vol_active(nt, 1), p_vol_active(np, 1);
    {
        std::vector<const float*> vs;
        std::vector<int*> dst;
        for (int t = 0; t < nt; ++t)
            if (wedge_t && wedge_t[t].kind == TOMGPU_WEDGE_VOLUME) { vs.push_back(wedge_t[t].volume); dst.push_back(&t_vol_active[t]); }
        for (int p = 0; p < np; ++p)
            if (wedge_p && wedge_p[p].kind == TOMGPU_WEDGE_VOLUME) { vs.push_back(wedge_p[p].volume); dst.push_back(&p_vol_active[p]); }
        if (!vs.empty()) {
            DevBuf ptrs, flags;
            std::vector<int> hf(vs.size());
            TG_CK(ptrs.get(sizeof(float*) * vs.size()));
            TG_CK(flags.get(sizeof(int) * vs.size()));
            TG_CK(cudaMemcpyAsync(ptrs.p, vs.data(), sizeof(float*) * vs.size(), cudaMemcpyHostToDevice, st));
            k_not_all_ones<<<(unsigned)vs.size(), 256, 0, st>>>((const float* const*)ptrs.p, N, (int*)flags.p);
            TG_CK(cudaMemcpyAsync(hf.data(), flags.p, sizeof(int) * vs.size(), cudaMemcpyDeviceToHost, st));
            TG_CK(cudaStreamSynchronize(st));
            for (size_t q = 0; q < vs.size(); ++q) *dst[q] = hf[q];
        }
    }
    std::vector<int> wp_index(np, -1);
    int n_wp = 0;
    for (int p = 0; p < np; ++p)
        if (wedge_p && wedge_active(&wedge_p[p]) && (wedge_p[p].kind != TOMGPU_WEDGE_VOLUME || p_vol_active[p]))
            wp_index[p] = n_wp++;
    DevBuf d_wp, d_sw, d_pose, d_src;
    TG_CK(d_wp.get(sizeof(float) * N * std::max(1, n_wp)));
    auto simple_params = [&](double phi, double psi, double theta, float angle_deg) {
        SimpleW w;
        double R[9];
        cpp_rotmat(phi, theta, psi, R);
        const float c[3] = {(float)std::ceil((d.x - 1) / 2.), (float)std::ceil((d.y - 1) / 2.),
                            (float)std::ceil((d.z - 1) / 2.)};
        for (int r = 0; r < 3; ++r) {
            for (int q = 0; q < 3; ++q) w.p[4 * r + q] = (float)R[3 * r + q];
            w.p[4 * r + 3] = (float)(-(R[3 * r] * c[0] + R[3 * r + 1] * c[1] + R[3 * r + 2] * c[2]));
        }
        const float maxdist = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        w.tan_a = (float)std::tan(angle_deg * deg);
        w.cut = (cutoff > 0 && (float)cutoff < maxdist) ? (float)cutoff : 0.f;
        return w;
    };
    if (n_wp) {
        std::vector<SimpleW> sw;
        std::vector<int> swi;
        std::vector<const float*> vsrc;
        std::vector<int> vi;
        for (int p = 0; p < np; ++p) {
            if (wp_index[p] < 0) continue;
            if (wedge_p[p].kind == TOMGPU_WEDGE_SIMPLE) {
                sw.push_back(simple_params(0, 0, 0, wedge_p[p].angle_deg));
                swi.push_back(wp_index[p]);
            } else {
                vsrc.push_back(wedge_p[p].volume);
                vi.push_back(wp_index[p]);
            }
        }
        if (!sw.empty()) {
            DevBuf tmp, par;
            TG_CK(par.get(sizeof(SimpleW) * sw.size()));
            TG_CK(tmp.get(sizeof(float) * N * sw.size()));
            TG_CK(cudaMemcpyAsync(par.p, sw.data(), sizeof(SimpleW) * sw.size(), cudaMemcpyHostToDevice, st));
            k_simple_wedge<<<dim3(grid_n(N), (unsigned)sw.size()), 256, 0, st>>>((const SimpleW*)par.p, (float*)tmp.p, d);
            for (size_t q = 0; q < sw.size(); ++q)
                TG_CK(cudaMemcpyAsync((float*)d_wp.p + (long long)swi[q] * N, (float*)tmp.p + (long long)q * N,
                                      sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
            TG_CK(cudaStreamSynchronize(st));
        }
        if (!vsrc.empty()) {
            DevBuf tmp, ptrs, pose;
            const Pose id = make_pose(d, 0, 0, 0);
            TG_CK(ptrs.get(sizeof(float*) * vsrc.size()));
            TG_CK(pose.get(sizeof(Pose)));
            TG_CK(tmp.get(sizeof(float) * N * vsrc.size()));
            TG_CK(cudaMemcpyAsync(ptrs.p, vsrc.data(), sizeof(float*) * vsrc.size(), cudaMemcpyHostToDevice, st));
            TG_CK(cudaMemcpyAsync(pose.p, &id, sizeof(Pose), cudaMemcpyHostToDevice, st));
            k_cpp_rotate<<<dim3(grid_n(N), (unsigned)vsrc.size()), 256, 0, st>>>((const float* const*)ptrs.p, 1,
                                                                                 (const Pose*)pose.p, (float*)tmp.p, d);
            DevBuf sh;
            TG_CK(sh.get(sizeof(float) * N * vsrc.size()));
            k_ifftshift_batch<<<dim3(grid_n(N), (unsigned)vsrc.size()), 256, 0, st>>>((float*)tmp.p, (float*)sh.p, d);
            for (size_t q = 0; q < vsrc.size(); ++q)
                TG_CK(cudaMemcpyAsync((float*)d_wp.p + (long long)vi[q] * N, (float*)sh.p + (long long)q * N,
                                      sizeof(float) * N, cudaMemcpyDeviceToDevice, st));
            TG_CK(cudaStreamSynchronize(st));
        }
    }

    // angle chunks: E angles x nt templates of spectra and wedges at a time
    const long long budget = 1LL << 24;  // voxels per work array
    const int E = (int)std::max<long long>(1, std::min<long long>(nang, budget / std::max<long long>(1, N * nt)));
    const int PB = (int)std::max<long long>(1, std::min<long long>((long long)nt * np * E, budget / N));
    DevBuf d_rot, d_tspec, d_ttvar, d_wt, d_jobs, d_C, d_scale, d_val, d_pos, d_ptab;
    TG_CK(d_rot.get(sizeof(float) * N * nt * E));
    TG_CK(d_tspec.get(sizeof(float2) * N * nt * E));
    TG_CK(d_ttvar.get(sizeof(double) * nt * E));
    TG_CK(d_wt.get(sizeof(float) * N * nt * E));
    TG_CK(d_jobs.get(sizeof(PairJob) * PB));
    TG_CK(d_C.get(sizeof(float2) * N * PB));
    TG_CK(d_scale.get(sizeof(double) * PB));
    TG_CK(d_val.get(sizeof(float) * PB));
    TG_CK(d_pos.get(sizeof(long long) * PB));
    TG_CK(d_pose.get(sizeof(Pose) * E));
    TG_CK(d_sw.get(sizeof(SimpleW) * nt * E));
    // template pointers into the normalised copies; template wedge volumes
    std::vector<const float*> tnp(nt), twv;
    for (int t = 0; t < nt; ++t) tnp[t] = (const float*)d_tn.p + (long long)t * N;
    TG_CK(d_ptab.get(sizeof(float*) * nt));
    TG_CK(cudaMemcpyAsync(d_ptab.p, tnp.data(), sizeof(float*) * nt, cudaMemcpyHostToDevice, st));
    std::vector<int> tw_kind(nt, 0);
    for (int t = 0; t < nt; ++t)
        if (wedge_t && wedge_active(&wedge_t[t]) && (wedge_t[t].kind != TOMGPU_WEDGE_VOLUME || t_vol_active[t]))
            tw_kind[t] = wedge_t[t].kind;

    std::vector<Pose> poses(E);
    std::vector<SimpleW> sws(nt * E);
    std::vector<double> ttvar(nt * E);
    std::vector<PairJob> jobs;
    std::vector<int> job_angle, job_t;
    std::vector<float> hval(PB);
    std::vector<long long> hpos(PB);
    for (int a0 = 0; a0 < nang; a0 += E) {
        const int ea = std::min(E, nang - a0);
        for (int q = 0; q < ea; ++q) {
            const double* an = angles_deg + 3 * (long long)(a0 + q);
            poses[q] = make_pose(d, an[0] * deg, an[1] * deg, an[2] * deg);
            for (int t = 0; t < nt; ++t)
                if (tw_kind[t] == TOMGPU_WEDGE_SIMPLE)
                    sws[t * ea + q] = simple_params(an[0] * deg, an[1] * deg, an[2] * deg, wedge_t[t].angle_deg);
        }
        TG_CK(cudaMemcpyAsync(d_pose.p, poses.data(), sizeof(Pose) * ea, cudaMemcpyHostToDevice, st));
        // rotated templates [t][e], normalised, spectra with DC 0
        k_cpp_rotate<<<dim3(grid_n(N), (unsigned)(nt * ea)), 256, 0, st>>>((const float* const*)d_ptab.p, ea,
                                                                           (const Pose*)d_pose.p, (float*)d_rot.p, d);
        k_normalise<<<nt * ea, NORM_THREADS, 0, st>>>(nullptr, (float*)d_rot.p, mask, N, mask ? 0 : 1,
                                                      (double*)d_ttvar.p);
        k_real_to_c<<<grid_n(N * nt * ea), 256, 0, st>>>((const float*)d_rot.p, (float2*)d_tspec.p, N * nt * ea);
        TG_CK(c2c3d_batch((float2*)d_tspec.p, n, nt * ea, -1, 1.0, st));
        k_dc_zero<<<(nt * ea + 127) / 128, 128, 0, st>>>((float2*)d_tspec.p, N, nt * ea);
        // template wedges [t][e]
        bool any_simple = false, any_vol = false;
        for (int t = 0; t < nt; ++t) {
            any_simple |= tw_kind[t] == TOMGPU_WEDGE_SIMPLE;
            any_vol |= tw_kind[t] == TOMGPU_WEDGE_VOLUME;
        }
        if (any_simple) {
            TG_CK(cudaMemcpyAsync(d_sw.p, sws.data(), sizeof(SimpleW) * nt * ea, cudaMemcpyHostToDevice, st));
            k_simple_wedge<<<dim3(grid_n(N), (unsigned)(nt * ea)), 256, 0, st>>>((const SimpleW*)d_sw.p, (float*)d_wt.p, d);
        }
        if (any_vol) {
            // rotated, ifftshifted weight volumes of the templates that have one
            std::vector<const float*> vs;
            std::vector<int> vt;
            for (int t = 0; t < nt; ++t)
                if (tw_kind[t] == TOMGPU_WEDGE_VOLUME) {
                    vs.push_back(wedge_t[t].volume);
                    vt.push_back(t);
                }
            const int nv = (int)vs.size();
            DevBuf tmp, sh, ptrs;
            TG_CK(ptrs.get(sizeof(float*) * nv));
            TG_CK(tmp.get(sizeof(float) * N * nv * ea));
            TG_CK(sh.get(sizeof(float) * N * nv * ea));
            TG_CK(cudaMemcpyAsync(ptrs.p, vs.data(), sizeof(float*) * nv, cudaMemcpyHostToDevice, st));
            k_cpp_rotate<<<dim3(grid_n(N), (unsigned)(nv * ea)), 256, 0, st>>>((const float* const*)ptrs.p, ea,
                                                                               (const Pose*)d_pose.p, (float*)tmp.p, d);
            k_ifftshift_batch<<<dim3(grid_n(N), (unsigned)(nv * ea)), 256, 0, st>>>((float*)tmp.p, (float*)sh.p, d);
            for (int v = 0; v < nv; ++v)
                TG_CK(cudaMemcpyAsync((float*)d_wt.p + (long long)vt[v] * ea * N, (float*)sh.p + (long long)v * ea * N,
                                      sizeof(float) * N * ea, cudaMemcpyDeviceToDevice, st));
            TG_CK(cudaStreamSynchronize(st));
        }
        TG_CK(cudaMemcpyAsync(ttvar.data(), d_ttvar.p, sizeof(double) * nt * ea, cudaMemcpyDeviceToHost, st));
        TG_CK(cudaStreamSynchronize(st));
        // pairs in angle order
        jobs.clear();
        job_angle.clear();
        job_t.clear();
        for (int q = 0; q < ea; ++q)
            for (int t = 0; t < nt; ++t) {
                if (tvar[t] == 0.0) continue;  // template not loaded
                for (int p = 0; p < np; ++p) {
                    if (pvar[p] == 0.0) continue;  // particle not loaded
                    PairJob j;
                    j.t_spec = t * ea + q;
                    j.p = p;
                    j.wt = tw_kind[t] ? t * ea + q : -1;
                    j.wp = wp_index[p];
                    j.var_t = ttvar[t * ea + q];
                    j.var_p = pvar[p];
                    jobs.push_back(j);
                    job_angle.push_back(a0 + q);
                    job_t.push_back(t);
                }
            }
        for (size_t j0 = 0; j0 < jobs.size(); j0 += PB) {
            const int nb = (int)std::min<size_t>(PB, jobs.size() - j0);
            TG_CK(cudaMemcpyAsync(d_jobs.p, jobs.data() + j0, sizeof(PairJob) * nb, cudaMemcpyHostToDevice, st));
            k_pair_product<<<nb, PAIR_THREADS, 0, st>>>((const PairJob*)d_jobs.p, (const float2*)d_tspec.p,
                                                        (const float2*)d_pspec.p, (const float*)d_wt.p,
                                                        (const float*)d_wp.p, (float2*)d_C.p, (double*)d_scale.p, d);
            TG_CK(c2c3d_batch((float2*)d_C.p, n, nb, +1, 1.0, st));
            k_pair_peak<<<nb, PAIR_THREADS, 0, st>>>((const float2*)d_C.p, (const double*)d_scale.p,
                                                     (const float*)d_mcc.p, N, (float*)d_val.p, (long long*)d_pos.p);
            TG_CK(cudaGetLastError());
            TG_CK(cudaMemcpyAsync(hval.data(), d_val.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, st));
            TG_CK(cudaMemcpyAsync(hpos.data(), d_pos.p, sizeof(long long) * nb, cudaMemcpyDeviceToHost, st));
            TG_CK(cudaStreamSynchronize(st));
            ctx->launches += 3 + 3;
            for (int b = 0; b < nb; ++b) {
                if (hpos[b] < 0) continue;  // empty mask: no peak
                const PairJob& j = jobs[j0 + b];
                const int t = job_t[j0 + b];
                const long long k = (long long)j.p * nt + t;
                const double v = (double)hval[b];
                if (v > val[k] || angle_idx[k] == 0) {
                    val[k] = v;
                    angle_idx[k] = job_angle[j0 + b] + 1;
                    peak[3 * k] = (double)(hpos[b] % d.x);
                    peak[3 * k + 1] = (double)((hpos[b] / d.x) % d.y);
                    peak[3 * k + 2] = (double)(hpos[b] / ((long long)d.x * d.y));
                }
            }
        }
        ctx->launches += 6;
    }
#undef TG_CK
    return TOMGPU_OK;
}

}  // namespace tg
