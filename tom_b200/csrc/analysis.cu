// Peak analysis of FLCF maps: the peak-to-sidelobe ratio (PSR) and the
// second-order ("Autocorrelation") map of
// Oscar3/matlabPicker/analyze/tom_os3_analyzePeak.m, and the per-rotation
// search that carries them (tom_os3_findTemplate.m:255-307 with
// search/tom_os3_bestPeak.m).
//
// PSR (tom_os3_analyzePeak.m:61-101): the mask is tom_os3_sphereMask(template)
// with a centred floor(T/4) box zeroed, pasted at the centre of the map; the
// map's local mean and std under it (tom_os3_mean/std, convolution through
// the FFT) give (peak - mean)/std where std > 1000 eps(max std), else 0.
//
// Autocorrelation (tom_os3_analyzePeak.m:174-190): A = tom_os3_corr(t, t)
// (same-size FLCF with the default sphere mask, circular, divided at every
// voxel), then tom_os3_corr(peak, A) with the correlation mask and A's own
// statistics (the FLCF of the search, sizes differ).
//
// Both run in FP64 (the local variances E[x^2] - E[x]^2 and the
// correlation), each output rounded once to float.  The scalar statistics of
// a rotation (template mean/std, the 'numeric artefact' tests of
// tom_os3_corr.m:108-127) stay on the device, so a rotation issues no host
// synchronisation.
#include <cfloat>
#include <cmath>
#include <vector>

#include "analysis.h"
#include "common.cuh"
#include "fft3d.h"
#include "match.h"
#include "misc.h"

namespace tg {

namespace {

// device scalar slots of one analysis step
enum {
    S_AC_TSUM = 0,   // sum of t under the sphere (autocorrelation template statistics)
    S_AC_TSQ,        // sum of t^2 under the sphere
    S_AC_GSUM,       // sum of t over the box (tom_norm of the artefact branch)
    S_AC_GSQ,
    S_AC_STDSUM,     // sum of the local std of t
    S_AC_HOT,        // hot-pixel threshold on the local std, or -1
    S_PK_SUM,        // sum of the peak map
    S_PK_SQ,
    S_SOC_STDSUM,    // sum of the peak map's local std under the correlation mask
    S_SOC_HOT,
    S_A_SUM,         // sum of A under the correlation mask
    S_A_SQ,
    S_PSR_MAXBITS,   // max local std under the PSR mask (float bits, as an unsigned)
    S_COUNT
};

unsigned grid_n(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

#define TG_GRID_STRIDE(i, n) \
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// K sums over n voxels of f(i, v[K]) added to out[0..K) (one atomicAdd per block and sum).
template <int K, typename F>
__global__ void __launch_bounds__(256) k_msum(F f, long long n, double* out) {
    double acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0;
    TG_GRID_STRIDE(i, n) {
        double v[K];
        f(i, v);
#pragma unroll
        for (int k = 0; k < K; ++k) acc[k] += v[k];
    }
    __shared__ double ws[8][K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double a = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5][k] = a;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w][threadIdx.x];
        atomicAdd(out + threadIdx.x, s);
    }
}
template <int K, typename F> cudaError_t msum(F f, long long n, double* out, cudaStream_t st) {
    long long b = (n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    k_msum<K><<<(unsigned)(b < 1 ? 1 : b), 256, 0, st>>>(f, n, out);
    return cudaGetLastError();
}

// sum and sum of squares over the mask's nonzeros (all voxels without a mask)
struct Moments {
    const float* a;
    const float* m;
    __device__ void operator()(long long i, double* v) const {
        const double x = (double)a[i];
        const double w = (m == nullptr || m[i] != 0.f) ? 1.0 : 0.0;
        v[0] = x * w;
        v[1] = x * x * w;
    }
};
struct FloatSum {
    const float* a;
    __device__ void operator()(long long i, double* v) const { v[0] = (double)a[i]; }
};
struct DoubleSum {
    const double* a;
    __device__ void operator()(long long i, double* v) const { v[0] = a[i]; }
};

// ------------------------------------------------------------- elementwise
__global__ void k_f32_f64_sq(const float* __restrict__ a, double* __restrict__ b, long long n, int square) {
    TG_GRID_STRIDE(i, n) {
        const double x = (double)a[i];
        b[i] = square ? x * x : x;
    }
}
// c = a * b or c = a * conj(b)
__global__ void k_cmul3(const double2* __restrict__ a, const double2* __restrict__ b, double2* __restrict__ c,
                        long long n, int conj_b) {
    TG_GRID_STRIDE(i, n) c[i] = conj_b ? cmulc(a[i], b[i]) : cmul(a[i], b[i]);
}
// a = a * conj(b)   (a holds the peak spectrum's product in place)
__global__ void k_cmulc_inplace_b(const double2* __restrict__ a, double2* __restrict__ b, long long n) {
    TG_GRID_STRIDE(i, n) b[i] = cmulc(a[i], b[i]);
}

__device__ __forceinline__ float matlab_eps_single(float x) {
    // eps(single(x)) for x >= 0: the spacing of floats at x; 2^-149 below the normal range
    const unsigned e = (__float_as_uint(x) >> 23) & 0xffu;
    return (float)ldexp(1.0, (e == 0u ? 1 : (int)e) - 150);
}

// PSR: local std (float) and its maximum
__global__ void k_psr_std(const double* __restrict__ m1, const double* __restrict__ m2, float* __restrict__ sd,
                          long long n, unsigned* maxbits) {
    unsigned best = 0;
    TG_GRID_STRIDE(i, n) {
        const double a = m1[i];
        const double var = m2[i] - a * a;
        const float s = (float)sqrt(var > 0 ? var : 0.0);
        sd[i] = s;
        best = max(best, __float_as_uint(s));  // s >= 0: the bit patterns order like the values
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, best);
}
__global__ void k_psr_final(const float* __restrict__ pk, const double* __restrict__ m1, const float* __restrict__ sd,
                            float* __restrict__ out, long long n, const unsigned* maxbits) {
    const float tol = (float)(1000.0 * (double)matlab_eps_single(__uint_as_float(*maxbits)));
    TG_GRID_STRIDE(i, n) {
        const float s = sd[i];
        out[i] = s > tol ? (float)(((double)pk[i] - m1[i]) / (double)s) : 0.f;
    }
}

// the second test of tom_os3_corr.m:108-127 after the (value-preserving)
// tom_norm of the first: threshold on the original local std, or -1
__device__ double hot_threshold(double std_sum, double n, double gsum, double gsq) {
    if (std_sum / n >= 0.01) return -1.0;
    const double gm = gsum / n;
    double var = gsq / n - gm * gm;
    const double s = sqrt(var > 0 ? var : 0.0);
    const double scale = s != 0 ? 1.0 / s : 2.0;
    if (std_sum / n * scale >= 0.01) return -1.0;
    return 0.05 / scale;
}
__global__ void k_hot(double* sc, int std_slot, int gsum_slot, int gsq_slot, int out_slot, double n) {
    if (threadIdx.x == 0 && blockIdx.x == 0)
        sc[out_slot] = hot_threshold(sc[std_slot], n, sc[gsum_slot], sc[gsq_slot]);
}

// gamma = 1/(sigma_T sigma_I) with the reference's eps rule, sigma_T from the device slots
__global__ void k_gamma_dev(const float* __restrict__ sig, float* __restrict__ gam, long long n, const double* sc,
                            int sum_slot, int sq_slot, double msize) {
    const double mean = sc[sum_slot] / msize;
    const double var = sc[sq_slot] / msize - mean * mean;
    // a non-finite template (0/0 in its autocorrelation) gives NaN: no voxel divides
    const double tstd = isnan(var) ? var : sqrt(fmax(var, 0.0));
    TG_GRID_STRIDE(i, n) {
        const double den = (double)(float)(tstd * (double)sig[i] * 10000.0);
        gam[i] = fabs(den - DBL_EPSILON) > DBL_EPSILON ? (float)(1.0 / (tstd * (double)sig[i])) : 0.f;
    }
}
__global__ void k_soc_final(const double* __restrict__ num, const float* __restrict__ mu,
                            const float* __restrict__ gam, const float* __restrict__ sig, float* __restrict__ out,
                            long long n, const double* sc, double msize) {
    const double tmean = sc[S_A_SUM] / msize;
    const double hot = sc[S_SOC_HOT];
    TG_GRID_STRIDE(i, n) {
        // tom_os3_corr assigns only where the denominator passes its test (res starts at 0)
        const float g = gam[i];
        float r = g != 0.f ? (float)((num[i] - (double)mu[i] * tmean) * (double)g) : 0.f;
        if ((double)sig[i] < hot) r = 0.f;
        out[i] = r;
    }
}

// ------------------------------------------------------ template autocorrelation
// z[0] = t, z[1] = t^2, z[2] = t * sphere (complex, three contiguous volumes)
__global__ void k_ac_prep(const float* __restrict__ t, const float* __restrict__ sph, double2* __restrict__ z,
                          long long tn) {
    TG_GRID_STRIDE(i, tn) {
        const double x = (double)t[i];
        z[i] = make_double2(x, 0.0);
        z[tn + i] = make_double2(x * x, 0.0);
        z[2 * tn + i] = make_double2(x * (double)sph[i], 0.0);
    }
}
// mean spectrum z0*zs, square spectrum z1*zs, correlation spectrum z0*conj(z2)
__global__ void k_ac_mul(double2* __restrict__ z, const double2* __restrict__ zs, long long tn) {
    TG_GRID_STRIDE(i, tn) {
        const double2 a = z[i], b = z[tn + i], c = z[2 * tn + i], s = zs[i];
        z[i] = cmul(a, s);
        z[tn + i] = cmul(b, s);
        z[2 * tn + i] = cmulc(a, c);
    }
}
// ifftshift index of a voxel: (x + floor(T/2)) mod T per axis
__device__ __forceinline__ long long ac_src(long long v, int tx, int ty, int tz) {
    const int i = (int)(v % tx), j = (int)((v / tx) % ty), k = (int)(v / ((long long)tx * ty));
    const int si = (i + tx / 2) % tx, sj = (j + ty / 2) % ty, sk = (k + tz / 2) % tz;
    return si + (long long)tx * (sj + (long long)ty * sk);
}
__global__ void k_ac_std(const double2* __restrict__ z, double* __restrict__ sd, int tx, int ty, int tz,
                         double inv_m) {
    const long long tn = (long long)tx * ty * tz;
    TG_GRID_STRIDE(v, tn) {
        const long long s = ac_src(v, tx, ty, tz);
        const double mean = z[s].x * inv_m;
        const double var = z[tn + s].x * inv_m - mean * mean;
        sd[v] = sqrt(var > 0 ? var : 0.0);
    }
}
__global__ void k_ac_final(const double2* __restrict__ z, const double* __restrict__ sd, float* __restrict__ A,
                           int tx, int ty, int tz, double inv_m, const double* sc, double msize) {
    const long long tn = (long long)tx * ty * tz;
    const double tmean = sc[S_AC_TSUM] / msize;
    const double tvar = sc[S_AC_TSQ] / msize - tmean * tmean;
    const double tstd = sqrt(tvar > 0 ? tvar : 0.0);
    const double hot = sc[S_AC_HOT];
    TG_GRID_STRIDE(v, tn) {
        const long long s = ac_src(v, tx, ty, tz);
        const double num = z[2 * tn + s].x * inv_m;
        const double mean = z[s].x * inv_m;
        float r = (float)((num - mean * tmean) / (tstd * sd[v]));
        if (sd[v] < hot) r = 0.f;
        A[v] = r;
    }
}
__global__ void k_mul_f32(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ c,
                          long long n) {
    TG_GRID_STRIDE(i, n) c[i] = a[i] * b[i];
}

// ------------------------------------------------------------- search update
// tom_os3_bestPeak: replace where every selected criterion strictly improves
__global__ void k_analysis_update(const float* __restrict__ cc, const float* __restrict__ psr,
                                  const float* __restrict__ soc, long long n, int flags, int index,
                                  float* __restrict__ o_cc, int* __restrict__ o_idx, float* __restrict__ o_psr,
                                  float* __restrict__ o_soc) {
    TG_GRID_STRIDE(i, n) {
        const float c = cc[i], p = psr[i], a = soc[i];
        bool upd = true;
        if (flags & TOMGPU_ANALYSIS_CCC) upd = upd && (o_cc[i] < c);
        if (flags & TOMGPU_ANALYSIS_PSR) upd = upd && (o_psr[i] < p);
        if (flags & TOMGPU_ANALYSIS_AUTOCORR) upd = upd && (o_soc[i] < a);
        if (upd) {
            o_cc[i] = c;
            o_psr[i] = p;
            o_soc[i] = a;
            o_idx[i] = index;
        }
    }
}
__global__ void k_fill4(float* a, int* idx, float* b, float* c, long long n) {
    TG_GRID_STRIDE(i, n) {
        a[i] = -1000.f;
        idx[i] = -1;
        b[i] = -1000.f;
        c[i] = -1000.f;
    }
}

}  // namespace

// tom_os3_sphereMask of a template-sized box (search/tom_os3_sphereMask.m:4-37)
void os3_sphere_mask_host(const int T[3], std::vector<float>& m) {
    const long long tn = (long long)T[0] * T[1] * T[2];
    m.assign((size_t)tn, 1.f);
    if (T[0] != T[1] || T[1] != T[2]) return;  // non-cubic: ones
    const long long r = T[0] / 2 - 1;
    const long long c = T[0] / 2;  // 0-based centre floor(n/2)
    for (int k = 0; k < T[2]; ++k)
        for (int j = 0; j < T[1]; ++j)
            for (int i = 0; i < T[0]; ++i) {
                const long long d2 = (i - c) * (i - c) + (j - c) * (j - c) + (k - c) * (k - c);
                // zero where distance >= radius
                const bool zero = r <= 0 || d2 >= r * r;
                if (zero) m[i + (size_t)T[0] * (j + (size_t)T[1] * k)] = 0.f;
            }
}

void PeakAnalysis::release() {
    void* bufs[] = {f_psr, f_msk, f1, f2, f3, v64, m1, m2, mu, sig, gam, d_mask, d_sph, d_am, d_psrbox,
                    z, zs, acsd, sc, tmp_t};
    for (void* p : bufs)
        if (p) cudaFree(p);
    f_psr = f_msk = f1 = f2 = f3 = nullptr;
    v64 = m1 = m2 = nullptr;
    mu = sig = gam = d_mask = d_sph = d_am = d_psrbox = tmp_t = nullptr;
    z = zs = nullptr;
    acsd = sc = nullptr;
}

PeakAnalysis::~PeakAnalysis() { release(); }

int PeakAnalysis::alloc(void** p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(ctx, TOMGPU_ERR_OOM, "peak-analysis allocation of " + std::to_string(bytes) + " bytes failed");
    }
    return TOMGPU_OK;
}

int PeakAnalysis::create(tomgpu_ctx* c, const int vol[3], const int tm[3], const float* mask_dev) {
    ctx = c;
    for (int d = 0; d < 3; ++d) { N[d] = vol[d]; T[d] = tm[d]; }
    for (int d = 0; d < 3; ++d)
        if (!fft_length_supported(N[d]) || !fft_length_supported(T[d]) || T[d] > N[d])
            return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "peak-analysis sizes not supported by the FFT kernels");
    nvox = (long long)N[0] * N[1] * N[2];
    hs = (long long)(N[0] / 2 + 1) * N[1] * N[2];
    tn = (long long)T[0] * T[1] * T[2];
    cudaStream_t st = ctx->stream;
    TG_TRY(alloc((void**)&f_psr, sizeof(double2) * hs));
    TG_TRY(alloc((void**)&f_msk, sizeof(double2) * hs));
    TG_TRY(alloc((void**)&f1, sizeof(double2) * hs));
    TG_TRY(alloc((void**)&f2, sizeof(double2) * hs));
    TG_TRY(alloc((void**)&f3, sizeof(double2) * hs));
    TG_TRY(alloc((void**)&v64, sizeof(double) * nvox));
    TG_TRY(alloc((void**)&m1, sizeof(double) * nvox));
    TG_TRY(alloc((void**)&m2, sizeof(double) * nvox));
    TG_TRY(alloc((void**)&mu, sizeof(float) * nvox));
    TG_TRY(alloc((void**)&sig, sizeof(float) * nvox));
    TG_TRY(alloc((void**)&gam, sizeof(float) * nvox));
    TG_TRY(alloc((void**)&d_mask, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_sph, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_am, sizeof(float) * tn));
    TG_TRY(alloc((void**)&d_psrbox, sizeof(float) * tn));
    TG_TRY(alloc((void**)&tmp_t, sizeof(float) * tn));
    TG_TRY(alloc((void**)&z, sizeof(double2) * 3 * tn));
    TG_TRY(alloc((void**)&zs, sizeof(double2) * tn));
    TG_TRY(alloc((void**)&acsd, sizeof(double) * tn));
    TG_TRY(alloc((void**)&sc, sizeof(double) * S_COUNT));

    // host masks: default sphere, PSR box (sphere with a centred floor(T/4) box zeroed)
    std::vector<float> sph, box;
    os3_sphere_mask_host(T, sph);
    box = sph;
    const int q[3] = {T[0] / 4, T[1] / 4, T[2] / 4};
    if (q[0] > 0 && q[1] > 0 && q[2] > 0) {
        const int o[3] = {T[0] / 2 - q[0] / 2, T[1] / 2 - q[1] / 2, T[2] / 2 - q[2] / 2};
        for (int k = o[2]; k < o[2] + q[2]; ++k)
            for (int j = o[1]; j < o[1] + q[1]; ++j)
                for (int i = o[0]; i < o[0] + q[0]; ++i) box[i + (size_t)T[0] * (j + (size_t)T[1] * k)] = 0.f;
    }
    std::vector<float> mk(sph);
    if (mask_dev) {
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(mk.data(), mask_dev, sizeof(float) * tn, cudaMemcpyDeviceToHost, st));
        TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    }
    m_psr = m_msk = m_sph = 0;
    for (long long i = 0; i < tn; ++i) {
        m_psr += box[i] != 0.f;
        m_msk += mk[i] != 0.f;
        m_sph += sph[i] != 0.f;
    }
    if (m_msk <= 0 || m_psr <= 0 || m_sph <= 0) return fail(ctx, TOMGPU_ERR_ARG, "a mask has no nonzero voxel");
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_sph, sph.data(), sizeof(float) * tn, cudaMemcpyHostToDevice, st));
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_psrbox, box.data(), sizeof(float) * tn, cudaMemcpyHostToDevice, st));
    TG_TRY_CUDA(ctx, cudaMemcpyAsync(d_mask, mk.data(), sizeof(float) * tn, cudaMemcpyHostToDevice, st));
    // convolution kernels of tom_os3_mean/std: the pasted mask shifted by
    // -floor(N/2), i.e. its box placed at -floor(T/2) (mod N)
    const int off[3] = {-(T[0] / 2), -(T[1] / 2), -(T[2] / 2)};
    TG_TRY_CUDA(ctx, cudaMemsetAsync(v64, 0, sizeof(double) * nvox, st));
    TG_TRY_CUDA(ctx, place_f64(d_psrbox, T, v64, N, off, st));
    TG_TRY_CUDA(ctx, r2c3d<double2>(v64, f_psr, N, st));
    TG_TRY_CUDA(ctx, cudaMemsetAsync(v64, 0, sizeof(double) * nvox, st));
    TG_TRY_CUDA(ctx, place_f64(d_mask, T, v64, N, off, st));
    TG_TRY_CUDA(ctx, r2c3d<double2>(v64, f_msk, N, st));
    // spectrum of the default sphere for the template autocorrelation
    {
        std::vector<double2> hz((size_t)tn);
        for (long long i = 0; i < tn; ++i) hz[i] = make_double2((double)sph[i], 0.0);
        TG_TRY_CUDA(ctx, cudaMemcpyAsync(zs, hz.data(), sizeof(double2) * tn, cudaMemcpyHostToDevice, st));
        TG_TRY_CUDA(ctx, c2c3d_batch64(zs, T, 1, -1, 1.0, st));
        TG_TRY_CUDA(ctx, cudaStreamSynchronize(st));  // hz leaves scope
    }
    ctx->launches += 12;
    return TOMGPU_OK;
}

int PeakAnalysis::autocorr(const float* t, float* A) {
    cudaStream_t st = ctx->stream;
    TG_TRY_CUDA(ctx, cudaMemsetAsync(sc, 0, sizeof(double) * (S_AC_HOT + 1), st));
    k_ac_prep<<<grid_n(tn), 256, 0, st>>>(t, d_sph, z, tn);
    TG_TRY_CUDA(ctx, msum<2>(Moments{t, d_sph}, tn, sc + S_AC_TSUM, st));
    TG_TRY_CUDA(ctx, msum<2>(Moments{t, nullptr}, tn, sc + S_AC_GSUM, st));
    TG_TRY_CUDA(ctx, c2c3d_batch64(z, T, 3, -1, 1.0, st));
    k_ac_mul<<<grid_n(tn), 256, 0, st>>>(z, zs, tn);
    TG_TRY_CUDA(ctx, c2c3d_batch64(z, T, 3, +1, 1.0 / (double)tn, st));
    k_ac_std<<<grid_n(tn), 256, 0, st>>>(z, acsd, T[0], T[1], T[2], 1.0 / m_sph);
    TG_TRY_CUDA(ctx, msum<1>(DoubleSum{acsd}, tn, sc + S_AC_STDSUM, st));
    k_hot<<<1, 32, 0, st>>>(sc, S_AC_STDSUM, S_AC_GSUM, S_AC_GSQ, S_AC_HOT, (double)tn);
    k_ac_final<<<grid_n(tn), 256, 0, st>>>(z, acsd, A, T[0], T[1], T[2], 1.0 / m_sph, sc, m_sph);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 14;
    return TOMGPU_OK;
}

int PeakAnalysis::spectra(const float* pk) {
    cudaStream_t st = ctx->stream;
    k_f32_f64_sq<<<grid_n(nvox), 256, 0, st>>>(pk, v64, nvox, 0);
    TG_TRY_CUDA(ctx, r2c3d<double2>(v64, f1, N, st));
    k_f32_f64_sq<<<grid_n(nvox), 256, 0, st>>>(pk, v64, nvox, 1);
    TG_TRY_CUDA(ctx, r2c3d<double2>(v64, f2, N, st));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 8;
    return TOMGPU_OK;
}

int PeakAnalysis::local_moments(const double2* fk, double msize) {
    cudaStream_t st = ctx->stream;
    const double s = 1.0 / ((double)nvox * msize);
    k_cmul3<<<grid_n(hs), 256, 0, st>>>(f1, fk, f3, hs, 0);
    TG_TRY_CUDA(ctx, c2r3d<double2>(f3, m1, N, s, st));
    k_cmul3<<<grid_n(hs), 256, 0, st>>>(f2, fk, f3, hs, 0);
    TG_TRY_CUDA(ctx, c2r3d<double2>(f3, m2, N, s, st));
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 8;
    return TOMGPU_OK;
}

int PeakAnalysis::psr(const float* pk, float* out) {
    cudaStream_t st = ctx->stream;
    TG_TRY(local_moments(f_psr, m_psr));
    unsigned* maxbits = reinterpret_cast<unsigned*>(sc + S_PSR_MAXBITS);
    TG_TRY_CUDA(ctx, cudaMemsetAsync(maxbits, 0, sizeof(unsigned), st));
    k_psr_std<<<grid_n(nvox), 256, 0, st>>>(m1, m2, sig, nvox, maxbits);
    k_psr_final<<<grid_n(nvox), 256, 0, st>>>(pk, m1, sig, out, nvox, maxbits);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 2;
    return TOMGPU_OK;
}

int PeakAnalysis::soc(const float* pk, const float* A, float* out) {
    cudaStream_t st = ctx->stream;
    TG_TRY_CUDA(ctx, cudaMemsetAsync(sc + S_PK_SUM, 0, sizeof(double) * (S_A_SQ - S_PK_SUM + 1), st));
    TG_TRY(local_moments(f_msk, m_msk));
    TG_TRY_CUDA(ctx, stats_final(m1, m2, mu, sig, nvox, st));
    // artefact test of tom_os3_corr.m:108-127 on the peak map
    TG_TRY_CUDA(ctx, msum<2>(Moments{pk, nullptr}, nvox, sc + S_PK_SUM, st));
    TG_TRY_CUDA(ctx, msum<1>(FloatSum{sig}, nvox, sc + S_SOC_STDSUM, st));
    k_hot<<<1, 32, 0, st>>>(sc, S_SOC_STDSUM, S_PK_SUM, S_PK_SQ, S_SOC_HOT, (double)nvox);
    // A's statistics under the correlation mask and gamma
    k_mul_f32<<<grid_n(tn), 256, 0, st>>>(A, d_mask, d_am, tn);
    TG_TRY_CUDA(ctx, msum<2>(Moments{A, d_mask}, tn, sc + S_A_SUM, st));
    k_gamma_dev<<<grid_n(nvox), 256, 0, st>>>(sig, gam, nvox, sc, S_A_SUM, S_A_SQ, m_msk);
    // numerator: sum_k pk(x + d0 + k) (A m)(k) / M, d0 = (2 floor(N/2) - floor(T/2)) mod N
    int d0[3];
    for (int d = 0; d < 3; ++d) d0[d] = ((2 * (N[d] / 2) - T[d] / 2) % N[d] + N[d]) % N[d];
    TG_TRY_CUDA(ctx, cudaMemsetAsync(v64, 0, sizeof(double) * nvox, st));
    TG_TRY_CUDA(ctx, place_f64(d_am, T, v64, N, d0, st));
    TG_TRY_CUDA(ctx, r2c3d<double2>(v64, f3, N, st));
    k_cmulc_inplace_b<<<grid_n(hs), 256, 0, st>>>(f1, f3, hs);
    TG_TRY_CUDA(ctx, c2r3d<double2>(f3, m1, N, 1.0 / ((double)nvox * m_msk), st));
    k_soc_final<<<grid_n(nvox), 256, 0, st>>>(m1, mu, gam, sig, out, nvox, sc, m_msk);
    TG_TRY_CUDA(ctx, cudaGetLastError());
    ctx->launches += 18;
    return TOMGPU_OK;
}

int analysis_update(tomgpu_ctx* ctx, const float* cc, const float* psr, const float* soc, long long n, int flags,
                    int index, float* o_cc, int* o_idx, float* o_psr, float* o_soc) {
    k_analysis_update<<<grid_n(n), 256, 0, ctx->stream>>>(cc, psr, soc, n, flags, index, o_cc, o_idx, o_psr, o_soc);
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cudaGetLastError());
    return TOMGPU_OK;
}

int analysis_init(tomgpu_ctx* ctx, long long n, float* o_cc, int* o_idx, float* o_psr, float* o_soc) {
    k_fill4<<<grid_n(n), 256, 0, ctx->stream>>>(o_cc, o_idx, o_psr, o_soc, n);
    ctx->launches += 1;
    TG_TRY_CUDA(ctx, cudaGetLastError());
    return TOMGPU_OK;
}

}  // namespace tg
