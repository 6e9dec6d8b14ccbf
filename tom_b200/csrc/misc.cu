// Weighting functions, masks, reductions and elementwise helpers.
#include <cfloat>

#include "common.cuh"
#include "misc.h"

namespace tg {

// ------------------------------------------------------------- weight3d
// Radermacher exact weighting (Filtrans/tom_calc_weight_functioninc.c:152-252).
// The per-axis frequency coordinates are the reference's accumulated float
// sequences (computed on the host), the tilt normals too; per voxel the sum
// over tilts runs in float in tilt order like the reference.
__global__ void k_weight3d(float* __restrict__ w, int nx, int ny, int nz, const float* __restrict__ fx,
                           const float* __restrict__ fy, const float* __restrict__ fz,
                           const float* __restrict__ nrm, int n_tilt) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((long long)nx * ny));
    const float x = fx[i], y = fy[j], z = fz[k];
    const float width = 3.1416f;
    float sum = 0.f;
    for (int t = 0; t < n_tilt; ++t) {
        const float arg = __fadd_rn(__fadd_rn(__fmul_rn(x, nrm[3 * t]), __fmul_rn(y, nrm[3 * t + 1])),
                                    __fmul_rn(z, nrm[3 * t + 2]));
        const float a = fabsf(arg);
        float add;
        if (a < 1e-6f) add = 1.f;
        else if ((double)a > 1e-6 && a < width) add = __fdiv_rn((float)sin((double)arg), arg);
        else add = 0.f;
        sum = __fadd_rn(sum, add);
    }
    w[v] = sum > 1.0f ? (float)(1.0 / (double)sum) : 1.0f;
}

cudaError_t weight3d(float* w, const int dims[3], const float* d_fx, const float* d_fy, const float* d_fz,
                     const float* d_nrm, int n_tilt, cudaStream_t st) {
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    k_weight3d<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(w, dims[0], dims[1], dims[2], d_fx, d_fy, d_fz,
                                                            d_nrm, n_tilt);
    return cudaGetLastError();
}

// ----------------------------------------------------------------- wedge
// tom_wedge (Filtrans/tom_wedge.m:62-77) and av3_wedge (av3/utils/av3_wedge.m:23-26)
// on the centred grid x = i - floor(n/2); IEEE division gives the z = 0 plane
// the reference's Inf/NaN behaviour (kept).
__global__ void k_wedge(float* __restrict__ out, int nx, int ny, int nz, double t1, double t2, int av3) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int i = (int)(v % nx), k = (int)(v / ((long long)nx * ny));
    const double x = (double)(i - nx / 2), z = (double)(k - nz / 2);
    float w = 1.f;
    if (!av3) {
        const double r = __ddiv_rn(fabs(x), fabs(z));
        if (t1 > r) w = 0.f;
    } else {
        const double r = __ddiv_rn(x, z);
        if (t1 > r && t2 < r) w = 0.f;
    }
    out[v] = w;
}

cudaError_t wedge(float* out, const int dims[3], double t1, double t2, int av3, cudaStream_t st) {
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    k_wedge<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, dims[0], dims[1], dims[2], t1, t2, av3);
    return cudaGetLastError();
}

// ifftshift of a real volume: out[i] = in[(i + floor(n/2)) mod n] per axis
__global__ void k_ifftshift(const float* __restrict__ in, float* __restrict__ out, int nx, int ny, int nz) {
    const long long n = (long long)nx * ny * nz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((long long)nx * ny));
    const int si = (i + nx / 2) % nx, sj = (j + ny / 2) % ny, sk = (k + nz / 2) % nz;
    out[v] = in[si + (long long)nx * (sj + (long long)ny * sk)];
}

cudaError_t ifftshift_real(const float* in, float* out, const int dims[3], cudaStream_t st) {
    const long long n = (long long)dims[0] * dims[1] * dims[2];
    k_ifftshift<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, out, dims[0], dims[1], dims[2]);
    return cudaGetLastError();
}

// ------------------------------------------------------------ reductions
// Sum over n doubles produced by f(i) into *out (atomicAdd per block).
template <typename F>
__global__ void __launch_bounds__(256) k_sum(F f, long long n, double* out) {
    double acc = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) acc += f(i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += ws[w];
        atomicAdd(out, s);
    }
}

template <typename F> static cudaError_t launch_sum(F f, long long n, double* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    if (e) return e;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_sum<<<(unsigned)blocks, 256, 0, st>>>(f, n, out);
    return cudaGetLastError();
}

struct FVal { const float* a; double s, o; __device__ double operator()(long long i) const { return (double)a[i] * s + o; } };
struct FSq { const float* a; double s, o, m; __device__ double operator()(long long i) const { double d = (double)a[i] * s + o - m; return d * d; } };
struct DVal { const double* a; __device__ double operator()(long long i) const { return a[i]; } };
struct Nz { const float* a; __device__ double operator()(long long i) const { return a[i] != 0.f ? 1.0 : 0.0; } };
// normUnderMask (mask = mask~=0 first): mean numerator sum(v*m*(v~=0)), variance numerator
struct NumMean { const double* v; const float* m; __device__ double operator()(long long i) const { double x = v[i]; return (x != 0.0 && m[i] != 0.f) ? x : 0.0; } };
struct NumVar { const double* v; const float* m; double mea; __device__ double operator()(long long i) const {
    const double mk = m[i] != 0.f ? 1.0 : 0.0; const double t = (mk == 0.0 ? mea : 0.0) + v[i] * mk - mea; return t * t; } };

cudaError_t sum_affine_f32(const float* a, long long n, double s, double o, double* out, cudaStream_t st) {
    return launch_sum(FVal{a, s, o}, n, out, st);
}
cudaError_t sum_sqdev_f32(const float* a, long long n, double s, double o, double mean, double* out, cudaStream_t st) {
    return launch_sum(FSq{a, s, o, mean}, n, out, st);
}
cudaError_t sum_f64(const double* a, long long n, double* out, cudaStream_t st) {
    return launch_sum(DVal{a}, n, out, st);
}
cudaError_t count_nonzero(const float* a, long long n, double* out, cudaStream_t st) {
    return launch_sum(Nz{a}, n, out, st);
}
cudaError_t norm_under_mask_sums(const double* v, const float* m, long long n, double* d_mean_num,
                                 double* d_var_num, double mea, int which, cudaStream_t st) {
    if (which == 0) return launch_sum(NumMean{v, m}, n, d_mean_num, st);
    return launch_sum(NumVar{v, m, mea}, n, d_var_num, st);
}

// ------------------------------------------------------------ elementwise
__global__ void k_affine_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, long long n, double s,
                                    double o) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i] * s + o;
}
__global__ void k_affine_f32_to_f32(const float* __restrict__ a, float* __restrict__ b, long long n, double s,
                                    double o, double m, double inv) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)((((double)a[i] * s + o) - m) * inv);
}
__global__ void k_square_f64(double* __restrict__ a, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = a[i] * a[i];
}
__global__ void k_mul_c64(double2* __restrict__ a, const double2* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = cmul(a[i], b[i]);
}
__global__ void k_real_to_c64(const float* __restrict__ a, double2* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = make_double2((double)a[i], 0.0);
}
__global__ void k_mul_weight_c64(double2* __restrict__ a, const float* __restrict__ w, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = cscale(a[i], (double)w[i]);
}
__global__ void k_re_c64(const double2* __restrict__ a, double* __restrict__ b, long long n, double s) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i].x * s;
}
// place a small real volume (t dims) into a zeroed big one at (j + off) mod N
__global__ void k_place_f64(const float* __restrict__ small, int tx, int ty, int tz, double* __restrict__ big,
                            int nx, int ny, int nz, int ox, int oy, int oz) {
    const long long n = (long long)tx * ty * tz;
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int i = (int)(v % tx), j = (int)((v / tx) % ty), k = (int)(v / ((long long)tx * ty));
    const int x = pmod(i + ox, nx), y = pmod(j + oy, ny), z = pmod(k + oz, nz);
    big[x + (long long)nx * (y + (long long)ny * z)] = (double)small[v];
}
// mean and std from FP64 sums: mu = m1, sigma = sqrt(max(m2 - mu^2, 0))
__global__ void k_stats_final(const double* __restrict__ m1, const double* __restrict__ m2, float* __restrict__ mu,
                              float* __restrict__ sig, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double a = m1[i];
        const double var = m2[i] - a * a;
        mu[i] = (float)a;
        sig[i] = (float)sqrt(var > 0 ? var : 0.0);
    }
}
// gamma = 1/(sigma_T sigma_I) where tom_os3_corr divides (|den - eps| > eps,
// den = single(sigma_T * sigma_I * 1e4)), else 0 (search/tom_os3_corr.m:157-176).
__global__ void k_gamma(const float* __restrict__ sig, float* __restrict__ gam, long long n, double tstd) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double den = (double)(float)(tstd * (double)sig[i] * 10000.0);
        gam[i] = fabs(den - DBL_EPSILON) > DBL_EPSILON ? (float)(1.0 / (tstd * (double)sig[i])) : 0.f;
    }
}

static unsigned grid_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

#define TG_LAUNCH(kern, n, ...)                                         \
    do {                                                                \
        kern<<<grid_for(n), 256, 0, st>>>(__VA_ARGS__);                 \
        return cudaGetLastError();                                      \
    } while (0)

cudaError_t affine_f32_to_f64(const float* a, double* b, long long n, double s, double o, cudaStream_t st) {
    TG_LAUNCH(k_affine_f32_to_f64, n, a, b, n, s, o);
}
cudaError_t normalize_f32(const float* a, float* b, long long n, double s, double o, double m, double inv,
                          cudaStream_t st) {
    TG_LAUNCH(k_affine_f32_to_f32, n, a, b, n, s, o, m, inv);
}
cudaError_t square_f64(double* a, long long n, cudaStream_t st) { TG_LAUNCH(k_square_f64, n, a, n); }
cudaError_t mul_c64(double2* a, const double2* b, long long n, cudaStream_t st) { TG_LAUNCH(k_mul_c64, n, a, b, n); }
cudaError_t real_to_c64(const float* a, double2* b, long long n, cudaStream_t st) { TG_LAUNCH(k_real_to_c64, n, a, b, n); }
cudaError_t mul_weight_c64(double2* a, const float* w, long long n, cudaStream_t st) {
    TG_LAUNCH(k_mul_weight_c64, n, a, w, n);
}
cudaError_t re_c64(const double2* a, double* b, long long n, double s, cudaStream_t st) { TG_LAUNCH(k_re_c64, n, a, b, n, s); }
__global__ void k_d2f(const double* __restrict__ a, float* __restrict__ b, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
cudaError_t double_to_float(const double* a, float* b, long long n, cudaStream_t st) { TG_LAUNCH(k_d2f, n, a, b, n); }
cudaError_t stats_final(const double* m1, const double* m2, float* mu, float* sig, long long n, cudaStream_t st) {
    TG_LAUNCH(k_stats_final, n, m1, m2, mu, sig, n);
}
cudaError_t gamma_from_sigma(const float* sig, float* gam, long long n, double tstd, cudaStream_t st) {
    TG_LAUNCH(k_gamma, n, sig, gam, n, tstd);
}
cudaError_t place_f64(const float* small, const int t[3], double* big, const int nn[3], const int off[3],
                      cudaStream_t st) {
    const long long n = (long long)t[0] * t[1] * t[2];
    k_place_f64<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(small, t[0], t[1], t[2], big, nn[0], nn[1], nn[2],
                                                             off[0], off[1], off[2]);
    return cudaGetLastError();
}

}  // namespace tg
