// Batched subtomogram alignment with tom_av3_align's semantics
// (av3_new/tom_av3_align.m:97-189, tom_corr 'norm' of Analysis/tom_corr.m:51-121).
//
// Per job (reference, particle, masks, wedges, angle ranges) and per Euler
// triplet of its scan, in the reference's loop order (phi outer, psi, theta
// inner):
//   ref_rot = rot3d(ref, R)            R = tom_angles2rotmatrix, matrix mode
//   w_rot   = rot3d(wedge_ref, euler)  Euler mode
//   a = ref_rot*mask (*) psf_part,  b = part*mask (*) psf_ref   (cross-wedging)
//   a, b normalised inside the mask (mean over the mask, std with n - 1)
//   ccf = real(fftshift(ifftn(F(b) conj F(a)))) / n
//   ccf_max = strict max, angle_max = index where ccf >= the updated max
// The convolutions with the wedge PSFs are products in Fourier space: the
// spectrum of psf = real(ifftn(ifftshift(w))) is the Hermitian part
// (W'(k) + W'(-k))/2 of W' = ifftshift(w), for the particle's wedge and for the
// rotated reference wedge alike.
// After the scan: first maximum of ccf_max*mask_ccf gives the angle index;
// the reference rotated by those angles is correlated once more without
// wedges and tom_peak(.,'spline') of ccf*mask_ccf gives shift and peak.
//
// The rotation batch of a job runs as batched template-sized real-to-half
// and half-to-real FFTs (fft3d.cu): every volume of the scan is real and every
// spectral factor (the Hermitian wedge parts, F(b) conj F(a)) keeps Hermitian
// symmetry, so the half spectrum carries the whole computation.  Per-entry
// statistics are FP64 segmented reductions.
#include <cfloat>
#include <cmath>
#include <string>
#include <vector>

#include "common.cuh"
#include "ctx.h"
#include "fft3d.h"
#include "match.h"
#include "misc.h"
#include "peak.h"
#include "rotate_sample.cuh"
#include "wedge_pair.cuh"

namespace tg {

namespace {

unsigned grid_for(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b < 1 ? 1 : b);
}

TG_D long long shifted(long long v, int nx, int ny, int nz, int sgn) {
    // sgn = +1: ifftshift source index (i + floor(n/2)); -1: fftshift (i - floor(n/2))
    const int i = (int)(v % nx), j = (int)((v / nx) % ny), k = (int)(v / ((long long)nx * ny));
    const int si = pmod(i + sgn * (nx / 2), nx), sj = pmod(j + sgn * (ny / 2), ny), sk = pmod(k + sgn * (nz / 2), nz);
    return si + (long long)nx * (sj + (long long)ny * sk);
}

// A[e] = rot(ref, mref_e) * mask (complex), W[e] = rot(wedge_ref, mw_e)
__global__ void k_al_rotate(const float* __restrict__ ref, const float* __restrict__ wref,
                            const float* __restrict__ mask, const float* __restrict__ mref,
                            const float* __restrict__ mw, int nx, int ny, int nz, float cx, float cy, float cz,
                            int mask_ref, float* __restrict__ Ar, float2* __restrict__ A, float* __restrict__ W) {
    const int nn = nx * ny * nz;  // boxes hold fewer than 2^31 voxels
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    const int e = blockIdx.y;
    if (v >= nn) return;
    const int i = v % nx, t = v / nx, j = t % ny, k = t / ny;
    float m[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) m[q] = mref[9 * e + q];
    float a = rot_sample(ref, nx, ny, nz, m, cx, cy, cz, i, j, k);
    if (mask_ref) a = __fmul_rn(a, mask[v]);
    if (Ar) Ar[(long long)e * nn + v] = a;
    else A[(long long)e * nn + v] = make_float2(a, 0.f);
    if (W) {
#pragma unroll
        for (int q = 0; q < 9; ++q) m[q] = mw[9 * e + q];
        W[(long long)e * nn + v] = rot_sample(wref, nx, ny, nz, m, cx, cy, cz, i, j, k);
    }
}

// A[e][k] *= (W'(k) + W'(-k)) / 2 with W' = ifftshift(wedge_part) (the
// spectrum of psf_part), and B[e][k] = B0[k] (W'(k) + W'(-k)) / 2 with
// W' = ifftshift(W[e]), on half spectra ((nx/2+1) ny nz per entry): half
// index h is the full-grid frequency kx + nx (ky + ny kz) with kx <= nx/2.
// The index pair is computed once per frequency for the AL_EG entries of the
// block's group (blockIdx.y).
constexpr int AL_EG = 16;
__global__ void k_al_wpart_h(float2* __restrict__ A, const float* __restrict__ wpart, int nx, int ny, int nz, int E) {
    const int nh = nx / 2 + 1, nhn = nh * ny * nz;
    const int e0 = blockIdx.y * AL_EG, e1 = min(E, e0 + AL_EG);
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < nhn; h += gridDim.x * blockDim.x) {
        const int kx = h % nh, t = h / nh;
        int s1, s2;
        wedge_pair(kx + nx * t, nx, ny, nz, s1, s2);
        const float ws = 0.5f * (wpart[s1] + wpart[s2]);
        for (int e = e0; e < e1; ++e) {
            float2* a = A + (long long)e * nhn + h;
            *a = cscale(*a, ws);
        }
    }
}

__global__ void k_al_bside_h(float2* __restrict__ B, const float2* __restrict__ B0, const float* __restrict__ W,
                             int nx, int ny, int nz, int E) {
    const int nh = nx / 2 + 1, nhn = nh * ny * nz, nn = nx * ny * nz;
    const int e0 = blockIdx.y * AL_EG, e1 = min(E, e0 + AL_EG);
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < nhn; h += gridDim.x * blockDim.x) {
        const int kx = h % nh, t = h / nh;
        int s1, s2;
        wedge_pair(kx + nx * t, nx, ny, nz, s1, s2);
        const float2 b0 = B0[h];
        for (int e = e0; e < e1; ++e) {
            const float* w = W + (long long)e * nn;
            B[(long long)e * nhn + h] = cscale(b0, 0.5f * (w[s1] + w[s2]));
        }
    }
}

// the particle in every entry (no wedges)
__global__ void k_al_bcast(float* __restrict__ B, const float* __restrict__ part, int nn, int E) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (long long)nn * E;
         t += (long long)gridDim.x * blockDim.x)
        B[t] = part[t % nn];
}

// per-entry FP64 sums of norm_inside_mask on real volumes: pass 0: sum x m,
// pass 1: sum over m of (x - mea)^2
__global__ void __launch_bounds__(256) k_al_stats_r(const float* __restrict__ X, const float* __restrict__ mask,
                                                    long long nn, const double* __restrict__ mea, int pass,
                                                    double* __restrict__ out) {
    const int e = blockIdx.y;
    const float* x = X + (long long)e * nn;
    double acc = 0;
    const double me = pass ? mea[e] : 0.0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x) {
        if (mask[v] != 0.f) {
            const double r = (double)x[v];
            acc += pass ? (r - me) * (r - me) : r;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0;
        for (int k = 0; k < 8; ++k) sum += ws[k];
        atomicAdd(out + e, sum);
    }
}

__global__ void k_al_normalize_r(float* __restrict__ X, const float* __restrict__ mask, long long nn, int E,
                                 const double* __restrict__ mea, const double* __restrict__ var, double n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn * E; t += (long long)gridDim.x * blockDim.x) {
        const long long v = t % nn, e = t / nn;
        const double st = sqrt(var[e] / (n - 1.0));
        X[t] = mask[v] != 0.f ? (float)(((double)X[t] - mea[e]) / st) : 0.f;
    }
}

// running max over the E entries in scan order; ccf = fftshift(C) / n, C real
__global__ void k_al_update_r(const float* __restrict__ C, int nx, int ny, int nz, int E, double inv_n,
                              const int* __restrict__ aidx, float* __restrict__ cmax, float* __restrict__ amax) {
    const long long nn = (long long)nx * ny * nz;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x) {
        const long long src = shifted(v, nx, ny, nz, -1);
        float m = cmax[v], a = amax[v];
        for (int e = 0; e < E; ++e) {
            const float c = (float)((double)C[(long long)e * nn + src] * inv_n);
            if (c > m) m = c;
            if (c >= m) a = (float)aidx[e];
        }
        cmax[v] = m;
        amax[v] = a;
    }
}

// per-entry FP64 sums of norm_inside_mask: pass 0: sum re*m, pass 1: sum over m of (re - mea)^2
__global__ void __launch_bounds__(256) k_al_stats(const float2* __restrict__ X, const float* __restrict__ mask,
                                                  long long nn, const double* __restrict__ mea, int pass,
                                                  double* __restrict__ out) {
    const int e = blockIdx.y;
    const float2* x = X + (long long)e * nn;
    double acc = 0;
    const double me = pass ? mea[e] : 0.0;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x) {
        if (mask[v] != 0.f) {
            const double r = (double)x[v].x;
            acc += pass ? (r - me) * (r - me) : r;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0;
        for (int w = 0; w < 8; ++w) s += ws[w];
        atomicAdd(out + e, s);
    }
}

__global__ void k_al_mean(const double* __restrict__ s, double* __restrict__ mea, int E, double n) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E) mea[e] = s[e] / n;
}

// X[e] = ((re - mea)/st) * (mask != 0), st = sqrt(var_sum / (n - 1))
__global__ void k_al_normalize(float2* __restrict__ X, const float* __restrict__ mask, long long nn, int E,
                               const double* __restrict__ mea, const double* __restrict__ var, double n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn * E; t += (long long)gridDim.x * blockDim.x) {
        const long long v = t % nn, e = t / nn;
        const double st = sqrt(var[e] / (n - 1.0));
        const double r = (double)X[t].x;
        X[t] = make_float2(mask[v] != 0.f ? (float)((r - mea[e]) / st) : 0.f, 0.f);
    }
}

// C = B * conj(A)
__global__ void k_al_cross(float2* __restrict__ B, const float2* __restrict__ A, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        B[t] = cmulc(B[t], A[t]);
}

// single map: out = real(fftshift(C)) / n * mask_ccf
__global__ void k_al_map(const float2* __restrict__ C, int nx, int ny, int nz, double inv_n,
                         const float* __restrict__ mccf, float* __restrict__ out) {
    const long long nn = (long long)nx * ny * nz;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nn; v += (long long)gridDim.x * blockDim.x) {
        const float c = (float)((double)C[shifted(v, nx, ny, nz, -1)].x * inv_n);
        out[v] = mccf ? c * mccf[v] : c;
    }
}

__global__ void k_al_fill(float* __restrict__ a, float* __restrict__ b, long long n, float va, float vb) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        a[t] = va;
        b[t] = vb;
    }
}

__global__ void k_al_mul(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ out, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = b ? a[t] * b[t] : a[t];
}

__global__ void k_al_r2c_masked(const float* __restrict__ a, const float* __restrict__ m, float2* __restrict__ out,
                                long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        out[t] = make_float2(m ? a[t] * m[t] : a[t], 0.f);
}

// matrix of tom_angles2rotmatrix (Sptrans/tom_sum_rotation.m): Rz(psi) Rx(theta) Rz(phi)
// in double, passed to rot3d's matrix mode as single in column-major order
}  // namespace

void rotmatrix_as_float(double phi, double psi, double theta, float m9[9]) {
    const double d = 3.14159265358979323846 / 180.0;
    const double cf = std::cos(phi * d), sf = std::sin(phi * d), cp = std::cos(psi * d), sp = std::sin(psi * d);
    const double ct = std::cos(theta * d), st = std::sin(theta * d);
    const double Rzpsi[3][3] = {{cp, -sp, 0}, {sp, cp, 0}, {0, 0, 1}};
    const double Rx[3][3] = {{1, 0, 0}, {0, ct, -st}, {0, st, ct}};
    const double Rzphi[3][3] = {{cf, -sf, 0}, {sf, cf, 0}, {0, 0, 1}};
    double T1[3][3], R[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            T1[a][b] = 0;
            for (int c = 0; c < 3; ++c) T1[a][b] += Rzpsi[a][c] * Rx[c][b];
        }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            R[a][b] = 0;
            for (int c = 0; c < 3; ++c) R[a][b] += T1[a][c] * Rzphi[c][b];
        }
    // column-major: m[0] = R(1,1), m[1] = R(2,1), m[2] = R(3,1), m[3] = R(1,2), ...
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) m9[3 * col + row] = (float)R[row][col];
}

std::vector<double> axis_values(const float r[3]) {
    std::vector<double> v;
    const double s = r[0], inc = r[1], e = r[2];
    if (inc == 0) {
        v.push_back(s);
        return v;
    }
    const long n = (long)std::floor((e - s) / inc + 1e-9) + 1;
    for (long i = 0; i < n; ++i) v.push_back(s + inc * (double)i);
    return v;
}

namespace {

struct Workspace {
    float2 *A = nullptr, *B = nullptr, *B0 = nullptr;  // the scan: half spectra; the refinement: complex
    float *Ar = nullptr, *Br = nullptr;                // the scan's real volumes
    float *W = nullptr, *cmax = nullptr, *amax = nullptr, *tmp = nullptr, *mats = nullptr;
    int* aidx = nullptr;
    double *sums = nullptr, *mea = nullptr, *var = nullptr, *spline = nullptr;
    unsigned long long* key = nullptr;
    void release() {
        void* p[] = {A, B, B0, Ar, Br, W, cmax, amax, tmp, mats, aidx, sums, mea, var, spline, key};
        for (void* q : p)
            if (q) cudaFree(q);
    }
};

}  // namespace

// The alignment workspace of one tomgpu_av3_align_dev call: grown to the
// largest job, reused by the following jobs.
struct AlignScratch {
    Workspace w;
    size_t cap[16] = {0};
    std::vector<void*> pool;  // the batched engine's buffers, by index
    std::vector<size_t> pool_cap;
    void release() {
        w.release();
        w = Workspace();
        for (size_t& c : cap) c = 0;
        for (void* p : pool)
            if (p) cudaFree(p);
        pool.clear();
        pool_cap.clear();
    }
    // grow-only buffer i to at least b bytes (the contents are not kept)
    bool grow(int i, void** p, size_t b) {
        if (b <= cap[i]) return true;
        if (*p) cudaFree(*p);
        *p = nullptr;
        cap[i] = 0;
        if (cudaMalloc(p, b) != cudaSuccess) return false;
        cap[i] = b;
        return true;
    }
};

// norm_inside_mask on E complex volumes X (real parts), in place
static cudaError_t normalize_entries(float2* X, const float* mask, long long nn, int E, double nmask, Workspace& w,
                                     cudaStream_t st, int64_t* launches) {
    cudaError_t e = cudaMemsetAsync(w.sums, 0, sizeof(double) * E, st);
    if (!e) e = cudaMemsetAsync(w.var, 0, sizeof(double) * E, st);
    dim3 g((unsigned)std::min<long long>((nn + 255) / 256, 64), E);
    if (!e) {
        k_al_stats<<<g, 256, 0, st>>>(X, mask, nn, nullptr, 0, w.sums);
        k_al_mean<<<(E + 127) / 128, 128, 0, st>>>(w.sums, w.mea, E, nmask);
        k_al_stats<<<g, 256, 0, st>>>(X, mask, nn, w.mea, 1, w.var);
        k_al_normalize<<<grid_for(nn * E), 256, 0, st>>>(X, mask, nn, E, w.mea, w.var, nmask);
        e = cudaGetLastError();
    }
    *launches += 4;
    return e;
}

// norm_inside_mask on E real volumes X, in place
static cudaError_t normalize_entries_r(float* X, const float* mask, long long nn, int E, double nmask, Workspace& w,
                                       cudaStream_t st, int64_t* launches) {
    cudaError_t e = cudaMemsetAsync(w.sums, 0, sizeof(double) * E, st);
    if (!e) e = cudaMemsetAsync(w.var, 0, sizeof(double) * E, st);
    dim3 g((unsigned)std::min<long long>((nn + 255) / 256, 64), E);
    if (!e) {
        k_al_stats_r<<<g, 256, 0, st>>>(X, mask, nn, nullptr, 0, w.sums);
        k_al_mean<<<(E + 127) / 128, 128, 0, st>>>(w.sums, w.mea, E, nmask);
        k_al_stats_r<<<g, 256, 0, st>>>(X, mask, nn, w.mea, 1, w.var);
        k_al_normalize_r<<<grid_for(nn * E), 256, 0, st>>>(X, mask, nn, E, w.mea, w.var, nmask);
        e = cudaGetLastError();
    }
    *launches += 4;
    return e;
}

namespace {
__global__ void k_cmul(float2* __restrict__ a, const float2* __restrict__ b, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a[t] = cmul(a[t], b[t]);
}
__global__ void k_re_keep(float2* __restrict__ a, long long n) {
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
        a[t].y = 0.f;
}
}  // namespace

// tom_corr (Analysis/tom_corr.m:51-95): mode 0 plain ccf / numel, mode 1 'norm'
// with mask (norm_inside_mask, n - 1 std) and optional psfs (a (*) psf2,
// b (*) psf1 first).  All device buffers of size n; out real.
int corr_norm(tomgpu_ctx* ctx, const float* a, const float* b, const int n[3], const float* mask, const float* psf1,
              const float* psf2, float* out) {
    const long long nn = (long long)n[0] * n[1] * n[2];
    cudaStream_t st = ctx->stream;
    for (int d = 0; d < 3; ++d)
        if (n[d] > 1 && !fft_length_supported(n[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "size not an FFT length");
    if ((psf1 == nullptr) != (psf2 == nullptr)) return fail(ctx, TOMGPU_ERR_ARG, "give both psfs or none");
    if (psf1 && !mask) return fail(ctx, TOMGPU_ERR_ARG, "the psf form needs a mask");
    float2 *A = nullptr, *B = nullptr, *P = nullptr;
    double *sums = nullptr, *mea = nullptr, *var = nullptr;
    auto cleanup = [&]() {
        void* p[] = {A, B, P, sums, mea, var};
        for (void* q : p)
            if (q) cudaFree(q);
    };
    if (cudaMalloc(&A, sizeof(float2) * nn) || cudaMalloc(&B, sizeof(float2) * nn) ||
        (psf1 && cudaMalloc(&P, sizeof(float2) * nn)) || cudaMalloc(&sums, 8) || cudaMalloc(&mea, 8) ||
        cudaMalloc(&var, 8)) {
        cudaGetLastError();
        cleanup();
        return fail(ctx, TOMGPU_ERR_OOM, "tom_corr workspace");
    }
    cudaError_t e = cudaSuccess;
    int rc = TOMGPU_OK;
    double nmask = (double)nn;
    do {
        k_al_r2c_masked<<<grid_for(nn), 256, 0, st>>>(a, nullptr, A, nn);
        k_al_r2c_masked<<<grid_for(nn), 256, 0, st>>>(b, nullptr, B, nn);
        if (psf1) {
            // a <- a (*) psf2, b <- b (*) psf1 (real parts kept)
            if ((e = c2c3d<float2>(A, n, -1, 1.0, st))) break;
            k_al_r2c_masked<<<grid_for(nn), 256, 0, st>>>(psf2, nullptr, P, nn);
            if ((e = c2c3d<float2>(P, n, -1, 1.0, st))) break;
            k_cmul<<<grid_for(nn), 256, 0, st>>>(A, P, nn);
            if ((e = c2c3d<float2>(A, n, +1, 1.0 / (double)nn, st))) break;
            k_re_keep<<<grid_for(nn), 256, 0, st>>>(A, nn);
            if ((e = c2c3d<float2>(B, n, -1, 1.0, st))) break;
            k_al_r2c_masked<<<grid_for(nn), 256, 0, st>>>(psf1, nullptr, P, nn);
            if ((e = c2c3d<float2>(P, n, -1, 1.0, st))) break;
            k_cmul<<<grid_for(nn), 256, 0, st>>>(B, P, nn);
            if ((e = c2c3d<float2>(B, n, +1, 1.0 / (double)nn, st))) break;
            k_re_keep<<<grid_for(nn), 256, 0, st>>>(B, nn);
            ctx->launches += 6 + 18;
        }
        if (mask) {
            if ((e = count_nonzero(mask, nn, sums, st))) break;
            if ((e = cudaMemcpyAsync(&nmask, sums, 8, cudaMemcpyDeviceToHost, st))) break;
            if ((e = cudaStreamSynchronize(st))) break;
            if (nmask < 2) { rc = fail(ctx, TOMGPU_ERR_ARG, "mask needs at least two voxels"); break; }
            Workspace w;
            w.sums = sums; w.mea = mea; w.var = var;
            if ((e = normalize_entries(A, mask, nn, 1, nmask, w, st, &ctx->launches))) break;
            if ((e = normalize_entries(B, mask, nn, 1, nmask, w, st, &ctx->launches))) break;
        }
        if ((e = c2c3d<float2>(A, n, -1, 1.0, st))) break;
        if ((e = c2c3d<float2>(B, n, -1, 1.0, st))) break;
        k_al_cross<<<grid_for(nn), 256, 0, st>>>(B, A, nn);
        if ((e = c2c3d<float2>(B, n, +1, 1.0 / (double)nn, st))) break;
        k_al_map<<<grid_for(nn), 256, 0, st>>>(B, n[0], n[1], n[2], 1.0 / nmask, nullptr, out);
        e = cudaGetLastError();
        ctx->launches += 2 + 9 + 2;
    } while (0);
    if (e && !rc) rc = cuda_fail(ctx, e, "tom_corr");
    cleanup();
    return rc;
}

// After the scan (av3_new/tom_av3_align.m:160-189): the first maximum of
// ccf_max * mask_ccf gives the angle index (tom_av3_index2angle); the
// reference rotated by those angles is correlated once more with the particle
// (tom_corr 'norm' inside the mask, no wedges) and tom_peak(., 'spline') of
// ccf * mask_ccf gives the shift and the peak.  cmax / amax are the scan's
// running maximum and angle index volumes, nmask the mask's non-zero count.
int align_finish(tomgpu_ctx* ctx, cudaStream_t st, const tomgpu_align_job& job, int nph, int nps,
                 const float* cmax, const float* amax, double nmask, AlignScratch* sc, float angles_out[3],
                 float shifts_out[3], float* peak_out) {
    const int* n = job.n;
    const long long nn = (long long)n[0] * n[1] * n[2];
    const bool wedges = job.wedge_ref != nullptr;
    Workspace& w = sc->w;
    if (!sc->grow(0, (void**)&w.A, sizeof(float2) * nn) || !sc->grow(1, (void**)&w.B, sizeof(float2) * nn) ||
        !sc->grow(6, (void**)&w.tmp, sizeof(float) * nn) || !sc->grow(7, (void**)&w.mats, sizeof(float) * 18) ||
        !sc->grow(8, (void**)&w.aidx, sizeof(int)) || !sc->grow(9, (void**)&w.sums, sizeof(double)) ||
        !sc->grow(10, (void**)&w.mea, sizeof(double)) || !sc->grow(11, (void**)&w.var, sizeof(double)) ||
        !sc->grow(12, (void**)&w.spline, sizeof(double) * 8) ||
        !sc->grow(13, (void**)&w.key, sizeof(unsigned long long))) {
        cudaGetLastError();
        sc->release();
        return fail(ctx, TOMGPU_ERR_OOM, "alignment workspace allocation failed");
    }
    const float cx = (float)((n[0] + 1) / 2), cy = (float)((n[1] + 1) / 2), cz = (float)((n[2] + 1) / 2);
    int rc = TOMGPU_OK;
    cudaError_t e = cudaSuccess;
    do {
        // first maximum of ccf_max * mask_ccf
        k_al_mul<<<grid_for(nn), 256, 0, st>>>(cmax, job.mask_ccf, w.tmp, nn);
        if ((e = argmax_key(w.tmp, nn, w.key, st))) break;
        unsigned long long key = 0;
        if ((e = cudaMemcpyAsync(&key, w.key, sizeof key, cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaStreamSynchronize(st))) break;
        if (!key) { rc = fail(ctx, TOMGPU_ERR_DEVICE, "no correlation peak above -99999"); break; }
        const long long pv = (long long)(0xFFFFFFFFull - (key & 0xFFFFFFFFull));
        float ai = 0;
        if ((e = cudaMemcpyAsync(&ai, amax + pv, sizeof(float), cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaStreamSynchronize(st))) break;
        // tom_av3_index2angle
        const double a3 = std::floor(ai / (double)(nph * nps));
        const double rest = ai - a3 * nph * nps;
        const double a2 = std::floor(rest / nph);
        const double a1 = rest - a2 * nph;
        const float eul[3] = {(float)(a1 * job.phi[1] + job.phi[0]), (float)(a2 * job.psi[1] + job.psi[0]),
                              (float)(a3 * job.theta[1] + job.theta[0])};
        // ccf_s = tom_corr(rot(ref, angles), part, 'norm', mask)
        float em[9];
        euler_matrix_host(eul, em);
        if ((e = cudaMemcpyAsync(w.mats, em, sizeof em, cudaMemcpyHostToDevice, st))) break;
        int zero = 0;
        if ((e = cudaMemcpyAsync(w.aidx, &zero, sizeof zero, cudaMemcpyHostToDevice, st))) break;
        k_al_rotate<<<dim3((unsigned)((nn + 255) / 256), 1), 256, 0, st>>>(job.ref, nullptr, job.mask, w.mats, nullptr,
                                                                            n[0], n[1], n[2], cx, cy, cz, 0, nullptr,
                                                                            w.A, nullptr);
        k_al_r2c_masked<<<grid_for(nn), 256, 0, st>>>(job.part, wedges ? job.mask : nullptr, w.B, nn);
        if ((e = normalize_entries(w.A, job.mask, nn, 1, nmask, w, st, &ctx->launches))) break;
        if ((e = normalize_entries(w.B, job.mask, nn, 1, nmask, w, st, &ctx->launches))) break;
        if ((e = c2c3d<float2>(w.A, n, -1, 1.0, st))) break;
        if ((e = c2c3d<float2>(w.B, n, -1, 1.0, st))) break;
        k_al_cross<<<grid_for(nn), 256, 0, st>>>(w.B, w.A, nn);
        if ((e = c2c3d<float2>(w.B, n, +1, 1.0 / (double)nn, st))) break;
        k_al_map<<<grid_for(nn), 256, 0, st>>>(w.B, n[0], n[1], n[2], 1.0 / nmask, job.mask_ccf, w.tmp);
        if ((e = argmax_key(w.tmp, nn, w.key, st))) break;
        if ((e = cudaMemcpyAsync(&key, w.key, sizeof key, cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaStreamSynchronize(st))) break;
        ctx->launches += 16;
        if (!key) { rc = fail(ctx, TOMGPU_ERR_DEVICE, "no refinement peak above -99999"); break; }
        const long long pv2 = (long long)(0xFFFFFFFFull - (key & 0xFFFFFFFFull));
        const int p0[3] = {(int)(pv2 % n[0]), (int)((pv2 / n[0]) % n[1]), (int)(pv2 / ((long long)n[0] * n[1]))};
        if ((e = spline_peak(w.tmp, n, p0, w.spline, st))) break;
        double h[6];
        if ((e = cudaMemcpyAsync(h, w.spline, sizeof h, cudaMemcpyDeviceToHost, st))) break;
        if ((e = cudaStreamSynchronize(st))) break;
        for (int d = 0; d < 3; ++d) {
            angles_out[d] = eul[d];
            shifts_out[d] = (float)(h[d] - (std::floor(n[d] / 2.0) + 1.0));
        }
        *peak_out = (float)std::fmax(h[3], std::fmax(h[4], h[5]));
    } while (0);
    if (e && !rc) rc = cuda_fail(ctx, e, "av3_align");
    return rc;
}

int align_job(tomgpu_ctx* ctx, const tomgpu_align_job& job, float angles_out[3], float shifts_out[3], float* peak_out,
              size_t budget_voxels, AlignScratch* scratch) {
    const int* n = job.n;
    const long long nn = (long long)n[0] * n[1] * n[2];
    cudaStream_t st = ctx->stream;
    const bool wedges = job.wedge_ref != nullptr;
    const float* wpart = job.wedge_part ? job.wedge_part : job.wedge_ref;
    if (!job.ref || !job.part || !job.mask) return fail(ctx, TOMGPU_ERR_ARG, "job needs ref, part and mask");
    for (int d = 0; d < 3; ++d)
        if (!fft_length_supported(n[d])) return fail(ctx, TOMGPU_ERR_UNSUPPORTED, "box edge not an FFT length");
    // scan in the reference's loop order
    std::vector<double> ph = axis_values(job.phi), ps = axis_values(job.psi), th = axis_values(job.theta);
    struct Ang { double phi, psi, theta; int idx; };
    std::vector<Ang> scan;
    const int nph = (int)ph.size(), nps = (int)ps.size();
    for (size_t a = 0; a < ph.size(); ++a)
        for (size_t b = 0; b < ps.size(); ++b)
            for (size_t c = 0; c < th.size(); ++c)
                scan.push_back({ph[a], ps[b], th[c], (int)(c * nph * nps + b * nph + a)});
    const int R = (int)scan.size();
    int E = (int)std::max<long long>(1, std::min<long long>(256, (long long)budget_voxels / nn));
    E = std::min(E, R);
    AlignScratch local;
    AlignScratch& sc = scratch ? *scratch : local;
    Workspace& w = sc.w;
    // grow-only buffers, kept for the next job of the call
    auto G = [&](int i, void** p, size_t b) { return sc.grow(i, p, b); };
    const long long nhn = (long long)(n[0] / 2 + 1) * n[1] * n[2];  // one half spectrum
    const long long ncx = std::max<long long>(nn, nhn * E);         // complex slots: E half spectra or one volume
    if (!G(0, (void**)&w.A, sizeof(float2) * ncx) || !G(1, (void**)&w.B, sizeof(float2) * ncx) ||
        !G(14, (void**)&w.Ar, sizeof(float) * nn * E) || !G(15, (void**)&w.Br, sizeof(float) * nn * E) ||
        !G(2, (void**)&w.B0, sizeof(float2) * nn) || (wedges && !G(3, (void**)&w.W, sizeof(float) * nn * E)) ||
        !G(4, (void**)&w.cmax, sizeof(float) * nn) || !G(5, (void**)&w.amax, sizeof(float) * nn) ||
        !G(6, (void**)&w.tmp, sizeof(float) * nn) || !G(7, (void**)&w.mats, sizeof(float) * 18 * R) ||
        !G(8, (void**)&w.aidx, sizeof(int) * R) || !G(9, (void**)&w.sums, sizeof(double) * E) ||
        !G(10, (void**)&w.mea, sizeof(double) * E) || !G(11, (void**)&w.var, sizeof(double) * E) ||
        !G(12, (void**)&w.spline, sizeof(double) * 8) || !G(13, (void**)&w.key, sizeof(unsigned long long))) {
        cudaGetLastError();
        sc.release();
        return fail(ctx, TOMGPU_ERR_OOM, "alignment workspace allocation failed");
    }
    int rc = TOMGPU_OK;
    cudaError_t e = cudaSuccess;
    const float cx = (float)((n[0] + 1) / 2), cy = (float)((n[1] + 1) / 2), cz = (float)((n[2] + 1) / 2);
    do {
        // mask size and B0 = F(part*mask) (the loop's part = part .* mask)
        double nmask = 0;
        {
            double* d = w.sums;
            if ((e = count_nonzero(job.mask, nn, d, st))) break;
            if ((e = cudaMemcpyAsync(&nmask, d, sizeof(double), cudaMemcpyDeviceToHost, st))) break;
            if ((e = cudaStreamSynchronize(st))) break;
        }
        if (nmask < 2) { rc = fail(ctx, TOMGPU_ERR_ARG, "mask needs at least two voxels"); break; }
        // B0: half spectrum of part (* mask where wedges are given)
        k_al_mul<<<grid_for(nn), 256, 0, st>>>(job.part, wedges ? job.mask : nullptr, w.Br, nn);
        if ((e = r2c3d_batch<float2>(w.Br, w.B0, n, 1, st))) break;
        k_al_fill<<<grid_for(nn), 256, 0, st>>>(w.cmax, w.amax, nn, -2.f, -2.f);
        ctx->launches += 5;
        // every rotation's matrices and angle index, uploaded once: [R] matrix-mode
        // matrices, then [R] Euler-mode matrices
        std::vector<float> mats(18 * (size_t)R);
        std::vector<int> aid(R);
        for (int q = 0; q < R; ++q) {
            const Ang& g = scan[q];
            rotmatrix_as_float(g.phi, g.psi, g.theta, mats.data() + 9 * q);
            const float eul[3] = {(float)g.phi, (float)g.psi, (float)g.theta};
            euler_matrix_host(eul, mats.data() + 9 * (size_t)R + 9 * q);
            aid[q] = g.idx;
        }
        if ((e = cudaMemcpyAsync(w.mats, mats.data(), sizeof(float) * 18 * R, cudaMemcpyHostToDevice, st))) break;
        if ((e = cudaMemcpyAsync(w.aidx, aid.data(), sizeof(int) * R, cudaMemcpyHostToDevice, st))) break;
        for (int off = 0; off < R && !e; off += E) {
            const int nb = std::min(E, R - off);
            dim3 g((unsigned)((nn + 255) / 256), nb);
            k_al_rotate<<<g, 256, 0, st>>>(job.ref, job.wedge_ref, job.mask, w.mats + 9 * off,
                                           w.mats + 9 * (size_t)R + 9 * off, n[0], n[1], n[2], cx, cy, cz,
                                           wedges ? 1 : 0, w.Ar, nullptr, wedges ? w.W : nullptr);
            ctx->launches += 1;
            const dim3 gh(grid_for(nhn), (nb + AL_EG - 1) / AL_EG);
            if (wedges) {
                // a = ref_rot*mask (*) psf_part
                if ((e = r2c3d_batch<float2>(w.Ar, w.A, n, nb, st))) break;
                k_al_wpart_h<<<gh, 256, 0, st>>>(w.A, wpart, n[0], n[1], n[2], nb);
                if ((e = c2r3d_batch<float2>(w.A, w.Ar, n, nb, 1.0 / (double)nn, st))) break;
                // b = part*mask (*) psf_ref
                k_al_bside_h<<<gh, 256, 0, st>>>(w.B, w.B0, w.W, n[0], n[1], n[2], nb);
                if ((e = c2r3d_batch<float2>(w.B, w.Br, n, nb, 1.0 / (double)nn, st))) break;
                ctx->launches += 2 + 9;
            } else {
                // b = part for every entry
                k_al_bcast<<<grid_for(nn * nb), 256, 0, st>>>(w.Br, job.part, (int)nn, nb);
                ctx->launches += 1;
            }
            if ((e = normalize_entries_r(w.Ar, job.mask, nn, nb, nmask, w, st, &ctx->launches))) break;
            if ((e = normalize_entries_r(w.Br, job.mask, nn, nb, nmask, w, st, &ctx->launches))) break;
            if ((e = r2c3d_batch<float2>(w.Ar, w.A, n, nb, st))) break;
            if ((e = r2c3d_batch<float2>(w.Br, w.B, n, nb, st))) break;
            k_al_cross<<<grid_for(nhn * nb), 256, 0, st>>>(w.B, w.A, nhn * nb);
            if ((e = c2r3d_batch<float2>(w.B, w.Br, n, nb, 1.0 / (double)nn, st))) break;
            k_al_update_r<<<grid_for(nn), 256, 0, st>>>(w.Br, n[0], n[1], n[2], nb, 1.0 / nmask, w.aidx + off,
                                                        w.cmax, w.amax);
            e = cudaGetLastError();
            ctx->launches += 2 + 9;
        }
        if (e) break;
        rc = align_finish(ctx, st, job, nph, nps, w.cmax, w.amax, nmask, &sc, angles_out, shifts_out, peak_out);
    } while (0);
    if (e && !rc) rc = cuda_fail(ctx, e, "av3_align");
    if (!scratch) local.release();
    return rc;
}

AlignScratch* align_scratch_new() { return new AlignScratch(); }

void* align_scratch_buffer(AlignScratch* s, int i, size_t bytes) {
    if ((size_t)i >= s->pool.size()) {
        s->pool.resize(i + 1, nullptr);
        s->pool_cap.resize(i + 1, 0);
    }
    if (bytes == 0) bytes = 1;
    if (bytes <= s->pool_cap[i]) return s->pool[i];
    if (s->pool[i]) cudaFree(s->pool[i]);
    s->pool[i] = nullptr;
    s->pool_cap[i] = 0;
    if (cudaMalloc(&s->pool[i], bytes) != cudaSuccess) {
        s->pool[i] = nullptr;
        return nullptr;
    }
    s->pool_cap[i] = bytes;
    return s->pool[i];
}

void align_scratch_free(AlignScratch* s) {
    if (!s) return;
    s->release();
    delete s;
}

}  // namespace tg
