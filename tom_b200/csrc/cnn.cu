// Kernels of the learned candidate proposer: a dilated 3-D convolutional
// network trained on the search's own results (tom_b200/proposer.py).
//
// Volumes are [C][Z][Y][X] FP32 (x fastest), one sample.  A layer is a 3x3x3
// convolution with dilation d and zero padding ("same" size), bias and an
// optional ReLU.  Forward: out[co][v] = b[co] + sum_ci sum_t w[co][ci][t]
// in[ci][v + d off(t)], off(t) = (t%3-1, t/3%3-1, t/9-1).  The input gradient
// is the same convolution with the taps mirrored and the channel roles
// swapped (the host passes the re-arranged weights); the weight gradient is a
// reduction over voxels per (co, ci, tap).
//
// conv_fwd (k_conv_fwd2): one block per 32 x 8 x 4 output tile and group of
// up to 16 output channels; per input channel the tile plus its halo is
// staged in shared memory and every thread applies the 27 taps to its 4
// voxels and the group's channels (4 x 16 multiply-adds per tap for 4 staged
// values and 4 float4 weight reads).
#include <cstdint>

#include "common.cuh"
#include "ctx.h"

namespace tg {

namespace {

// Register-blocked forward convolution: a 32 x 8 x 4 output tile per block,
// each thread 4 voxels along y (lanes along x, so every shared-memory read of
// a warp is 32 consecutive floats) for a group of up to 16 output channels
// (the group is blockIdx.z / ztiles).  Per input channel the tile and its halo
// are staged row by row (one division per row), the group's weights tap-major
// so that a tap's channel weights are read as float4.
constexpr int FX = 32, FY = 8, FZ = 4, FR = 4, FCG = 16;

template <int CO>
__global__ void __launch_bounds__(256) k_conv_fwd2(const float* __restrict__ in, int ci_n, int nx, int ny, int nz,
                                                   const float* __restrict__ w, const float* __restrict__ bias,
                                                   int dil, int relu, float* __restrict__ out, int ztiles) {
    constexpr int CG = CO < FCG ? CO : FCG;
    extern __shared__ __align__(16) float smf[];
    const int hx = FX + 2 * dil, hy = FY + 2 * dil, hz = FZ + 2 * dil;
    float* tile = smf;                                // [hz][hy][hx]
    float* ws = smf + ((hz * hy * hx + 3) & ~3);      // [27][CG]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ty = (tid >> 5) & 1, tz = tid >> 6;
    const int g = blockIdx.z / ztiles, zt = blockIdx.z - g * ztiles;
    const int bx = blockIdx.x * FX, by = blockIdx.y * FY, bz = zt * FZ, c0 = g * CG;
    const long long nv = (long long)nx * ny * nz;
    float acc[FR][CG];
#pragma unroll
    for (int r = 0; r < FR; ++r)
#pragma unroll
        for (int c = 0; c < CG; ++c) acc[r][c] = 0.f;
    const int rows = hz * hy;
    for (int ci = 0; ci < ci_n; ++ci) {
        const float* src = in + (long long)ci * nv;
        for (int row = warp; row < rows; row += 8) {
            const int iz = row / hy, iy = row - iz * hy;
            const int gy = by + iy - dil, gz = bz + iz - dil;
            const bool rok = gy >= 0 && gy < ny && gz >= 0 && gz < nz;
            const float* srow = src + ((long long)gz * ny + gy) * nx;
            for (int ix = lane; ix < hx; ix += 32) {
                const int gx = bx + ix - dil;
                tile[row * hx + ix] = (rok && gx >= 0 && gx < nx) ? __ldg(srow + gx) : 0.f;
            }
        }
        for (int i = tid; i < 27 * CG; i += 256) {
            const int t = i / CG, c = i - t * CG;
            ws[i] = __ldg(w + ((long long)(c0 + c) * ci_n + ci) * 27 + t);
        }
        __syncthreads();
#pragma unroll
        for (int t = 0; t < 27; ++t) {
            const int ox = (t % 3) * dil, oy = ((t / 3) % 3) * dil, oz = (t / 9) * dil;
            const float* trow = tile + ((tz + oz) * hy + (ty * FR + oy)) * hx + lane + ox;
            float v[FR];
#pragma unroll
            for (int r = 0; r < FR; ++r) v[r] = trow[r * hx];
            if constexpr (CG % 4 == 0) {
                const float4* wr = reinterpret_cast<const float4*>(ws + t * CG);
#pragma unroll
                for (int c4 = 0; c4 < CG / 4; ++c4) {
                    const float4 wv = wr[c4];
#pragma unroll
                    for (int r = 0; r < FR; ++r) {
                        acc[r][4 * c4] = fmaf(wv.x, v[r], acc[r][4 * c4]);
                        acc[r][4 * c4 + 1] = fmaf(wv.y, v[r], acc[r][4 * c4 + 1]);
                        acc[r][4 * c4 + 2] = fmaf(wv.z, v[r], acc[r][4 * c4 + 2]);
                        acc[r][4 * c4 + 3] = fmaf(wv.w, v[r], acc[r][4 * c4 + 3]);
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < CG; ++c) {
                    const float wv = ws[t * CG + c];
#pragma unroll
                    for (int r = 0; r < FR; ++r) acc[r][c] = fmaf(wv, v[r], acc[r][c]);
                }
            }
        }
        __syncthreads();
    }
    const int x = bx + lane, z = bz + tz;
    if (x >= nx || z >= nz) return;
#pragma unroll
    for (int r = 0; r < FR; ++r) {
        const int y = by + ty * FR + r;
        if (y >= ny) continue;
        const long long o = ((long long)z * ny + y) * nx + x;
#pragma unroll
        for (int c = 0; c < CG; ++c) {
            float res = acc[r][c] + (bias ? __ldg(bias + c0 + c) : 0.f);
            if (relu) res = fmaxf(res, 0.f);
            out[(long long)(c0 + c) * nv + o] = res;
        }
    }
}

// gw[co][ci][t] += sum_v gout[co][v] in[ci][v + d off(t)]; blockIdx.y = co * ci_n + ci
__global__ void __launch_bounds__(256) k_conv_wgrad(const float* __restrict__ in, int ci_n, int nx, int ny, int nz,
                                                    const float* __restrict__ gout, int dil, float* __restrict__ gw) {
    const int co = blockIdx.y / ci_n, ci = blockIdx.y - co * ci_n;
    const long long nv = (long long)nx * ny * nz;
    const float* g = gout + (long long)co * nv;
    const float* a = in + (long long)ci * nv;
    float acc[27];
#pragma unroll
    for (int t = 0; t < 27; ++t) acc[t] = 0.f;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x) {
        const float gv = g[v];
        if (gv == 0.f) continue;
        const int x = (int)(v % nx), y = (int)((v / nx) % ny), z = (int)(v / ((long long)nx * ny));
#pragma unroll
        for (int t = 0; t < 27; ++t) {
            const int sx = x + ((t % 3) - 1) * dil, sy = y + (((t / 3) % 3) - 1) * dil, sz = z + ((t / 9) - 1) * dil;
            if (sx >= 0 && sx < nx && sy >= 0 && sy < ny && sz >= 0 && sz < nz)
                acc[t] = fmaf(gv, __ldg(a + ((long long)sz * ny + sy) * nx + sx), acc[t]);
        }
    }
    __shared__ float red[8][27];
#pragma unroll
    for (int t = 0; t < 27; ++t) {
        float s = acc[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][t] = s;
    }
    __syncthreads();
    if (threadIdx.x < 27) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
        atomicAdd(gw + ((long long)co * ci_n + ci) * 27 + threadIdx.x, s);
    }
}

// gb[c] += sum_v g[c][v]
__global__ void __launch_bounds__(256) k_bias_grad(const float* __restrict__ g, long long nv, float* __restrict__ gb) {
    const float* a = g + (long long)blockIdx.y * nv;
    float s = 0.f;
    for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += (long long)gridDim.x * blockDim.x)
        s += a[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(gb + blockIdx.y, t);
    }
}

// the input-gradient weights: wt[ci][co][t] = w[co][ci][26 - t]
__global__ void k_flip_weights(const float* __restrict__ w, int co_n, int ci_n, float* __restrict__ wt) {
    const long long n = (long long)co_n * ci_n * 27;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(i % 27);
        const long long r = i / 27;
        const int co = (int)(r % co_n), ci = (int)(r / co_n);
        wt[i] = w[((long long)co * ci_n + ci) * 27 + (26 - t)];
    }
}

// g *= (act > 0)   (ReLU backward on the layer's output)
__global__ void k_relu_bwd(float* __restrict__ g, const float* __restrict__ act, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!(act[i] > 0.f)) g[i] = 0.f;
}

// binary cross-entropy with logits, positive weight pw: per voxel loss and
// d loss / d logit (divided by n); loss sum into *loss (FP64)
__global__ void __launch_bounds__(256) k_bce(const float* __restrict__ logit, const float* __restrict__ target,
                                             long long n, float pw, float* __restrict__ grad, double* __restrict__ loss) {
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float z = logit[i], y = target[i];
        // log(1 + exp(-|z|)) + max(-z, 0) = softplus(-z)
        const float sp_neg = log1pf(expf(-fabsf(z))) + fmaxf(-z, 0.f);  // -log sigmoid(z)
        const float sp_pos = sp_neg + z;                                 // -log(1 - sigmoid(z))
        const float wgt = y > 0.f ? pw : 1.f;
        s += (double)(wgt * (y * sp_neg + (1.f - y) * sp_pos));
        const float sg = 1.f / (1.f + expf(-z));
        grad[i] = wgt * (sg - y) / (float)n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(loss, t / (double)n);
    }
}

// softmax cross-entropy over K classes for P samples: logits [K][P] (channel
// major like the volumes), labels[P]; grad = (softmax - onehot) / P
__global__ void k_softmax_ce(const float* __restrict__ logits, const int* __restrict__ labels, int K, int P,
                             float* __restrict__ grad, double* __restrict__ loss) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    float mx = -INFINITY;
    for (int k = 0; k < K; ++k) mx = fmaxf(mx, logits[(long long)k * P + p]);
    float den = 0.f;
    for (int k = 0; k < K; ++k) den += expf(logits[(long long)k * P + p] - mx);
    const int y = labels[p];
    for (int k = 0; k < K; ++k) {
        const float sm = expf(logits[(long long)k * P + p] - mx) / den;
        grad[(long long)k * P + p] = (sm - (k == y ? 1.f : 0.f)) / (float)P;
    }
    atomicAdd(loss, (double)(-(logits[(long long)y * P + p] - mx - logf(den))) / (double)P);
}

// Adam step with bias correction (lr, b1, b2, eps), t = step number (1-based)
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// features at P voxels: out[c][p] = f[c][idx[p]]; scatter-add back for the gradient
__global__ void k_gather(const float* __restrict__ f, int C, long long nv, const long long* __restrict__ idx, int P,
                         float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)C * P) return;
    const int c = (int)(i / P), p = (int)(i - (long long)c * P);
    out[i] = f[(long long)c * nv + idx[p]];
}
__global__ void k_scatter_add(const float* __restrict__ g, int C, long long nv, const long long* __restrict__ idx,
                              int P, float* __restrict__ gf) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)C * P) return;
    const int c = (int)(i / P), p = (int)(i - (long long)c * P);
    atomicAdd(gf + (long long)c * nv + idx[p], g[i]);
}

// dense layer over P samples (a 1x1x1 convolution): out[k][p] = b[k] + sum_c W[k][c] F[c][p]
__global__ void k_dense_fwd(const float* __restrict__ W, const float* __restrict__ b, const float* __restrict__ F,
                            int K, int C, long long P, int relu, float* __restrict__ out) {
    const long long n = (long long)K * P;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / P);
        const long long p = i - (long long)k * P;
        float s = b ? b[k] : 0.f;
        for (int c = 0; c < C; ++c) s = fmaf(__ldg(W + (long long)k * C + c), F[(long long)c * P + p], s);
        out[i] = relu ? fmaxf(s, 0.f) : s;
    }
}
// gF[c][p] = sum_k W[k][c] g[k][p]
__global__ void k_dense_bwd_in(const float* __restrict__ W, const float* __restrict__ g, int K, int C, long long P,
                               float* __restrict__ gF) {
    const long long n = (long long)C * P;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i / P);
        const long long p = i - (long long)c * P;
        float s = 0.f;
        for (int k = 0; k < K; ++k) s = fmaf(__ldg(W + (long long)k * C + c), g[(long long)k * P + p], s);
        gF[i] = s;
    }
}
// gW[k][c] += sum_p g[k][p] F[c][p]; blockIdx.y = k * C + c
__global__ void __launch_bounds__(256) k_dense_bwd_w(const float* __restrict__ g, const float* __restrict__ F, int C,
                                                     long long P, float* __restrict__ gW) {
    const int k = blockIdx.y / C, c = blockIdx.y - k * C;
    float s = 0.f;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x)
        s = fmaf(g[(long long)k * P + p], F[(long long)c * P + p], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ float red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        atomicAdd(gW + blockIdx.y, t);
    }
}

unsigned gridn(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (unsigned)(b < 1 ? 1 : b);
}

template <int CO>
cudaError_t launch_fwd(const float* in, int ci, const int d[3], const float* w, const float* b, int dil, int relu,
                       float* out, cudaStream_t st) {
    constexpr int CG = CO < FCG ? CO : FCG, NG = CO / CG;
    const size_t tile = (size_t)(FX + 2 * dil) * (FY + 2 * dil) * (FZ + 2 * dil);
    const size_t smem = sizeof(float) * (((tile + 3) & ~(size_t)3) + 27 * CG);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    cudaFuncSetAttribute(k_conv_fwd2<CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int ztiles = (d[2] + FZ - 1) / FZ;
    dim3 g((d[0] + FX - 1) / FX, (d[1] + FY - 1) / FY, ztiles * NG);
    k_conv_fwd2<CO><<<g, 256, smem, st>>>(in, ci, d[0], d[1], d[2], w, b, dil, relu, out, ztiles);
    return cudaGetLastError();
}

}  // namespace

cudaError_t cnn_conv_fwd(const float* in, int ci, const int d[3], const float* w, const float* b, int co, int dil,
                         int relu, float* out, cudaStream_t st) {
    switch (co) {
        case 1: return launch_fwd<1>(in, ci, d, w, b, dil, relu, out, st);
        case 8: return launch_fwd<8>(in, ci, d, w, b, dil, relu, out, st);
        case 16: return launch_fwd<16>(in, ci, d, w, b, dil, relu, out, st);
        case 32: return launch_fwd<32>(in, ci, d, w, b, dil, relu, out, st);
        case 64: return launch_fwd<64>(in, ci, d, w, b, dil, relu, out, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t cnn_conv_wgrad(const float* in, int ci, const int d[3], const float* gout, int co, int dil, float* gw,
                           float* gb, cudaStream_t st) {
    const long long nv = (long long)d[0] * d[1] * d[2];
    long long bx = (nv + 255) / 256;
    if (bx > 64) bx = 64;
    k_conv_wgrad<<<dim3((unsigned)bx, (unsigned)(co * ci)), 256, 0, st>>>(in, ci, d[0], d[1], d[2], gout, dil, gw);
    if (gb) k_bias_grad<<<dim3((unsigned)bx, (unsigned)co), 256, 0, st>>>(gout, nv, gb);
    return cudaGetLastError();
}

cudaError_t cnn_flip_weights(const float* w, int co, int ci, float* wt, cudaStream_t st) {
    k_flip_weights<<<gridn((long long)co * ci * 27), 256, 0, st>>>(w, co, ci, wt);
    return cudaGetLastError();
}

cudaError_t cnn_relu_bwd(float* g, const float* act, long long n, cudaStream_t st) {
    k_relu_bwd<<<gridn(n), 256, 0, st>>>(g, act, n);
    return cudaGetLastError();
}

cudaError_t cnn_bce(const float* logit, const float* target, long long n, float pw, float* grad, double* loss,
                    cudaStream_t st) {
    k_bce<<<gridn(n), 256, 0, st>>>(logit, target, n, pw, grad, loss);
    return cudaGetLastError();
}

cudaError_t cnn_softmax_ce(const float* logits, const int* labels, int K, int P, float* grad, double* loss,
                           cudaStream_t st) {
    k_softmax_ce<<<(P + 127) / 128, 128, 0, st>>>(logits, labels, K, P, grad, loss);
    return cudaGetLastError();
}

cudaError_t cnn_adam(float* p, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                     int step, cudaStream_t st) {
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<gridn(n), 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t cnn_dense_fwd(const float* W, const float* b, const float* F, int K, int C, long long P, int relu,
                          float* out, cudaStream_t st) {
    k_dense_fwd<<<gridn((long long)K * P), 256, 0, st>>>(W, b, F, K, C, P, relu, out);
    return cudaGetLastError();
}

cudaError_t cnn_dense_bwd(const float* W, const float* F, const float* g, int K, int C, long long P, float* gF,
                          float* gW, float* gb, cudaStream_t st) {
    if (gF) k_dense_bwd_in<<<gridn((long long)C * P), 256, 0, st>>>(W, g, K, C, P, gF);
    long long bx = (P + 255) / 256;
    if (bx > 64) bx = 64;
    if (gW) k_dense_bwd_w<<<dim3((unsigned)bx, (unsigned)(K * C)), 256, 0, st>>>(g, F, C, P, gW);
    if (gb) k_bias_grad<<<dim3((unsigned)bx, (unsigned)K), 256, 0, st>>>(g, P, gb);
    return cudaGetLastError();
}

cudaError_t cnn_gather(const float* f, int C, long long nv, const long long* idx, int P, float* out, cudaStream_t st) {
    k_gather<<<(unsigned)(((long long)C * P + 255) / 256), 256, 0, st>>>(f, C, nv, idx, P, out);
    return cudaGetLastError();
}

cudaError_t cnn_scatter_add(const float* g, int C, long long nv, const long long* idx, int P, float* gf,
                            cudaStream_t st) {
    k_scatter_add<<<(unsigned)(((long long)C * P + 255) / 256), 256, 0, st>>>(g, C, nv, idx, P, gf);
    return cudaGetLastError();
}

}  // namespace tg
