// Line FFTs of any length in shared memory (sm_100a, FP32 or FP64).
//
// The compile-time engine (fft_engine.cuh) covers the lengths the benchmark
// sizes need, with the stage count and butterflies-per-thread known to the
// compiler.  This engine takes the length at run time, so a tomogram or a
// template of any edge can be transformed (MATLAB's fftn takes any size):
//
// * lengths whose prime factors are all in {2, 3, 5, 7, 11, 13}: a Stockham
//   mixed-radix transform (radices 16, 8, 4, 2, 3, 5, 7, 11, 13), each stage
//   reading one shared-memory buffer and writing the other (ping-pong), so a
//   thread may own any number of butterflies;
// * any other length L: Bluestein's chirp-z form, X_k = c_k sum_n (x_n c_n)
//   conj(c_{k-n}) with c_n = exp(-i pi n^2 / L), the convolution done
//   cyclically over a {2,3,5,7}-smooth length M >= 2L - 1 by two mixed-radix
//   transforms and a product with the precomputed spectrum of conj(c).
//
// The block holds NL lines at s + l LS and a second buffer of the same shape
// at s2; LS >= the length the stages run over (L, or M for Bluestein).  The
// inverse (DIR = +1) is unnormalised, as in fft_engine.cuh.
#pragma once
#include "fft_engine.cuh"
#include "fft_plan.h"

namespace tgrt {

// One Stockham stage of radix R over lines of length L: butterfly j of a line
// reads src[j + r L/R] (r < R), applies the stage twiddles, runs the R-point
// DFT and writes dst[(j - k) R + k + r NS] with k = j mod NS.
template <int R, int DIR, typename C>
TG_D void stage_r(const C* __restrict__ src, C* __restrict__ dst, int L, int NS, int NL, int LS,
                  const C* __restrict__ tw, int tid, int nt) {
    const int NBL = L / R;
    const int NB = NL * NBL;
    const int tstep = L / (NS * R);
    for (int b = tid; b < NB; b += nt) {
        const int line = b / NBL, j = b - line * NBL;
        const C* sp = src + line * LS;
        C v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = sp[j + r * NBL];
        const int k = j % NS;
        if (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                C w = tgfft::ldtw(tw, r * k * tstep);
                if (DIR > 0) w = cconj(w);
                v[r] = cmul(v[r], w);
            }
        }
        tgfft::dft<R, DIR>(v, tw, L / R);
        C* dp = dst + line * LS;
        const int p0 = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dp[p0 + r * NS] = v[r];
    }
}

// The mixed-radix stages over length L; the caller has synchronised after
// filling a.  Returns the buffer that holds the result (a or b); ends with a
// barrier.
template <int DIR, typename C>
TG_D C* run_direct(C* a, C* b, const Plan& p, int NL, int LS, const C* __restrict__ tw, int tid, int nt) {
    const int L = p.M;
    int NS = 1;
    for (int i = 0; i < p.nst; ++i) {
        const int R = p.r[i];
        switch (R) {
            case 2: stage_r<2, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 3: stage_r<3, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 4: stage_r<4, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 5: stage_r<5, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 7: stage_r<7, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 8: stage_r<8, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 11: stage_r<11, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            case 13: stage_r<13, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
            default: stage_r<16, DIR>(a, b, L, NS, NL, LS, tw, tid, nt); break;
        }
        __syncthreads();
        C* t = a;
        a = b;
        b = t;
        NS *= R;
    }
    return a;
}

// Transform NL lines of length p.L held at s + l LS (natural order); s2 is the
// second buffer.  Returns the buffer holding the result, after a barrier.
template <int DIR, typename C>
TG_D C* fft(C* s, C* s2, const Plan& p, const Tabs<C>& t, int NL, int LS, int tid, int nt) {
    if (!p.blue) return run_direct<DIR>(s, s2, p, NL, LS, t.tw, tid, nt);
    const int L = p.L, M = p.M;
    // a_n = x_n c_n (the inverse conjugates in and out), zero-padded to M
    for (int i = tid; i < NL * M; i += nt) {
        const int l = i / M, n = i - l * M;
        C v = CTraits<C>::make(0, 0);
        if (n < L) {
            C x = s[l * LS + n];
            if (DIR > 0) x = cconj(x);
            v = cmul(x, __ldg(t.chirp + n));
        }
        s[l * LS + n] = v;
    }
    __syncthreads();
    C* X = run_direct<-1>(s, s2, p, NL, LS, t.tw, tid, nt);
    C* Y = X == s ? s2 : s;
    for (int i = tid; i < NL * M; i += nt) {
        const int l = i / M, m = i - l * M;
        X[l * LS + m] = cmul(X[l * LS + m], __ldg(t.bspec + m));
    }
    __syncthreads();
    X = run_direct<+1>(X, Y, p, NL, LS, t.tw, tid, nt);
    for (int i = tid; i < NL * L; i += nt) {
        const int l = i / L, k = i - l * L;
        C y = cmul(X[l * LS + k], __ldg(t.chirp + k));
        if (DIR > 0) y = cconj(y);
        X[l * LS + k] = y;
    }
    __syncthreads();
    return X;
}

}  // namespace tgrt
