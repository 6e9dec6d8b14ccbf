// Batched line FFTs in shared memory (sm_100a, FP32 or FP64).
//
// All threads of a block cooperate on NL lines of length L held in shared
// memory at s[l * LS + e].  Each stage is a Stockham autosort step of radix R:
// every thread loads its butterflies' R inputs into registers, applies the
// stage twiddles, runs the R-point DFT in registers, and after a barrier
// writes the outputs to their self-sorted positions, so the transform runs in
// place without a second buffer and leaves the result in natural order.
//
// Twiddles come from a per-length table tw[m] = exp(-2 pi i m / L) computed on
// the host in double precision (so the FP32 table is correctly rounded); the
// inverse direction uses the conjugate.  DIR = -1 is the forward transform,
// DIR = +1 the unnormalised inverse.
#pragma once
#include "common.cuh"

namespace tgfft {

template <int... Rs> struct seq {};
template <int A, int... Rs> struct seq_first { static constexpr int value = A; };

// Radix plans: odd radices last so that every stride NS before them is a power
// of two.  Other lengths run on the run-time engine (fft_rt.cuh).
template <int L> struct Radices;
template <> struct Radices<8> { typedef seq<8> type; };
template <> struct Radices<12> { typedef seq<4, 3> type; };
template <> struct Radices<16> { typedef seq<16> type; };
template <> struct Radices<20> { typedef seq<4, 5> type; };
template <> struct Radices<24> { typedef seq<8, 3> type; };
template <> struct Radices<32> { typedef seq<8, 4> type; };
template <> struct Radices<40> { typedef seq<8, 5> type; };
template <> struct Radices<48> { typedef seq<16, 3> type; };
template <> struct Radices<64> { typedef seq<8, 8> type; };
template <> struct Radices<80> { typedef seq<16, 5> type; };
template <> struct Radices<96> { typedef seq<3, 4, 8> type; };  // measured 6 % faster than 8, 4, 3
template <> struct Radices<128> { typedef seq<16, 8> type; };
template <> struct Radices<160> { typedef seq<16, 2, 5> type; };
template <> struct Radices<192> { typedef seq<16, 4, 3> type; };
template <> struct Radices<232> { typedef seq<8, 29> type; };
template <> struct Radices<256> { typedef seq<16, 16> type; };
template <> struct Radices<464> { typedef seq<16, 29> type; };
template <> struct Radices<512> { typedef seq<8, 8, 8> type; };
template <> struct Radices<928> { typedef seq<8, 4, 29> type; };
template <> struct Radices<1024> { typedef seq<16, 8, 8> type; };

template <typename C> TG_D C ldtw(const C* tw, int m) { return __ldg(tw + m); }

// ------------------------------------------------------------ small DFTs
template <int DIR, typename C> TG_D void dft2(C& a, C& b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR, typename C> TG_D void dft4(C& a0, C& a1, C& a2, C& a3) {
    C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3);
    C t3 = cmul_i<DIR>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

#define TG_SQRT1_2 0.70710678118654752440
#define TG_COS_PI8 0.92387953251128675613
#define TG_SIN_PI8 0.38268343236508977173

template <int DIR, typename C> TG_D void dft8(C* v) {
    typedef typename CTraits<C>::R Rt;
    const Rt h = (Rt)TG_SQRT1_2;
    dft4<DIR>(v[0], v[2], v[4], v[6]);
    dft4<DIR>(v[1], v[3], v[5], v[7]);
    // odd half times w8^k, w8 = exp(DIR i pi / 4)
    C o1 = v[3], o2 = v[5], o3 = v[7];
    o1 = CTraits<C>::make(h * (o1.x - DIR * o1.y), h * (o1.y + DIR * o1.x));
    o2 = cmul_i<DIR>(o2);
    o3 = CTraits<C>::make(h * (-o3.x - DIR * o3.y), h * (DIR * o3.x - o3.y));
    C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

template <int DIR, typename C> TG_D C w16(C a, int e) {
    // a * exp(DIR * 2 pi i e / 16) for the exponents a 4x4 split needs
    typedef typename CTraits<C>::R Rt;
    Rt c, s;
    switch (e) {
        case 1: c = (Rt)TG_COS_PI8; s = (Rt)TG_SIN_PI8; break;
        case 2: c = (Rt)TG_SQRT1_2; s = (Rt)TG_SQRT1_2; break;
        case 3: c = (Rt)TG_SIN_PI8; s = (Rt)TG_COS_PI8; break;
        case 4: return cmul_i<DIR>(a);
        case 6: c = -(Rt)TG_SQRT1_2; s = (Rt)TG_SQRT1_2; break;
        case 9: c = -(Rt)TG_COS_PI8; s = -(Rt)TG_SIN_PI8; break;
        default: return a;
    }
    s = DIR * s;
    return CTraits<C>::make(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <int DIR, typename C> TG_D void dft16(C* v) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<DIR>(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) v[n2 + 4 * k1] = w16<DIR>(v[n2 + 4 * k1], n2 * k1);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<DIR>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // v[k2 + 4 k1] holds X[k1 + 4 k2]: transpose the 4x4 index
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = a + 1; b < 4; ++b) {
            C t = v[a + 4 * b];
            v[a + 4 * b] = v[b + 4 * a];
            v[b + 4 * a] = t;
        }
}

// 32-point DFT: two 16-point DFTs of the even and odd samples and a radix-2
// combination with the 32nd roots of unity.
template <int DIR, typename C> TG_D void dft32(C* v) {
    typedef typename CTraits<C>::R Rt;
    // cos(pi k / 16), k = 0..8
    const Rt c[9] = {(Rt)1.0, (Rt)0.98078528040323044913, (Rt)0.92387953251128675613, (Rt)0.83146961230254523708,
                     (Rt)0.70710678118654752440, (Rt)0.55557023301960222474, (Rt)0.38268343236508977173,
                     (Rt)0.19509032201612826785, (Rt)0.0};
    C e[16], o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        e[i] = v[2 * i];
        o[i] = v[2 * i + 1];
    }
    dft16<DIR>(e);
    dft16<DIR>(o);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        // w = exp(DIR 2 pi i k / 32) = cos(pi k/16) + DIR i sin(pi k/16)
        const Rt cr = k <= 8 ? c[k] : -c[16 - k];
        const Rt si = k <= 8 ? c[8 - k] : c[k - 8];
        const Rt sn = DIR * si;
        const C t = CTraits<C>::make(o[k].x * cr - o[k].y * sn, o[k].x * sn + o[k].y * cr);
        v[k] = cadd(e[k], t);
        v[k + 16] = csub(e[k], t);
    }
}

template <int DIR, typename C> TG_D void dft3(C* v) {
    typedef typename CTraits<C>::R Rt;
    const Rt c = (Rt)-0.5, s = (Rt)(DIR * 0.86602540378443864676);
    C a = v[0], sm = cadd(v[1], v[2]), df = csub(v[1], v[2]);
    C m = CTraits<C>::make(a.x + c * sm.x, a.y + c * sm.y);
    C r = CTraits<C>::make(-s * df.y, s * df.x);  // i * s * df
    v[0] = cadd(a, sm);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}

template <int DIR, typename C> TG_D void dft5(C* v) {
    typedef typename CTraits<C>::R Rt;
    const Rt c1 = (Rt)0.30901699437494742410, c2 = (Rt)-0.80901699437494742410;
    const Rt s1 = (Rt)(DIR * 0.95105651629515357212), s2 = (Rt)(DIR * 0.58778525229247312917);
    C a = v[0];
    C p1 = cadd(v[1], v[4]), m1 = csub(v[1], v[4]);
    C p2 = cadd(v[2], v[3]), m2 = csub(v[2], v[3]);
    C b1 = CTraits<C>::make(a.x + c1 * p1.x + c2 * p2.x, a.y + c1 * p1.y + c2 * p2.y);
    C b2 = CTraits<C>::make(a.x + c2 * p1.x + c1 * p2.x, a.y + c2 * p1.y + c1 * p2.y);
    // i * (s1 m1 + s2 m2) and i * (s2 m1 - s1 m2)
    C q1 = CTraits<C>::make(-(s1 * m1.y + s2 * m2.y), s1 * m1.x + s2 * m2.x);
    C q2 = CTraits<C>::make(-(s2 * m1.y - s1 * m2.y), s2 * m1.x - s1 * m2.x);
    v[0] = cadd(a, cadd(p1, p2));
    v[1] = cadd(b1, q1);
    v[4] = csub(b1, q1);
    v[2] = cadd(b2, q2);
    v[3] = csub(b2, q2);
}

// 6 = 2 x 3 by the prime-factor mapping (no twiddles): inputs n = 3 n1 + 2 n2
// (mod 6) into two 3-point DFTs, then 2-point DFTs; output k = 3 k1 + 4 k2.
template <int DIR, typename C> TG_D void dft6(C* v) {
    C a[3] = {v[0], v[2], v[4]}, b[3] = {v[3], v[5], v[1]};
    dft3<DIR>(a);
    dft3<DIR>(b);
    v[0] = cadd(a[0], b[0]);
    v[3] = csub(a[0], b[0]);
    v[4] = cadd(a[1], b[1]);
    v[1] = csub(a[1], b[1]);
    v[2] = cadd(a[2], b[2]);
    v[5] = csub(a[2], b[2]);
}

// Prime radix P by direct summation, pairing k with P-k (real/imag symmetry):
// X_k = a0 + sum_{n=1}^{(P-1)/2} [ (a_n + a_{P-n}) cos + i DIR (a_n - a_{P-n}) sin ].
// Cos/sin of 2 pi m / P are read from the line's table (P divides L).
template <int P, int DIR, typename C>
TG_D void dft_prime(C* v, const C* __restrict__ tw, int q) {
    constexpr int H = (P - 1) / 2;
    C p[H], m[H];
#pragma unroll
    for (int n = 1; n <= H; ++n) {
        p[n - 1] = cadd(v[n], v[P - n]);
        m[n - 1] = csub(v[n], v[P - n]);
    }
    C out[P];
    C s0 = v[0];
#pragma unroll
    for (int n = 0; n < H; ++n) s0 = cadd(s0, p[n]);
    out[0] = s0;
#pragma unroll 1
    for (int k = 1; k <= H; ++k) {
        C re = v[0];
        C im = CTraits<C>::make(0, 0);
        int mk = 0;
#pragma unroll
        for (int n = 1; n <= H; ++n) {
            mk += k;
            if (mk >= P) mk -= P;
            const C w = ldtw(tw, mk * q);  // (cos, -sin) of 2 pi mk / P
            re = CTraits<C>::make(re.x + w.x * p[n - 1].x, re.y + w.x * p[n - 1].y);
            im = CTraits<C>::make(im.x - w.y * m[n - 1].x, im.y - w.y * m[n - 1].y);
        }
        // im holds sum sin * (a_n - a_{P-n}); forward multiplies by -i, inverse by +i
        C t = cmul_i<DIR>(im);
        out[k] = cadd(re, t);
        out[P - k] = csub(re, t);
    }
#pragma unroll
    for (int k = 0; k < P; ++k) v[k] = out[k];
}

template <int R, int DIR, typename C>
TG_D void dft(C* v, const C* __restrict__ tw, int q) {
    if constexpr (R == 2) dft2<DIR>(v[0], v[1]);
    else if constexpr (R == 3) dft3<DIR>(v);
    else if constexpr (R == 4) dft4<DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) dft5<DIR>(v);
    else if constexpr (R == 6) dft6<DIR>(v);
    else if constexpr (R == 8) dft8<DIR>(v);
    else if constexpr (R == 16) dft16<DIR>(v);
    else if constexpr (R == 32) dft32<DIR>(v);
    else dft_prime<R, DIR>(v, tw, q);
}

// ------------------------------------------------------------ one stage
// Position of element p of a line in shared memory: p + (p >> SK) (one
// padding slot every 2^SK elements, SK = 0: none), which spreads the
// power-of-two strides of the Stockham stages over the banks.
template <int SK> TG_HD constexpr int skew(int p) { return SK ? p + (p >> SK) : p; }

template <int L, int R, int NS, int DIR, int NL, int NT, int LS, typename C, int SK = 0>
TG_D void stage(C* s, const C* __restrict__ tw, int tid) {
    constexpr int NBL = L / R;
    constexpr int NB = NL * NBL;
    constexpr int BPT = (NB + NT - 1) / NT;
    C v[BPT][R];
#pragma unroll
    for (int q = 0; q < BPT; ++q) {
        const int b = tid + q * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = b / NBL, j = b - line * NBL;
            const C* src = s + line * LS;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = src[skew<SK>(j + r * NBL)];
            if (NS > 1) {
                const int k = j % NS;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    C w = ldtw(tw, r * k * (L / (NS * R)));
                    if (DIR > 0) w = cconj(w);
                    v[q][r] = cmul(v[q][r], w);
                }
            }
            dft<R, DIR>(v[q], tw, L / R);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < BPT; ++q) {
        const int b = tid + q * NT;
        if (NB % NT == 0 || b < NB) {
            const int line = b / NBL, j = b - line * NBL;
            const int k = j % NS;
            C* dst = s + line * LS;
            const int p0 = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[skew<SK>(p0 + r * NS)] = v[q][r];
        }
    }
    __syncthreads();
}

template <int L, int DIR, int NL, int NT, int LS, typename C, int SK, int NS, int R, int... Rest>
TG_D void run_stages(C* s, const C* __restrict__ tw, int tid) {
    stage<L, R, NS, DIR, NL, NT, LS, C, SK>(s, tw, tid);
    if constexpr (sizeof...(Rest) > 0) run_stages<L, DIR, NL, NT, LS, C, SK, NS * R, Rest...>(s, tw, tid);
}

template <int L, int DIR, int NL, int NT, int LS, typename C, int SK, int... Rs>
TG_D void smem_fft_impl(C* s, const C* __restrict__ tw, int tid, seq<Rs...>) {
    run_stages<L, DIR, NL, NT, LS, C, SK, 1, Rs...>(s, tw, tid);
}

// Transform NL lines in shared memory (line i at s + i LS, element p at
// skew<SK>(p) within it).  The caller must have synchronised after filling
// s; the routine ends with a barrier.
template <int L, int DIR, int NL, int NT, int LS, typename C, int SK = 0>
TG_D void smem_fft(C* s, const C* __restrict__ tw, int tid) {
    smem_fft_impl<L, DIR, NL, NT, LS, C, SK>(s, tw, tid, typename Radices<L>::type{});
}

}  // namespace tgfft
