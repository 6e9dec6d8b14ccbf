// Half-warp-owned line FFTs with the data in registers (sm_100a, FP32).
//
// Sixteen lanes hold one line of length L (EPT = L/16 values per lane), so a
// warp carries two independent lines.  Longer per-lane vectors let a 512-point
// transform run as radix 16 x 32 and a 256-point one as 16 x 16: one exchange
// through shared memory per transform instead of two for the warp-owned
// layout, and one twiddle stage.  Stages follow the Stockham indexing of
// warp_fft.cuh with butterfly j = l + 16 q.
//
// Exchange slot p lives at p ^ ((p >> 4) & 15): each half-warp's 16 float2
// accesses of both plans fall in distinct bank pairs, and because the map is
// linear over GF(2) an address splits into a per-lane part and a
// compile-time part (one XOR per access).
#pragma once
#include "fft_engine.cuh"

namespace tghfft {

using tgfft::seq;

template <int L> struct HPlan;
template <> struct HPlan<512> { typedef seq<16, 32> type; static constexpr int R1 = 16, RL = 32; };
template <> struct HPlan<256> { typedef seq<16, 16> type; static constexpr int R1 = 16, RL = 16; };

__host__ __device__ constexpr int hswz(int p) { return p ^ ((p >> 4) & 15); }

// stage tables T_s[r NS + k] = w_(NS R)^(r k), stages after the first
template <int L, int NS, int R, int... Rest>
TG_D void htabs_rec(float2* dst, const float2* __restrict__ tw) {
    if constexpr (NS > 1) {
        for (int i = threadIdx.x; i < NS * R; i += blockDim.x) {
            const int r = i / NS, k = i - r * NS;
            dst[i] = __ldg(tw + (k * r) * (L / (NS * R)));
        }
        dst += NS * R;
    }
    if constexpr (sizeof...(Rest) > 0) htabs_rec<L, NS * R, Rest...>(dst, tw);
}
template <int L, int... Rs> TG_D void htabs_impl(float2* dst, const float2* __restrict__ tw, seq<Rs...>) {
    htabs_rec<L, 1, Rs...>(dst, tw);
}
template <int L> TG_D void build_stage_tables(float2* dst, const float2* __restrict__ tw) {
    htabs_impl<L>(dst, tw, typename HPlan<L>::type{});
}
template <int L> constexpr int tab_size() { return L; }  // both plans: one twiddle stage of NS*R = L

template <int L, int R, int NS, int DIR>
TG_D void hstage(float2* v, const float2* tab, int l) {
    constexpr int EPT = L / 16, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        if constexpr (NS > 1) {
            const int k = (l + 16 * q) % NS;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tab[r * NS + k];
                if (DIR > 0) w = cconj(w);
                v[q * R + r] = cmul(v[q * R + r], w);
            }
        }
        tgfft::dft<R, DIR>(v + q * R, static_cast<const float2*>(nullptr), L / R);
    }
}

template <int L, int R, int NS>
TG_D void hstore(const float2* v, float2* buf, int l) {
    constexpr int EPT = L / 16, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int j = l + 16 * q, k = j % NS;
        const int a = hswz((j - k) * R + k);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[a ^ hswz(r * NS)] = v[q * R + r];
    }
}

template <int L, int R>
TG_D void hload(float2* v, const float2* buf, int l) {
    constexpr int EPT = L / 16, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int a = hswz(l + 16 * q);
#pragma unroll
        for (int r = 0; r < R; ++r) v[q * R + r] = buf[a ^ hswz(r * (L / R))];
    }
}

template <int L, int DIR, int NS, int R, int... Rest>
TG_D void hrun(float2* v, float2* buf, const float2* tab, int l) {
    hstage<L, R, NS, DIR>(v, tab, l);
    if constexpr (sizeof...(Rest) > 0) {
        constexpr int Rn = tgfft::seq_first<Rest...>::value;
        hstore<L, R, NS>(v, buf, l);
        __syncwarp();
        hload<L, Rn>(v, buf, l);
        __syncwarp();
        hrun<L, DIR, NS * R, Rest...>(v, buf, NS > 1 ? tab + NS * R : tab, l);
    }
}
template <int L, int DIR, int... Rs>
TG_D void hfft_impl(float2* v, float2* buf, const float2* tab, int l, seq<Rs...>) {
    hrun<L, DIR, 1, Rs...>(v, buf, tab, l);
}
// One line per half-warp; buf: L float2 private to the line; l: lane within the line.
// Every lane of the warp must call (the exchanges use __syncwarp()).
template <int L, int DIR> TG_D void hfft(float2* v, float2* buf, const float2* tab, int l) {
    hfft_impl<L, DIR>(v, buf, tab, l, typename HPlan<L>::type{});
}

template <int L> TG_D int in_pos(int i, int l) {
    constexpr int R = HPlan<L>::R1;
    return l + 16 * (i / R) + (i % R) * (L / R);
}
template <int L> TG_D int out_pos(int i, int l) {
    constexpr int R = HPlan<L>::RL;
    return l + 16 * (i / R) + (i % R) * (L / R);
}
// Register of the forward output that holds the input position of register i
// of the next transform (a compile-time permutation).
template <int L> __host__ __device__ constexpr int out_index_of_in(int i) {
    constexpr int R1 = HPlan<L>::R1, RL = HPlan<L>::RL;
    // in position: l + 16 (i / R1) + (i % R1) (L / R1) = l + 16 m with
    // m = i / R1 + (i % R1) (L / R1) / 16; out register of l + 16 m: m = q + r L/(16 RL)
    const int m = i / R1 + (i % R1) * (L / R1) / 16;
    const int per = L / (16 * RL);  // out positions l + 16 (q + r * per)
    return (m % per) * RL + m / per;
}

}  // namespace tghfft
