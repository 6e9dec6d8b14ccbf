// Warp-owned line FFTs with the data in registers (sm_100a, FP32).
//
// One warp holds one line of length L: lane `l` keeps EPT = L/32 complex
// values.  A stage of radix R runs EPT/R Stockham butterflies per lane
// (butterfly j = l + 32 q); its inputs sit at positions j + r L/R and its
// outputs go to (j - j mod NS) R + j mod NS + r NS.  Between stages the warp
// exchanges its line through a private shared-memory buffer (write outputs,
// __syncwarp, read next inputs), so a transform of S stages costs S-1
// exchanges and no block-wide barrier, and the first stage reads, and the last
// stage writes, registers directly.
//
// Register pattern: before the first stage v[q R1 + r] is x[l + 32 q + r L/R1];
// after the last stage v[q RL + r] is X[l + 32 q + r L/RL].  Plans with
// R1 == RL leave the spectrum in the same pattern the inverse transform
// starts from, so a product between a forward and an inverse transform needs
// no exchange.
//
// Bank conflicts: slot p of the exchange buffer lives at p ^ S(p >> 4) with S
// linear over GF(2) on the row bits (coefficients 15, 14, 10, 15, 13); this
// places every half-warp's 16 float2 accesses of every stage of the plans
// below in 16 distinct bank pairs (checked exhaustively on the host).
//
// Twiddles: every stage s > 1 (stride NS, radix R) has its own table
// T_s[r NS + k] = w_(NS R)^(r k) in shared memory, built once per block from
// the double-precision line table, so a lane reads the R-1 twiddles of its
// butterfly at consecutive k across the warp (no bank conflicts, no
// products).
#pragma once
#include "fft_engine.cuh"

namespace tgwfft {

using tgfft::seq;

template <int L> struct WPlan;
template <> struct WPlan<512> { typedef seq<8, 8, 8> type; static constexpr int R1 = 8, RL = 8; };
template <> struct WPlan<256> { typedef seq<8, 4, 8> type; static constexpr int R1 = 8, RL = 8; };
template <> struct WPlan<128> { typedef seq<4, 2, 4, 4> type; static constexpr int R1 = 4, RL = 4; };

__host__ __device__ constexpr int swz(int p) {
    return p ^ (((p >> 4) & 1 ? 15 : 0) ^ ((p >> 5) & 1 ? 14 : 0) ^ ((p >> 6) & 1 ? 10 : 0) ^
                ((p >> 7) & 1 ? 15 : 0) ^ ((p >> 8) & 1 ? 13 : 0));
}
// swz is linear over GF(2): for bit-disjoint a and c, swz(a + c) = swz(a) ^ swz(c).
// Exchange positions split into a per-lane part and a compile-time part with
// disjoint bits (power-of-two plans), so each access costs one XOR.

// w[r] = tw^(r m) (forward sign), conjugated for DIR > 0.  tw is a table of
// L entries, in shared memory in the hot kernels.
template <int R, int DIR>
TG_D void twiddle_powers(const float2* tw, int m, float2* w) {
    w[0] = make_float2(1.f, 0.f);
    if constexpr (R >= 2) w[1] = tw[m];
    if constexpr (R >= 4) {
        w[2] = tw[2 * m];
        w[3] = cmul(w[1], w[2]);
    }
    if constexpr (R >= 8) {
        w[4] = tw[4 * m];
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
    }
    if constexpr (R >= 16) {
        w[8] = tw[8 * m];
#pragma unroll
        for (int i = 9; i < 16; ++i) w[i] = cmul(w[8], w[i - 8]);
    }
    if constexpr (DIR > 0) {
#pragma unroll
        for (int i = 1; i < R; ++i) w[i] = cconj(w[i]);
    }
}

// Offset of stage s's table (stages numbered from 0; stage 0 needs none) and
// total size of the per-line stage tables of a plan.
template <int NS, int... Rs> struct TabSize;
template <int NS> struct TabSize<NS> { static constexpr int value = 0; };
template <int NS, int R, int... Rest> struct TabSize<NS, R, Rest...> {
    static constexpr int value = (NS > 1 ? NS * R : 0) + TabSize<NS * R, Rest...>::value;
};
template <int L, int... Rs> constexpr int tab_size(seq<Rs...>) { return TabSize<1, Rs...>::value; }
template <int L> struct WTab { static constexpr int size = tab_size<L>(typename WPlan<L>::type{}); };

// Build the stage tables of plan L from the line table tw (L entries), all threads of the block.
template <int L, int NS, int R, int... Rest>
TG_D void build_tabs_rec(float2* dst, const float2* __restrict__ tw) {
    if constexpr (NS > 1) {
        for (int i = threadIdx.x; i < NS * R; i += blockDim.x) {
            const int r = i / NS, k = i - r * NS;
            dst[i] = __ldg(tw + (k * r) * (L / (NS * R)));
        }
        dst += NS * R;
    }
    if constexpr (sizeof...(Rest) > 0) build_tabs_rec<L, NS * R, Rest...>(dst, tw);
}
template <int L, int... Rs> TG_D void build_tabs_impl(float2* dst, const float2* __restrict__ tw, seq<Rs...>) {
    build_tabs_rec<L, 1, Rs...>(dst, tw);
}
template <int L> TG_D void build_stage_tables(float2* dst, const float2* __restrict__ tw) {
    build_tabs_impl<L>(dst, tw, typename WPlan<L>::type{});
}

template <int L, int R, int NS, int DIR>
TG_D void wstage(float2* v, const float2* tab, int lane) {
    constexpr int EPT = L / 32, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        if constexpr (NS > 1) {
            const int k = (lane + 32 * q) % NS;
#pragma unroll
            for (int r = 1; r < R; ++r) {
                float2 w = tab[r * NS + k];
                if (DIR > 0) w = cconj(w);
                v[q * R + r] = cmul(v[q * R + r], w);
            }
        }
        tgfft::dft<R, DIR>(v + q * R, static_cast<const float2*>(nullptr), L / R);  // radices <= 16: no table
    }
}

// Copy a twiddle table into shared memory (all threads of the block).
TG_D void stage_table(float2* dst, const float2* __restrict__ src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

template <int L, int R, int NS>
TG_D void wstore(const float2* v, float2* buf, int lane) {
    constexpr int EPT = L / 32, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int j = lane + 32 * q, k = j % NS;
        const int a = swz((j - k) * R + k);  // bits below NS and from NS*R up
#pragma unroll
        for (int r = 0; r < R; ++r) buf[a ^ swz(r * NS)] = v[q * R + r];  // r*NS: the bits between
    }
}

template <int L, int R>
TG_D void wload(float2* v, const float2* buf, int lane) {
    constexpr int EPT = L / 32, NB = EPT / R;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int a = swz(lane + 32 * q);  // j < L/R
#pragma unroll
        for (int r = 0; r < R; ++r) v[q * R + r] = buf[a ^ swz(r * (L / R))];
    }
}

template <int L, int DIR, int NS, int R, int... Rest>
TG_D void wrun(float2* v, float2* buf, const float2* tab, int lane) {
    wstage<L, R, NS, DIR>(v, tab, lane);
    if constexpr (sizeof...(Rest) > 0) {
        constexpr int Rn = tgfft::seq_first<Rest...>::value;
        wstore<L, R, NS>(v, buf, lane);
        __syncwarp();
        wload<L, Rn>(v, buf, lane);
        __syncwarp();
        wrun<L, DIR, NS * R, Rest...>(v, buf, NS > 1 ? tab + NS * R : tab, lane);
    }
}

template <int L, int DIR, int... Rs>
TG_D void warp_fft_impl(float2* v, float2* buf, const float2* tw, int lane, seq<Rs...>) {
    wrun<L, DIR, 1, Rs...>(v, buf, tw, lane);
}

// In-register transform of one line per warp; buf: L float2 private to the
// warp; tabs: the plan's stage tables (build_stage_tables).
template <int L, int DIR>
TG_D void warp_fft(float2* v, float2* buf, const float2* tw, int lane) {
    warp_fft_impl<L, DIR>(v, buf, tw, lane, typename WPlan<L>::type{});
}

// Position of register i (0 <= i < L/32) before the first / after the last stage.
template <int L> TG_D int in_pos(int i, int lane) {
    constexpr int R = WPlan<L>::R1;
    return lane + 32 * (i / R) + (i % R) * (L / R);
}
template <int L> TG_D int out_pos(int i, int lane) {
    constexpr int R = WPlan<L>::RL;
    return lane + 32 * (i / R) + (i % R) * (L / R);
}

}  // namespace tgwfft
