// Run-time line-FFT plans (host side of fft_rt.cuh): which radices a length
// takes, or the Bluestein convolution length, and the device tables.
#pragma once
#include <cuda_runtime.h>

namespace tgrt {

constexpr int kMaxStages = 24;
// Dynamic shared memory a line kernel may ask for: 224 KB of the 227 KB a
// block may hold on sm_100a, leaving room for the kernels' static arrays.
constexpr int kMaxBlockSmem = 229376;

// A line transform: the radices of the stages over M (M = L for the
// mixed-radix form, the convolution length for Bluestein).
struct Plan {
    int L;
    int blue;
    int M;
    int nst;
    unsigned char r[kMaxStages];
};

template <typename C> struct Tabs {
    const C* tw;     // exp(-2 pi i m / M), m < M
    const C* chirp;  // Bluestein: exp(-i pi n^2 / L), n < L
    const C* bspec;  // Bluestein: FFT_M of the cyclic conj(chirp), times 1/M
};

// Line pitch (elements) of a plan's shared-memory lines: M + 1.
inline int pitch(const Plan& p) { return p.M + 1; }

}  // namespace tgrt

namespace tg {
// Plan for length L: the mixed-radix form when every prime factor of L is in
// {2, 3, 5, 7, 11, 13}, else Bluestein over the smallest {2,3,5,7}-smooth
// M >= 2L - 1.  False for L < 1 or when two lines of the plan's pitch with
// elements of elem_bytes do not fit one block's shared memory.
bool rt_plan(int L, int elem_bytes, tgrt::Plan* p);
// Device tables of a plan on the current device (built once per device and
// length, kept for the life of the process).  False on allocation failure.
template <typename C> bool rt_tabs(const tgrt::Plan& p, tgrt::Tabs<C>* t);
}  // namespace tg
