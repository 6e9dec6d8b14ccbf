// Asynchronous copy of a c2r tile (the x line of YT consecutive y at one z,
// all NH1 half-spectrum columns kx) from global memory into shared memory
// rows tile[yl * TS + kx], with cp.async (8 bytes per element).
//
// Element e = tid + NTHR i of the tile is (kx, yl) = (e / YT, e % YT); with
// NTHR a multiple of YT a thread keeps yl = tid % YT and steps kx by
// NTHR / YT, so its copies are one base address plus compile-time offsets in
// shared memory and a fixed stride in global memory.
#pragma once
#include "common.cuh"

namespace tgtile {

TG_D void cp_async8(unsigned smem_dst, const void* gsrc, int bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_dst), "l"(gsrc), "r"(bytes) : "memory");
}
TG_D void commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> TG_D void wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int YT, int NH1, int NTHR>
struct TileCopy {
    static_assert(NTHR % YT == 0, "threads per block a multiple of the lines per tile");
    static constexpr int KS = NTHR / YT, NF = NH1 / KS, REM = NH1 % KS;
    unsigned dst;         // shared address of this thread's first element
    const float2* src;    // H at (kx0, z, y0 + yl) of rotation 0
    long long kx_stride;  // elements between consecutive kx (Nz Ny)
    long long rot_stride; // elements between rotations (NH1 Nz Ny)
    int bytes;            // 8, or 0 (zero fill) past the last y
    bool tail;            // this thread copies the element kx = NF KS + kx0 (kx0 < REM)

    // tile: the shared buffer of stage 0; TS: its row stride (float2)
    TG_D TileCopy(float2* tile, int TS, const float2* H, int tid, int y0, int z, int Ny, int Nz) {
        const int yl = tid % YT, kx0 = tid / YT;
        const bool ok = y0 + yl < Ny;
        kx_stride = (long long)Nz * Ny;
        rot_stride = (long long)NH1 * kx_stride;
        src = H + (long long)kx0 * kx_stride + (long long)z * Ny + (ok ? y0 + yl : 0);
        dst = (unsigned)__cvta_generic_to_shared(tile + yl * TS + kx0);
        bytes = ok ? 8 : 0;
        tail = REM > 0 && kx0 < REM;
    }

    // copy rotation b into the stage starting stage_bytes after stage 0
    TG_D void issue(int b, unsigned stage_bytes) const {
        const float2* s = src + (long long)b * rot_stride;
        const unsigned d = dst + stage_bytes;
#pragma unroll
        for (int i = 0; i < NF; ++i) cp_async8(d + i * KS * 8, s + (long long)i * KS * kx_stride, bytes);
        if (tail) cp_async8(d + NF * KS * 8, s + (long long)NF * KS * kx_stride, bytes);
        commit();
    }
};

}  // namespace tgtile
