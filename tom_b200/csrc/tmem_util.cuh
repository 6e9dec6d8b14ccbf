// Tensor-memory (TMEM) helpers (sm_100a): allocation and 32x32b loads and
// stores, with which a thread keeps per-lane constants in its own TMEM lane
// instead of shared memory.  A warp w reaches lanes 32 (w mod 4) .. + 31; a
// 32x32b access moves one lane per thread.
#pragma once
#include "common.cuh"

namespace tgtm {

// Allocate ncols columns (a power of two, 32..512) for the block; one warp
// calls it; the base address lands in *slot (shared memory).
template <int NCOLS> TG_D void alloc(unsigned* slot) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(slot)),
                 "n"(NCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
template <int NCOLS> TG_D void dealloc(unsigned base) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "n"(NCOLS));
}
TG_D void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
TG_D void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

TG_D void st16(unsigned taddr, const float (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};\n" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]),
        "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]));
}
TG_D void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// load 16 columns of this thread's lane and wait for them
TG_D void ld16(unsigned taddr, float (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
          "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
// TMEM address of this warp's lane quadrant (warp mod 4) at column col
TG_D unsigned lane_addr(unsigned base, int warp, unsigned col) {
    return base + ((unsigned)(32 * (warp & 3)) << 16) + col;
}

}  // namespace tgtm
