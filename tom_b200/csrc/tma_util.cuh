// mbarrier and tiled-TMA helpers (sm_100a), and the host-side tensor-map
// encoder obtained from the driver at run time.  Loads here never multicast;
// the tensor maps the library builds cover the calling GPU's own buffers.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"

namespace tgtma {

TG_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

TG_D void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
TG_D void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
TG_D bool mbar_try_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
TG_D bool mbar_test_wait(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait on one phase; false when `limit` polls ran out
TG_D bool mbar_wait_bounded(unsigned bar, unsigned parity, long long limit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
TG_D void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
TG_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
TG_D void prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<unsigned long long>(map)) : "memory");
}
// tiled 4-D load of one box into shared memory, completing on bar
TG_D void load_4d(unsigned dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, unsigned bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

}  // namespace tgtma

namespace tg {
// cuTensorMapEncodeTiled from the driver (nullptr when it cannot be had).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();
// A 4-D FP32 tensor map over a half-spectrum batch H[b][kx][z][y] (float2
// elements viewed as float pairs): dims {2 Ny, Nz, nh1, nb}, box {2 yt, 1,
// rows, 1}, the given swizzle.  False when the driver refuses it.
bool encode_h_map(CUtensorMap* map, const void* H, int Ny, int Nz, int nh1, int nb, int yt, int rows,
                  CUtensorMapSwizzle swizzle);
}  // namespace tg
