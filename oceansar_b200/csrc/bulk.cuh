// mbarrier and one-dimensional bulk-copy primitives (CTA scope; the kernels that use them
// are launched without clusters, and every source is this GPU's own global memory).
#pragma once
#include "common.cuh"

namespace ocs {

constexpr unsigned kWaitLimit = 1u << 20;   // try_wait polls before a bounded wait gives up

OCS_D unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

OCS_D void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
OCS_D void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
OCS_D bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity; false if it did not complete.
OCS_D bool mbar_wait(unsigned long long *bar, unsigned parity) {
    for (unsigned n = 0; n < kWaitLimit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// Global -> shared bulk copy of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) completing on `bar`.
OCS_D void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
OCS_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

}  // namespace ocs

namespace ocs {

// Tiled tensor copies global -> shared (cp.async.bulk.tensor) completing on `bar`; `map` is
// the generic address of a CUtensorMap in parameter or global memory, (x, y[, z]) the
// box origin in elements (x times the element size a multiple of 16 bytes).  Boxes that
// reach past the tensor are filled with zeros and count their full size.
OCS_D void tma_load_2d(void *dst, const void *map, int x, int y, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
OCS_D void tma_load_3d(void *dst, const void *map, int x, int y, int z, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace ocs
