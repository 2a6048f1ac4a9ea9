// ocfd_tma.cuh -- bulk tensor copies into shared memory (sm_100a): mbarrier
// helpers, the 4-D tile load and the host-side tensor-map encoder.  Every
// tensor map here covers this GPU's own memory, and no load multicasts
// across a cluster.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace ocfd {
namespace tma {

// polls of an mbarrier phase before a kernel gives up on a staged copy
// (each poll suspends the thread for a hardware-chosen time)
constexpr long long WAIT_LIMIT = 1LL << 22;

__device__ __forceinline__ unsigned smem_u32(const void *ptr) {
    return (unsigned)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of the given parity, at most WAIT_LIMIT polls
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    for (long long it = 0; it <= WAIT_LIMIT; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// one box of a 4-D tensor map into shared memory, completion counted on bar
__device__ __forceinline__ void load_4d(void *dst, const CUtensorMap *tm, int c0, int c1, int c2, int c3,
                                        unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<unsigned long long>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void prefetch_l1(const void *ptr) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(ptr));
}

}  // namespace tma

// A 4-D tiled tensor map (FP64 or FP32 elements, no swizzle, out-of-range
// elements read as zero): dims[0] innermost, strides in bytes of dims 1..3,
// box in elements.  Returns false when the driver entry point is missing or
// the layout breaks the copy engine's rules (16-byte aligned base and
// strides, inner box a multiple of 16 bytes).
bool encode_map_4d(const void *base, int elem_bytes, const unsigned long long dims[4],
                   const unsigned long long strides[3], const unsigned box[4], CUtensorMap *out);

}  // namespace ocfd
