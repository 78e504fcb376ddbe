// Asynchronous copies into this CTA's shared memory that complete on an
// mbarrier: TMA tensor boxes (cp.async.bulk.tensor) from this GPU's own
// global memory, never with cluster multicast. Every wait is bounded: a copy that never completes
// ends in a false return (the caller flags the run), not in a hang.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace zfv {

// try_wait polls of an mbarrier before a wait gives up (each poll may block
// for a hardware-defined interval)
constexpr int kMaxBarrierPolls = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised barriers visible to the copy engine
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
    uint32_t ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait for the barrier's phase; false when the polls ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
    for (int it = 0; it < kMaxBarrierPolls; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}
// One 3-D box of a tensor map (x, y, plane) into shared memory, completing
// on `bar`. x must be a multiple of 4 floats (16 bytes).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace zfv
