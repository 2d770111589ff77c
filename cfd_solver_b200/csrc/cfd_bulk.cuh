// cfd_bulk.cuh -- bulk asynchronous global -> shared copies (the TMA engine's 1-D mode)
// completed on an mbarrier, with bounded waits.
//
// Rules kept here: source and destination 16-byte aligned, sizes a multiple of 16 bytes;
// no multicast (every copy reads this GPU's own memory into this CTA's shared memory);
// every wait gives up after a bounded number of polls and reports through a flag instead
// of spinning forever. A kernel whose wait gave up still waits, at the long default
// limit, for the copies it issued before its CTA leaves, so no copy lands in shared
// memory that another CTA owns.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfd {

constexpr unsigned kWaitPolls = 1u << 24;  // ~0.1-1 s of polling before a wait gives up (default)

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared-memory accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// plain arrival (no transaction bytes), release semantics at CTA scope
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
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

// 3-D tiled tensor load (box from a CUtensorMap in global memory) into shared memory;
// x must be a multiple of 16 bytes / element size (2 for float64), other coordinates free
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// bounded wait for phase `parity` of `bar`, at most `polls` polls (0: none, the wait gives
// up at once); false when it gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned polls = kWaitPolls) {
    for (unsigned n = 0; n < polls; n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace cfd
