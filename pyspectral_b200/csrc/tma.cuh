// Tensor-memory-accelerator (TMA) helpers for sm_100a: tiled 2D loads from global memory into
// shared memory completing on an mbarrier, and bulk L2 prefetches.  No multicast form is used:
// every load reads this GPU's own memory into this CTA's shared memory only.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "tcgen05.cuh"

namespace sp {
namespace tma {

// Make an mbarrier initialised by this thread visible to the async proxy (TMA completions).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once on the barrier and add `bytes` to the transaction count its phase waits for.
__device__ __forceinline__ void arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Box (x, y) of a 2D tensor map -> shared memory at `dst`; completes `bytes` on `bar`.
// x is in elements of the map's innermost dimension; x * element size must be a multiple of
// 16 bytes.
__device__ __forceinline__ void load_2d(void* dst, const void* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(tc::smem_u32(dst)),
        "l"((uint64_t)(uintptr_t)map), "r"(x), "r"(y), "r"(tc::smem_u32(bar))
        : "memory");
}

// `bytes` (a multiple of 16) of global memory at `src` -> shared memory at `dst` (both 16-byte
// aligned), completing on `bar`.
__device__ __forceinline__ void load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(tc::smem_u32(dst)), "l"((uint64_t)(uintptr_t)src), "r"(bytes),
        "r"(tc::smem_u32(bar))
        : "memory");
}

// Start moving `bytes` (a multiple of 16, 16-byte aligned source) of global memory into L2.
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((uint64_t)(uintptr_t)src),
                 "r"(bytes)
                 : "memory");
}

}  // namespace tma
}  // namespace sp
