// Minimal sm_100a tensor-core toolkit: tcgen05 MMA (BF16 x BF16 -> FP32 in tensor memory),
// shared-memory matrix descriptors for the no-swizzle canonical layout, TMEM allocation and
// loads, mbarrier completion with bounded waits.
//
// Operand layout in shared memory ("core-matrix" layout, no swizzle): a tile of R rows x C
// columns of bf16 (C contiguous = the K direction for a K-major operand) is stored as 8 x 8
// blocks of 128 bytes, block (r/8, c/8) at ((r/8) * (C/8) + c/8) * 128, row r%8 of a block at
// 16 * (r%8), element c%8 at 2 * (c%8).  The same bytes read with an MN-major descriptor are the
// transposed tile (rows c, K = r): one buffer serves both orientations.
//
// Descriptor field layout (shared memory descriptor, 64 bit): start address >> 4 in bits
// 0..13, leading-dimension byte offset >> 4 in bits 16..29, stride-dimension byte offset >> 4
// in bits 32..45, version 1 in bits 46..47, layout type (0 = no swizzle) in bits 61..63.
// Instruction descriptor (32 bit): accumulator format (1 = F32) at bit 4, A and B formats
// (1 = BF16) at bits 7 and 10, A / B major (0 = K, 1 = MN) at bits 15 / 16, N >> 3 at bit 17,
// M >> 4 at bit 24.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace sp {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, c) in a core-matrix tile with C columns
__host__ __device__ __forceinline__ uint32_t core_offset(int r, int c, int C) {
    return (uint32_t)(((r >> 3) * (C >> 3) + (c >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, legacy LBO mode, no swizzle
}

// Descriptor of the K-slab [16 k, 16 k + 16) of a tile with R rows (the M or N operand rows)
// and C columns, stored in the core layout, used as a K-major operand (K = columns).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t tile, int C, int kstep) {
    // two 8-column core blocks per slab: LBO = 128 B between them; SBO = one row of blocks
    return smem_desc(tile + (uint32_t)(2 * kstep) * 128u, 128u, (uint32_t)(C / 8) * 128u);
}

// Descriptor of the K-slab [16 k, 16 k + 16) when the same tile (R rows x C columns) is read
// transposed: operand rows = tile columns, K = tile rows (MN-major).
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t tile, int C, int kstep) {
    // K runs over tile rows: 16 rows = 2 row-blocks, LBO = distance between row-blocks;
    // MN runs over tile columns in blocks of 8: SBO = 128 B between column blocks
    return smem_desc(tile + (uint32_t)(2 * kstep) * (uint32_t)(C / 8) * 128u,
                     (uint32_t)(C / 8) * 128u, 128u);
}

__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T, one 128 x N x 16 MMA issued by the calling thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                         uint32_t idesc, bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    const uint32_t z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

// Arrive on an mbarrier once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Wait for phase `parity` of the mbarrier; gives up after `limit` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_to_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// One warp allocates `ncols` (power of two >= 32) TMEM columns; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

// Eight consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32 (w%4) ..).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// Sixteen consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// TMEM address of (lane, column) relative to an allocation base
__device__ __forceinline__ uint32_t tmem_at(uint32_t base, uint32_t lane, uint32_t col) {
    return base + (lane << 16) + col;
}

}  // namespace tc
}  // namespace sp
