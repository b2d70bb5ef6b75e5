// Closure network kernels on the tensor cores (tcgen05, BF16 operands, FP32 accumulation).
//
// This file holds the tile-level GEMM check (one 128 x N x K tile through shared memory, TMEM
// and back) used to validate descriptors and operand orientations against a reference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "spectral_b200.h"
#include "tcgen05.cuh"

namespace sp {
void set_thread_error(const char* why);  // spectral_b200.cu
}

using namespace sp;

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls before a wait gives up

// D[128 x N] = A[128 x K] * B[N x K]^T.  a_mn: A is given as [K][128] (read MN-major);
// b_mn: B is given as [K][N].  N in {16..256} multiple of 16, K multiple of 16, <= 256.
__global__ void __launch_bounds__(128) k_mma_tile_check(const __nv_bfloat16* __restrict__ A,
                                                        const __nv_bfloat16* __restrict__ B,
                                                        float* __restrict__ D, int N, int K,
                                                        int a_mn, int b_mn, int ncols,
                                                        int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    unsigned char* tA = smem;
    unsigned char* tB = smem + 128 * K * 2;
    const int t = threadIdx.x, warp = t >> 5;
    // stage A and B into the core layout
    for (int e = t; e < 128 * K; e += blockDim.x) {
        int r, c, C;
        if (!a_mn) { r = e / K; c = e % K; C = K; }    // A[m][k]: rows m, columns k
        else { r = e / 128; c = e % 128; C = 128; }    // A[k][m]: rows k, columns m
        *reinterpret_cast<__nv_bfloat16*>(tA + tc::core_offset(r, c, C)) = A[e];
    }
    for (int e = t; e < N * K; e += blockDim.x) {
        int r, c, C;
        if (!b_mn) { r = e / K; c = e % K; C = K; }
        else { r = e / N; c = e % N; C = N; }
        *reinterpret_cast<__nv_bfloat16*>(tB + tc::core_offset(r, c, C)) = B[e];
    }
    if (t == 0) {
        tc::mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tslot, (uint32_t)ncols);
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    if (t == 0) {
        const uint32_t a = tc::smem_u32(tA), b = tc::smem_u32(tB);
        const uint32_t idesc = tc::instr_desc_bf16(128, N, a_mn, b_mn);
        for (int s = 0; s < K / 16; ++s) {
            const uint64_t da = a_mn ? tc::desc_mnmajor(a, 128, s) : tc::desc_kmajor(a, K, s);
            const uint64_t db = b_mn ? tc::desc_mnmajor(b, N, s) : tc::desc_kmajor(b, K, s);
            tc::mma_bf16(tmem, da, db, idesc, s > 0);
        }
        tc::mma_commit(&bar);
    }
    // a warp reads TMEM only if all its lanes saw the MMAs complete (tcgen05.ld is warp-wide)
    const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&bar, 0, kWaitLimit));
    if (!ok && (t & 31) == 0) atomicExch(err, 1);
    tc::fence_after_sync();
    if (ok) {
        const int row = 32 * warp + (t & 31);
        for (int c = 0; c < N; c += 8) {
            float v[8];
            tc::tmem_ld8(tc::tmem_at(tmem, 32 * warp, c), v);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) D[row * N + c + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)ncols);
}

}  // namespace

extern "C" {

int sp_mma_tile_check(const void* A, const void* B, float* D, int N, int K, int a_mn, int b_mn,
                      void* stream) {
    if (!A || !B || !D || N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16) {
        sp::set_thread_error("sp_mma_tile_check: N, K multiples of 16 in 16..256");
        return SP_ERR_ARG;
    }
    int ncols = 32;
    while (ncols < N) ncols *= 2;
    int* err = nullptr;
    auto st = (cudaStream_t)stream;
    // the check is a test utility: a 4-byte flag is allocated per call
    if (cudaMallocAsync(&err, sizeof(int), st) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) {
        sp::set_thread_error("sp_mma_tile_check: flag allocation failed");
        return SP_ERR_CUDA;
    }
    const size_t smem = (size_t)(128 + N) * K * 2;
    cudaFuncSetAttribute(k_mma_tile_check, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mma_tile_check<<<1, 128, smem, st>>>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, D,
                                          N, K, a_mn, b_mn, ncols, err);
    cudaError_t e = cudaGetLastError();
    int host_err = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&host_err, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(err, st);
    if (e != cudaSuccess) {
        sp::set_thread_error(cudaGetErrorString(e));
        return SP_ERR_CUDA;
    }
    if (host_err) {
        sp::set_thread_error("sp_mma_tile_check: MMA completion wait timed out");
        return SP_ERR_CUDA;
    }
    return SP_OK;
}

}  // extern "C"
