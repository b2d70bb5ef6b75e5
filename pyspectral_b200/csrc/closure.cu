// Learned closure: training (forward + backward on the tensor cores), gradient reduction and
// Adam, inference fused with the coarse step's products, the filtered-DNS snapshot bank, and the
// spectral filter that defines the coarse field.
//
// Tensor-memory plan of the training kernel (512 columns, 128 lanes, fp32):
//   Z1 [0,64)  Z2 [64,128)  Z3/DH [128,208)  GW1 [208,288)  GW2 [288,368)  GW3 [368,448)
// Z* are the layer pre-activations (M = 128 points), DH the data gradient of a layer input
// (M = 128, N = 80), GW* the weight gradients (M = 64 outputs, N = 80 inputs) accumulated over
// every tile the CTA processes.  An M = 64 accumulator occupies lanes 0-15 of each 32-lane
// sub-partition: row m sits in lane (m % 16) + 32 (m / 16).
//
// Shared-memory operands use the no-swizzle core-matrix layout (tcgen05.cuh); a single buffer
// serves as a K-major operand in the forward pass and as an MN-major operand (its transpose) in
// the backward pass.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "closure.cuh"
#include "common.cuh"
#include "spectral_b200.h"
#include "tcgen05.cuh"

namespace sp {
void set_thread_error(const char* why);  // spectral_b200.cu
}

using namespace sp;
using namespace sp::cl;

namespace {

constexpr uint32_t kWait = 1u << 22;  // mbarrier polls before a wait gives up

// ------------------------------------------------------------------------ device helpers
// GELU, tanh form (Hendrycks and Gimpel): 0.5 z (1 + tanh u) with u = c0 (z + c1 z^3), written
// as z s with the logistic factor s = (1 + tanh u) / 2 = 1 / (1 + exp(-2u)); its derivative is
// s + 2 z s (1 - s) c0 (1 + 3 c1 z^2).
constexpr float kGc0 = 0.7978845608028654f, kGc1 = 0.044715f;
__device__ __forceinline__ float gelu_s(float z) {
    // the exponent is capped so that 1 + exp stays finite (s is 0 to fp32 precision there)
    const float a = fminf(-2.f * kGc0 * z * (1.f + kGc1 * z * z), 80.f);
    return __fdividef(1.f, 1.f + __expf(a));
}
__device__ __forceinline__ float gelu(float z) { return z * gelu_s(z); }
__device__ __forceinline__ float gelu_d(float z, float& g) {
    const float s = gelu_s(z);
    g = z * s;
    return s + 2.f * z * s * (1.f - s) * kGc0 * (1.f + 3.f * kGc1 * z * z);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a in the low half = lower column
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ void st_row8(unsigned char* tile, int r, int c, int C, const float* v) {
    uint4 q;
    q.x = pack_bf16(v[0], v[1]);
    q.y = pack_bf16(v[2], v[3]);
    q.z = pack_bf16(v[4], v[5]);
    q.w = pack_bf16(v[6], v[7]);
    *reinterpret_cast<uint4*>(tile + tc::core_offset(r, c, C)) = q;
}

// Shared-memory writes and TMEM reads of all threads are complete and visible to the tensor
// core before thread 0 issues the next MMAs.
__device__ __forceinline__ void sync_for_mma() {
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
}

// Waits for the MMAs committed to `bar`; the CTA agrees on the outcome.
__device__ __forceinline__ bool wait_mma(uint64_t* bar, uint32_t& phase) {
    const bool ok = tc::mbar_wait(bar, phase, kWait);
    phase ^= 1u;
    const bool all = __syncthreads_and(ok) != 0;
    tc::fence_after_sync();
    return all;
}

// D (+)= A * B^T over `ksteps` K-slabs of 16; operands in core layout with a_C / b_C columns.
__device__ __forceinline__ void issue(uint32_t d, uint32_t a, int a_mn, int a_C, uint32_t b,
                                      int b_mn, int b_C, int M, int N, int ksteps, bool acc) {
    const uint32_t idesc = tc::instr_desc_bf16(M, N, a_mn, b_mn);
    for (int s = 0; s < ksteps; ++s) {
        const uint64_t da = a_mn ? tc::desc_mnmajor(a, a_C, s) : tc::desc_kmajor(a, a_C, s);
        const uint64_t db = b_mn ? tc::desc_mnmajor(b, b_C, s) : tc::desc_kmajor(b, b_C, s);
        tc::mma_bf16(d, da, db, idesc, acc || s > 0);
    }
}

// Stages the 3 x 5 x 132 stencil rows of one tile (periodic wrap, n a power of two), scaled.
// A tile's stencil in two halves: stencil_load issues all of a thread's loads into registers
// (one memory latency per tile, and none at all when they are issued a tile ahead);
// stencil_store scales them into shared memory.
template <int THREADS>
constexpr int stencil_per_thread() { return (kStencil + THREADS - 1) / THREADS; }

template <int THREADS>
__device__ __forceinline__ void stencil_load(float (&v)[stencil_per_thread<THREADS>()],
                                             const float* f0, size_t fstride, int rstride, int n,
                                             int row, int y0) {
#pragma unroll
    for (int i = 0; i < stencil_per_thread<THREADS>(); ++i) {
        const int e = threadIdx.x + i * THREADS;
        if (e < kStencil) {
            const int f = e / (5 * kSpan);
            const int r = (e / kSpan) % 5;
            const int c = e % kSpan;
            const int xr = (row + r - kHalo) & (n - 1);
            const int yc = (y0 + c - kHalo) & (n - 1);
            v[i] = f0[(size_t)f * fstride + (size_t)xr * rstride + yc];
        }
    }
}

template <int THREADS>
__device__ __forceinline__ void stencil_store(float* sSt,
                                              const float (&v)[stencil_per_thread<THREADS>()],
                                              const Consts& cc) {
#pragma unroll
    for (int i = 0; i < stencil_per_thread<THREADS>(); ++i) {
        const int e = threadIdx.x + i * THREADS;
        if (e < kStencil) {
            const int f = e / (5 * kSpan);
            const float sc = f == 0 ? cc.inscale[0] : (f == 1 ? cc.inscale[1] : cc.inscale[2]);
            sSt[e] = v[i] * sc;
        }
    }
}

// Inference staging: the scaled stencil rounded to bf16 once (the value X receives).
template <int THREADS>
__device__ __forceinline__ void stage_stencil_bf16(__nv_bfloat16* sSt, const float* f0,
                                                   size_t fstride, int rstride, int n, int row,
                                                   int y0, const Consts& cc) {
    constexpr int kPer = (kStencil + THREADS - 1) / THREADS;
    float v[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {  // all loads first
        const int e = threadIdx.x + i * THREADS;
        if (e < kStencil) {
            const int f = e / (5 * kSpan);
            const int r = (e / kSpan) % 5;
            const int c = e % kSpan;
            const int xr = (row + r - kHalo) & (n - 1);
            const int yc = (y0 + c - kHalo) & (n - 1);
            v[i] = f0[(size_t)f * fstride + (size_t)xr * rstride + yc];
        }
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int e = threadIdx.x + i * THREADS;
        if (e < kStencil) {
            const int f = e / (5 * kSpan);
            const float sc = f == 0 ? cc.inscale[0] : (f == 1 ? cc.inscale[1] : cc.inscale[2]);
            sSt[e] = __float2bfloat16_rn(v[i] * sc);
        }
    }
}

template <int G0, int G1>
__device__ __forceinline__ void build_x_bf16(unsigned char* sX, const __nv_bfloat16* sSt, int p) {
    const unsigned short* src = reinterpret_cast<const unsigned short*>(sSt);
#pragma unroll
    for (int g = G0; g < G1; ++g) {
        uint32_t h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int f = 8 * g + i;
            if (f < kIn) {
                const int fld = f / 25, rr = (f % 25) / 5, cc = f % 5;
                h[i] = src[fld * 5 * kSpan + rr * kSpan + p + cc];
            } else {
                h[i] = f == kBiasIn ? 0x3F80u : 0u;  // bf16 1.0
            }
        }
        uint4 q;
        q.x = h[0] | (h[1] << 16);
        q.y = h[2] | (h[3] << 16);
        q.z = h[4] | (h[5] << 16);
        q.w = h[6] | (h[7] << 16);
        *reinterpret_cast<uint4*>(sX + tc::core_offset(p, 8 * g, kK)) = q;
    }
}

// Feature groups [G0, G1) (8 inputs each: 75 stencil values, the constant one, zero padding) of
// point p into the X tile.
template <int G0 = 0, int G1 = kK / 8>
__device__ __forceinline__ void build_x(unsigned char* sX, const float* sSt, int p) {
#pragma unroll
    for (int g = G0; g < G1; ++g) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int f = 8 * g + i;
            if (f < kIn) {
                const int fld = f / 25, rr = (f % 25) / 5, cc = f % 5;
                v[i] = sSt[fld * 5 * kSpan + rr * kSpan + p + cc];
            } else {
                v[i] = f == kBiasIn ? 1.f : 0.f;
            }
        }
        st_row8(sX, p, 8 * g, kK, v);
    }
}

// Hidden tiles carry the constant-one column 64 and zero columns 65..79.
__device__ __forceinline__ void init_hidden_bias(unsigned char* sHt, int p) {
    float v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = 0.f;
    v[0] = 1.f;
    st_row8(sHt, p, 64, kK, v);
    v[0] = 0.f;
    st_row8(sHt, p, 72, kK, v);
}

// Element index, in the bf16 weight copy, of parameter j < 3 * 5120: the three [64][80]
// matrices are kept in the core-matrix layout their shared-memory operand tiles use, so that
// staging them is a contiguous copy.
__host__ __device__ __forceinline__ int wb_index(int j) {
    const int l = j / kWsz, e = j % kWsz;
    return l * kWsz + (int)(tc::core_offset(e / kK, e % kK, kK) / 2);
}

// Copies the three bf16 weight tiles (already in core layout) into shared memory; every
// thread's loads are issued before its stores.
template <int THREADS>
__device__ __forceinline__ void stage_weights(unsigned char* sW, const __nv_bfloat16* wb) {
    constexpr int kQ = kLayers * kWsz / 8;  // 16-byte chunks
    constexpr int kPer = (kQ + THREADS - 1) / THREADS;
    const uint4* src = reinterpret_cast<const uint4*>(wb);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    uint4 v[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = threadIdx.x + i * THREADS;
        if (q < kQ) v[i] = src[q];
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        const int q = threadIdx.x + i * THREADS;
        if (q < kQ) dst[q] = v[i];
    }
}

// Forward epilogue of a hidden layer: row p of Z (64 columns) -> GELU -> bf16 hidden tile.
__device__ __forceinline__ void epi_forward(uint32_t tbase, uint32_t zcol, unsigned char* sHt,
                                            int p, int warp) {
#pragma unroll 1
    for (int c = 0; c < kH; c += 8) {
        float z[8];
        tc::tmem_ld8(tc::tmem_at(tbase, 32 * warp, zcol + c), z);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 8; ++i) z[i] = gelu(z[i]);
        st_row8(sHt, p, c, kK, z);
    }
}

// Sum over a warp of 8 values per lane; lanes with (lane & 3) == 0 return the sum of column
// 4 b4 + 2 b3 + b2 (b_k = bit k of the lane) in v[0].
__device__ __forceinline__ int warp_sum8(float (&v)[8], int lane) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const bool hi = lane & 16;
        const float send = hi ? v[i] : v[i + 4], keep = hi ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const bool hi = lane & 8;
        const float send = hi ? v[i] : v[i + 2], keep = hi ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    {
        const bool hi = lane & 4;
        const float send = hi ? v[0] : v[1], keep = hi ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 2);
    v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
    return ((lane >> 4) & 1) * 4 + ((lane >> 3) & 1) * 2 + ((lane >> 2) & 1);
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------------ training kernel
struct TrainSmem {
    static constexpr int W = 0;                                  // 3 x [64 x 80] bf16
    static constexpr int X = W + kLayers * kWsz * 2;             // [128 x 80]
    static constexpr int H1 = X + kTile * kK * 2;                // [128 x 80]
    static constexpr int H2 = H1 + kTile * kK * 2;               // [128 x 80]
    static constexpr int DZ = H2 + kTile * kK * 2;               // [128 x 64]
    static constexpr int ST = DZ + kTile * kH * 2;               // stencil floats
    static constexpr int W4 = ST + kStencil * 4;                 // w4 fp32 [80]
    static constexpr int DW4 = W4 + kK * 4;                      // dw4 partials fp32 [4][80]
    static constexpr int BYTES = DW4 + 4 * kK * 4;
};
static_assert(TrainSmem::W4 % 16 == 0, "alignment");
// A CTA's row of the partials buffer: the 15440 gradient sums, then its loss sum.
constexpr int kPartStride = kNParam + 16;

constexpr uint32_t kZ1 = 0, kZ2 = 64, kZ3 = 128, kDH = 128, kGW1 = 208, kGW2 = 288, kGW3 = 368;
constexpr uint32_t kTrainCols = 512;

// One CTA per SM; each CTA runs forward + backward over its share of the batch's tiles and
// writes its summed gradient to partials[blockIdx.x][15440].
__global__ void __launch_bounds__(128, 1)
    k_train(const float* __restrict__ bank, int n, int count, const __nv_bfloat16* __restrict__ wb,
            const float* __restrict__ params, const Consts* __restrict__ ccp,
            const int* __restrict__ step_dev, int64_t step_override, uint64_t seed, int ntiles,
            float inv_batch, float* __restrict__ partials, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    __shared__ float sLoss[4];
    unsigned char* sW = smem + TrainSmem::W;
    unsigned char* sX = smem + TrainSmem::X;
    unsigned char* sH1 = smem + TrainSmem::H1;
    unsigned char* sH2 = smem + TrainSmem::H2;
    unsigned char* sDZ = smem + TrainSmem::DZ;
    float* sSt = reinterpret_cast<float*>(smem + TrainSmem::ST);
    float* sW4 = reinterpret_cast<float*>(smem + TrainSmem::W4);
    float* sDW4 = reinterpret_cast<float*>(smem + TrainSmem::DW4);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const Consts cc = *ccp;
    const int64_t step = step_override >= 0 ? step_override : (int64_t)*step_dev;

    // the stencil and target of the CTA's next tile are loaded while the current one computes
    // (the first tile's while the weights are staged)
    float nxt[stencil_per_thread<128>()];
    float nxt_target = 0.f;
    auto load_tile = [&](int tl) {
        const TilePick pk = pick_tile(seed, step, tl, count, n);
        const int y0 = pk.seg * kTile;
        const float* snap = bank + (size_t)pk.snap * 4 * n * n;
        nxt_target = snap[3 * (size_t)n * n + (size_t)pk.row * n + y0 + t];
        stencil_load<128>(nxt, snap, (size_t)n * n, n, n, pk.row, y0);
    };
    if (blockIdx.x < ntiles) load_tile(blockIdx.x);
    stage_weights<128>(sW, wb);
    if (t < kK) sW4[t] = params[kLayers * kWsz + t];
    for (int i = t; i < 4 * kK; i += blockDim.x) sDW4[i] = 0.f;  // one row per warp
    init_hidden_bias(sH1, t);
    init_hidden_bias(sH2, t);
    if (t == 0) {
        tc::mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tslot, kTrainCols);
    sync_for_mma();
    const uint32_t tb = tslot;
    const uint32_t aX = tc::smem_u32(sX), aH1 = tc::smem_u32(sH1), aH2 = tc::smem_u32(sH2);
    const uint32_t aDZ = tc::smem_u32(sDZ), aW = tc::smem_u32(sW);
    const uint32_t aW1 = aW, aW2 = aW + kWsz * 2, aW3 = aW + 2 * kWsz * 2;

    uint32_t phase = 0;
    bool ok = true, first = true;
    float loss = 0.f;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        stencil_store<128>(sSt, nxt, cc);
        const float target = nxt_target * cc.inv_outscale;
        if (tile + (int)gridDim.x < ntiles) load_tile(tile + gridDim.x);
        __syncthreads();
        build_x(sX, sSt, t);

        // ---- forward: three tensor-core layers
        sync_for_mma();
        if (t == 0) {
            issue(tb + kZ1, aX, 0, kK, aW1, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        epi_forward(tb, kZ1, sH1, t, warp);
        sync_for_mma();
        if (t == 0) {
            issue(tb + kZ2, aH1, 0, kK, aW2, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        epi_forward(tb, kZ2, sH2, t, warp);
        sync_for_mma();
        if (t == 0) {
            issue(tb + kZ3, aH2, 0, kK, aW3, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;

        // ---- output layer, loss, and the layer-3 gradient
        float y = sW4[kBiasH];
#pragma unroll 1
        for (int c = 0; c < kH; c += 8) {
            float z[8];
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kZ3 + c), z);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) y += gelu(z[i]) * sW4[c + i];
        }
        const float r = y - target;
        const float dy = 2.f * r * inv_batch;
        loss += r * r;
#pragma unroll 1
        for (int c = 0; c < kH; c += 8) {
            float z[8], dz[8];
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kZ3 + c), z);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float h;
                const float d = gelu_d(z[i], h);
                dz[i] = dy * sW4[c + i] * d;
                z[i] = dy * h;  // output-layer weight gradient contribution
            }
            st_row8(sDZ, t, c, kH, dz);
            const int col = warp_sum8(z, lane);
            // lanes 0, 4, .., 28 hold distinct columns: this warp's row, no atomics
            if ((lane & 3) == 0) sDW4[warp * kK + c + col] += z[0];
        }
        {
            const float sdy = warp_sum(dy);
            if (lane == 0) sDW4[warp * kK + kBiasH] += sdy;
        }

        // ---- backward through layers 3, 2, 1
        sync_for_mma();
        if (t == 0) {
            issue(tb + kGW3, aDZ, 1, kH, aH2, 1, kK, 64, kK, kTile / 16, !first);
            issue(tb + kDH, aDZ, 0, kH, aW3, 1, kK, 128, kK, kH / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
#pragma unroll 1
        for (int c = 0; c < kH; c += 8) {
            float dh[8], z[8];
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kDH + c), dh);
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kZ2 + c), z);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float h;
                dh[i] *= gelu_d(z[i], h);
            }
            st_row8(sDZ, t, c, kH, dh);
        }
        sync_for_mma();
        if (t == 0) {
            issue(tb + kGW2, aDZ, 1, kH, aH1, 1, kK, 64, kK, kTile / 16, !first);
            issue(tb + kDH, aDZ, 0, kH, aW2, 1, kK, 128, kK, kH / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
#pragma unroll 1
        for (int c = 0; c < kH; c += 8) {
            float dh[8], z[8];
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kDH + c), dh);
            tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, kZ1 + c), z);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float h;
                dh[i] *= gelu_d(z[i], h);
            }
            st_row8(sDZ, t, c, kH, dh);
        }
        sync_for_mma();
        if (t == 0) {
            issue(tb + kGW1, aDZ, 1, kH, aX, 1, kK, 64, kK, kTile / 16, !first);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        first = false;
    }

    if (ok) {
        float* out = partials + (size_t)blockIdx.x * kPartStride;
        const uint32_t gw[3] = {kGW1, kGW2, kGW3};
        for (int l = 0; l < kLayers; ++l) {
#pragma unroll 1
            for (int c = 0; c < kK; c += 8) {
                float v[8];
                tc::tmem_ld8(tc::tmem_at(tb, 32 * warp, gw[l] + c), v);
                tc::tmem_wait_ld();
                if (lane < 16) {
                    float* dst = out + l * kWsz + (16 * warp + lane) * kK + c;
#pragma unroll
                    for (int i = 0; i < 8; ++i) dst[i] = v[i];
                }
            }
        }
        loss = warp_sum(loss);
        if (lane == 0) sLoss[warp] = loss;
        __syncthreads();
        // fixed summation orders throughout: the gradient and loss are bit-reproducible
        if (t < kK) out[kLayers * kWsz + t] = ((sDW4[t] + sDW4[kK + t]) + sDW4[2 * kK + t]) +
                                              sDW4[3 * kK + t];
        if (t == 0) out[kNParam] = (((sLoss[0] + sLoss[1]) + sLoss[2]) + sLoss[3]) * inv_batch;
    } else if (t == 0) {
        atomicExch(err, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tb, kTrainCols);
}

// ------------------------------------------------------------------------ optimiser
struct AdamCfg {
    float lr, lr_min, b1, b2, eps;
    int total, warmup;
};

// Sums the CTAs' partial rows in order; thread kNParam also records the step's loss and (when
// `advance`) moves the step counter on — one thread reads and writes it.
__global__ void k_grad_reduce(const float* __restrict__ partials, int nblk, float* __restrict__ grad,
                              int* __restrict__ step_dev, int64_t step_override,
                              float* __restrict__ loss_ring, int advance) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > kNParam) return;
    float s = 0.f;
    for (int b = 0; b < nblk; ++b) s += partials[(size_t)b * kPartStride + j];
    if (j < kNParam) {
        grad[j] = s;
        return;
    }
    const int64_t step = step_override >= 0 ? step_override : (int64_t)*step_dev;
    loss_ring[step & (kLossRing - 1)] = s;
    if (advance) *step_dev = (int)step + 1;
}

// Adam (Kingma and Ba) with a linear warm-up and cosine decay of the learning rate; step_dev
// holds the 1-based step number of this update.
__global__ void k_adam(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, __nv_bfloat16* __restrict__ wb,
                       const int* __restrict__ step_dev, AdamCfg cfg) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kNParam) return;
    const int t = *step_dev;
    float lr;
    if (cfg.warmup > 0 && t <= cfg.warmup) {
        lr = cfg.lr * (float)t / (float)cfg.warmup;
    } else {
        const float span = (float)(cfg.total > cfg.warmup ? cfg.total - cfg.warmup : 1);
        const float x = fminf((float)(t - cfg.warmup) / span, 1.f);
        lr = cfg.lr_min + 0.5f * (cfg.lr - cfg.lr_min) * (1.f + cospif(x));
    }
    const float g = grad[j];
    const float mj = cfg.b1 * m[j] + (1.f - cfg.b1) * g;
    const float vj = cfg.b2 * v[j] + (1.f - cfg.b2) * g * g;
    m[j] = mj;
    v[j] = vj;
    const float mh = mj / (1.f - powf(cfg.b1, (float)t));
    const float vh = vj / (1.f - powf(cfg.b2, (float)t));
    const float p = params[j] - lr * mh / (sqrtf(vh) + cfg.eps);
    params[j] = p;
    if (j < kLayers * kWsz) wb[wb_index(j)] = __float2bfloat16_rn(p);
}

__global__ void k_to_bf16(const float* __restrict__ params, __nv_bfloat16* __restrict__ wb) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < kLayers * kWsz) wb[wb_index(j)] = __float2bfloat16_rn(params[j]);
}

// ------------------------------------------------------------------------ inference kernel
// Eight warps per CTA: warps w and w + 4 serve the TMEM lanes (points) 32 (w % 4) .. + 31 and
// split the 64 hidden columns in halves; X and the hidden activations share one operand buffer
// (each layer's epilogue runs after the MMA that read the buffer has completed), so three CTAs
// fit on an SM.
struct InferSmem {
    static constexpr int W = 0;                                  // 3 x [64 x 80] bf16
    static constexpr int A = W + kLayers * kWsz * 2;             // X, then H1, H2 [128 x 80]
    static constexpr int ST = A + kTile * kK * 2;                // stencil, bf16
    static constexpr int W4 = ST + ((kStencil * 2 + 15) / 16) * 16;  // w4 fp32 [80]
    static constexpr int YP = W4 + kK * 4;                       // upper-half output partials
    static constexpr int BYTES = YP + kTile * 4;
};
constexpr uint32_t kInferCols = 64;
// four CTAs per SM: one wave of 128-point tiles covers 256^2 on 148 SMs
constexpr int kInferThreads = 256, kInferCtasPerSm = 4;

// Hidden epilogue of one column half: 32 columns of row p -> GELU -> bf16 operand buffer.
__device__ __forceinline__ void epi_half(uint32_t tb, int quad, int ch, unsigned char* sA, int p) {
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        float z[16];
        tc::tmem_ld16(tc::tmem_at(tb, 32 * quad, 32 * ch + 16 * h), z);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) z[i] = gelu(z[i]);
        st_row8(sA, p, 32 * ch + 16 * h, kK, z);
        st_row8(sA, p, 32 * ch + 16 * h + 8, kK, z + 8);
    }
}

// Closure term at every point of an n x n field, one 128-point row segment per tile.
// fields: omega, d omega/dx, d omega/dy at f0 + k * fstride (row stride rstride); out gets
// outscale * network (row stride out_rstride).  With uv set, the Basdevant products of the
// velocity pair at uv, uv + uv_stride (same row stride) are formed in place as well.
__global__ void __launch_bounds__(kInferThreads, kInferCtasPerSm)
    k_infer(const float* __restrict__ f0, size_t fstride, int rstride, int n,
            const __nv_bfloat16* __restrict__ wb, const float* __restrict__ params,
            const Consts* __restrict__ ccp, float* __restrict__ out, int out_rstride,
            float* __restrict__ uv, size_t uv_stride, int* __restrict__ err) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tslot;
    unsigned char* sW = smem + InferSmem::W;
    unsigned char* sA = smem + InferSmem::A;
    __nv_bfloat16* sSt = reinterpret_cast<__nv_bfloat16*>(smem + InferSmem::ST);
    float* sW4 = reinterpret_cast<float*>(smem + InferSmem::W4);
    float* sYP = reinterpret_cast<float*>(smem + InferSmem::YP);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int quad = warp & 3, ch = warp >> 2;  // TMEM lane quadrant, hidden column half
    const int p = 32 * quad + lane;             // this thread's point in the tile
    const Consts cc = *ccp;

    stage_weights<kInferThreads>(sW, wb);
    if (t < kK) sW4[t] = params[kLayers * kWsz + t];
    if (t == 0) {
        tc::mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tslot, kInferCols);
    sync_for_mma();
    const uint32_t tb = tslot;
    const uint32_t aA = tc::smem_u32(sA), aW = tc::smem_u32(sW);

    uint32_t phase = 0;
    bool ok = true;
    const int segs = n / kTile;
    const int ntiles = n * segs;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int row = tile / segs, y0 = (tile % segs) * kTile;
        stage_stencil_bf16<kInferThreads>(sSt, f0, fstride, rstride, n, row, y0, cc);
        if (uv && ch == 0) {
            float* pu = uv + (size_t)row * rstride + y0 + p;
            const float u = pu[0], v = pu[uv_stride];
            pu[0] = (v - u) * (v + u);
            pu[uv_stride] = u * v;
        }
        __syncthreads();
        if (ch == 0) build_x_bf16<0, kK / 16>(sA, sSt, p);
        else build_x_bf16<kK / 16, kK / 8>(sA, sSt, p);
        sync_for_mma();
        if (t == 0) {
            issue(tb, aA, 0, kK, aW, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        epi_half(tb, quad, ch, sA, p);
        if (ch == 1) init_hidden_bias(sA, p);  // X's inputs 64..79 become the bias column
        sync_for_mma();
        if (t == 0) {
            issue(tb, aA, 0, kK, aW + kWsz * 2, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        epi_half(tb, quad, ch, sA, p);
        sync_for_mma();
        if (t == 0) {
            issue(tb, aA, 0, kK, aW + 2 * kWsz * 2, 0, kK, 128, kH, kK / 16, false);
            tc::mma_commit(&bar);
        }
        if (!(ok = wait_mma(&bar, phase))) break;
        float y = 0.f;
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            float z[16];
            tc::tmem_ld16(tc::tmem_at(tb, 32 * quad, 32 * ch + 16 * h), z);
            tc::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) y += gelu(z[i]) * sW4[32 * ch + 16 * h + i];
        }
        if (ch == 1) sYP[p] = y;
        __syncthreads();
        if (ch == 0) {
            float S = cc.outscale * (sW4[kBiasH] + y + sYP[p]);
            if (cc.clip) {
                const float w = f0[(size_t)row * rstride + y0 + p];
                if (S * w > 0.f) S = 0.f;
            }
            out[(size_t)row * out_rstride + y0 + p] = S;
        }
        // the next tile's MMA and partials must not overtake this tile's TMEM and sYP reads
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    if (!ok && t == 0) atomicExch(err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tb, kInferCols);
}

// ------------------------------------------------------------------------ spectral helpers
__device__ __forceinline__ int sgn_k(int i, int n) { return i <= n / 2 ? i : i - n; }

// pad_spectrum (validation.py:24-35): keep |k| < min(n_src, n_dst) / 2 on the full axes and
// k < that on the half axis, rescale by (n_dst / n_src)^dim; optionally apply the destination's
// 2/3 dealiasing mask as well.
template <typename T>
__global__ void k_filter(const cplx<T>* __restrict__ src, int ns, cplx<T>* __restrict__ dst,
                         int nd, int dim, int dealias, T scale, uint64_t total) {
    const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int nhd = nd / 2 + 1, nhs = ns / 2 + 1;
    const int m = (ns < nd ? ns : nd) / 2;
    const int j = (int)(idx % (uint64_t)nhd);
    uint64_t rest = idx / (uint64_t)nhd;
    int k1 = 0, k0;
    if (dim == 3) {
        k1 = sgn_k((int)(rest % (uint64_t)nd), nd);
        rest /= (uint64_t)nd;
    }
    k0 = sgn_k((int)rest, nd);
    const int a0 = k0 < 0 ? -k0 : k0, a1 = k1 < 0 ? -k1 : k1;
    bool keep = j < m && a0 < m && a1 < m;
    if (dealias) keep = keep && 3 * j < nd && 3 * a0 < nd && 3 * a1 < nd;
    cplx<T> v;
    v.x = 0;
    v.y = 0;
    if (keep) {
        const int i0 = (k0 + ns) % ns;
        uint64_t s;
        if (dim == 3) {
            const int i1 = (k1 + ns) % ns;
            s = ((uint64_t)i0 * ns + i1) * nhs + j;
        } else {
            s = (uint64_t)i0 * nhs + j;
        }
        v = src[s];
        v.x *= scale;
        v.y *= scale;
    }
    dst[idx] = v;
}

// Spectral inputs of one bank entry: omega, i kx omega, i ky omega and the subgrid term
// (filtered fine nonlinear term - coarse nonlinear term), dealiased and scaled by 1/n^2.
__global__ void k_snap_spec(const cplx<float>* __restrict__ w, const cplx<float>* __restrict__ fN,
                            const cplx<float>* __restrict__ cN, cplx<float>* __restrict__ spec,
                            int n, uint32_t fsc) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= fsc) return;
    const int nh = n / 2 + 1;
    const int i = (int)(idx / (uint32_t)nh), j = (int)(idx % (uint32_t)nh);
    const int kx = sgn_k(i, n);
    const bool keep = 3 * (kx < 0 ? -kx : kx) < n && 3 * j < n;
    const float sc = keep ? 1.f / ((float)n * (float)n) : 0.f;
    const cplx<float> a = w[idx];
    cplx<float> o;
    o.x = sc * a.x;
    o.y = sc * a.y;
    spec[idx] = o;
    o.x = -sc * (float)kx * a.y;
    o.y = sc * (float)kx * a.x;
    spec[fsc + idx] = o;
    o.x = -sc * (float)j * a.y;
    o.y = sc * (float)j * a.x;
    spec[2 * (size_t)fsc + idx] = o;
    const cplx<float> f = fN[idx], c = cN[idx];
    o.x = sc * (f.x - c.x);
    o.y = sc * (f.y - c.y);
    spec[3 * (size_t)fsc + idx] = o;
}

}  // namespace

// ============================================================================ closure object
struct sp_closure {
    int n = 0, nh = 0, capacity = 0, count = 0, sms = 0;
    uint32_t fsc = 0;
    float* bank = nullptr;
    float* params = nullptr;
    float* adam_m = nullptr;
    float* adam_v = nullptr;
    float* grad = nullptr;
    float* partials = nullptr;
    float* loss = nullptr;
    __nv_bfloat16* wb = nullptr;
    int* step_dev = nullptr;
    int* err = nullptr;
    Consts* consts_dev = nullptr;
    float* shell_gain = nullptr;  // per-shell gain of the closure term in the coarse step
    int nshell = 0;
    int every_stage = 1;  // evaluate the network at every RK stage (1) or at the first only (0)
    Consts consts{};
    AdamCfg adam{1e-3f, 1e-5f, 0.9f, 0.999f, 1e-8f, 20000, 200};
    int64_t host_step = 0;
    // snapshot transforms: batch-4 out-of-place C2R into the bank
    cufftHandle plan = 0;
    bool have_plan = false;
    void* plan_ws = nullptr;
    cplx<float>* spec = nullptr;
    // training graph: kChunk optimiser steps per replay
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_tiles = 0;
    uint64_t graph_seed = 0;
    int64_t launches = 0;
    std::string errstr;
};

namespace {

int cfail(sp_closure* c, int code, const std::string& what) {
    if (c) c->errstr = what;
    return code;
}

#define CL_CUDA(call)                                                                      \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return cfail(c, SP_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

int check_err_flag(sp_closure* c, cudaStream_t st, const char* what) {
    int h = 0;
    CL_CUDA(cudaMemcpyAsync(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CL_CUDA(cudaStreamSynchronize(st));
    if (h) {
        CL_CUDA(cudaMemsetAsync(c->err, 0, sizeof(int), st));
        return cfail(c, SP_ERR_CUDA, std::string(what) + ": tensor-core completion wait timed out");
    }
    return SP_OK;
}

int launch_train_step(sp_closure* c, int ntiles, uint64_t seed, int64_t step_override,
                      bool advance, bool adam, cudaStream_t st) {
    const int grid = ntiles < c->sms ? ntiles : c->sms;
    const float inv_batch = 1.f / ((float)ntiles * (float)kTile);
    k_train<<<grid, 128, TrainSmem::BYTES, st>>>(c->bank, c->n, c->count, c->wb, c->params,
                                                 c->consts_dev, c->step_dev, step_override, seed,
                                                 ntiles, inv_batch, c->partials, c->err);
    CL_CUDA(cudaGetLastError());
    k_grad_reduce<<<(kNParam + 1 + 255) / 256, 256, 0, st>>>(
        c->partials, grid, c->grad, c->step_dev, step_override, c->loss, advance ? 1 : 0);
    CL_CUDA(cudaGetLastError());
    c->launches += 2;
    if (adam) {
        k_adam<<<(kNParam + 255) / 256, 256, 0, st>>>(c->params, c->adam_m, c->adam_v, c->grad,
                                                      c->wb, c->step_dev, c->adam);
        CL_CUDA(cudaGetLastError());
        c->launches += 1;
    }
    return SP_OK;
}

void drop_train_graph(sp_closure* c) {
    if (c->exec) {
        cudaGraphExecDestroy(c->exec);
        c->exec = nullptr;
    }
}

int upload_consts(sp_closure* c) {
    CL_CUDA(cudaMemcpy(c->consts_dev, &c->consts, sizeof(Consts), cudaMemcpyHostToDevice));
    return SP_OK;
}

int infer_grid(const sp_closure* c, int n) {
    const int ntiles = n * (n / kTile);
    return ntiles < kInferCtasPerSm * c->sms ? ntiles : kInferCtasPerSm * c->sms;
}

}  // namespace

namespace sp {
namespace closure {

int grid_n(const sp_closure* c) { return c ? c->n : 0; }

const float* shell_gain(const sp_closure* c) { return c->shell_gain; }
bool every_stage(const sp_closure* c) { return c->every_stage != 0; }
int shell_count(const sp_closure* c) { return c->nshell; }

cudaError_t les_phase(const sp_closure* c, float* R, int n, uint32_t fsr, cudaStream_t st) {
    const int rs = n + 2;
    k_infer<<<infer_grid(c, n), kInferThreads, InferSmem::BYTES, st>>>(
        R + 3 * (size_t)fsr, fsr, rs, n, c->wb, c->params, c->consts_dev, R, rs, R + fsr, fsr,
        c->err);
    return cudaGetLastError();
}

}  // namespace closure
}  // namespace sp

extern "C" {

int sp_closure_param_count(void) { return kNParam; }

sp_closure* sp_closure_create(int n, int capacity, int* status) {
    auto set = [&](int code, const std::string& why) -> sp_closure* {
        if (status) *status = code;
        sp::set_thread_error(why.c_str());
        return nullptr;
    };
    if (n < kTile || n > 4096 || (n & (n - 1)))
        return set(SP_ERR_ARG, "closure grid must be a power of two in 128..4096");
    if (capacity < 1) return set(SP_ERR_ARG, "capacity must be positive");
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return set(SP_ERR_CUDA, "no CUDA device");
    auto* c = new sp_closure();
    c->n = n;
    c->nh = n / 2 + 1;
    c->fsc = (uint32_t)(n * c->nh);
    c->capacity = capacity;
    c->sms = sms;
    auto fail_create = [&](const char* why) {
        std::string w = std::string(why) + (c->errstr.empty() ? "" : ": " + c->errstr);
        sp_closure_destroy(c);
        return set(SP_ERR_CUDA, w);
    };
    const size_t nn = (size_t)n * n;
    if (cudaMalloc(&c->bank, (size_t)capacity * 4 * nn * sizeof(float)) != cudaSuccess)
        return fail_create("bank allocation failed");
    bool okm = cudaMalloc(&c->params, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->adam_m, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->adam_v, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->grad, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->partials, (size_t)sms * kPartStride * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->loss, kLossRing * sizeof(float)) == cudaSuccess &&
               cudaMalloc(&c->wb, kLayers * kWsz * sizeof(__nv_bfloat16)) == cudaSuccess &&
               cudaMalloc(&c->step_dev, sizeof(int)) == cudaSuccess &&
               cudaMalloc(&c->err, sizeof(int)) == cudaSuccess &&
               cudaMalloc(&c->consts_dev, sizeof(Consts)) == cudaSuccess &&
               cudaMalloc(&c->spec, 4 * (size_t)c->fsc * sizeof(cplx<float>)) == cudaSuccess;
    c->nshell = (int)std::floor(std::sqrt(2.0) * (double)(n / 2) + 0.5) + 1;
    okm = okm && cudaMalloc(&c->shell_gain, c->nshell * sizeof(float)) == cudaSuccess;
    if (!okm) return fail_create("allocation failed");
    bool okz = cudaMemset(c->params, 0, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMemset(c->adam_m, 0, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMemset(c->adam_v, 0, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMemset(c->grad, 0, kNParam * sizeof(float)) == cudaSuccess &&
               cudaMemset(c->loss, 0, kLossRing * sizeof(float)) == cudaSuccess &&
               cudaMemset(c->wb, 0, kLayers * kWsz * sizeof(__nv_bfloat16)) == cudaSuccess &&
               cudaMemset(c->step_dev, 0, sizeof(int)) == cudaSuccess &&
               cudaMemset(c->err, 0, sizeof(int)) == cudaSuccess;
    if (!okz) return fail_create("initialisation failed");
    {
        std::vector<float> ones(c->nshell, 1.f);
        if (cudaMemcpy(c->shell_gain, ones.data(), c->nshell * sizeof(float),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            return fail_create("initialisation failed");
    }
    for (int f = 0; f < 3; ++f) c->consts.inscale[f] = 1.f;
    c->consts.outscale = 1.f;
    c->consts.inv_outscale = 1.f;
    c->consts.clip = 0;
    if (upload_consts(c)) return fail_create("constant upload failed");
    if (cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             TrainSmem::BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(k_infer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             InferSmem::BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(k_infer, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return fail_create("cudaFuncSetAttribute failed");
    // batch of 4 out-of-place C2R transforms: spectral scratch -> unpadded bank fields
    long long shape[2] = {n, n}, cemb[2] = {n, c->nh}, remb[2] = {n, n};
    size_t ws = 0;
    if (cufftCreate(&c->plan) != CUFFT_SUCCESS) return fail_create("cufftCreate failed");
    c->have_plan = true;
    if (cufftSetAutoAllocation(c->plan, 0) != CUFFT_SUCCESS ||
        cufftMakePlanMany64(c->plan, 2, shape, cemb, 1, (long long)c->fsc, remb, 1, (long long)nn,
                            CUFFT_C2R, 4, &ws) != CUFFT_SUCCESS)
        return fail_create("cuFFT plan failed");
    if (ws && cudaMalloc(&c->plan_ws, ws) != cudaSuccess) return fail_create("cuFFT workspace");
    if (ws && cufftSetWorkArea(c->plan, c->plan_ws) != CUFFT_SUCCESS)
        return fail_create("cuFFT work area");
    if (cudaDeviceSynchronize() != cudaSuccess) return fail_create("initialisation failed");
    if (status) *status = SP_OK;
    return c;
}

void sp_closure_destroy(sp_closure* c) {
    if (!c) return;
    drop_train_graph(c);
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->have_plan) cufftDestroy(c->plan);
    for (void* p : {(void*)c->bank, (void*)c->params, (void*)c->adam_m, (void*)c->adam_v,
                    (void*)c->grad, (void*)c->partials, (void*)c->loss, (void*)c->wb,
                    (void*)c->step_dev, (void*)c->err, (void*)c->consts_dev, (void*)c->spec,
                    (void*)c->shell_gain, c->plan_ws})
        if (p) cudaFree(p);
    delete c;
}

const char* sp_closure_last_error(const sp_closure* c) { return c ? c->errstr.c_str() : "null handle"; }

int64_t sp_closure_kernel_launches(const sp_closure* c) { return c ? c->launches : -1; }

int sp_closure_set_params(sp_closure* c, const float* host) {
    if (!c || !host) return SP_ERR_ARG;
    drop_train_graph(c);
    CL_CUDA(cudaMemcpy(c->params, host, kNParam * sizeof(float), cudaMemcpyHostToDevice));
    CL_CUDA(cudaMemset(c->adam_m, 0, kNParam * sizeof(float)));
    CL_CUDA(cudaMemset(c->adam_v, 0, kNParam * sizeof(float)));
    CL_CUDA(cudaMemset(c->step_dev, 0, sizeof(int)));
    CL_CUDA(cudaMemset(c->loss, 0, kLossRing * sizeof(float)));
    c->host_step = 0;
    k_to_bf16<<<(kLayers * kWsz + 255) / 256, 256>>>(c->params, c->wb);
    CL_CUDA(cudaGetLastError());
    c->launches += 1;
    CL_CUDA(cudaDeviceSynchronize());
    return SP_OK;
}

int sp_closure_get_params(sp_closure* c, float* host) {
    if (!c || !host) return SP_ERR_ARG;
    CL_CUDA(cudaDeviceSynchronize());
    CL_CUDA(cudaMemcpy(host, c->params, kNParam * sizeof(float), cudaMemcpyDeviceToHost));
    return SP_OK;
}

int sp_closure_get_grad(sp_closure* c, float* host) {
    if (!c || !host) return SP_ERR_ARG;
    CL_CUDA(cudaDeviceSynchronize());
    CL_CUDA(cudaMemcpy(host, c->grad, kNParam * sizeof(float), cudaMemcpyDeviceToHost));
    return SP_OK;
}

int sp_closure_set_scales(sp_closure* c, const float* inscale, float outscale, int clip) {
    if (!c || !inscale || !(outscale > 0.f)) return SP_ERR_ARG;
    for (int f = 0; f < 3; ++f) c->consts.inscale[f] = inscale[f];
    c->consts.outscale = outscale;
    c->consts.inv_outscale = 1.f / outscale;
    c->consts.clip = clip ? 1 : 0;
    return upload_consts(c);
}

int sp_closure_get_scales(const sp_closure* c, float* out5) {
    if (!c || !out5) return SP_ERR_ARG;
    for (int f = 0; f < 3; ++f) out5[f] = c->consts.inscale[f];
    out5[3] = c->consts.outscale;
    out5[4] = (float)c->consts.clip;
    return SP_OK;
}

int sp_closure_set_shell_gain(sp_closure* c, const float* host, int nshell) {
    if (!c || !host || nshell != c->nshell) return SP_ERR_ARG;
    CL_CUDA(cudaMemcpy(c->shell_gain, host, nshell * sizeof(float), cudaMemcpyHostToDevice));
    return SP_OK;
}

int sp_closure_shell_count(const sp_closure* c) { return c ? c->nshell : -1; }

int sp_closure_set_update(sp_closure* c, int every_stage) {
    if (!c) return SP_ERR_ARG;
    c->every_stage = every_stage ? 1 : 0;
    return SP_OK;
}

int sp_closure_set_adam(sp_closure* c, double lr, double lr_min, double beta1, double beta2,
                        double eps, int total_steps, int warmup) {
    if (!c || !(lr > 0) || lr_min < 0 || total_steps < 1 || warmup < 0) return SP_ERR_ARG;
    drop_train_graph(c);
    c->adam = AdamCfg{(float)lr, (float)lr_min, (float)beta1, (float)beta2, (float)eps,
                      total_steps, warmup};
    return SP_OK;
}

int sp_closure_bank_load(sp_closure* c, const float* host, int count) {
    if (!c || !host || count < 1 || count > c->capacity) return SP_ERR_ARG;
    CL_CUDA(cudaMemcpy(c->bank, host, (size_t)count * 4 * c->n * c->n * sizeof(float),
                       cudaMemcpyHostToDevice));
    c->count = count;
    drop_train_graph(c);
    return SP_OK;
}

int sp_closure_bank_read(sp_closure* c, int index, float* host) {
    if (!c || !host || index < 0 || index >= c->count) return SP_ERR_ARG;
    CL_CUDA(cudaDeviceSynchronize());
    const size_t nn = (size_t)c->n * c->n;
    CL_CUDA(cudaMemcpy(host, c->bank + (size_t)index * 4 * nn, 4 * nn * sizeof(float),
                       cudaMemcpyDeviceToHost));
    return SP_OK;
}

int sp_closure_bank_count(const sp_closure* c) { return c ? c->count : -1; }

int sp_closure_bank_reset(sp_closure* c) {
    if (!c) return SP_ERR_ARG;
    c->count = 0;
    drop_train_graph(c);
    return SP_OK;
}

int sp_closure_add_snapshot(sp_closure* c, const void* wbar_hat, const void* fine_nl_hat,
                            const void* coarse_nl_hat, void* stream) {
    if (!c || !wbar_hat || !fine_nl_hat || !coarse_nl_hat) return SP_ERR_ARG;
    if (c->count >= c->capacity) return cfail(c, SP_ERR_STATE, "snapshot bank is full");
    auto st = (cudaStream_t)stream;
    k_snap_spec<<<(c->fsc + 255) / 256, 256, 0, st>>>(
        (const cplx<float>*)wbar_hat, (const cplx<float>*)fine_nl_hat,
        (const cplx<float>*)coarse_nl_hat, c->spec, c->n, c->fsc);
    CL_CUDA(cudaGetLastError());
    c->launches += 1;
    float* dst = c->bank + (size_t)c->count * 4 * c->n * c->n;
    if (cufftSetStream(c->plan, st) != CUFFT_SUCCESS ||
        cufftExecC2R(c->plan, (cufftComplex*)c->spec, (cufftReal*)dst) != CUFFT_SUCCESS)
        return cfail(c, SP_ERR_CUFFT, "snapshot C2R failed");
    c->count += 1;
    drop_train_graph(c);
    return SP_OK;
}

int sp_closure_grad(sp_closure* c, int64_t step, int batch_tiles, uint64_t seed, void* stream) {
    if (!c || step < 0 || batch_tiles < 1) return SP_ERR_ARG;
    if (c->count < 1) return cfail(c, SP_ERR_STATE, "snapshot bank is empty");
    auto st = (cudaStream_t)stream;
    int r = launch_train_step(c, batch_tiles, seed, step, false, false, st);
    if (r) return r;
    return check_err_flag(c, st, "sp_closure_grad");
}

int sp_closure_train(sp_closure* c, int steps, int batch_tiles, uint64_t seed, void* stream) {
    if (!c || steps < 0 || batch_tiles < 1) return SP_ERR_ARG;
    if (c->count < 1) return cfail(c, SP_ERR_STATE, "snapshot bank is empty");
    auto st = (cudaStream_t)stream;
    constexpr int kChunk = 50;
    int done = 0;
    if (steps >= kChunk) {
        if (c->exec && (c->graph_tiles != batch_tiles || c->graph_seed != seed)) drop_train_graph(c);
        if (!c->exec) {
            if (!c->cap_stream)
                CL_CUDA(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
            CL_CUDA(cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal));
            const int64_t before = c->launches;
            int r = 0;
            for (int i = 0; i < kChunk && !r; ++i)
                r = launch_train_step(c, batch_tiles, seed, -1, true, true, c->cap_stream);
            c->launches = before;
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(c->cap_stream, &g);
            if (r) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            if (e != cudaSuccess) return cfail(c, SP_ERR_CUDA, cudaGetErrorString(e));
            e = cudaGraphInstantiate(&c->exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                c->exec = nullptr;
                return cfail(c, SP_ERR_CUDA, cudaGetErrorString(e));
            }
            c->graph_tiles = batch_tiles;
            c->graph_seed = seed;
        }
        for (; done + kChunk <= steps; done += kChunk) {
            CL_CUDA(cudaGraphLaunch(c->exec, st));
            c->launches += 3 * kChunk;
        }
    }
    for (; done < steps; ++done) {
        int r = launch_train_step(c, batch_tiles, seed, -1, true, true, st);
        if (r) return r;
    }
    c->host_step += steps;
    return check_err_flag(c, st, "sp_closure_train");
}

int sp_closure_train_begin(sp_closure* c, int batch_tiles, uint64_t seed, void* stream) {
    if (!c || batch_tiles < 1) return SP_ERR_ARG;
    if (c->count < 1) return cfail(c, SP_ERR_STATE, "snapshot bank is empty");
    return launch_train_step(c, batch_tiles, seed, -1, true, false, (cudaStream_t)stream);
}

int sp_closure_train_finish(sp_closure* c, void* stream) {
    if (!c) return SP_ERR_ARG;
    k_adam<<<(kNParam + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        c->params, c->adam_m, c->adam_v, c->grad, c->wb, c->step_dev, c->adam);
    CL_CUDA(cudaGetLastError());
    c->launches += 1;
    c->host_step += 1;
    return SP_OK;
}

void* sp_closure_grad_buffer(sp_closure* c) { return c ? (void*)c->grad : nullptr; }

int64_t sp_closure_step_count(const sp_closure* c) { return c ? c->host_step : -1; }

int sp_closure_check(sp_closure* c, void* stream) {
    if (!c) return SP_ERR_ARG;
    return check_err_flag(c, (cudaStream_t)stream, "closure step");
}

int sp_closure_losses(sp_closure* c, int64_t first, int count, float* host) {
    if (!c || !host || first < 0 || count < 0 || count > kLossRing) return SP_ERR_ARG;
    CL_CUDA(cudaDeviceSynchronize());
    std::vector<float> ring(kLossRing);
    CL_CUDA(cudaMemcpy(ring.data(), c->loss, kLossRing * sizeof(float), cudaMemcpyDeviceToHost));
    for (int i = 0; i < count; ++i) host[i] = ring[(first + i) & (kLossRing - 1)];
    return SP_OK;
}

int sp_closure_infer_async(sp_closure* c, const float* fields, int64_t field_stride,
                           int row_stride, float* out, int out_row_stride, void* stream) {
    if (!c || !fields || !out || field_stride <= 0 || row_stride < c->n || out_row_stride < c->n)
        return SP_ERR_ARG;
    auto st = (cudaStream_t)stream;
    const int n = c->n;
    k_infer<<<infer_grid(c, n), kInferThreads, InferSmem::BYTES, st>>>(
        fields, (size_t)field_stride, row_stride, n, c->wb, c->params, c->consts_dev, out,
        out_row_stride, nullptr, 0, c->err);
    CL_CUDA(cudaGetLastError());
    c->launches += 1;
    return SP_OK;
}

int sp_closure_infer(sp_closure* c, const float* fields, int64_t field_stride, int row_stride,
                     float* out, int out_row_stride, void* stream) {
    int r = sp_closure_infer_async(c, fields, field_stride, row_stride, out, out_row_stride, stream);
    if (r) return r;
    return check_err_flag(c, (cudaStream_t)stream, "sp_closure_infer");
}

int sp_filter_spectrum(const void* src, int n_src, void* dst, int n_dst, int dim, int fp64,
                       int dealias, void* stream) {
    if (!src || !dst || (dim != 2 && dim != 3) || n_src < 2 || n_dst < 2 || n_src % 2 ||
        n_dst % 2) {
        sp::set_thread_error("sp_filter_spectrum: bad arguments");
        return SP_ERR_ARG;
    }
    const uint64_t total = (uint64_t)n_dst * (dim == 3 ? (uint64_t)n_dst : 1ull) *
                           (uint64_t)(n_dst / 2 + 1);
    const double scale = std::pow((double)n_dst / (double)n_src, dim);
    const unsigned grid = (unsigned)((total + 255) / 256);
    auto st = (cudaStream_t)stream;
    if (fp64)
        k_filter<double><<<grid, 256, 0, st>>>((const cplx<double>*)src, n_src, (cplx<double>*)dst,
                                               n_dst, dim, dealias, scale, total);
    else
        k_filter<float><<<grid, 256, 0, st>>>((const cplx<float>*)src, n_src, (cplx<float>*)dst,
                                              n_dst, dim, dealias, (float)scale, total);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        sp::set_thread_error(cudaGetErrorString(e));
        return SP_ERR_CUDA;
    }
    return SP_OK;
}

}  // extern "C"
