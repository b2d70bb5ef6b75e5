// Learned subgrid closure for coarse 2D runs: network geometry, the shared device-side pieces
// (tile sampling, constants) and the launch interface used by the solver step.
//
// Network: 75 inputs (5 x 5 stencils of the filtered vorticity and its two derivatives) ->
// 64 -> 64 -> 64 (GELU, tanh form) -> 1.  Layers 1-3 run as BF16 tcgen05 GEMMs with FP32
// accumulation in tensor memory; the 64 -> 1 output layer runs in FP32 on the CUDA cores.
// Every GEMM layer is stored as W[64][80]: the bias is the weight of a constant-one input
// column (input 75 for layer 1, input 64 for layers 2 and 3), the remaining columns are zero
// padding up to K = 80.  The output layer is w4[80] with its bias at index 64.  Parameter
// vector (fp32): [W1 | W2 | W3 | w4] = 3 * 5120 + 80 = 15440 values.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct sp_closure;

namespace sp {
namespace cl {

constexpr int kIn = 75;                              // stencil features
constexpr int kK = 80;                               // GEMM K (inputs + bias + padding)
constexpr int kH = 64;                               // hidden width = GEMM N
constexpr int kTile = 128;                           // points per tile = MMA M
constexpr int kLayers = 3;                           // tensor-core layers
constexpr int kWsz = kH * kK;                        // 5120
constexpr int kNParam = kLayers * kWsz + kK;         // 15440
constexpr int kBiasIn = 75, kBiasH = 64;             // constant-one columns
constexpr int kHalo = 2, kSpan = kTile + 2 * kHalo;  // stencil row segment
constexpr int kStencil = 3 * 5 * kSpan;              // staged floats per tile
constexpr int kLossRing = 1 << 16;

// Input scales and the output scale: feature = field * inscale[f]; the network predicts the
// subgrid term divided by outscale.  clip: drop predictions that feed enstrophy back to the
// resolved field (S * omega > 0).
struct Consts {
    float inscale[3];
    float outscale;
    float inv_outscale;
    int clip;
};

// splitmix64 finaliser
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Training tile i of step `step`: (snapshot, row, 128-point segment) drawn from a counter hash.
struct TilePick {
    int snap, row, seg;
};
__host__ __device__ __forceinline__ TilePick pick_tile(uint64_t seed, int64_t step, int i,
                                                       int count, int n) {
    const uint64_t h = mix64(seed + mix64(((uint64_t)step << 32) | (uint32_t)i));
    const uint32_t lo = (uint32_t)h;
    TilePick p;
    p.snap = (int)((h >> 32) % (uint64_t)count);
    p.row = (int)(lo % (uint32_t)n);
    p.seg = (int)((lo / (uint32_t)n) % (uint32_t)(n / kTile));
    return p;
}

}  // namespace cl

namespace closure {
// Coarse-step phase of a solver with the closure attached: R is the solver's work array in
// the padded real layout with slots [S, u, v, omega, d omega/dx, d omega/dy] of fsr reals each.
// Writes the Basdevant products into the u, v slots in place and the closure term into S.
cudaError_t les_phase(const sp_closure* c, float* R, int n, uint32_t fsr, cudaStream_t st);
int grid_n(const sp_closure* c);
// Per-shell gains (shell = round(|k|), shell_count entries) applied to the closure term.
const float* shell_gain(const sp_closure* c);
int shell_count(const sp_closure* c);
// Whether the network runs at every RK stage or only at the first stage of each step (its term
// then held for the step's other stages).
bool every_stage(const sp_closure* c);
}  // namespace closure
}  // namespace sp
