// Diagnostics reductions: energy / enstrophy / palinstrophy / band energy of a spectral state,
// the shell spectrum E(k), and max|u_i| over a padded physical field.
//
// The spectral sums follow src/pyspectral/diagnostics.py:48-97 (Hermitian weights 1,2,..,2,1 on
// the last axis divided by n^(2d); 2D energy divides by k^2), accumulated in fp64.  They run as
// a fixed grid of blocks writing one partial per block, then one block summing the partials in
// a fixed order, so repeated calls give bit-identical results.
#pragma once

#include "common.cuh"

namespace sp {

constexpr int kRedBlocks = 148 * 4;  // 4 resident 256-thread blocks per SM on 148 SMs
constexpr int kRedThreads = 256;

template <int NQ>
__device__ __forceinline__ void block_sum(double (&v)[NQ], double* smem /* [NQ][32] */) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) smem[q * 32 + warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            v[q] = lane < nw ? smem[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
        }
    }
}

// Per-mode wavenumbers for either dimension: last axis index l (weight axis), k^2.
struct ModeK {
    int last;
    double k2;
};
__device__ __forceinline__ ModeK mode_k(uint32_t idx, int n, int nh, int dim) {
    ModeK r;
    uint32_t t = idx / (uint32_t)nh;
    uint32_t l = idx - t * (uint32_t)nh;
    double kz = (double)l;
    double s;
    if (dim == 2) {
        double kx = (double)signed_k((int)t, n);
        s = kx * kx + kz * kz;
    } else {
        uint32_t i = t / (uint32_t)n, j = t - i * (uint32_t)n;
        double kx = (double)signed_k((int)i, n), ky = (double)signed_k((int)j, n);
        s = kx * kx + ky * ky + kz * kz;
    }
    r.last = (int)l;
    r.k2 = s;
    return r;
}

template <typename T>
__device__ __forceinline__ double mode_density(const cplx<T>* __restrict__ st, uint32_t idx,
                                               uint32_t fsc, int ncomp) {
    double a = 0.0;
    for (int c = 0; c < ncomp; ++c) {
        cplx<T> z = st[(size_t)c * fsc + idx];
        double x = (double)z.x, y = (double)z.y;
        a += x * x + y * y;
    }
    return a;
}

// partials[blockIdx.x * 4 + q], q = energy, enstrophy, palinstrophy, band energy (each x2).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_reduce_spectral(
    const cplx<T>* __restrict__ st, int n, int nh, int dim, uint32_t fsc, double w_edge,
    double w_mid, double klo2, double khi2, double* __restrict__ partials) {
    __shared__ double smem[4 * 32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int ncomp = dim == 2 ? 1 : 3;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < fsc;
         idx += gridDim.x * blockDim.x) {
        ModeK m = mode_k(idx, n, nh, dim);
        double w = (m.last == 0 || m.last == nh - 1) ? w_edge : w_mid;
        double d = mode_density<T>(st, idx, fsc, ncomp) * w;
        double de, z, p;
        if (dim == 2) {
            double inv = m.k2 > 0.0 ? 1.0 / m.k2 : 0.0;
            de = d * inv;
            z = d;
            p = d * m.k2;
        } else {
            de = d;
            z = d * m.k2;
            p = d * m.k2 * m.k2;
        }
        v[0] += de;
        v[1] += z;
        v[2] += p;
        if (m.k2 >= klo2 && m.k2 <= khi2) v[3] += de;
    }
    block_sum<4>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) partials[blockIdx.x * 4 + q] = v[q];
    }
}

// Sums nblk partial rows of width NQ in a fixed order; out[q] = factor * sum.
template <int NQ>
__global__ void __launch_bounds__(kRedThreads) k_finish_sum(const double* __restrict__ partials,
                                                            int nblk, double factor,
                                                            double* __restrict__ out) {
    __shared__ double smem[NQ * 32];
    double v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) v[q] += partials[b * NQ + q];
    }
    block_sum<NQ>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) out[q] = factor * v[q];
    }
}

// Shell spectrum: E[s] += 0.5 * energy density, s = int(sqrt(k^2) + 0.5)
// (diagnostics.py:90-97).  Shared-memory histogram when it fits, global atomics otherwise.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_spectrum(const cplx<T>* __restrict__ st, int n,
                                                          int nh, int dim, uint32_t fsc,
                                                          double w_edge, double w_mid,
                                                          int nshell, int use_smem,
                                                          double* __restrict__ spec) {
    extern __shared__ double hist[];
    if (use_smem) {
        for (int s = threadIdx.x; s < nshell; s += blockDim.x) hist[s] = 0.0;
        __syncthreads();
    }
    const int ncomp = dim == 2 ? 1 : 3;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < fsc;
         idx += gridDim.x * blockDim.x) {
        ModeK m = mode_k(idx, n, nh, dim);
        double w = (m.last == 0 || m.last == nh - 1) ? w_edge : w_mid;
        double d = mode_density<T>(st, idx, fsc, ncomp) * w;
        if (dim == 2) d = d * (m.k2 > 0.0 ? 1.0 / m.k2 : 0.0);
        int s = (int)(sqrt(m.k2) + 0.5);
        if (s < nshell && d != 0.0) {
            if (use_smem) atomicAdd(&hist[s], 0.5 * d);
            else atomicAdd(&spec[s], 0.5 * d);
        }
    }
    if (use_smem) {
        __syncthreads();
        for (int s = threadIdx.x; s < nshell; s += blockDim.x)
            if (hist[s] != 0.0) atomicAdd(&spec[s], hist[s]);
    }
}

// One velocity component of a state, scaled by 1/n^d, into a complex field (no dealiasing,
// as Diagnostics.max_velocity_sum transforms the state as it is, diagnostics.py:99-109).
// 2D: comp 0 -> i ky omega/k^2, comp 1 -> -i kx omega/k^2; 3D: comp c -> u_c.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_velocity_component(
    const cplx<T>* __restrict__ st, cplx<T>* __restrict__ out, int n, int nh, int dim,
    uint32_t fsc, int comp, T scale) {
    uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= fsc) return;
    if (dim == 3) {
        out[idx] = scl(scale, st[(size_t)comp * fsc + idx]);
        return;
    }
    uint32_t i = idx / (uint32_t)nh, j = idx - i * (uint32_t)nh;
    T kx = (T)signed_k((int)i, n), ky = (T)j;
    T k2 = kx * kx + ky * ky;
    T ik2 = k2 > (T)0 ? scale / k2 : (T)0;
    cplx<T> psi = scl(ik2, st[idx]);
    out[idx] = comp == 0 ? scl(ky, mul_i(psi)) : scl(kx, mul_mi(psi));
}

// max |x| over the n physical entries of each padded row (row stride 2*nh reals), as the bit
// pattern of a non-negative double (orders like an unsigned integer; NaN wins, as in a max
// that propagates NaN).
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_max_abs_padded(const T* __restrict__ R, int n,
                                                                int row_stride, uint32_t rows,
                                                                unsigned long long* out) {
    __shared__ unsigned long long smem[32];
    unsigned long long best = 0ull;
    const uint32_t half = (uint32_t)n >> 1;  // pairs per row (n even)
    const uint32_t total = rows * half;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += gridDim.x * blockDim.x) {
        uint32_t r = q / half, x = 2u * (q - r * half);
        const T* p = R + (size_t)r * row_stride + x;
        double a = fabs((double)p[0]), b = fabs((double)p[1]);
        unsigned long long ba = (unsigned long long)__double_as_longlong(a);
        unsigned long long bb = (unsigned long long)__double_as_longlong(b);
        best = max(best, max(ba, bb));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = best;
    __syncthreads();
    if (warp == 0) {
        int nw = (blockDim.x + 31) >> 5;
        best = lane < nw ? smem[lane] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
        if (lane == 0) atomicMax(out, best);
    }
}

}  // namespace sp
