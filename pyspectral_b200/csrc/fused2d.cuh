// Fused 2D IF-RK4 stage on hand-written FFTs: two HBM round trips per stage.
//
// Only the dealiased columns ky < kc (kc = number of ky with 3 ky < n, about n/3) are ever
// non-zero in the transforms' inputs or needed from their outputs, so the work array keeps
// just those: X holds (n rows x kc columns) of Pair<T> — at stage boundaries the pair
// (u~, v~)(x, ky) of the two velocity fields transformed back along x only; after a row pass
// the products (P~, Q~)(x, ky) transformed forward along y only.  Rows are interleaved in
// pairs, X[x/2][ky][x%2] (xidx): a column access then moves whole 32-byte sectors (rows x and
// x+1 of one column are adjacent) and a row-pair access is contiguous.
//
// Row pass (one CTA sub-block per row; two CTAs per SM):
//   Z(k) = U(k) + i V(k) (Hermitian completion of both half spectra), z = IFFT_n(Z) gives
//   z = u + i v; the products (v^2 - u^2) + i (u v) are formed in registers; Z' = FFT_n of
//   that; P(k) = (Z'(k) + conj Z'(n-k)) / 2, Q(k) = (Z'(k) - conj Z'(n-k)) / 2i for k < kc.
//   One complex transform pair per row replaces the two C2R + two R2C of the reference stage.
// Column pass (one sub-block per column ky):
//   forward FFT along x of (P~, Q~) -> (P, Q)(kx, ky); in registers: nonlinear term
//   N = kx ky P + (kx^2 - ky^2) Q (dealiased), Lawson stage update of the state and the
//   accumulator, next inputs u = i ky psi, v = -i kx psi (scaled by 1/n^2); inverse FFT along x
//   -> X.  State and accumulator are kept transposed (ky-major, u0t[ky][x], acct[ky][x]) so the
//   column pass reads them contiguously; the NumPy-layout state u0 is refreshed on demand.
#pragma once

#include "common.cuh"
#include "fft_block.cuh"
#include "fused2d.h"
#include "reduce.cuh"
#include "tma.cuh"

namespace sp {

// Sub-blocks (columns) per CTA: one sequence per CTA once a sequence has at least 16 threads
// (n >= 256), so small grids still spread over every SM; smaller n packs sequences into one
// warp.  Never more sub-blocks than sequences.
constexpr int sub_blocks(int t, int count) {
    const int b = t >= 16 ? 1 : 32 / t;
    return b < count ? b : count;
}

// BX: tile multiplier chosen by the ensemble autotuner (1, 2 or 4 times the default sub-blocks
// per CTA; the single-run engine uses 1).
constexpr int tiled_blocks(int t, int count, int bx) {
    const int b = sub_blocks(t, count) * bx;
    return b < count ? b : count;
}

template <int N, int BX = 1>
struct Fused2D {
    static constexpr int T = N / 16;
    static constexpr int B = tiled_blocks(T, N, BX);
    static constexpr int THREADS = T * B;
    template <typename E>
    static constexpr size_t smem_bytes() { return (size_t)B * FftPlan<N>::SMEM * sizeof(E); }
};

// Index of element (x, ky) in the row-pair interleaved work array, in Pair<T> units.
__device__ __forceinline__ size_t xidx(int x, int ky, int kc) {
    return ((size_t)(x >> 1) * kc + ky) * 2 + (x & 1);
}

// ------------------------------------------------------------------------------- row pass
// Z(k) of one row from its stored (U, V)(k): Hermitian completion of both half spectra.
template <typename T, int N>
__device__ __forceinline__ cplx<T> row_input(const Pair<T>* __restrict__ X, int p, int k,
                                             int kc, int half) {
    if (k < kc) {
        Pair<T> q = X[((size_t)p * kc + k) * 2 + half];
        if (k == 0) return mk<T>(q.a.x, q.b.x);  // c2r ignores Im at k = 0
        return mk<T>(q.a.x - q.b.y, q.a.y + q.b.x);
    }
    if (k > N - kc) {
        Pair<T> q = X[((size_t)p * kc + (N - k)) * 2 + half];
        return mk<T>(q.a.x + q.b.y, q.b.x - q.a.y);
    }
    return mk<T>(0, 0);
}

// The same for register slot M of the first inverse pass (radix 16: slot M of thread t holds
// k = t + M n/16), with the kept columns kc = (n + 2) / 3 known at compile time: each slot's
// k range lies wholly in the low half spectrum, the dealiased gap (zero) or the high half for
// all but the two slots straddling +-kc, so the branches and zeros resolve when compiled.
// Xr: the row's first element, X + (p kc) 2 + half; column k is Xr[2 k].
template <typename T, int N, int M>
__device__ __forceinline__ cplx<T> row_input_slot(const Pair<T>* __restrict__ Xr, int t) {
    constexpr int KC = (N + 2) / 3;
    constexpr int L = N / 16;
    constexpr int LO = M * L, HI = LO + L - 1;  // k range of the slot
    const int k = t + LO;
    auto low = [&](int kk) {
        Pair<T> q = Xr[2 * kk];
        if (M == 0 && kk == 0) return mk<T>(q.a.x, q.b.x);  // c2r ignores Im at k = 0
        return mk<T>(q.a.x - q.b.y, q.a.y + q.b.x);
    };
    auto high = [&](int kk) {
        Pair<T> q = Xr[2 * (N - kk)];
        return mk<T>(q.a.x + q.b.y, q.b.x - q.a.y);
    };
    if constexpr (HI < KC) {
        return low(k);
    } else if constexpr (LO > N - KC) {
        return high(k);
    } else if constexpr (LO >= KC && HI <= N - KC) {
        return mk<T>(0, 0);
    } else {
        if (k < KC) return low(k);
        if (k > N - KC) return high(k);
        return mk<T>(0, 0);
    }
}

template <typename T, int N, int M = 0>
__device__ __forceinline__ void row_inputs(cplx<T> (&v)[16], const Pair<T>* __restrict__ Xr,
                                           int t) {
    if constexpr (M < 16) {
        v[M] = row_input_slot<T, N, M>(Xr, t);
        row_inputs<T, N, M + 1>(v, Xr, t);
    }
}

// Row pairs per CTA: the sub-block structure of Fused2D over n/2 row pairs.
template <int N>
struct RowPairs {
    static constexpr int T = N / 16;
    static constexpr int B = sub_blocks(T, N / 2);
    static constexpr int THREADS = T * B;
    static constexpr size_t smem_bytes(size_t elem) { return (size_t)B * FftPlan<N>::SMEM * elem; }
};

// Rows per CTA for the row pass: single-row sub-blocks (see sub_blocks), two CTAs resident
// per SM at n = 8192 (64 registers per thread at 512 threads).
template <int N, int BX = 1>
struct RowSingle {
    static constexpr int T = N / 16;
    static constexpr int B = tiled_blocks(T, N, BX);
    static constexpr int THREADS = T * B;
    static constexpr size_t smem_bytes(size_t elem) { return (size_t)B * FftPlan<N>::SMEM * elem; }
};

// The row pass of B consecutive rows row0 .. row0 + B - 1 of one run's X, by the CTA's
// B (n/16)-thread sub-blocks (every thread of the CTA calls it: barriers inside); smem_raw
// holds B exchange buffers.
template <typename T, int N, int B>
__device__ __forceinline__ void row_pass_rows(Pair<T>* __restrict__ X, int row0,
                                              const cplx<T>* __restrict__ tw,
                                              unsigned char* smem_raw) {
    constexpr int TT = N / 16;
    constexpr int RI = first_radix<N, true>();   // inverse input pattern
    constexpr int RF = last_radix<N, false>();   // forward output pattern
    static_assert(last_radix<N, true>() == first_radix<N, false>(), "register hand-off");
    const int sub = threadIdx.x / TT, t = threadIdx.x % TT;
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smem_raw) + sub * FftPlan<N>::SMEM;
    const int row = row0 + sub;
    const int p = row >> 1, half = row & 1;

    static_assert(RI == 16, "first inverse pass is radix 16: slot m holds k = t + m n/16");
    constexpr int KC = (N + 2) / 3;  // == kc: the dealiased columns, fixed by n
    // n = 2 16^k: split transforms (fft_block.cuh), whose slot m holds k = k0 + m n/16 on input
    // and output with k0 = spec_base(t); otherwise k0 = t.
    constexpr bool SPLIT = split_plan<N>();
    const int k0 = spec_base<N>(t);
    cplx<T> v[16];
    row_inputs<T, N>(v, X + (size_t)p * KC * 2 + half, k0);
    seq_fft<N, true>(v, sm, t, tw);
    // physical space: z = u + i v  ->  (v^2 - u^2) + i (u v)
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        T u = v[e].x, w = v[e].y;
        v[e] = mk<T>((w - u) * (w + u), u * w);
    }
    if constexpr (SPLIT) {
        seq_fft<N, false>(v, sm, t, tw);  // its last shared reads end at a barrier
    } else {
        __syncthreads();
        seq_fft<N, false>(v, sm, t, tw);
        __syncthreads();
    }
    static_assert(RF == 16, "last forward pass is radix 16: slot m holds k = t + m n/16");
    {
        cplx<T>* st = sm + spad(k0);
#pragma unroll
        for (int m = 0; m < 16; ++m) {
            const int c = m * TT;
            if (c % 16 == 0) st[c + (c >> 4)] = v[m];
            else sm[spad(k0 + c)] = v[m];
        }
    }
    __syncthreads();
    // P(k) = (Z'(k) + conj Z'(n-k)) / 2, Q(k) = (Z'(k) - conj Z'(n-k)) / 2i
    Pair<T>* Xo = X + (size_t)p * KC * 2 + half;
    // n - k = (n - (j+1) TT) + (TT - t): a padded base for TT - t plus a constant (TT a
    // multiple of 16); k = 0 (t = 0, j = 0) reads element 0
    const int pk = spad(t), pnk = spad(TT - t);
#pragma unroll
    for (int j = 0; j < (KC + TT - 1) / TT; ++j) {
        const int k = t + j * TT;
        if ((j + 1) * TT <= KC || k < KC) {
            cplx<T> a, b;
            if constexpr (TT % 16 == 0) {
                const int ca = j * TT, cb = N - (j + 1) * TT;
                a = sm[pk + ca + (ca >> 4)];
                b = sm[(j == 0 && t == 0) ? 0 : pnk + cb + (cb >> 4)];
            } else {
                a = sm[spad(k)];
                b = sm[spad((N - k) & (N - 1))];
            }
            Pair<T> o;
            o.a = mk<T>((T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y));
            o.b = mk<T>((T)0.5 * (a.y + b.y), (T)0.5 * (b.x - a.x));
            Xo[2 * k] = o;
        }
    }
}

// Batched launches: blockIdx.y selects the member; each member's arrays start `stride`
// elements after the previous member's (stride 0 for a single run).
template <typename T, int N, int BX = 1>
__global__ void __launch_bounds__(RowSingle<N, BX>::THREADS, 2) k_row_pass(
    Pair<T>* __restrict__ X, int kc, const cplx<T>* __restrict__ tw, size_t x_stride) {
    using F = RowSingle<N, BX>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    (void)kc;  // fixed by n: (n + 2) / 3
    row_pass_rows<T, N, F::B>(X + blockIdx.y * x_stride, blockIdx.x * F::B, tw, smem_raw);
}

// CFL bound from the stage-0 inputs: max |u|, max |v| over the physical rows (no write-back).
template <typename T, int N>
__global__ void __launch_bounds__(RowPairs<N>::THREADS) k_row_max(const Pair<T>* __restrict__ X,
                                                                 int kc,
                                                                 const cplx<T>* __restrict__ tw,
                                                                 unsigned long long* umax,
                                                                 size_t x_stride) {
    using F = RowPairs<N>;
    constexpr int TT = F::T;
    constexpr int RI = first_radix<N, true>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int sub = threadIdx.x / TT, t = threadIdx.x % TT;
    Pair<T>* sm = reinterpret_cast<Pair<T>*>(smem_raw) + sub * FftPlan<N>::SMEM;
    const int p = blockIdx.x * F::B + sub;
    X += blockIdx.y * x_stride;
    umax += 2 * blockIdx.y;
    static_assert(RI == 16, "slot m holds k = k0 + m n/16");
    const int k0 = spec_base<N>(t);  // see seq_fft; the maximum needs no sample order
    Pair<T> v[16];
#pragma unroll
    for (int g = 0; g < 16 / RI; ++g)
#pragma unroll
        for (int m = 0; m < RI; ++m) {
            const int k = in_pos<N, RI>(k0, g, m);
            v[g * RI + m] = Pair<T>{row_input<T, N>(X, p, k, kc, 0), row_input<T, N>(X, p, k, kc, 1)};
        }
    seq_fft<N, true>(v, sm, t, tw);
    double mu = 0.0, mv = 0.0;
    bool nan_u = false, nan_v = false;
#pragma unroll
    for (int e = 0; e < 16; ++e) {
        const double a0 = (double)v[e].a.x, b0 = (double)v[e].a.y;
        const double a1 = (double)v[e].b.x, b1 = (double)v[e].b.y;
        nan_u |= (a0 != a0) || (a1 != a1);
        nan_v |= (b0 != b0) || (b1 != b1);
        mu = fmax(mu, fmax(fabs(a0), fabs(a1)));
        mv = fmax(mv, fmax(fabs(b0), fabs(b1)));
    }
    unsigned long long bu = (unsigned long long)__double_as_longlong(mu);
    unsigned long long bv = (unsigned long long)__double_as_longlong(mv);
    // a NaN anywhere wins the max, as in a NaN-propagating maximum
    if (nan_u) bu = 0x7ff8000000000000ull;
    if (nan_v) bv = 0x7ff8000000000000ull;
    if constexpr (F::THREADS % 32 == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bu = max(bu, __shfl_down_sync(0xffffffffu, bu, o));
            bv = max(bv, __shfl_down_sync(0xffffffffu, bv, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(umax + 0, bu);
            atomicMax(umax + 1, bv);
        }
    } else {  // tiny grids: a partial warp, no shuffles
        atomicMax(umax + 0, bu);
        atomicMax(umax + 1, bv);
    }
}

// Streaming store of one Pair (written once, read by the next pass: not kept in L1).
__device__ __forceinline__ void st_stream(Pair<float>* p, const Pair<float>& v) {
    __stcs(reinterpret_cast<float4*>(p), make_float4(v.a.x, v.a.y, v.b.x, v.b.y));
}
__device__ __forceinline__ void st_stream(Pair<double>* p, const Pair<double>& v) {
    __stcs(reinterpret_cast<double2*>(p), v.a);
    __stcs(reinterpret_cast<double2*>(p) + 1, v.b);
}

// ------------------------------------------------------------------------------- column pass
// Next inverse-FFT inputs (u, v) of a vorticity mode, scaled and dealiased (velocity2).
template <typename T>
__device__ __forceinline__ Pair<T> next_inputs(T kx, T ky, T k2, bool keep, cplx<T> w, T scale) {
    T ik2 = (keep && k2 > (T)0) ? scale / k2 : (T)0;
    cplx<T> psi = scl(ik2, w);
    Pair<T> o;
    o.a = scl(ky, mul_i(psi));
    o.b = scl(kx, mul_mi(psi));
    return o;
}

// The pointwise middle of a column pass, on the forward transform's output held in registers:
// v[m] belongs to row index i = k0 + m n/16 (the forward's last pass is radix 16; k0 =
// spec_base(t)).  Nonlinear term, Lawson stage update of u0t / acct, and the next
// inverse-transform inputs written back into v.
// ld_u(i, o) / ld_c(i, o): the state / accumulator value of kept row i (o = its global index);
// the updated values go to global memory.
template <typename T, int N, int STAGE, typename LdU, typename LdC>
__device__ __forceinline__ void col_update_from(Pair<T> (&v)[16], int k0, int ky, bool active,
                                                cplx<T>* __restrict__ u0t,
                                                cplx<T>* __restrict__ acct,
                                                const T* __restrict__ tab,
                                                const StepParams<T>& p, LdU&& ld_u, LdC&& ld_c) {
    constexpr int RL = last_radix<N, false>();
    static_assert(RL == 16, "slot m holds row index k0 + m n/16");
    const T kyr = (T)ky;
    const int nh = N / 2 + 1;
#pragma unroll
    for (int g = 0; g < 16 / RL; ++g)
#pragma unroll
        for (int m = 0; m < RL; ++m) {
            const int i = in_pos<N, RL>(k0, g, m);
            const int kxi = signed_k(i, N);
            const int akx = kxi < 0 ? -kxi : kxi;
            const bool keep = active && (3 * akx < N);
            const T kx = (T)kxi, k2 = kx * kx + kyr * kyr;
            cplx<T> nxt = mk<T>(0, 0);
            if (keep) {
                const size_t o = (size_t)ky * N + i;
                cplx<T> U = ld_u(i, o);
                if constexpr (STAGE < 0) {
                    nxt = U;
                } else {
                    Pair<T> e = v[g * RL + m];
                    cplx<T> Nl = axpy(kx * kyr, e.a, scl(kx * kx - kyr * kyr, e.b));
                    IFac<T> f = if_factors(tab, nh, akx, ky, -1, k2, p);
                    cplx<T> C = STAGE > 0 ? ld_c(i, o) : mk<T>(0, 0);
                    nxt = lawson_stage<T, (STAGE < 0 ? 0 : STAGE)>(p.dt, f, Nl, U, C);
                    if (STAGE == 3) __stcs(u0t + o, nxt);
                    else __stcs(acct + o, C);
                }
            }
            v[g * RL + m] = next_inputs<T>(kx, kyr, k2, keep, nxt, p.scale);
        }
}

// col_update_from with the state and accumulator read from global memory (streamed once:
// L1 keeps the twiddles).
template <typename T, int N, int STAGE>
__device__ __forceinline__ void col_update(Pair<T> (&v)[16], int k0, int ky, bool active,
                                           cplx<T>* __restrict__ u0t, cplx<T>* __restrict__ acct,
                                           const T* __restrict__ tab, const StepParams<T>& p) {
    col_update_from<T, N, STAGE>(v, k0, ky, active, u0t, acct, tab, p,
                                 [&](int, size_t o) { return __ldcs(u0t + o); },
                                 [&](int, size_t o) { return __ldcs(acct + o); });
}

// STAGE 0..3: Lawson stage; STAGE = -1: set-up (no forward transform, no update: the inputs of
// stage 0 from the state u0t).
// The column pass of columns ky0 .. ky0 + B - 1 of one run (B (n/16)-thread sub-blocks;
// every thread of the CTA calls it: barriers inside).  Sub-blocks past kc take part in every
// barrier and write nothing.
template <typename T, int N, int STAGE, int B>
__device__ __forceinline__ void col_pass_cols(Pair<T>* __restrict__ X, int kc,
                                              cplx<T>* __restrict__ u0t,
                                              cplx<T>* __restrict__ acct,
                                              const T* __restrict__ tab, const StepParams<T>& p,
                                              const cplx<T>* __restrict__ tw, int ky0,
                                              unsigned char* smem_raw) {
    constexpr int TT = N / 16;
    constexpr int RF0 = first_radix<N, false>();  // forward input pattern
    constexpr int RIL = last_radix<N, true>();    // inverse output pattern
    static_assert(first_radix<N, true>() == last_radix<N, false>(), "register hand-off");
    const int sub = threadIdx.x / TT, t = threadIdx.x % TT;
    Pair<T>* sm = reinterpret_cast<Pair<T>*>(smem_raw) + sub * FftPlan<N>::SMEM;
    const int ky = ky0 + sub;
    const bool active = ky < kc;
    // rows x = in_pos(xb, g, m) at the ends, k0 + m n/16 in the middle (see seq_fft)
    const int xb = phys_base<N>(t), k0 = spec_base<N>(t);

    Pair<T> v[16];
    if constexpr (STAGE >= 0) {
#pragma unroll
        for (int g = 0; g < 16 / RF0; ++g)
#pragma unroll
            for (int m = 0; m < RF0; ++m) {
                const int x = in_pos<N, RF0>(xb, g, m);
                v[g * RF0 + m] = active ? X[xidx(x, ky, kc)] : Pair<T>{mk<T>(0, 0), mk<T>(0, 0)};
            }
        seq_fft<N, false>(v, sm, t, tw);
    }
    col_update<T, N, STAGE>(v, k0, ky, active, u0t, acct, tab, p);
    __syncthreads();
    seq_fft<N, true>(v, sm, t, tw);
    if (active) {
#pragma unroll
        for (int g = 0; g < 16 / RIL; ++g)
#pragma unroll
            for (int m = 0; m < RIL; ++m) {
                const int x = in_pos<N, RIL>(xb, g, m);
                X[xidx(x, ky, kc)] = v[g * RIL + m];
            }
    }
}

template <typename T, int N, int STAGE, int BX = 1>
__global__ void __launch_bounds__(Fused2D<N, BX>::THREADS) k_col_pass(
    Pair<T>* __restrict__ X, int kc, cplx<T>* __restrict__ u0t, cplx<T>* __restrict__ acct,
    const T* __restrict__ tab, const StepParams<T>* __restrict__ P,
    const cplx<T>* __restrict__ tw, size_t x_stride, size_t u_stride, int tab_stride) {
    using F = Fused2D<N, BX>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const StepParams<T> p = P[blockIdx.y];
    col_pass_cols<T, N, STAGE, F::B>(X + blockIdx.y * x_stride, kc, u0t + blockIdx.y * u_stride,
                                     acct + blockIdx.y * u_stride,
                                     tab + blockIdx.y * tab_stride, p, tw, blockIdx.x * F::B,
                                     smem_raw);
}

// ------------------------------------------------------------------------------- streamed column pass
// Persistent form of k_col_pass for one run (stages 0..3): CTA b takes columns b, b + grid, ...
// The X data of a column (n Pairs at a stride of one row pair) comes into shared memory by TMA
// (boxes of 2 Pairs x up to 256 row pairs) while the previous column's inverse transform runs;
// once it is in registers, the same buffer takes the column's kept state / accumulator rows
// (bulk copies, prefetched into L2 beforehand) while the forward transform runs, so the update
// reads them from shared memory, and the next column's X data is asked for after the update.  The two transforms exchange through a buffer of single
// complex values (exchange_halves), which leaves room for the prefetch buffer.  (Exchanging
// whole Pairs through the prefetch buffer in the forward transform and starting the next copy
// after it saves half the barriers but leaves the copy too little time: slower at n = 8192.)
// The tensor map
// views X as float32 words: row pair q is row q of width kc * 2 * sizeof(Pair) / 4; column ky
// is the box column at x = ky * stream_box_w<T>().
template <typename T>
constexpr int stream_box_w() { return 2 * (int)sizeof(Pair<T>) / 4; }  // words per row pair
template <int N>
constexpr int stream_box_h() { return N / 2 < 256 ? N / 2 : 256; }     // row pairs per box

template <typename T, int N>
struct ColStream {
    static constexpr int THREADS = N / 16;
    static constexpr size_t PB_BYTES = (size_t)N * sizeof(Pair<T>);
    static constexpr size_t EX_BYTES = (size_t)FftPlan<N>::SMEM * sizeof(cplx<T>);
    static constexpr size_t SMEM = PB_BYTES + EX_BYTES + 16;  // + the mbarrier
    // CTAs per SM that shared memory (228 KB, 1 KB reserved per CTA) and 128 registers per
    // thread allow: 1 at n = 8192 fp32, 2 at 4096, 4 at 2048
    static constexpr int by_smem = (int)(233472 / (SMEM + 1024));
    static constexpr int by_regs = 65536 / (THREADS * 128);
    static constexpr int MIN_BLOCKS = by_smem < 1 ? 1 : (by_smem < by_regs ? by_smem : by_regs);
};

constexpr uint32_t kStreamWait = 1u << 22;  // mbarrier polls before a wait gives up

// Error bit set by a streamed column pass whose TMA data never arrived (the pass then returns).
constexpr unsigned kStreamTimeout = 1u;

template <typename T, int N, int STAGE>
__global__ void __launch_bounds__(ColStream<T, N>::THREADS, ColStream<T, N>::MIN_BLOCKS)
k_col_stream(const __grid_constant__ CUtensorMap xmap, Pair<T>* __restrict__ X, int kc,
             cplx<T>* __restrict__ u0t, cplx<T>* __restrict__ acct, const T* __restrict__ tab,
             const StepParams<T>* __restrict__ P, const cplx<T>* __restrict__ tw,
             unsigned* __restrict__ err) {
    static_assert(STAGE >= 0, "the set-up pass reads no X");
    using CS = ColStream<T, N>;
    constexpr int RF0 = first_radix<N, false>();
    constexpr int RIL = last_radix<N, true>();
    constexpr int BW = stream_box_w<T>(), BH = stream_box_h<N>();
    constexpr int NBOX = (N / 2) / BH;
    static_assert(first_radix<N, true>() == last_radix<N, false>(), "register hand-off");
    extern __shared__ __align__(128) unsigned char stream_smem[];
    Pair<T>* pb = reinterpret_cast<Pair<T>*>(stream_smem);
    cplx<T>* ex = reinterpret_cast<cplx<T>*>(stream_smem + CS::PB_BYTES);
    // bar[0]: the X data of a column; bar[1]: its kept state (and accumulator) rows
    uint64_t* bar = reinterpret_cast<uint64_t*>(stream_smem + CS::PB_BYTES + CS::EX_BYTES);
    const int t = threadIdx.x;
    const int xb = phys_base<N>(t), k0 = spec_base<N>(t);  // see seq_fft
    const StepParams<T> p = *P;

    // kept rows of a state column: i < LO and i >= HI (|kx| < n/3), rounded out to 16 bytes
    constexpr int EPB = 16 / (int)sizeof(cplx<T>);  // elements per 16 bytes
    constexpr int LO = (((N - 1) / 3 + 1) + EPB - 1) / EPB * EPB;
    constexpr int HI = (N - (N - 1) / 3) / EPB * EPB;
    // staged in the X buffer once the column's X data is in registers: [0, LO) then [HI, n)
    // of the state, the same of the accumulator after them
    constexpr int KEPT = LO + (N - HI);
    constexpr uint32_t ROWS_BYTES = (uint32_t)(KEPT * sizeof(cplx<T>));
    static_assert(2 * (size_t)ROWS_BYTES <= CS::PB_BYTES, "state rows fit the X buffer");
    cplx<T>* sU = reinterpret_cast<cplx<T>*>(stream_smem);
    cplx<T>* sC = sU + KEPT;
    // thread 0: column c's X data into the buffer (completing on bar[0]) and its kept state
    // rows into L2 (for the copy into shared memory that follows)
    auto fetch_x = [&](int c) {
        tma::arrive_expect_tx(bar, (uint32_t)CS::PB_BYTES);
#pragma unroll 1
        for (int b = 0; b < NBOX; ++b)
            tma::load_2d(pb + (size_t)b * BH * 2, &xmap, c * BW, b * BH, bar);
        tma::prefetch_l2(u0t + (size_t)c * N, (uint32_t)(LO * sizeof(cplx<T>)));
        tma::prefetch_l2(u0t + (size_t)c * N + HI, (uint32_t)((N - HI) * sizeof(cplx<T>)));
        if (STAGE > 0) {
            tma::prefetch_l2(acct + (size_t)c * N, (uint32_t)(LO * sizeof(cplx<T>)));
            tma::prefetch_l2(acct + (size_t)c * N + HI, (uint32_t)((N - HI) * sizeof(cplx<T>)));
        }
    };
    // thread 0: column c's kept state (and accumulator) rows into the buffer (bar[1])
    auto fetch_rows = [&](int c) {
        tma::arrive_expect_tx(bar + 1, (STAGE > 0 ? 2u : 1u) * ROWS_BYTES);
        tma::load_1d(sU, u0t + (size_t)c * N, (uint32_t)(LO * sizeof(cplx<T>)), bar + 1);
        tma::load_1d(sU + LO, u0t + (size_t)c * N + HI, (uint32_t)((N - HI) * sizeof(cplx<T>)),
                     bar + 1);
        if (STAGE > 0) {
            tma::load_1d(sC, acct + (size_t)c * N, (uint32_t)(LO * sizeof(cplx<T>)), bar + 1);
            tma::load_1d(sC + LO, acct + (size_t)c * N + HI,
                         (uint32_t)((N - HI) * sizeof(cplx<T>)), bar + 1);
        }
    };
    auto srow = [](int i) { return i < LO ? i : LO + (i - HI); };  // kept row -> staged index

    int ky = blockIdx.x;
    if (t == 0) {
        tc::mbar_init(bar, 1);
        tc::mbar_init(bar + 1, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (t == 0 && ky < kc) fetch_x(ky);
    uint32_t px = 0, pr = 0;
    for (; ky < kc; ky += gridDim.x) {
        const bool ok = tc::mbar_wait(bar, px, kStreamWait);
        if (!__syncthreads_and(ok)) {
            // the copy never completed: report, give it one more bounded wait, leave
            if (t == 0) {
                atomicOr(err, kStreamTimeout);
                tc::mbar_wait(bar, px, kStreamWait);
            }
            return;
        }
        px ^= 1u;
        Pair<T> v[16];
#pragma unroll
        for (int g = 0; g < 16 / RF0; ++g)
#pragma unroll
            for (int m = 0; m < RF0; ++m) v[g * RF0 + m] = pb[in_pos<N, RF0>(xb, g, m)];
        __syncthreads();  // every thread has its column: the buffer takes the state rows
        if (t == 0) {
            tc::fence_smem_to_async();
            fetch_rows(ky);
        }
        seq_fft<N, false>(v, ex, t, tw);
        const bool ok_rows = tc::mbar_wait(bar + 1, pr, kStreamWait);
        if (!__syncthreads_and(ok_rows)) {
            if (t == 0) {
                atomicOr(err, kStreamTimeout);
                tc::mbar_wait(bar + 1, pr, kStreamWait);
            }
            return;  // the next column's X data was not asked for yet
        }
        pr ^= 1u;
        col_update_from<T, N, STAGE>(v, k0, ky, true, u0t, acct, tab, p,
                                     [&](int i, size_t) { return sU[srow(i)]; },
                                     [&](int i, size_t) { return sC[srow(i)]; });
        __syncthreads();  // every thread has its rows: the buffer may take the next column
        if (t == 0 && ky + (int)gridDim.x < kc) {
            tc::fence_smem_to_async();
            fetch_x(ky + gridDim.x);
        }
        seq_fft<N, true>(v, ex, t, tw);
#pragma unroll
        for (int g = 0; g < 16 / RIL; ++g)
#pragma unroll
            for (int m = 0; m < RIL; ++m)
                st_stream(X + xidx(in_pos<N, RIL>(xb, g, m), ky, (N + 2) / 3), v[g * RIL + m]);
    }
}

// The time-out path of the streamed passes on its own: one block arms an mbarrier for a copy
// that is never issued, waits `polls` polls (bounded, as the passes do), records
// kStreamTimeout and returns.  Nothing is in flight when it exits.
__global__ void __launch_bounds__(32) k_wait_probe(unsigned* __restrict__ err, uint32_t polls) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) tma::arrive_expect_tx(&bar, 16);  // 16 bytes that never arrive
    const bool ok = tc::mbar_wait(&bar, 0, polls);
    if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicOr(err, kStreamTimeout);
}

// ------------------------------------------------------------------------------- work lists
// Persistent passes of a batched group over a packed list of items, one launch per phase for
// every size class: a CTA of MT threads takes items blockIdx.x, blockIdx.x + gridDim.x, ...;
// an item is 16 MT / n rows (or columns) of one member, so every item fills the CTA and uses
// the same shared memory whatever its n.  The row and column work per item is the single-run
// passes' own (row_pass_rows, col_pass_cols).
template <int MT, int N>
constexpr bool multi_fits() {
    return N >= 16 && (N & (N - 1)) == 0 && N / 16 <= MT && 16 * MT / N <= N;
}

template <typename T, int MT, int N>
__device__ __forceinline__ void row_item(const fused::MultiClass& c, const fused::MultiItem& it,
                                         unsigned char* smem) {
    if constexpr (multi_fits<MT, N>())
        row_pass_rows<T, N, 16 * MT / N>(reinterpret_cast<Pair<T>*>(c.X) + (size_t)it.member * c.x_stride,
                                         it.first, reinterpret_cast<const cplx<T>*>(c.tw), smem);
}

template <typename T, int MT, int N, int STAGE>
__device__ __forceinline__ void col_item(const fused::MultiClass& c, const fused::MultiItem& it,
                                         unsigned char* smem) {
    if constexpr (multi_fits<MT, N>()) {
        const size_t m = (size_t)it.member;
        const StepParams<T> p = reinterpret_cast<const StepParams<T>*>(c.params)[m];
        col_pass_cols<T, N, STAGE, 16 * MT / N>(
            reinterpret_cast<Pair<T>*>(c.X) + m * c.x_stride, c.kc,
            reinterpret_cast<cplx<T>*>(c.u0t) + m * c.u_stride,
            reinterpret_cast<cplx<T>*>(c.acct) + m * c.u_stride,
            reinterpret_cast<const T*>(c.tab) + m * (size_t)c.tab_stride, p,
            reinterpret_cast<const cplx<T>*>(c.tw), it.first, smem);
    }
}

template <typename T, int MT>
__global__ void __launch_bounds__(MT, 1024 / MT) k_row_multi(const fused::MultiClass* __restrict__ cls,
                                                             const fused::MultiItem* __restrict__ items,
                                                             int nitems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const fused::MultiItem it = items[w];
        const fused::MultiClass c = cls[it.cls];
        switch (c.n) {  // uniform over the CTA: one item is one class
            case 32: row_item<T, MT, 32>(c, it, smem_raw); break;
            case 64: row_item<T, MT, 64>(c, it, smem_raw); break;
            case 128: row_item<T, MT, 128>(c, it, smem_raw); break;
            case 256: row_item<T, MT, 256>(c, it, smem_raw); break;
            case 512: row_item<T, MT, 512>(c, it, smem_raw); break;
            case 1024: row_item<T, MT, 1024>(c, it, smem_raw); break;
            default: break;
        }
        __syncthreads();  // the next item reuses the exchange buffers
    }
}

template <typename T, int MT, int STAGE>
__global__ void __launch_bounds__(MT, 512 / MT) k_col_multi(const fused::MultiClass* __restrict__ cls,
                                                            const fused::MultiItem* __restrict__ items,
                                                            int nitems) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int w = blockIdx.x; w < nitems; w += gridDim.x) {
        const fused::MultiItem it = items[w];
        const fused::MultiClass c = cls[it.cls];
        switch (c.n) {
            case 32: col_item<T, MT, 32, STAGE>(c, it, smem_raw); break;
            case 64: col_item<T, MT, 64, STAGE>(c, it, smem_raw); break;
            case 128: col_item<T, MT, 128, STAGE>(c, it, smem_raw); break;
            case 256: col_item<T, MT, 256, STAGE>(c, it, smem_raw); break;
            case 512: col_item<T, MT, 512, STAGE>(c, it, smem_raw); break;
            case 1024: col_item<T, MT, 1024, STAGE>(c, it, smem_raw); break;
            default: break;
        }
        __syncthreads();
    }
}

// Shared memory of one work-list CTA: 16 MT / n exchange buffers of n + n/16 elements.
template <typename E, int MT>
constexpr size_t multi_smem() { return (size_t)MT * 17 * sizeof(E); }

// ------------------------------------------------------------------------------- layout moves
// u0 (n, nh) NumPy layout -> u0t (kc, n): 32 x 32 tiles through shared memory.
template <typename T>
__global__ void __launch_bounds__(256) k_transpose_in(const cplx<T>* __restrict__ u0,
                                                      cplx<T>* __restrict__ u0t, int n, int nh,
                                                      int kc, size_t u0_stride, size_t u_stride) {
    __shared__ cplx<T> tile[32][33];
    u0 += blockIdx.z * u0_stride;
    u0t += blockIdx.z * u_stride;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;  // i = row (x index), j = ky
    for (int r = threadIdx.y; r < 32; r += 8) {
        int i = i0 + r, j = j0 + threadIdx.x;
        tile[r][threadIdx.x] = (i < n && j < kc) ? u0[(size_t)i * nh + j] : mk<T>(0, 0);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        int j = j0 + r, i = i0 + threadIdx.x;
        if (j < kc && i < n) u0t[(size_t)j * n + i] = tile[threadIdx.x][r];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_transpose_out(const cplx<T>* __restrict__ u0t,
                                                       cplx<T>* __restrict__ u0, int n, int nh,
                                                       int kc, size_t u_stride, size_t u0_stride) {
    __shared__ cplx<T> tile[32][33];
    u0t += blockIdx.z * u_stride;
    u0 += blockIdx.z * u0_stride;
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        int j = j0 + r, i = i0 + threadIdx.x;
        tile[r][threadIdx.x] = (j < kc && i < n) ? u0t[(size_t)j * n + i] : mk<T>(0, 0);
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        int i = i0 + r, j = j0 + threadIdx.x;
        if (i < n && j < kc) u0[(size_t)i * nh + j] = tile[threadIdx.x][r];
    }
}

// dealias a 2D state in place (zero every mode outside 3|kx| < n, 3 ky < n)
template <typename T>
__global__ void __launch_bounds__(256) k_mask2d(cplx<T>* __restrict__ u0, int n, int nh,
                                                uint32_t fsc) {
    uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= fsc) return;
    u0 += (size_t)blockIdx.y * fsc;
    uint32_t i = idx / (uint32_t)nh, j = idx - i * (uint32_t)nh;
    int kxi = signed_k((int)i, n);
    int akx = kxi < 0 ? -kxi : kxi;
    if (!(3 * akx < n && 3 * (int)j < n)) u0[idx] = mk<T>(0, 0);
}

// Spectral sums of each member's transposed state (kept modes only; the others are zero):
// partials[(m * nblk + b) * 4 + q], q = energy, enstrophy, palinstrophy, band energy (x2, the
// 1/2 is applied when the partials are summed).  2D: energy density |w|^2 / k^2.
template <typename T>
__global__ void __launch_bounds__(256) k_reduce_t(const cplx<T>* __restrict__ u0t, int n, int kc,
                                                  size_t u_stride, double inv_norm, double klo2,
                                                  double khi2, double* __restrict__ partials) {
    __shared__ double smem[4 * 32];
    const cplx<T>* st = u0t + blockIdx.y * u_stride;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const uint32_t total = (uint32_t)kc * (uint32_t)n;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += gridDim.x * blockDim.x) {
        const uint32_t ky = e / (uint32_t)n, i = e - ky * (uint32_t)n;
        const int kxi = signed_k((int)i, n);
        const int akx = kxi < 0 ? -kxi : kxi;
        if (3 * akx >= n) continue;
        const cplx<T> z = st[e];
        const double kx = (double)kxi, kyd = (double)ky, k2 = kx * kx + kyd * kyd;
        const double w = (ky == 0 || 2 * (int)ky == n) ? inv_norm : 2.0 * inv_norm;
        const double d = ((double)z.x * z.x + (double)z.y * z.y) * w;
        const double de = k2 > 0.0 ? d * (1.0 / k2) : 0.0;
        v[0] += de;
        v[1] += d;
        v[2] += d * k2;
        if (k2 >= klo2 && k2 <= khi2) v[3] += de;
    }
    block_sum<4>(v, smem);
    if (threadIdx.x == 0) {
        double* out = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * 4;
#pragma unroll
        for (int q = 0; q < 4; ++q) out[q] = v[q];
    }
}

// out[m * 4 + q] = 0.5 * sum over member m's nblk partial rows, fixed order.
__global__ void __launch_bounds__(256) k_reduce_t_finish(const double* __restrict__ partials,
                                                         int nblk, double* __restrict__ out) {
    __shared__ double smem[4 * 32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const double* pm = partials + (size_t)blockIdx.x * nblk * 4;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
#pragma unroll
        for (int q = 0; q < 4; ++q) v[q] += pm[b * 4 + q];
    block_sum<4>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) out[blockIdx.x * 4 + q] = 0.5 * v[q];
}

}  // namespace sp
