// Block-level complex FFT of length N (power of two, 16..8192) in shared memory and registers.
//
// A sub-block of T = N/16 threads transforms one length-N sequence; every thread keeps 16
// elements in registers across all passes.  The transform is a Stockham (self-sorting) radix
// sequence: radix-16 passes plus at most one radix-2/4/8 pass, so 8192 = 16*16*16*2 takes four
// passes with three shared-memory exchanges.  Pass p with radix R and stride S reads element m
// of group j at j + m*N/R, multiplies it by w_{S R}^{(j mod S) m}, does an R-point DFT and
// writes output m to (j div S) S R + (j mod S) + m S.  The last pass of a transform therefore
// leaves output j + m*N/R in the same thread and register that the first pass of a transform
// with the same radix reads its input from: an inverse transform ending with radix R feeds a
// forward transform starting with radix R without any exchange (and vice versa).
//
// Elements are either one complex sequence (cplx<T>) or two sequences sharing the transform
// (Pair<T>).  Twiddles come from a per-pass table (FftPlan::tw_offset, built in fp64 on the
// host and rounded to T); the forward transform conjugates them.  DIR = +1: inverse (e^{+}),
// DIR = -1: forward.  For N = 2 16^k, split_inverse / split_forward (below) run the transform
// as two length-N/2 halves joined by a radix-2 step whose partners trade through warp shuffles.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace sp {

// Two complex values moved as one unit: aligned to its size so a Pair<float> is one 128-bit
// access (and a Pair<double> two) instead of separate 64-bit halves.
template <typename T>
struct alignas(4 * sizeof(T) <= 16 ? 4 * sizeof(T) : 16) Pair {
    cplx<T> a, b;
};

// ---------------------------------------------------------------------------- element algebra
template <typename C>
__device__ __forceinline__ C cmul(C x, C w) {
    C r;
    r.x = fma(x.x, w.x, -x.y * w.y);
    r.y = fma(x.x, w.y, x.y * w.x);
    return r;
}
template <typename C>
__device__ __forceinline__ C csub(C x, C y) {
    C r;
    r.x = x.x - y.x;
    r.y = x.y - y.y;
    return r;
}
// x * (dir * i)
template <int DIR, typename C>
__device__ __forceinline__ C cmul_i(C x) {
    C r;
    if (DIR > 0) { r.x = -x.y; r.y = x.x; }
    else { r.x = x.y; r.y = -x.x; }
    return r;
}

__device__ __forceinline__ float2 eadd(float2 x, float2 y) { return add(x, y); }
__device__ __forceinline__ double2 eadd(double2 x, double2 y) { return add(x, y); }
__device__ __forceinline__ float2 esub(float2 x, float2 y) { return csub(x, y); }
__device__ __forceinline__ double2 esub(double2 x, double2 y) { return csub(x, y); }
__device__ __forceinline__ float2 emul(float2 x, float2 w) { return cmul(x, w); }
__device__ __forceinline__ double2 emul(double2 x, double2 w) { return cmul(x, w); }
template <int DIR> __device__ __forceinline__ float2 emul_i(float2 x) { return cmul_i<DIR>(x); }
template <int DIR> __device__ __forceinline__ double2 emul_i(double2 x) { return cmul_i<DIR>(x); }
__device__ __forceinline__ float2 escale(float2 x, float s) { return scl(s, x); }
__device__ __forceinline__ double2 escale(double2 x, double s) { return scl(s, x); }

template <typename T>
__device__ __forceinline__ Pair<T> eadd(Pair<T> x, Pair<T> y) { return {add(x.a, y.a), add(x.b, y.b)}; }
template <typename T>
__device__ __forceinline__ Pair<T> esub(Pair<T> x, Pair<T> y) { return {csub(x.a, y.a), csub(x.b, y.b)}; }
template <typename T>
__device__ __forceinline__ Pair<T> emul(Pair<T> x, cplx<T> w) { return {cmul(x.a, w), cmul(x.b, w)}; }
template <int DIR, typename T>
__device__ __forceinline__ Pair<T> emul_i(Pair<T> x) { return {cmul_i<DIR>(x.a), cmul_i<DIR>(x.b)}; }
template <typename T>
__device__ __forceinline__ Pair<T> escale(Pair<T> x, T s) { return {scl(s, x.a), scl(s, x.b)}; }

template <typename E> struct ElemReal;
template <> struct ElemReal<float2> { using type = float; };
template <> struct ElemReal<double2> { using type = double; };
template <> struct ElemReal<Pair<float>> { using type = float; };
template <> struct ElemReal<Pair<double>> { using type = double; };

// ---------------------------------------------------------------------------- small DFTs
// X_k = sum_n x_n w^{n k}, w = exp(DIR * 2 pi i / R), in place, natural order in and out.
template <int DIR, typename E>
__device__ __forceinline__ void dft2(E* x) {
    E t = esub(x[0], x[1]);
    x[0] = eadd(x[0], x[1]);
    x[1] = t;
}

template <int DIR, typename E>
__device__ __forceinline__ void dft4(E& x0, E& x1, E& x2, E& x3) {
    E a = eadd(x0, x2), b = esub(x0, x2), c = eadd(x1, x3), d = emul_i<DIR>(esub(x1, x3));
    x0 = eadd(a, c);
    x2 = esub(a, c);
    x1 = eadd(b, d);
    x3 = esub(b, d);
}

template <int DIR, typename E>
__device__ __forceinline__ void dft4(E* x) { dft4<DIR>(x[0], x[1], x[2], x[3]); }

// multiply by exp(DIR * 2 pi i * q / 16) for q in 0..15 given as a compile-time constant
template <int DIR, int Q, typename E>
__device__ __forceinline__ E rot16(E x) {
    using R = typename ElemReal<E>::type;
    constexpr int q = Q & 15;
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;  // cos, sin(pi/8)
    const R h = (R)0.70710678118654752440;                                     // sqrt(2)/2
    if (q == 0) return x;
    if (q == 4) return emul_i<DIR>(x);
    if (q == 8) return escale(x, (R)-1);
    if (q == 12) return emul_i<-DIR>(x);
    // generic: exp(i theta) with theta = DIR * q * pi / 8
    R cs, sn;
    switch (q) {
        case 1: cs = c1; sn = s1; break;
        case 2: cs = h; sn = h; break;
        case 3: cs = s1; sn = c1; break;
        case 5: cs = -s1; sn = c1; break;
        case 6: cs = -h; sn = h; break;
        case 7: cs = -c1; sn = s1; break;
        case 9: cs = -c1; sn = -s1; break;
        case 10: cs = -h; sn = -h; break;
        case 11: cs = -s1; sn = -c1; break;
        case 13: cs = s1; sn = -c1; break;
        case 14: cs = h; sn = -h; break;
        default: cs = c1; sn = -s1; break;  // 15
    }
    cplx<R> w = mk<R>(cs, DIR > 0 ? sn : -sn);
    return emul(x, w);
}

template <int DIR, typename E>
__device__ __forceinline__ void dft8(E* x) {
    // even/odd split: X_k = E_k + w8^k O_k, X_{k+4} = E_k - w8^k O_k
    E e[4] = {x[0], x[2], x[4], x[6]}, o[4] = {x[1], x[3], x[5], x[7]};
    dft4<DIR>(e);
    dft4<DIR>(o);
    o[1] = rot16<DIR, 2>(o[1]);
    o[2] = rot16<DIR, 4>(o[2]);
    o[3] = rot16<DIR, 6>(o[3]);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x[k] = eadd(e[k], o[k]);
        x[k + 4] = esub(e[k], o[k]);
    }
}

template <int DIR, typename E>
__device__ __forceinline__ void dft16(E* x) {
    // n = 4 n1 + n2, k = k1 + 4 k2: inner DFT4 over n1, twiddle w16^{n2 k1}, outer DFT4 over n2
    E y[16];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        E a = x[n2], b = x[4 + n2], c = x[8 + n2], d = x[12 + n2];
        dft4<DIR>(a, b, c, d);  // k1 = 0..3
        y[n2 * 4 + 0] = a;
        y[n2 * 4 + 1] = b;
        y[n2 * 4 + 2] = c;
        y[n2 * 4 + 3] = d;
    }
    y[1 * 4 + 1] = rot16<DIR, 1>(y[1 * 4 + 1]);
    y[1 * 4 + 2] = rot16<DIR, 2>(y[1 * 4 + 2]);
    y[1 * 4 + 3] = rot16<DIR, 3>(y[1 * 4 + 3]);
    y[2 * 4 + 1] = rot16<DIR, 2>(y[2 * 4 + 1]);
    y[2 * 4 + 2] = rot16<DIR, 4>(y[2 * 4 + 2]);
    y[2 * 4 + 3] = rot16<DIR, 6>(y[2 * 4 + 3]);
    y[3 * 4 + 1] = rot16<DIR, 3>(y[3 * 4 + 1]);
    y[3 * 4 + 2] = rot16<DIR, 6>(y[3 * 4 + 2]);
    y[3 * 4 + 3] = rot16<DIR, 9>(y[3 * 4 + 3]);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        E a = y[0 * 4 + k1], b = y[1 * 4 + k1], c = y[2 * 4 + k1], d = y[3 * 4 + k1];
        dft4<DIR>(a, b, c, d);  // k2 = 0..3
        x[k1 + 0] = a;
        x[k1 + 4] = b;
        x[k1 + 8] = c;
        x[k1 + 12] = d;
    }
}

template <int R, int DIR, typename E>
__device__ __forceinline__ void dftR(E* x) {
    if constexpr (R == 2) dft2<DIR>(x);
    else if constexpr (R == 4) dft4<DIR>(x);
    else if constexpr (R == 8) dft8<DIR>(x);
    else dft16<DIR>(x);
}

// ---------------------------------------------------------------------------- pass plan
constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

template <int N>
struct FftPlan {
    static constexpr int LOG = ilog2(N);
    static constexpr int A = LOG / 4;                 // radix-16 passes
    static constexpr int R0 = 1 << (LOG % 4);         // remainder radix (1 = none)
    static constexpr int NP = A + (R0 > 1 ? 1 : 0);   // passes per transform
    static constexpr int T = N / 16;                  // threads per sequence
    static constexpr int SMEM = N + N / 16;           // padded elements per sequence
    static_assert((1 << LOG) == N && N >= 16 && N <= 8192, "N must be a power of two, 16..8192");
    // inverse order: 16, 16, ..., R0 ; forward order: R0, 16, ..., 16
    static constexpr int radix(bool inv, int p) {
        return inv ? (p < A ? 16 : R0) : ((R0 > 1 && p == 0) ? R0 : 16);
    }
    static constexpr int stride(bool inv, int p) {  // product of the previous radices
        int s = 1;
        for (int q = 0; q < p; ++q) s *= radix(inv, q);
        return s;
    }
    // Per-pass twiddle table: for the inverse passes p = 1..NP-1, then the forward passes
    // p = 1..NP-1, a block of npow(R_p) S_p entries: the stored powers w^q (q = 1, 2, 3, 4, 8,
    // 12, the first npow of them) of w = exp(+2 pi i js / (S_p R_p)), js < S_p, laid out
    // [power][js].  tw_offset is the start of a pass's block; TW_SIZE the whole table.
    static constexpr int npow(int r) { return r == 2 ? 1 : r == 4 ? 3 : r == 8 ? 4 : 6; }
    static constexpr int tw_offset(bool inv, int p) {
        int o = 0;
        for (int q = 1; q < NP; ++q) {
            if (inv && q == p) return o;
            o += npow(radix(true, q)) * stride(true, q);
        }
        for (int q = 1; q < NP; ++q) {
            if (!inv && q == p) return o;
            o += npow(radix(false, q)) * stride(false, q);
        }
        return o;
    }
    static constexpr int TW_SIZE = tw_offset(false, NP) > 0 ? tw_offset(false, NP) : 1;
};

// Barrier between the passes of a transform: the whole CTA, or (WARP) only the calling warp,
// for kernels whose every sequence lies inside one warp (n <= 512) and whose warps exchange
// through buffers of their own.
template <bool WARP>
__device__ __forceinline__ void seq_sync() {
    if constexpr (WARP) __syncwarp();
    else __syncthreads();
}

// shared-memory index with one pad element every 16 (conflict-free strided access)
__device__ __forceinline__ int spad(int e) { return e + (e >> 4); }

// position of register v[g*R + m] for a pass of radix R: input pattern j + m N/R
template <int N, int R>
__device__ __forceinline__ int in_pos(int t, int g, int m) {
    return t + (N / 16) * g + m * (N / R);
}

template <int DIR, typename C>
__device__ __forceinline__ C tw_load(const C* __restrict__ tw, int idx) {
    C w = __ldg(tw + idx);
    if (DIR < 0) w.y = -w.y;
    return w;
}

// Powers of w stored per pass (see FftPlan::tw_offset): w^1, w^2, w^3 (radix >= 4), w^4
// (radix >= 8), w^8 and w^12 (radix 16).  Every other power is one product of two stored,
// correctly rounded values, so each twiddle is within about one rounding of exact.
template <int R>
constexpr int tw_powers() { return R == 2 ? 1 : R == 4 ? 3 : R == 8 ? 4 : 6; }

// Twiddles w^m, m = 1..R-1, of one group from this pass's block, laid out [power][js]: a warp
// (consecutive js) reads each stored power contiguously.
template <int R, int S, int DIR, typename C>
__device__ __forceinline__ void group_twiddles(C (&w)[16], const C* __restrict__ tw, int js) {
    w[1] = tw_load<DIR>(tw, js);
    if constexpr (R >= 4) {
        w[2] = tw_load<DIR>(tw, S + js);
        w[3] = tw_load<DIR>(tw, 2 * S + js);
    }
    if constexpr (R >= 8) {
        w[4] = tw_load<DIR>(tw, 3 * S + js);
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
    }
    if constexpr (R >= 16) {
        w[8] = tw_load<DIR>(tw, 4 * S + js);
        w[12] = tw_load<DIR>(tw, 5 * S + js);
        w[9] = cmul(w[8], w[1]);
        w[10] = cmul(w[8], w[2]);
        w[11] = cmul(w[8], w[3]);
        w[13] = cmul(w[12], w[1]);
        w[14] = cmul(w[12], w[2]);
        w[15] = cmul(w[12], w[3]);
    }
}

template <int N, int R, int S, int DIR, typename E, typename C>
__device__ __forceinline__ void pass_compute(E (&v)[16], int t, const C* __restrict__ tw) {
    constexpr int G = 16 / R;
    constexpr int T = N / 16;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if constexpr (S > 1) {
            // w_{S R}^{js m}, from this pass's block of the per-pass table
            const int js = (t + T * g) & (S - 1);
            C w[16];
            group_twiddles<R, S, DIR>(w, tw, js);
#pragma unroll
            for (int m = 1; m < R; ++m) v[g * R + m] = emul(v[g * R + m], w[m]);
        }
        dftR<R, DIR>(v + g * R);
    }
}

// Padded addresses with compile-time offsets.  A pass reads element t + c (c = T g + m N/R) and
// a pass writes element b_t + c (c = T g R + m S, b_t = (t / S) S R + (t mod S)).  Whenever the
// 16-element blocks of c line up (c's part from g a multiple of 16), spad(b + c) =
// spad(b) + c + c / 16, because b's low four bits plus c's never carry: for S >= 16 c's low
// bits are zero; for S < 16, b mod 16 < S when S R >= 16 (m S mod 16 <= 16 - S), and for S = 1,
// b = R t is a multiple of R with m < R.  Each thread then forms one padded base per exchange
// and every access is that base plus an immediate.
template <int R, int S>
constexpr bool blocks_line_up() { return S >= 16 || S * R >= 16 || S == 1; }

template <int N, int R, typename E>
__device__ __forceinline__ void pass_load(E (&v)[16], const E* sm, int t) {
    constexpr int G = 16 / R;
    constexpr int T = N / 16;
    const E* st = sm + spad(t);
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int m = 0; m < R; ++m) {
            const int c = T * g + m * (N / R);  // a constant once unrolled
            v[g * R + m] = (c % 16 == 0) ? st[c + (c >> 4)] : sm[spad(t + c)];
        }
}

template <int N, int R, int S, typename E>
__device__ __forceinline__ void pass_store(const E (&v)[16], E* sm, int t) {
    constexpr int G = 16 / R;
    constexpr int T = N / 16;
    if constexpr ((T % S == 0 || G == 1) && blocks_line_up<R, S>()) {
        const int bt = (t / S) * S * R + (t & (S - 1));
        E* sb = sm + spad(bt);
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int m = 0; m < R; ++m) {
                const int c = T * g * R + m * S;
                if ((T * g * R) % 16 == 0) sb[c + (c >> 4)] = v[g * R + m];
                else sm[spad(bt + c)] = v[g * R + m];
            }
    } else {
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const int j = t + T * g;
            const int base = (j / S) * S * R + (j & (S - 1));
#pragma unroll
            for (int m = 0; m < R; ++m) sm[spad(base + m * S)] = v[g * R + m];
        }
    }
}

// Group G of pass_radix2_half and the groups after it, each rotation formed where it is used
// (fewer live registers than forming all eight first).
template <int DIR, int G, typename E, typename C>
__device__ __forceinline__ void radix2_half_group(E (&v)[16], const C w1) {
    if constexpr (G < 8) {
        v[G * 2 + 1] = emul(v[G * 2 + 1], rot16<DIR, G>(w1));
        dft2<DIR>(v + G * 2);
        radix2_half_group<DIR, G + 1>(v, w1);
    }
}

// Twiddled pass of radix 2 at stride S = N/2 (the last inverse pass of N = 2 * 16^k): group g of
// thread t has js = t + (N/16) g, so w^js = w^t * exp(DIR 2 pi i g / 16): one table load per
// thread and constant rotations instead of one load per group.
template <int N, int DIR, typename E, typename C>
__device__ __forceinline__ void pass_radix2_half(E (&v)[16], int t, const C* __restrict__ tw) {
    const C w1 = tw_load<DIR>(tw, t);
    radix2_half_group<DIR, 0>(v, w1);
}

// pass_compute, with pass_radix2_half for the radix-2 pass at stride N/2.
template <int N, int R, int S, int DIR, typename E, typename C>
__device__ __forceinline__ void pass_compute_h(E (&v)[16], int t, const C* __restrict__ tw) {
    if constexpr (R == 2 && S == N / 2 && N / 16 * 8 == S) pass_radix2_half<N, DIR>(v, t, tw);
    else pass_compute<N, R, S, DIR>(v, t, tw);
}

// Full transform.  On entry v holds the input in the pattern of pass 0 (in_pos with radix
// radix(INV, 0)); on exit v holds the output at in_pos with the last pass's radix.  `sm` is this
// sequence's padded shared buffer; every thread of the CTA must call (barriers inside).  TWINV
// picks the table blocks: a forward transform whose passes have the inverse's radices and
// strides (N = 16^k) may read the inverse blocks, conjugated.
template <int N, bool INV, bool WARP = false, bool TWINV = INV, typename E, typename C>
__device__ __forceinline__ void block_fft(E (&v)[16], E* sm, int t, const C* __restrict__ tw) {
    using P = FftPlan<N>;
    static_assert(!WARP || P::T <= 32, "a warp-synchronised transform fits in one warp");
    constexpr int DIR = INV ? 1 : -1;
    static_assert(TWINV == INV || P::R0 == 1, "shared blocks need equal pass structures");
    constexpr int R0 = P::radix(INV, 0), S0 = P::stride(INV, 0);
    pass_compute<N, R0, S0, DIR>(v, t, tw);  // S0 = 1: no twiddles
    if constexpr (P::NP > 1) {
        constexpr int R1 = P::radix(INV, 1), S1 = P::stride(INV, 1);
        pass_store<N, R0, S0>(v, sm, t);
        seq_sync<WARP>();
        pass_load<N, R1>(v, sm, t);
        seq_sync<WARP>();
        pass_compute_h<N, R1, S1, DIR>(v, t, tw + P::tw_offset(TWINV, 1));
        if constexpr (P::NP > 2) {
            constexpr int R2 = P::radix(INV, 2), S2 = P::stride(INV, 2);
            pass_store<N, R1, S1>(v, sm, t);
            seq_sync<WARP>();
            pass_load<N, R2>(v, sm, t);
            seq_sync<WARP>();
            pass_compute_h<N, R2, S2, DIR>(v, t, tw + P::tw_offset(TWINV, 2));
            if constexpr (P::NP > 3) {
                constexpr int R3 = P::radix(INV, 3), S3 = P::stride(INV, 3);
                pass_store<N, R2, S2>(v, sm, t);
                seq_sync<WARP>();
                pass_load<N, R3>(v, sm, t);
                seq_sync<WARP>();
                pass_compute_h<N, R3, S3, DIR>(v, t, tw + P::tw_offset(TWINV, 3));
            }
        }
    }
}

// Exchange between two passes of a Pair transform through a buffer of single complex values
// (half the bytes of a Pair buffer): the `a` sequences move first, then the `b` sequences.
template <int N, int R0, int S0, int R1, bool WARP = false, typename T>
__device__ __forceinline__ void exchange_halves(Pair<T> (&v)[16], cplx<T>* sm, int t) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        cplx<T> u[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) u[e] = h == 0 ? v[e].a : v[e].b;
        pass_store<N, R0, S0>(u, sm, t);
        seq_sync<WARP>();
        pass_load<N, R1>(u, sm, t);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            if (h == 0) v[e].a = u[e];
            else v[e].b = u[e];
        }
        seq_sync<WARP>();
    }
}

// block_fft of Pair elements with the exchanges of exchange_halves: `sm` holds
// FftPlan<N>::SMEM complex values instead of Pairs.
template <int N, bool INV, bool WARP = false, bool TWINV = INV, typename T, typename C>
__device__ __forceinline__ void block_fft_halves(Pair<T> (&v)[16], cplx<T>* sm, int t,
                                                 const C* __restrict__ tw) {
    using P = FftPlan<N>;
    static_assert(TWINV == INV || P::R0 == 1, "shared blocks need equal pass structures");
    constexpr int DIR = INV ? 1 : -1;
    constexpr int R0 = P::radix(INV, 0), S0 = P::stride(INV, 0);
    pass_compute<N, R0, S0, DIR>(v, t, tw);
    if constexpr (P::NP > 1) {
        constexpr int R1 = P::radix(INV, 1), S1 = P::stride(INV, 1);
        exchange_halves<N, R0, S0, R1, WARP>(v, sm, t);
        pass_compute_h<N, R1, S1, DIR>(v, t, tw + P::tw_offset(TWINV, 1));
        if constexpr (P::NP > 2) {
            constexpr int R2 = P::radix(INV, 2), S2 = P::stride(INV, 2);
            exchange_halves<N, R1, S1, R2, WARP>(v, sm, t);
            pass_compute_h<N, R2, S2, DIR>(v, t, tw + P::tw_offset(TWINV, 2));
            if constexpr (P::NP > 3) {
                constexpr int R3 = P::radix(INV, 3), S3 = P::stride(INV, 3);
                exchange_halves<N, R2, S2, R3, WARP>(v, sm, t);
                pass_compute_h<N, R3, S3, DIR>(v, t, tw + P::tw_offset(TWINV, 3));
            }
        }
    }
}

// ---------------------------------------------------------------------------- split transforms
// A transform of length N = 2 M, M = 16^k (N = 32, 512, 8192), as two length-M halves, one per
// half of the sequence's T = N/16 threads, joined by one radix-2 step:
//   inverse (decimation in time): the halves transform the even and the odd inputs (E, O) and
//     x_n = E_n + w^n O_n, x_{n+M} = E_n - w^n O_n, w = exp(2 pi i / N);
//   forward (decimation in frequency): a_j = x_j + x_{j+M}, b_j = (x_j - x_{j+M}) w^-j, and
//     the halves transform a (the even outputs) and b (the odd outputs).
// A thread's role r: half h = r / (T/2), sub-role s = r mod (T/2).  The radix-2 step needs E_n and
// O_n in one thread while the halves leave them in roles s and s + T/2, so each thread keeps
// eight of its sixteen values and trades the other eight with role r ^ (T/2).  split_role puts
// the two roles in lanes l and l ^ 16 of one warp (T > 32: bits 4 and log2(T) - 1 of the
// thread index swapped; T <= 32: lanes l and l ^ (T/2)): eight warp shuffles of one element
// instead of a shared-memory exchange of sixteen, on each side of the pointwise work.
// Patterns: the inverse takes element tau + m N/16 in slot m and the forward leaves element
// tau + m N/16 in slot m, tau = split_tau(r) = 2 s + h; in between, slot 2g holds x_j and slot
// 2g + 1 holds x_{j+M}, j = r + T g.  Table: FftPlan<N>'s; the halves' passes (radix 16,
// strides 1, 16, 256) are its first inverse passes, and its radix-2 block holds w^js, js < M.
template <int N>
constexpr bool split_plan() { return FftPlan<N>::R0 == 2; }

template <int T>
__device__ __forceinline__ int split_role(int p) {
    if constexpr (T <= 32) {
        return p;
    } else {
        constexpr int HB = ilog2(T) - 1;
        const int b4 = (p >> 4) & 1, bt = (p >> HB) & 1;
        return (p & ~((1 << 4) | (1 << HB))) | (b4 << HB) | (bt << 4);
    }
}

template <int T>
__device__ __forceinline__ int split_tau(int r) { return 2 * (r % (T / 2)) + r / (T / 2); }

template <typename T>
__device__ __forceinline__ T shfl_xor_e(T x, int lm) { return __shfl_xor_sync(0xffffffffu, x, lm); }
__device__ __forceinline__ float2 shfl_xor_e(float2 x, int lm) {
    return make_float2(shfl_xor_e(x.x, lm), shfl_xor_e(x.y, lm));
}
__device__ __forceinline__ double2 shfl_xor_e(double2 x, int lm) {
    return make_double2(shfl_xor_e(x.x, lm), shfl_xor_e(x.y, lm));
}
template <typename T>
__device__ __forceinline__ Pair<T> shfl_xor_e(Pair<T> x, int lm) {
    return {shfl_xor_e(x.a, lm), shfl_xor_e(x.b, lm)};
}

// Half h = 0 keeps the even slots and takes its partner's even slots into its odd ones; half
// h = 1 keeps the odd slots and takes its partner's odd slots into its even ones.
template <int T, typename E>
__device__ __forceinline__ void half_trade(E (&v)[16], int h) {
    constexpr int LM = T > 32 ? 16 : T / 2;
#pragma unroll
    for (int g = 0; g < 8; ++g) {
        const E got = shfl_xor_e(h ? v[2 * g] : v[2 * g + 1], LM);
        if (h) v[2 * g] = got;
        else v[2 * g + 1] = got;
    }
}

template <int G, typename E, typename C>
__device__ __forceinline__ void dif_radix2_group(E (&v)[16], const C w1) {
    if constexpr (G < 8) {
        dft2<-1>(v + G * 2);
        v[G * 2 + 1] = emul(v[G * 2 + 1], rot16<-1, G>(w1));
        dif_radix2_group<G + 1>(v, w1);
    }
}

template <int N>
constexpr bool split_tables_agree() {
    using P = FftPlan<N>;
    using Q = FftPlan<N / 2>;
    for (int p = 1; p < Q::NP; ++p)
        if (Q::tw_offset(true, p) != P::tw_offset(true, p)) return false;
    return P::radix(true, P::NP - 1) == 2 && P::stride(true, P::NP - 1) == N / 2;
}

// One half's transform of a split transform: block_fft when the buffer holds the element type,
// block_fft_halves for Pair elements exchanged through a buffer of single complex values.
template <int N, bool INV, bool WARP, bool TWINV, typename E, typename S, typename C>
__device__ __forceinline__ void half_fft(E (&v)[16], S* sm, int s, const C* __restrict__ tw) {
    if constexpr (std::is_same_v<E, S>) block_fft<N, INV, WARP, TWINV>(v, sm, s, tw);
    else block_fft_halves<N, INV, WARP, TWINV>(v, sm, s, tw);
}

// Inverse split transform: slot m holds element split_tau(r) + m N/16 on entry; slot 2g holds
// x_j and slot 2g + 1 holds x_{j + N/2}, j = r + (N/16) g, on exit.  `sm`: FftPlan<N>::SMEM
// elements or, for Pair elements, single complex values (the two halves' buffers); every
// thread of the CTA calls (barriers inside).
template <int N, bool WARP = false, typename E, typename S, typename C>
__device__ __forceinline__ void split_inverse(E (&v)[16], S* sm, int r, const C* __restrict__ tw) {
    static_assert(split_plan<N>() && split_tables_agree<N>(), "N = 2 16^k");
    using P = FftPlan<N>;
    constexpr int H = P::T / 2;
    const int h = r / H;
    half_fft<N / 2, true, WARP, true>(v, sm + h * FftPlan<N / 2>::SMEM, r - h * H, tw);
    half_trade<P::T>(v, h);
    radix2_half_group<1, 0>(v, tw_load<1>(tw + P::tw_offset(true, P::NP - 1), r));
}

// Forward split transform: the exit pattern of split_inverse on entry; slot m holds element
// split_tau(r) + m N/16 on exit.
template <int N, bool WARP = false, typename E, typename S, typename C>
__device__ __forceinline__ void split_forward(E (&v)[16], S* sm, int r, const C* __restrict__ tw) {
    static_assert(split_plan<N>() && split_tables_agree<N>(), "N = 2 16^k");
    using P = FftPlan<N>;
    constexpr int H = P::T / 2;
    const int h = r / H;
    dif_radix2_group<0>(v, tw_load<-1>(tw + P::tw_offset(true, P::NP - 1), r));
    half_trade<P::T>(v, h);
    half_fft<N / 2, false, WARP, true>(v, sm + h * FftPlan<N / 2>::SMEM, r - h * H, tw);
}

// The transform of one sequence by thread t of its N/16: the split form when N = 2 16^k,
// block_fft (or block_fft_halves for Pair elements through a single complex buffer) otherwise.
// Frequency side (inverse input, forward output): slot m holds index spec_base(t) + m N/16.
// Sample side (inverse output, forward input): slot g R + m holds in_pos<N, R>(phys_base(t),
// g, m), R = last_radix<N, true>() = first_radix<N, false>().
template <int N, bool INV, bool WARP = false, typename E, typename S, typename C>
__device__ __forceinline__ void seq_fft(E (&v)[16], S* sm, int t, const C* __restrict__ tw) {
    if constexpr (split_plan<N>()) {
        if constexpr (INV) split_inverse<N, WARP>(v, sm, split_role<N / 16>(t), tw);
        else split_forward<N, WARP>(v, sm, split_role<N / 16>(t), tw);
    } else {
        half_fft<N, INV, WARP, INV>(v, sm, t, tw);
    }
}
template <int N>
__device__ __forceinline__ int spec_base(int t) {
    if constexpr (split_plan<N>()) return split_tau<N / 16>(split_role<N / 16>(t));
    else return t;
}
template <int N>
__device__ __forceinline__ int phys_base(int t) {
    if constexpr (split_plan<N>()) return split_role<N / 16>(t);
    else return t;
}

// radix of the last pass (output pattern) and of the first pass (input pattern)
template <int N, bool INV>
constexpr int first_radix() { return FftPlan<N>::radix(INV, 0); }
template <int N, bool INV>
constexpr int last_radix() { return FftPlan<N>::radix(INV, FftPlan<N>::NP - 1); }

}  // namespace sp
