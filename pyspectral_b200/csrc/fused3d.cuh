// Fused 3D IF-RK4 stage on hand-written FFTs: four passes per stage over the kept modes only.
//
// The 2/3 rule keeps |kx|, |ky| <= KM and kz <= KM (KM = (n-1)/3), so of the n x n x (n/2+1)
// modes only (2KM+1)^2 (KM+1) are ever non-zero — about 30 %.  The stage runs as four passes,
// each a sweep of 1D transforms along one axis with the pointwise work of that point fused in:
//
//   Y-inverse : B_spec -> B_phys   (inverse along y, f < n_inv)
//   Z         : per line (x, y): c2r along z of the velocity (and vorticity) fields, the
//               physical-space products (Basdevant stress / u x omega), r2c along z of the
//               products, kept kz only; in place in B_phys
//   Y-forward : B_phys -> B_spec (forward along y, kept ky only, f < n_fwd)
//   X         : per column (ky', kz pair): forward along x of the products, then for every
//               kept kx the divergence / Leray projection / integrating factor / Lawson update
//               of the state and accumulator and the next stage's inputs, then inverse along x
//               of those inputs; in place in B_spec
//
// ky' and kx' index the kept wavenumbers -KM..KM (0..KM, then -KM..-1); kz is padded to a
// multiple of four so two adjacent kz columns move as one Pair (16 bytes in fp32) and the
// pairs per row are even: every 1D transform of the Y and X passes is a Pair transform of two
// kz columns sharing twiddles.  B_spec interleaves x in pairs innermost,
// B_spec[x/2][f][ky'][q][x%2] (q = kz pair), and B_phys keeps whole z lines,
// B_phys[x][f][y][q].  An X-pass CTA holds two adjacent kz pairs of one ky' (its lanes t, t+1
// hold x, x+1): runs of 64 bytes of B_spec.  A Y-pass CTA holds (x, x+1) x two adjacent kz
// pairs: runs of 64 bytes of B_spec and 32 of B_phys.
// Each transform is one warp's (n <= 512: n/16 threads, 16 elements per thread; several
// transforms per warp below n = 512), and its exchanges are warp-synchronised.  The state and
// the accumulator live as compact copies of the kept modes, [c][ky'][kz][kx'] (kx' fastest, so
// the X pass reads and writes them in whole rows); the NumPy-layout state u0 is refreshed from
// the compact state only when it is read (k3_state_move).
//
// Equations (the reference's pre3d / phys3d_basd / phys3d_rot / post3d,
// src/pyspectral/kernels/spectral.cu:164-238): Basdevant T = (uu - q, vv - q, uv, uw, vw),
// q = |u|^2 / 3, N_i = -i k_j T_ij with T33 = -(T11 + T22); rotational N = (u x omega)^,
// omega = i k x u; Leray N <- N - k (k.N) / k^2; Lawson stage update (common.cuh).
#pragma once

#include <utility>

#include "common.cuh"
#include "fft_block.cuh"
#include "tma.cuh"

namespace sp {
namespace f3 {

template <int N>
struct Dims {
    static constexpr int KM = (N - 1) / 3;     // largest kept |k| (3 |k| < n)
    static constexpr int KZ = KM + 1;          // kept kz: 0..KM
    static constexpr int KK = 2 * KM + 1;      // kept kx, ky: -KM..KM
    static constexpr int NQ = (KZ + 3) / 4 * 2;  // kz pairs per row (even)
    static constexpr int KZP = 2 * NQ;            // kz extent, padded
    static constexpr int T = N / 16;           // threads per transform
    static constexpr int SEQ = T >= 32 ? 1 : 32 / T;  // transforms per warp
    static_assert(N >= 16 && N <= 512 && (N & (N - 1)) == 0, "n a power of two, 16..512");
};

// Field slots of the work arrays: Basdevant 5 (u, v, w in; 5 stress components out),
// rotational 6 (u, omega in; u x omega out).
template <bool ROT> constexpr int nslot() { return ROT ? 6 : 5; }
template <bool ROT> constexpr int ninv() { return ROT ? 6 : 3; }
template <bool ROT> constexpr int nfwd() { return ROT ? 3 : 5; }

// signed wavenumber of kept index ki, and the kept index of FFT index i (which must be kept)
template <int N>
__device__ __forceinline__ int kept_k(int ki) {
    return ki <= Dims<N>::KM ? ki : ki - Dims<N>::KK;
}
template <int N>
__device__ __forceinline__ int kept_of_fft(int i) {
    return i <= Dims<N>::KM ? i : i - N + Dims<N>::KK;
}

template <typename F, int... M>
__device__ __forceinline__ void for_slots_impl(F&& f, std::integer_sequence<int, M...>) {
    (f(std::integral_constant<int, M>{}), ...);
}
// f(integral_constant<int, M>) for the 16 register slots
template <typename F>
__device__ __forceinline__ void for_slots(F&& f) {
    for_slots_impl(f, std::make_integer_sequence<int, 16>{});
}

// Register slot M on the frequency side of a transform (inverse input, forward output) holds
// FFT index k = k0 + M n/16, k0 = spec_base(thread) < n/16.  Kind of the slot against the kept set [0, KM] u [n - KM, n): 0 = all kept
// low, 1 = all kept high, 2 = none kept, 3 = mixed (decided per thread).
template <int N, int M>
constexpr int slot_kind() {
    constexpr int KM = Dims<N>::KM, L = N / 16, LO = M * L, HI = LO + L - 1;
    if (HI <= KM) return 0;
    if (LO >= N - KM) return 1;
    if (LO > KM && HI < N - KM) return 2;
    return 3;
}

// value of slot M: load_lo(k) for a kept low k, load_hi(k) for a kept high k, else zero
template <int N, int M, typename E, typename Lo, typename Hi>
__device__ __forceinline__ E slot_value(int k0, Lo&& load_lo, Hi&& load_hi, E zero) {
    constexpr int kind = slot_kind<N, M>();
    const int k = k0 + M * (N / 16);
    if constexpr (kind == 0) return load_lo(k);
    else if constexpr (kind == 1) return load_hi(k);
    else if constexpr (kind == 2) return zero;
    else {
        if (k <= Dims<N>::KM) return load_lo(k);
        if (k >= N - Dims<N>::KM) return load_hi(k);
        return zero;
    }
}

// store(k) for slot M when its k is kept
template <int N, int M, typename St>
__device__ __forceinline__ void slot_store(int k0, St&& store) {
    constexpr int kind = slot_kind<N, M>();
    const int k = k0 + M * (N / 16);
    if constexpr (kind == 0 || kind == 1) store(k);
    else if constexpr (kind == 3) {
        if (k <= Dims<N>::KM || k >= N - Dims<N>::KM) store(k);
    }
}

template <typename T>
__device__ __forceinline__ Pair<T> pzero() {
    return Pair<T>{mk<T>(0, 0), mk<T>(0, 0)};
}

// Work-array indices in Pair units (two kz columns): B_spec [x/2][f][ky'][q][x%2],
// B_phys [x][f][y][q].
template <int N, bool ROT>
__device__ __forceinline__ size_t spec_idx(int x, int f, int ky, int q) {
    return (((((size_t)(x >> 1) * nslot<ROT>() + f) * Dims<N>::KK + ky) * Dims<N>::NQ + q) << 1) |
           (size_t)(x & 1);
}
template <int N, bool ROT>
__device__ __forceinline__ size_t phys_idx(int x, int f, int y, int q) {
    return (((size_t)x * nslot<ROT>() + f) * N + y) * Dims<N>::NQ + q;
}

// Unit of a Y pass: (x, f, q) with x % 2 fastest, then q, f, x / 2 — the consecutive units of
// one CTA are x, x+1 for adjacent kz pairs.
struct YUnit {
    int x, f, q;
};
template <int N>
__device__ __forceinline__ YUnit y_unit(long unit, int nfields) {
    const int xl = (int)(unit & 1);
    const long rest = unit >> 1;
    const int q = (int)(rest % Dims<N>::NQ);
    const long r2 = rest / Dims<N>::NQ;
    return YUnit{2 * (int)(r2 / nfields) + xl, (int)(r2 % nfields), q};
}

// Y passes: 4 warps per CTA (8 measured no faster at 512^3)
template <typename T>
constexpr int y_threads() { return 128; }
// Z pass: 4 warps (fp32) or 2 (fp64), so its static shared memory stays below 48 KB
template <typename T>
constexpr int z_threads() { return sizeof(T) == 4 ? 128 : 64; }

// ------------------------------------------------------------------------------- Y passes
// Inverse along y of fields f < nfields: one Pair transform per (x, f, kz pair).
template <typename T, int N, bool ROT>
__global__ void __launch_bounds__(y_threads<T>()) k3_yinv(const Pair<T>* __restrict__ Bs,
                                                        Pair<T>* __restrict__ Bp, int nfields,
                                                        const cplx<T>* __restrict__ tw) {
    using D = Dims<N>;
    constexpr int TT = D::T;
    constexpr int RIL = last_radix<N, true>();
    __shared__ __align__(16) cplx<T> exch[y_threads<T>() / TT][FftPlan<N>::SMEM];
    const int seq = threadIdx.x / TT, t = threadIdx.x % TT;
    const long units = (long)N * nfields * D::NQ;
    const long unit = (long)blockIdx.x * (y_threads<T>() / TT) + seq;
    const bool active = unit < units;
    const YUnit yu = y_unit<N>(unit, nfields);
    const int x = yu.x, f = yu.f, q = yu.q;
    const int kb = spec_base<N>(t), yb = phys_base<N>(t);
    Pair<T> v[16];
    for_slots([&](auto mc) {
        constexpr int M = decltype(mc)::value;
        auto lo = [&](int k) { return Bs[spec_idx<N, ROT>(x, f, k, q)]; };
        auto hi = [&](int k) { return Bs[spec_idx<N, ROT>(x, f, k - N + D::KK, q)]; };
        v[M] = active ? slot_value<N, M>(kb, lo, hi, pzero<T>()) : pzero<T>();
    });
    seq_fft<N, true, true>(v, exch[seq], t, tw);
    if (active) {
#pragma unroll
        for (int g = 0; g < 16 / RIL; ++g)
#pragma unroll
            for (int m = 0; m < RIL; ++m)
                Bp[phys_idx<N, ROT>(x, f, in_pos<N, RIL>(yb, g, m), q)] = v[g * RIL + m];
    }
}

// Forward along y of fields f < nfields, kept ky only.
template <typename T, int N, bool ROT>
__global__ void __launch_bounds__(y_threads<T>()) k3_yfwd(const Pair<T>* __restrict__ Bp,
                                                        Pair<T>* __restrict__ Bs, int nfields,
                                                        const cplx<T>* __restrict__ tw) {
    using D = Dims<N>;
    constexpr int TT = D::T;
    constexpr int RF0 = first_radix<N, false>();
    __shared__ __align__(16) cplx<T> exch[y_threads<T>() / TT][FftPlan<N>::SMEM];
    const int seq = threadIdx.x / TT, t = threadIdx.x % TT;
    const long units = (long)N * nfields * D::NQ;
    const long unit = (long)blockIdx.x * (y_threads<T>() / TT) + seq;
    const bool active = unit < units;
    const YUnit yu = y_unit<N>(unit, nfields);
    const int x = yu.x, f = yu.f, q = yu.q;
    const int kb = spec_base<N>(t), yb = phys_base<N>(t);
    Pair<T> v[16];
#pragma unroll
    for (int g = 0; g < 16 / RF0; ++g)
#pragma unroll
        for (int m = 0; m < RF0; ++m)
            v[g * RF0 + m] =
                active ? Bp[phys_idx<N, ROT>(x, f, in_pos<N, RF0>(yb, g, m), q)] : pzero<T>();
    seq_fft<N, false, true>(v, exch[seq], t, tw);
    if (active) {
        for_slots([&](auto mc) {
            constexpr int M = decltype(mc)::value;
            slot_store<N, M>(kb, [&](int k) { Bs[spec_idx<N, ROT>(x, f, kept_of_fft<N>(k), q)] = v[M]; });
        });
    }
}

// ------------------------------------------------------------------------------- Z pass
// Largest |value| as a bit pattern for atomicMax; a NaN wins, as in a NaN-propagating max.
__device__ __forceinline__ unsigned long long max_bits(double m, bool nan) {
    return nan ? 0x7ff8000000000000ull : (unsigned long long)__double_as_longlong(m);
}

// Hermitian completion along z of two real fields' half spectra a(kz), b(kz) (kz <= KM): the
// value at FFT index k of Z = A + i B.
template <typename T>
__device__ __forceinline__ cplx<T> herm_pair_lo(cplx<T> a, cplx<T> b, int k) {
    if (k == 0) return mk<T>(a.x, b.x);  // c2r ignores Im at k = 0
    return mk<T>(a.x - b.y, a.y + b.x);
}
template <typename T>
__device__ __forceinline__ cplx<T> herm_pair_hi(cplx<T> a, cplx<T> b) {  // a, b at n - k
    return mk<T>(a.x + b.y, b.x - a.y);
}

// MODE 0: the stage's Z pass (inverse, products, forward).  MODE 1: inverse of the velocity
// only and max |u_i| into umax[0..3) (CFL bound; nothing written back).
template <typename T, int N, bool ROT, int MODE>
__global__ void __launch_bounds__(z_threads<T>()) k3_z(Pair<T>* __restrict__ Bp,
                                                       const cplx<T>* __restrict__ tw,
                                                       unsigned long long* __restrict__ umax,
                                                       int want_max) {
    using D = Dims<N>;
    constexpr int TT = D::T;
    constexpr int ZT = z_threads<T>();
    constexpr int NS = ZT / TT;
    __shared__ __align__(16) cplx<T> exch[NS][FftPlan<N>::SMEM];
    // each thread's 16 points of (omega_y, omega_z) (rotational) or of v w (Basdevant), kept
    // in shared memory between the transforms (thread-private)
    __shared__ __align__(16) cplx<T> stash[MODE == 0 ? 16 : 1][MODE == 0 ? ZT : 1];
    const int seq = threadIdx.x / TT, t = threadIdx.x % TT;
    const long line = (long)blockIdx.x * NS + seq;
    const bool active = line < (long)N * N;
    const int x = (int)(line / N), y = (int)(line % N);
    cplx<T>* B = reinterpret_cast<cplx<T>*>(Bp);
    // complex index of (x, f, y, kz): B_phys rows of whole z lines
    auto at = [&](int f, int kz) -> size_t {
        return (((size_t)x * nslot<ROT>() + f) * N + y) * D::KZP + kz;
    };
    cplx<T>* sm = exch[seq];
    const cplx<T> z0 = mk<T>(0, 0);
    const int kb = spec_base<N>(t);  // the z line's samples stay in registers: no sample index

    Pair<T> v[16];
    if constexpr (ROT && MODE == 0) {
        // (omega_y, omega_z) first, kept in shared memory for the products
        cplx<T> w[16];
        for_slots([&](auto mc) {
            constexpr int M = decltype(mc)::value;
            auto lo = [&](int k) { return herm_pair_lo<T>(B[at(4, k)], B[at(5, k)], k); };
            auto hi = [&](int k) { return herm_pair_hi<T>(B[at(4, N - k)], B[at(5, N - k)]); };
            w[M] = active ? slot_value<N, M>(kb, lo, hi, z0) : z0;
        });
        seq_fft<N, true, true>(w, sm, t, tw);
#pragma unroll
        for (int e = 0; e < 16; ++e) stash[e][threadIdx.x] = w[e];
    }
    for_slots([&](auto mc) {
        constexpr int M = decltype(mc)::value;
        auto lo = [&](int k) {
            cplx<T> wz;
            if (ROT && MODE == 0) wz = herm_pair_lo<T>(B[at(2, k)], B[at(3, k)], k);
            else wz = k == 0 ? mk<T>(B[at(2, 0)].x, (T)0) : B[at(2, k)];
            return Pair<T>{herm_pair_lo<T>(B[at(0, k)], B[at(1, k)], k), wz};
        };
        auto hi = [&](int k) {
            const int kk = N - k;
            cplx<T> wz;
            if (ROT && MODE == 0) {
                wz = herm_pair_hi<T>(B[at(2, kk)], B[at(3, kk)]);
            } else {
                const cplx<T> c = B[at(2, kk)];
                wz = mk<T>(c.x, -c.y);
            }
            return Pair<T>{herm_pair_hi<T>(B[at(0, kk)], B[at(1, kk)]), wz};
        };
        v[M] = active ? slot_value<N, M>(kb, lo, hi, pzero<T>()) : pzero<T>();
    });
    seq_fft<N, true, true>(v, sm, t, tw);  // v[e] = (u + i v, w + i (omega_x or 0))

    if (want_max) {
        double mu = 0.0, mv = 0.0, mw = 0.0;
        bool nu = false, nv = false, nw = false;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const double a = (double)v[e].a.x, b = (double)v[e].a.y, c = (double)v[e].b.x;
            nu |= a != a;
            nv |= b != b;
            nw |= c != c;
            mu = fmax(mu, fabs(a));
            mv = fmax(mv, fabs(b));
            mw = fmax(mw, fabs(c));
        }
        unsigned long long bu = max_bits(mu, nu), bv = max_bits(mv, nv), bw = max_bits(mw, nw);
        if (!active) bu = bv = bw = 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bu = max(bu, __shfl_down_sync(0xffffffffu, bu, o));
            bv = max(bv, __shfl_down_sync(0xffffffffu, bv, o));
            bw = max(bw, __shfl_down_sync(0xffffffffu, bw, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(umax + 0, bu);
            atomicMax(umax + 1, bv);
            atomicMax(umax + 2, bw);
        }
    }

    if constexpr (MODE == 0) {
        // physical-space products, packed two real fields per complex sequence
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const T u = v[e].a.x, vv = v[e].a.y, w = v[e].b.x;
            if constexpr (ROT) {
                const T ox = v[e].b.y;
                const cplx<T> o = stash[e][threadIdx.x];  // (omega_y, omega_z)
                const T p1 = vv * o.y - w * o.x, p2 = w * ox - u * o.y, p3 = u * o.x - vv * ox;
                v[e].a = mk<T>(p1, p2);
                v[e].b = mk<T>(p3, (T)0);
            } else {
                const T q = (u * u + vv * vv + w * w) * ((T)1 / (T)3);
                stash[e][threadIdx.x] = mk<T>(vv * w, (T)0);
                v[e].a = mk<T>(u * u - q, vv * vv - q);
                v[e].b = mk<T>(u * vv, u * w);
            }
        }
        seq_fft<N, false, true>(v, sm, t, tw);  // output slot M: k = kb + M n/16
        // split Z' = F(p + i q): P(k) = (Z'(k) + conj Z'(n-k)) / 2,
        // Q(k) = (Z'(k) - conj Z'(n-k)) / 2i
        constexpr int NSPLIT = ROT ? 1 : 2;
#pragma unroll
        for (int h = 0; h < NSPLIT; ++h) {
            __syncwarp();
#pragma unroll
            for (int e = 0; e < 16; ++e) sm[spad(kb + e * TT)] = h == 0 ? v[e].a : v[e].b;
            __syncwarp();
#pragma unroll
            for (int j = 0; j < (D::KZ + TT - 1) / TT; ++j) {
                const int k = t + j * TT;
                if (active && ((j + 1) * TT <= D::KZ || k < D::KZ)) {
                    const cplx<T> a = sm[spad(k)], b = sm[spad((N - k) & (N - 1))];
                    B[at(2 * h, k)] = mk<T>((T)0.5 * (a.x + b.x), (T)0.5 * (a.y - b.y));
                    B[at(2 * h + 1, k)] = mk<T>((T)0.5 * (a.y + b.y), (T)0.5 * (b.x - a.x));
                }
            }
        }
        if constexpr (ROT) {
            // the third product had a zero imaginary part: its r2c coefficients are Z'(k)
            if (active) {
                for_slots([&](auto mc) {
                    constexpr int M = decltype(mc)::value;
                    const int k = kb + M * TT;
                    if (M * TT < D::KZ && k < D::KZ) B[at(2, k)] = v[M].b;
                });
            }
        } else {
            __syncwarp();
            cplx<T> w[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) w[e] = stash[e][threadIdx.x];  // (v w, 0)
            seq_fft<N, false, true>(w, sm, t, tw);
            if (active) {
                for_slots([&](auto mc) {
                    constexpr int M = decltype(mc)::value;
                    const int k = kb + M * TT;
                    if (M * TT < D::KZ && k < D::KZ) B[at(4, k)] = w[M];
                });
            }
        }
    }
}

// ------------------------------------------------------------------------------- X pass
// A CTA holds U units (ky', q) = blockIdx.x U + u: G groups of field warps (one warp per field
// slot), each warp SEQ transforms.  U = 2 (two adjacent kz pairs) except in fp64 at n = 512,
// where the shared memory holds one.  STAGE -1: the stage-0 inputs from the state (no forward
// transform, no update).
template <typename T, int N, bool ROT>
struct XPass {
    using D = Dims<N>;
    static constexpr int S = D::SEQ;
    // rotational form (six fields) at n = 512 in fp32: one kz pair per CTA and three CTAs per
    // SM, which leaves the pass its registers (two pairs of 12 warps at two CTAs spill)
    static constexpr bool ONE_PAIR_ROT = ROT && sizeof(T) == 4 && S == 1;
    static constexpr int G = (S >= 2 || sizeof(T) == 8 || ONE_PAIR_ROT) ? 1 : 2;
    static constexpr int MIN_BLOCKS = ONE_PAIR_ROT ? 3 : 2;
    static constexpr int U = G * S;
    static constexpr int WARPS = G * nslot<ROT>();
    static constexpr int THREADS = WARPS * 32;
    static constexpr size_t stage_bytes() {
        return (size_t)U * nslot<ROT>() * D::KK * sizeof(Pair<T>);
    }
    static constexpr size_t smem_bytes() {
        return stage_bytes() + (size_t)WARPS * S * FftPlan<N>::SMEM * sizeof(cplx<T>);
    }
    static constexpr long UNITS = (long)D::KK * D::NQ;
};

// Index of kept mode (c, ky', kz, kx') in the compact state / accumulator.
template <int N>
__device__ __forceinline__ size_t compact_idx(int c, int kyi, int kz, int kxi) {
    using D = Dims<N>;
    return (((size_t)c * D::KK + kyi) * D::KZ + kz) * D::KK + kxi;
}

template <typename T, int N, bool ROT, int STAGE>
__global__ void __launch_bounds__(XPass<T, N, ROT>::THREADS, XPass<T, N, ROT>::MIN_BLOCKS) k3_x(
    Pair<T>* __restrict__ Bs, cplx<T>* __restrict__ u0, cplx<T>* __restrict__ acc,
    const T* __restrict__ tab, const StepParams<T>* __restrict__ P,
    const cplx<T>* __restrict__ tw) {
    using D = Dims<N>;
    using X = XPass<T, N, ROT>;
    constexpr int TT = D::T, S = X::S, U = X::U, KK = D::KK, NF = nslot<ROT>();
    constexpr int NIN = ninv<ROT>(), NFW = nfwd<ROT>();
    constexpr int RF0 = first_radix<N, false>(), RIL = last_radix<N, true>();
    constexpr int NH = N / 2 + 1;
    extern __shared__ __align__(16) unsigned char xsm[];
    Pair<T>* stage = reinterpret_cast<Pair<T>*>(xsm);  // [u][f][kx']
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fw = warp % NF;                               // this warp's field slot
    const int sub = (warp / NF) * S + lane / TT, t = lane % TT;  // this sequence's unit in the CTA
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(xsm + X::stage_bytes()) +
                  (size_t)(warp * S + lane / TT) * FftPlan<N>::SMEM;
    const long unit = (long)blockIdx.x * U + sub;
    const bool active = unit < X::UNITS;
    const int q = (int)(unit % D::NQ), kyi = (int)(unit / D::NQ);
    const int kb = spec_base<N>(t), xb = phys_base<N>(t);
    const StepParams<T> p = *P;
    // thread 0: the CTA's compact state (and accumulator) rows into L2 while the forward
    // transforms run (bulk prefetches of whole 16-byte blocks inside each row range)
    if (threadIdx.x == 0) {
        constexpr size_t CS = (size_t)KK * D::KZ * KK;  // one component
        for (int s = 0; s < U; ++s) {
            const long us = (long)blockIdx.x * U + s;
            if (us >= X::UNITS) break;
            const int qs = (int)(us % D::NQ), kyis = (int)(us / D::NQ);
            const int nkz = D::KZ - 2 * qs < 2 ? D::KZ - 2 * qs : 2;
            if (nkz <= 0) continue;
            const size_t e0 = compact_idx<N>(0, kyis, 2 * qs, 0);
            for (int c = 0; c < (STAGE > 0 ? 6 : 3); ++c) {
                const cplx<T>* base = c < 3 ? u0 + c * CS : acc + (c - 3) * CS;
                const uintptr_t b0 = (uintptr_t)(base + e0);
                const uintptr_t b1 = b0 + (uintptr_t)nkz * KK * sizeof(cplx<T>);
                const uintptr_t a0 = (b0 + 15) & ~(uintptr_t)15, a1 = b1 & ~(uintptr_t)15;
                if (a1 > a0) tma::prefetch_l2((const void*)a0, (uint32_t)(a1 - a0));
            }
        }
    }
    auto st_at = [&](int s, int f, int kxi) -> Pair<T>& {
        return stage[((size_t)s * NF + f) * KK + kxi];
    };

    // forward along x of the products, kept kx into the staging buffer
    if constexpr (STAGE >= 0) {
        if (fw < NFW) {
            const int f = fw;
            Pair<T> v[16];
#pragma unroll
            for (int g = 0; g < 16 / RF0; ++g)
#pragma unroll
                for (int m = 0; m < RF0; ++m)
                    v[g * RF0 + m] = active ? Bs[spec_idx<N, ROT>(in_pos<N, RF0>(xb, g, m), f, kyi, q)]
                                            : pzero<T>();
            seq_fft<N, false, true>(v, sm, t, tw);
            for_slots([&](auto mc) {
                constexpr int M = decltype(mc)::value;
                slot_store<N, M>(kb, [&](int k) { st_at(sub, f, kept_of_fft<N>(k)) = v[M]; });
            });
        }
        __syncthreads();
    }

    // every kept kx of the CTA's columns, one kz column at a time (kx' fastest: the compact
    // state and accumulator rows are read and written contiguously): update and next inputs
#pragma unroll 2
    for (int e = threadIdx.x; e < U * 2 * KK; e += X::THREADS) {
        const int kxi = e % KK, sh = e / KK, s = sh >> 1, h = sh & 1;
        const long us = (long)blockIdx.x * U + s;
        if (us >= X::UNITS) continue;
        const int qs = (int)(us % D::NQ), kyis = (int)(us / D::NQ);
        const int kzi = 2 * qs + h;
        cplx<T> out[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) out[c] = mk<T>(0, 0);
        if (kzi < D::KZ) {  // else the padding column: zero inputs
            const int kxs = kept_k<N>(kxi), kys = kept_k<N>(kyis);
            const T kx = (T)kxs, ky = (T)kys, kz = (T)kzi, k2 = kx * kx + ky * ky + kz * kz;
            const size_t o = compact_idx<N>(0, kyis, kzi, kxi);
            constexpr size_t CS = (size_t)D::KK * D::KZ * D::KK;  // one component
            cplx<T> a = u0[o], b = u0[CS + o], c = u0[2 * CS + o];
            if constexpr (STAGE >= 0) {
                cplx<T> F[NFW];
#pragma unroll
                for (int f = 0; f < NFW; ++f) {
                    const Pair<T> pf = st_at(s, f, kxi);
                    F[f] = h ? pf.b : pf.a;
                }
                cplx<T> N0, N1, N2;
                if constexpr (ROT) {
                    N0 = F[0];
                    N1 = F[1];
                    N2 = F[2];
                } else {
                    const cplx<T> t11 = F[0], t22 = F[1], t12 = F[2], t13 = F[3], t23 = F[4];
                    const cplx<T> t33 = mk<T>(-(t11.x + t22.x), -(t11.y + t22.y));
                    N0 = mul_mi(add(add(scl(kx, t11), scl(ky, t12)), scl(kz, t13)));
                    N1 = mul_mi(add(add(scl(kx, t12), scl(ky, t22)), scl(kz, t23)));
                    N2 = mul_mi(add(add(scl(kx, t13), scl(ky, t23)), scl(kz, t33)));
                }
                // Leray projection N <- N - k (k.N) / k^2
                const T ik2 = k2 > (T)0 ? (T)1 / k2 : (T)0;
                const cplx<T> d = scl(ik2, add(add(scl(kx, N0), scl(ky, N1)), scl(kz, N2)));
                N0 = axpy(-kx, d, N0);
                N1 = axpy(-ky, d, N1);
                N2 = axpy(-kz, d, N2);
                const IFac<T> fac = if_factors(tab, NH, kxs < 0 ? -kxs : kxs,
                                               kys < 0 ? -kys : kys, kzi, k2, p);
                cplx<T> Ca = STAGE > 0 ? acc[o] : mk<T>(0, 0);
                cplx<T> Cb = STAGE > 0 ? acc[CS + o] : mk<T>(0, 0);
                cplx<T> Cc = STAGE > 0 ? acc[2 * CS + o] : mk<T>(0, 0);
                constexpr int SG = STAGE < 0 ? 0 : STAGE;
                a = lawson_stage<T, SG>(p.dt, fac, N0, a, Ca);
                b = lawson_stage<T, SG>(p.dt, fac, N1, b, Cb);
                c = lawson_stage<T, SG>(p.dt, fac, N2, c, Cc);
                if (STAGE == 3) {
                    u0[o] = a;
                    u0[CS + o] = b;
                    u0[2 * CS + o] = c;
                } else {
                    acc[o] = Ca;
                    acc[CS + o] = Cb;
                    acc[2 * CS + o] = Cc;
                }
            }
            // next inputs: u scaled; rotational form also omega = i k x u
            const T sc = p.scale;
            a = scl(sc, a);
            b = scl(sc, b);
            c = scl(sc, c);
            out[0] = a;
            out[1] = b;
            out[2] = c;
            if (ROT) {
                out[3] = mul_i(add(scl(ky, c), scl(-kz, b)));
                out[4] = mul_i(add(scl(kz, a), scl(-kx, c)));
                out[5] = mul_i(add(scl(kx, b), scl(-ky, a)));
            }
        }
#pragma unroll
        for (int c = 0; c < NIN; ++c) {
            Pair<T>& slot = st_at(s, c, kxi);
            if (h) slot.b = out[c];
            else slot.a = out[c];
        }
    }
    __syncthreads();

    // inverse along x of the next inputs
    if (fw < NIN) {
        const int f = fw;
        Pair<T> v[16];
        for_slots([&](auto mc) {
            constexpr int M = decltype(mc)::value;
            auto lo = [&](int k) { return st_at(sub, f, k); };
            auto hi = [&](int k) { return st_at(sub, f, k - N + KK); };
            v[M] = slot_value<N, M>(kb, lo, hi, pzero<T>());
        });
        seq_fft<N, true, true>(v, sm, t, tw);
        if (active) {
#pragma unroll
            for (int g = 0; g < 16 / RIL; ++g)
#pragma unroll
                for (int m = 0; m < RIL; ++m)
                    Bs[spec_idx<N, ROT>(in_pos<N, RIL>(xb, g, m), f, kyi, q)] = v[g * RIL + m];
        }
    }
}

// Compact state <-> NumPy layout: for each (c, ky'), a [kx'][kz] slab of u0 (kz contiguous)
// against the [kz][kx'] slab of the compact copy, through 32 x 33 shared tiles.  IN: u0 ->
// compact; otherwise compact -> u0 (kept modes only; the others stay as they are, zero).
template <typename T, bool IN>
__global__ void __launch_bounds__(256) k3_state_move(cplx<T>* __restrict__ u0,
                                                     cplx<T>* __restrict__ uc, int n) {
    __shared__ cplx<T> tile[32][33];
    const int km = (n - 1) / 3, kz_n = km + 1, kk = 2 * km + 1, nh = n / 2 + 1;
    const int c = blockIdx.z / kk, kyi = blockIdx.z % kk;
    const int ky = kyi <= km ? kyi : kyi - kk;
    const size_t fsc = (size_t)n * n * nh;
    cplx<T>* u = u0 + (size_t)c * fsc + (size_t)(ky < 0 ? ky + n : ky) * nh;  // + kx row * n nh
    cplx<T>* w = uc + ((size_t)c * kk + kyi) * kz_n * kk;                      // [kz][kx']
    const int x0 = blockIdx.y * 32, z0 = blockIdx.x * 32;
    auto kx_row = [&](int kxi) -> size_t {
        const int kx = kxi <= km ? kxi : kxi - kk;
        return (size_t)(kx < 0 ? kx + n : kx) * n * nh;
    };
    if (IN) {
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int kxi = x0 + r, kz = z0 + threadIdx.x;
            if (kxi < kk && kz < kz_n) tile[r][threadIdx.x] = u[kx_row(kxi) + kz];
        }
        __syncthreads();
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int kz = z0 + r, kxi = x0 + threadIdx.x;
            if (kxi < kk && kz < kz_n) w[(size_t)kz * kk + kxi] = tile[threadIdx.x][r];
        }
    } else {
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int kz = z0 + r, kxi = x0 + threadIdx.x;
            if (kxi < kk && kz < kz_n) tile[r][threadIdx.x] = w[(size_t)kz * kk + kxi];
        }
        __syncthreads();
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int kxi = x0 + r, kz = z0 + threadIdx.x;
            if (kxi < kk && kz < kz_n) u[kx_row(kxi) + kz] = tile[threadIdx.x][r];
        }
    }
}

// zero every mode outside the 2/3 mask of the three components (set_state's dealiasing)
template <typename T>
__global__ void __launch_bounds__(256) k3_mask(cplx<T>* __restrict__ u0, int n, int nh,
                                               uint32_t fsc) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= fsc) return;
    const uint32_t l = idx % (uint32_t)nh, r = idx / (uint32_t)nh;
    const uint32_t j = r % (uint32_t)n, i = r / (uint32_t)n;
    const int kx = signed_k((int)i, n), ky = signed_k((int)j, n);
    const bool keep =
        3 * (kx < 0 ? -kx : kx) < n && 3 * (ky < 0 ? -ky : ky) < n && 3 * (int)l < n;
    if (!keep) {
        u0[idx] = mk<T>(0, 0);
        u0[fsc + idx] = mk<T>(0, 0);
        u0[2 * (size_t)fsc + idx] = mk<T>(0, 0);
    }
}

}  // namespace f3
}  // namespace sp
