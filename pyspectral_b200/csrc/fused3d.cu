// Launchers of the fused 3D engine: runtime (n, precision, form, stage) -> kernel instantiation.
#include "fused3d.h"
#include "fused3d.cuh"

// the dispatch lambdas name their template parameters only in the body
#pragma nv_diag_suppress 445

namespace sp {
namespace fused3 {

namespace {

template <typename T, int N, bool ROT>
constexpr size_t spec_pairs() {
    using D = f3::Dims<N>;
    return (size_t)N * f3::nslot<ROT>() * D::KK * D::NQ;
}
template <typename T, int N, bool ROT>
constexpr size_t phys_pairs() {
    using D = f3::Dims<N>;
    return (size_t)N * f3::nslot<ROT>() * N * D::NQ;
}

template <typename T, int N, bool ROT>
cudaError_t attrs() {
    using X = f3::XPass<T, N, ROT>;
    const int smem = (int)X::smem_bytes();
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(f3::k3_x<T, N, ROT, -1>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem)))
        return e;
    if ((e = cudaFuncSetAttribute(f3::k3_x<T, N, ROT, 0>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem)))
        return e;
    if ((e = cudaFuncSetAttribute(f3::k3_x<T, N, ROT, 1>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem)))
        return e;
    if ((e = cudaFuncSetAttribute(f3::k3_x<T, N, ROT, 2>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem)))
        return e;
    return cudaFuncSetAttribute(f3::k3_x<T, N, ROT, 3>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <typename T, int N, bool ROT>
cudaError_t yinv(const void* Bs, void* Bp, int nfields, const void* tw, cudaStream_t st) {
    using D = f3::Dims<N>;
    constexpr int per = f3::y_threads<T>() / D::T;
    const long units = (long)N * nfields * D::NQ;
    const unsigned grid = (unsigned)((units + per - 1) / per);
    f3::k3_yinv<T, N, ROT><<<grid, f3::y_threads<T>(), 0, st>>>(
        (const Pair<T>*)Bs, (Pair<T>*)Bp, nfields, (const cplx<T>*)tw);
    return cudaGetLastError();
}

template <typename T, int N, bool ROT>
cudaError_t yfwd(const void* Bp, void* Bs, int nfields, const void* tw, cudaStream_t st) {
    using D = f3::Dims<N>;
    constexpr int per = f3::y_threads<T>() / D::T;
    const long units = (long)N * nfields * D::NQ;
    const unsigned grid = (unsigned)((units + per - 1) / per);
    f3::k3_yfwd<T, N, ROT><<<grid, f3::y_threads<T>(), 0, st>>>(
        (const Pair<T>*)Bp, (Pair<T>*)Bs, nfields, (const cplx<T>*)tw);
    return cudaGetLastError();
}

template <typename T, int N, bool ROT>
cudaError_t zp(int mode, void* Bp, const void* tw, unsigned long long* umax, int want_max,
               cudaStream_t st) {
    using D = f3::Dims<N>;
    constexpr int zt = f3::z_threads<T>();
    constexpr int per = zt / D::T;
    const long lines = (long)N * N;
    const unsigned grid = (unsigned)((lines + per - 1) / per);
    if (mode == 1)
        f3::k3_z<T, N, ROT, 1><<<grid, zt, 0, st>>>((Pair<T>*)Bp, (const cplx<T>*)tw, umax, 1);
    else
        f3::k3_z<T, N, ROT, 0><<<grid, zt, 0, st>>>((Pair<T>*)Bp, (const cplx<T>*)tw, umax,
                                                     want_max);
    return cudaGetLastError();
}

template <typename T, int N, bool ROT, int STAGE>
cudaError_t xs(void* Bs, void* u0, void* acc, const void* tab, const void* params,
               const void* tw, cudaStream_t st) {
    using X = f3::XPass<T, N, ROT>;
    const unsigned grid = (unsigned)((X::UNITS + X::U - 1) / X::U);
    f3::k3_x<T, N, ROT, STAGE><<<grid, X::THREADS, X::smem_bytes(), st>>>(
        (Pair<T>*)Bs, (cplx<T>*)u0, (cplx<T>*)acc, (const T*)tab,
        (const StepParams<T>*)params, (const cplx<T>*)tw);
    return cudaGetLastError();
}

template <typename T, int N, bool ROT>
cudaError_t xp(int stage, void* Bs, void* u0, void* acc, const void* tab, const void* params,
               const void* tw, cudaStream_t st) {
    switch (stage) {
        case -1: return xs<T, N, ROT, -1>(Bs, u0, acc, tab, params, tw, st);
        case 0: return xs<T, N, ROT, 0>(Bs, u0, acc, tab, params, tw, st);
        case 1: return xs<T, N, ROT, 1>(Bs, u0, acc, tab, params, tw, st);
        case 2: return xs<T, N, ROT, 2>(Bs, u0, acc, tab, params, tw, st);
        case 3: return xs<T, N, ROT, 3>(Bs, u0, acc, tab, params, tw, st);
        default: return cudaErrorInvalidValue;
    }
}

// Calls fn.operator()<T, N, ROT>() for the runtime (n, fp64, rot).
template <typename Fn>
cudaError_t dispatch(int n, int fp64, int rot, Fn&& fn) {
    auto by_n = [&]<typename T, bool ROT>() -> cudaError_t {
        switch (n) {
            case 16: return fn.template operator()<T, 16, ROT>();
            case 32: return fn.template operator()<T, 32, ROT>();
            case 64: return fn.template operator()<T, 64, ROT>();
            case 128: return fn.template operator()<T, 128, ROT>();
            case 256: return fn.template operator()<T, 256, ROT>();
            case 512: return fn.template operator()<T, 512, ROT>();
            default: return cudaErrorInvalidValue;
        }
    };
    if (fp64) {
        if (rot) return by_n.template operator()<double, true>();
        return by_n.template operator()<double, false>();
    }
    if (rot) return by_n.template operator()<float, true>();
    return by_n.template operator()<float, false>();
}

template <typename Fn>
size_t dispatch_size(int n, int fp64, int rot, Fn&& fn) {
    size_t out = 0;
    dispatch(n, fp64, rot, [&]<typename T, int N, bool ROT>() {
        out = fn.template operator()<T, N, ROT>();
        return cudaSuccess;
    });
    return out;
}

}  // namespace

bool supported(int n, int fp64) {
    (void)fp64;
    return n >= 16 && n <= 512 && (n & (n - 1)) == 0;
}

size_t spec_bytes(int n, int fp64, int rot) {
    return dispatch_size(n, fp64, rot, []<typename T, int N, bool ROT>() {
        return spec_pairs<T, N, ROT>() * sizeof(Pair<T>);
    });
}

size_t phys_bytes(int n, int fp64, int rot) {
    return dispatch_size(n, fp64, rot, []<typename T, int N, bool ROT>() {
        return phys_pairs<T, N, ROT>() * sizeof(Pair<T>);
    });
}

cudaError_t set_attributes(int n, int fp64, int rot) {
    return dispatch(n, fp64, rot, []<typename T, int N, bool ROT>() { return attrs<T, N, ROT>(); });
}

cudaError_t y_inverse(int n, int fp64, int rot, const void* Bs, void* Bp, int nfields,
                      const void* tw, cudaStream_t st) {
    return dispatch(n, fp64, rot, [&]<typename T, int N, bool ROT>() {
        return yinv<T, N, ROT>(Bs, Bp, nfields, tw, st);
    });
}

cudaError_t y_forward(int n, int fp64, int rot, const void* Bp, void* Bs, int nfields,
                      const void* tw, cudaStream_t st) {
    return dispatch(n, fp64, rot, [&]<typename T, int N, bool ROT>() {
        return yfwd<T, N, ROT>(Bp, Bs, nfields, tw, st);
    });
}

cudaError_t z_pass(int n, int fp64, int rot, int mode, void* Bp, const void* tw,
                   unsigned long long* umax, int want_max, cudaStream_t st) {
    if (mode != 0 && mode != 1) return cudaErrorInvalidValue;
    return dispatch(n, fp64, rot, [&]<typename T, int N, bool ROT>() {
        return zp<T, N, ROT>(mode, Bp, tw, umax, want_max, st);
    });
}

cudaError_t x_pass(int n, int fp64, int rot, int stage, void* Bs, void* u0, void* acc,
                   const void* tab, const void* params, const void* tw, cudaStream_t st) {
    return dispatch(n, fp64, rot, [&]<typename T, int N, bool ROT>() {
        return xp<T, N, ROT>(stage, Bs, u0, acc, tab, params, tw, st);
    });
}

size_t compact_bytes(int n, int fp64) {
    const size_t km = (size_t)(n - 1) / 3, kk = 2 * km + 1;
    return 3 * kk * (km + 1) * kk * (fp64 ? 16 : 8);
}

cudaError_t state_move(int fp64, void* u0, void* compact, int n, int in, cudaStream_t st) {
    const int km = (n - 1) / 3, kk = 2 * km + 1;
    const dim3 grid((km + 1 + 31) / 32, (kk + 31) / 32, 3 * kk), block(32, 8);
    if (fp64) {
        if (in) f3::k3_state_move<double, true><<<grid, block, 0, st>>>((cplx<double>*)u0, (cplx<double>*)compact, n);
        else f3::k3_state_move<double, false><<<grid, block, 0, st>>>((cplx<double>*)u0, (cplx<double>*)compact, n);
    } else {
        if (in) f3::k3_state_move<float, true><<<grid, block, 0, st>>>((cplx<float>*)u0, (cplx<float>*)compact, n);
        else f3::k3_state_move<float, false><<<grid, block, 0, st>>>((cplx<float>*)u0, (cplx<float>*)compact, n);
    }
    return cudaGetLastError();
}

cudaError_t mask(int fp64, void* u0, int n, cudaStream_t st) {
    const int nh = n / 2 + 1;
    const uint32_t fsc = (uint32_t)n * (uint32_t)n * (uint32_t)nh;
    const unsigned grid = (fsc + 255) / 256;
    if (fp64) f3::k3_mask<double><<<grid, 256, 0, st>>>((cplx<double>*)u0, n, nh, fsc);
    else f3::k3_mask<float><<<grid, 256, 0, st>>>((cplx<float>*)u0, n, nh, fsc);
    return cudaGetLastError();
}

}  // namespace fused3
}  // namespace sp
