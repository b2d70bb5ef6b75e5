// Shared device helpers of the B200 spectral engine: complex arithmetic, 16-byte paired loads,
// the device-resident parameter block and the Lawson IF-RK4 stage update.
#pragma once

#include <cmath>

#include <cuda_runtime.h>
#include <stdint.h>

namespace sp {

template <typename T> struct ComplexOf;
template <> struct ComplexOf<float> { using type = float2; };
template <> struct ComplexOf<double> { using type = double2; };
template <typename T> using cplx = typename ComplexOf<T>::type;

template <typename T>
__device__ __forceinline__ cplx<T> mk(T x, T y) {
    cplx<T> c;
    c.x = x;
    c.y = y;
    return c;
}
template <typename C> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };
template <typename C> using real_of = typename RealOf<C>::type;

template <typename C>
__device__ __forceinline__ C add(C a, C b) {
    C r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}
template <typename C>
__device__ __forceinline__ C scl(real_of<C> s, C a) {
    C r;
    r.x = s * a.x;
    r.y = s * a.y;
    return r;
}
// s*a + b
template <typename C>
__device__ __forceinline__ C axpy(real_of<C> s, C a, C b) {
    C r;
    r.x = fma(s, a.x, b.x);
    r.y = fma(s, a.y, b.y);
    return r;
}
// i*a and -i*a
template <typename C>
__device__ __forceinline__ C mul_i(C a) {
    C r;
    r.x = -a.y;
    r.y = a.x;
    return r;
}
template <typename C>
__device__ __forceinline__ C mul_mi(C a) {
    C r;
    r.x = a.y;
    r.y = -a.x;
    return r;
}

// Two consecutive complex values moved as 16-byte (fp32) or 2x16-byte (fp64) transactions.
// Every field starts at a multiple of fsc complex values and fsc is even, so pair addresses
// (even flat index) are 16-byte aligned for fp32 and 32-byte aligned for fp64.
__device__ __forceinline__ void ld2(const float2* p, float2& a, float2& b) {
    float4 v = *reinterpret_cast<const float4*>(p);
    a = make_float2(v.x, v.y);
    b = make_float2(v.z, v.w);
}
__device__ __forceinline__ void ld2(const double2* p, double2& a, double2& b) {
    a = p[0];
    b = p[1];
}
__device__ __forceinline__ void st2(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ void st2(double2* p, double2 a, double2 b) {
    p[0] = a;
    p[1] = b;
}

// Four consecutive reals (physical-space kernels): one float4 or two double2.
template <typename T> struct Real4 { T v[4]; };
__device__ __forceinline__ Real4<float> ld4(const float* p) {
    float4 q = *reinterpret_cast<const float4*>(p);
    return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ Real4<double> ld4(const double* p) {
    double2 a = reinterpret_cast<const double2*>(p)[0];
    double2 b = reinterpret_cast<const double2*>(p)[1];
    return {{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const Real4<float>& r) {
    *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
}
__device__ __forceinline__ void st4(double* p, const Real4<double>& r) {
    reinterpret_cast<double2*>(p)[0] = make_double2(r.v[0], r.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(r.v[2], r.v[3]);
}

// Scalars of one time step, written by the host into device memory before the step is
// launched, so a captured graph never bakes dt or the forcing amplitude into its nodes.
// Fields follow the scalar tuple of the reference (_update_table, cupy_cuda.py:151-161).
template <typename T>
struct StepParams {
    T dt;
    T ea1, eah;    // drag factors exp(-alpha dt), exp(-alpha dt/2)
    T eb1, ebh;    // band factors exp(A dt), exp(A dt/2)
    T klo2, khi2;  // forcing band in k^2 (klo2 > khi2 disables it)
    T ka2;         // drag acts on k^2 <= ka2
    T scale;       // 1 / n^d, folded into the inverse-FFT inputs
};

// Host side: the step scalars and the separable table, computed in fp64 and rounded to T
// (if_table / if_scalars of src/pyspectral/backends/_fused_common.py:10-19 and the band on/off
// rule of cupy_cuda.py:156-159).
template <typename T>
inline StepParams<T> make_step_params(double dt, double alpha, double amp, double klo,
                                      double khi, double drag_k2, double scale) {
    StepParams<T> p;
    p.dt = (T)dt;
    p.ea1 = (T)std::exp(-alpha * dt);
    p.eah = (T)std::exp(-alpha * 0.5 * dt);
    p.eb1 = (T)std::exp(amp * dt);
    p.ebh = (T)std::exp(amp * 0.5 * dt);
    const bool band_on = amp != 0.0;
    p.klo2 = band_on ? (T)(klo * klo) : (T)1;
    p.khi2 = band_on ? (T)(khi * khi) : (T)0;
    p.ka2 = (T)drag_k2;
    p.scale = (T)scale;
    return p;
}
// tab[m] = exp(-nu m^2 dt), tab[nh + m] = exp(-nu m^2 dt / 2), m < nh
template <typename T>
inline void make_if_table(double nu, double dt, int nh, T* tab) {
    for (int m = 0; m < nh; ++m) {
        const double mm = (double)m;
        tab[m] = (T)std::exp(-nu * mm * mm * dt);
        tab[nh + m] = (T)std::exp(-nu * mm * mm * 0.5 * dt);
    }
}

// Integrating factors exp(L dt) and exp(L dt/2) of one mode.  L is separable apart from the
// drag and band indicator terms, so the viscous part is a product of 1D table entries
// tab[m] = exp(-nu m^2 dt), tab[nh + m] = exp(-nu m^2 dt / 2)  (same factorisation as
// if_factors, spectral.cu:43-59).
template <typename T>
struct IFac {
    T E, Eh;
};
template <typename T>
__device__ __forceinline__ IFac<T> if_factors(const T* __restrict__ tab, int nh, int a0, int a1,
                                              int a2, T k2, const StepParams<T>& p) {
    IFac<T> f;
    f.E = tab[a0] * tab[a1];
    f.Eh = tab[nh + a0] * tab[nh + a1];
    if (a2 >= 0) {
        f.E *= tab[a2];
        f.Eh *= tab[nh + a2];
    }
    if (k2 <= p.ka2) {
        f.E *= p.ea1;
        f.Eh *= p.eah;
    }
    if (k2 >= p.klo2 && k2 <= p.khi2) {
        f.E *= p.eb1;
        f.Eh *= p.ebh;
    }
    return f;
}

// Lawson IF-RK4 (numpy_ref.py:145-153) as four stage updates of one mode.  acc carries
// E k1 + 2 Eh (k2 + k3); the value returned is the state the next nonlinear evaluation sees;
// stage 3 returns (and stores) the new state.
template <typename T, int STAGE>
__device__ __forceinline__ cplx<T> lawson_stage(T dt, const IFac<T>& f, cplx<T> N, cplx<T> u,
                                                cplx<T>& acc) {
    if (STAGE == 0) {
        acc = scl(f.E, N);
        return scl(f.Eh, axpy((T)0.5 * dt, N, u));
    } else if (STAGE == 1) {
        acc = axpy((T)2 * f.Eh, N, acc);
        return axpy((T)0.5 * dt, N, scl(f.Eh, u));
    } else if (STAGE == 2) {
        acc = axpy((T)2 * f.Eh, N, acc);
        return axpy(dt * f.Eh, N, scl(f.E, u));
    } else {
        return axpy(dt / (T)6, add(acc, N), scl(f.E, u));
    }
}

__device__ __forceinline__ int signed_k(int i, int n) { return i < (n >> 1) ? i : i - n; }

}  // namespace sp
