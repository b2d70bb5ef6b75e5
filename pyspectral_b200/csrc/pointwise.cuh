// Fused pointwise kernels of one IF-RK4 stage around the cuFFT transforms.
//
// Stage = inverse FFT (W: spectral -> padded physical, in place) -> phys kernel (in place)
//       -> forward FFT (in place) -> post kernel.
// The post kernel evaluates the nonlinear term from the transformed products, dealiases,
// projects (3D), performs the Lawson stage update and writes the next stage's FFT inputs, so
// the state is read exactly once per stage.  The pair decomposition (two modes per thread,
// 16-byte transactions) and device-resident StepParams are the B200-specific parts; the
// per-mode arithmetic is the one of spectral.cu:93-238 in the reference.
#pragma once

#include "common.cuh"

namespace sp {

constexpr int kBlock = 256;

// --------------------------------------------------------------------------------------- 2D
// (n, nh) spectral layout, mode idx = i*nh + j with kx = signed(i), ky = j.
template <typename T>
struct Mode2 {
    T kx, ky, k2;
    int akx, ky_i;
    bool keep;
};

template <typename T>
__device__ __forceinline__ Mode2<T> mode2(int i, int j, int n) {
    Mode2<T> m;
    int kxi = signed_k(i, n);
    m.akx = kxi < 0 ? -kxi : kxi;
    m.ky_i = j;
    m.kx = (T)kxi;
    m.ky = (T)j;
    m.k2 = m.kx * m.kx + m.ky * m.ky;
    m.keep = (3 * m.akx < n) && (3 * j < n);
    return m;
}

// Next-stage inverse-FFT inputs of a vorticity mode: u = i ky psi, v = -i kx psi with
// psi = omega / k^2, scaled by 1/n^2 and dealiased.
template <typename T>
__device__ __forceinline__ void velocity2(const Mode2<T>& m, cplx<T> w, T scale, cplx<T>& u,
                                          cplx<T>& v) {
    T ik2 = (m.keep && m.k2 > (T)0) ? scale / m.k2 : (T)0;
    cplx<T> psi = scl(ik2, w);
    u = scl(m.ky, mul_i(psi));
    v = scl(m.kx, mul_mi(psi));
}

// Closure layout of the 2D work array (a coarse run with the learned closure attached): slots
// [S, u, v, omega, d omega/dx, d omega/dy]; the plain layout is [u, v].  The vorticity and its
// gradient are the closure network's inputs, S its output.
template <typename T>
__device__ __forceinline__ void omega_set(const Mode2<T>& m, cplx<T> w, T scale, cplx<T>& o,
                                          cplx<T>& ox, cplx<T>& oy) {
    const T s = m.keep ? scale : (T)0;
    o = scl(s, w);
    ox = scl(m.kx * s, mul_i(w));
    oy = scl(m.ky * s, mul_i(w));
}

// Loads a state: dealiases u0 in place (the host-side check_state mask of base.py:134-139, done
// on the device) and writes the stage-0 inverse-FFT inputs.
template <typename T, bool CL = false>
__global__ void __launch_bounds__(kBlock) k_pre2d(cplx<T>* __restrict__ u0,
                                                  cplx<T>* __restrict__ W, int n, int nh,
                                                  uint32_t fsc,
                                                  const StepParams<T>* __restrict__ P) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    const T scale = P->scale;
    uint32_t i = idx0 / (uint32_t)nh;
    uint32_t j = idx0 - i * (uint32_t)nh;
    cplx<T> w[2], u[2], v[2], o[2], ox[2], oy[2];
    ld2(u0 + idx0, w[0], w[1]);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode2<T> m = mode2<T>((int)i, (int)j, n);
        if (!m.keep) w[e] = mk<T>(0, 0);
        velocity2(m, w[e], scale, u[e], v[e]);
        if (CL) omega_set(m, w[e], scale, o[e], ox[e], oy[e]);
        if (++j == (uint32_t)nh) { j = 0; ++i; }
    }
    st2(u0 + idx0, w[0], w[1]);
    cplx<T>* Wuv = CL ? W + fsc : W;
    st2(Wuv + idx0, u[0], u[1]);
    st2(Wuv + fsc + idx0, v[0], v[1]);
    if (CL) {
        st2(W + 3 * (size_t)fsc + idx0, o[0], o[1]);
        st2(W + 4 * (size_t)fsc + idx0, ox[0], ox[1]);
        st2(W + 5 * (size_t)fsc + idx0, oy[0], oy[1]);
    }
}

// Nonlinear term of a given state (no update): the velocity pair of `state` (left untouched)
// into the plain work layout ...
template <typename T>
__global__ void __launch_bounds__(kBlock) k_nl_pre2d(const cplx<T>* __restrict__ state,
                                                     cplx<T>* __restrict__ W, int n, int nh,
                                                     uint32_t fsc,
                                                     const StepParams<T>* __restrict__ P) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    const T scale = P->scale;
    uint32_t i = idx0 / (uint32_t)nh;
    uint32_t j = idx0 - i * (uint32_t)nh;
    cplx<T> w[2], u[2], v[2];
    ld2(state + idx0, w[0], w[1]);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode2<T> m = mode2<T>((int)i, (int)j, n);
        velocity2(m, w[e], scale, u[e], v[e]);
        if (++j == (uint32_t)nh) { j = 0; ++i; }
    }
    st2(W + idx0, u[0], u[1]);
    st2(W + fsc + idx0, v[0], v[1]);
}

// ... and, after the transforms and the products, the dealiased Basdevant term into `out`.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_nl_post2d(const cplx<T>* __restrict__ W,
                                                      cplx<T>* __restrict__ out, int n, int nh,
                                                      uint32_t fsc) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    cplx<T> A[2], B[2], N[2];
    ld2(W + idx0, A[0], A[1]);
    ld2(W + fsc + idx0, B[0], B[1]);
    uint32_t i = idx0 / (uint32_t)nh;
    uint32_t j = idx0 - i * (uint32_t)nh;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode2<T> m = mode2<T>((int)i, (int)j, n);
        N[e] = mk<T>(0, 0);
        if (m.keep) N[e] = axpy(m.kx * m.ky, A[e], scl(m.kx * m.kx - m.ky * m.ky, B[e]));
        if (++j == (uint32_t)nh) { j = 0; ++i; }
    }
    st2(out + idx0, N[0], N[1]);
}

// physical space, in place over the padded real fields: (u, v) -> (v^2 - u^2, u v)
template <typename T>
__global__ void __launch_bounds__(kBlock) k_phys2d(T* __restrict__ R, uint32_t fsr) {
    uint32_t p = 4u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p >= fsr) return;
    Real4<T> u = ld4(R + p), v = ld4(R + fsr + p), a, b;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        a.v[e] = (v.v[e] - u.v[e]) * (v.v[e] + u.v[e]);
        b.v[e] = u.v[e] * v.v[e];
    }
    st4(R + p, a);
    st4(R + fsr + p, b);
}

template <typename T, int STAGE, bool CL = false>
__global__ void __launch_bounds__(kBlock) k_post2d(cplx<T>* __restrict__ W,
                                                   cplx<T>* __restrict__ u0,
                                                   cplx<T>* __restrict__ acc,
                                                   const T* __restrict__ tab,
                                                   const StepParams<T>* __restrict__ P, int n,
                                                   int nh, uint32_t fsc,
                                                   const float* __restrict__ gain = nullptr,
                                                   int ngain = 0, int omega_out = 1) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    const StepParams<T> p = *P;
    cplx<T>* Wuv = CL ? W + fsc : W;
    cplx<T> A[2], B[2], U[2], C[2], S[2], nu_[2], nv_[2], o[2], ox[2], oy[2];
    ld2(Wuv + idx0, A[0], A[1]);
    ld2(Wuv + fsc + idx0, B[0], B[1]);
    if (CL) ld2(W + idx0, S[0], S[1]);
    ld2(u0 + idx0, U[0], U[1]);
    if (STAGE > 0) ld2(acc + idx0, C[0], C[1]);
    uint32_t i = idx0 / (uint32_t)nh;
    uint32_t j = idx0 - i * (uint32_t)nh;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode2<T> m = mode2<T>((int)i, (int)j, n);
        // Basdevant 2D nonlinear term: kx ky FFT(v^2-u^2) + (kx^2-ky^2) FFT(uv), plus the
        // transformed closure term when one is attached
        cplx<T> N = mk<T>(0, 0);
        if (m.keep) N = axpy(m.kx * m.ky, A[e], scl(m.kx * m.kx - m.ky * m.ky, B[e]));
        if (CL && m.keep && m.k2 > (T)0) {  // S is a divergence: no mean
            int sh = (int)(sqrt(m.k2) + (T)0.5);
            sh = sh < ngain ? sh : ngain - 1;
            N = axpy((T)gain[sh], S[e], N);
        }
        IFac<T> f = if_factors(tab, nh, m.akx, m.ky_i, -1, m.k2, p);
        cplx<T> nxt = lawson_stage<T, STAGE>(p.dt, f, N, U[e], C[e]);
        if (STAGE == 3) U[e] = nxt;
        velocity2(m, nxt, p.scale, nu_[e], nv_[e]);
        if (CL) omega_set(m, nxt, p.scale, o[e], ox[e], oy[e]);
        if (++j == (uint32_t)nh) { j = 0; ++i; }
    }
    if (STAGE == 3) st2(u0 + idx0, U[0], U[1]);
    else st2(acc + idx0, C[0], C[1]);
    st2(Wuv + idx0, nu_[0], nu_[1]);
    st2(Wuv + fsc + idx0, nv_[0], nv_[1]);
    if (CL && omega_out) {  // the network's inputs, when the next stage evaluates it
        st2(W + 3 * (size_t)fsc + idx0, o[0], o[1]);
        st2(W + 4 * (size_t)fsc + idx0, ox[0], ox[1]);
        st2(W + 5 * (size_t)fsc + idx0, oy[0], oy[1]);
    }
}

// --------------------------------------------------------------------------------------- 3D
// (n, n, nh) spectral layout per component, idx = (i*n + j)*nh + l; a ky slab of a distributed
// run holds (n, ny, nh) with local index jl and global ky index j = j0 + jl.
template <typename T>
struct Mode3 {
    T kx, ky, kz, k2;
    int akx, aky, kz_i;
    bool keep;
};

template <typename T>
__device__ __forceinline__ Mode3<T> mode3(int i, int j, int l, int n) {
    Mode3<T> m;
    int kxi = signed_k(i, n), kyi = signed_k(j, n);
    m.akx = kxi < 0 ? -kxi : kxi;
    m.aky = kyi < 0 ? -kyi : kyi;
    m.kz_i = l;
    m.kx = (T)kxi;
    m.ky = (T)kyi;
    m.kz = (T)l;
    m.k2 = m.kx * m.kx + m.ky * m.ky + m.kz * m.kz;
    m.keep = (3 * m.akx < n) && (3 * m.aky < n) && (3 * l < n);
    return m;
}

// Walks (i, jl, l) through consecutive flat indices of an (n, ny, nh) array; j() is the global
// ky index j0 + jl (ny = n, j0 = 0 for a whole grid).
struct Walk3 {
    uint32_t i, jl, l;
    int j0;
    __device__ __forceinline__ Walk3(uint32_t idx, int ny, int nh, int j0_) : j0(j0_) {
        uint32_t t = idx / (uint32_t)nh;
        l = idx - t * (uint32_t)nh;
        i = t / (uint32_t)ny;
        jl = t - i * (uint32_t)ny;
    }
    __device__ __forceinline__ int j() const { return j0 + (int)jl; }
    __device__ __forceinline__ void next(int ny, int nh) {
        if (++l == (uint32_t)nh) {
            l = 0;
            if (++jl == (uint32_t)ny) { jl = 0; ++i; }
        }
    }
};

// Next-stage inputs of one velocity mode: u (scaled, dealiased) and for the rotational form
// omega = i k x u.
template <typename T, bool ROT>
__device__ __forceinline__ void inputs3(const Mode3<T>& m, T scale, cplx<T> a, cplx<T> b,
                                        cplx<T> c, cplx<T> out[6]) {
    T s = m.keep ? scale : (T)0;
    a = scl(s, a);
    b = scl(s, b);
    c = scl(s, c);
    out[0] = a;
    out[1] = b;
    out[2] = c;
    if (ROT) {
        out[3] = mul_i(add(scl(m.ky, c), scl(-m.kz, b)));
        out[4] = mul_i(add(scl(m.kz, a), scl(-m.kx, c)));
        out[5] = mul_i(add(scl(m.kx, b), scl(-m.ky, a)));
    }
}

template <typename T, bool ROT>
__global__ void __launch_bounds__(kBlock) k_pre3d(cplx<T>* __restrict__ u0,
                                                  cplx<T>* __restrict__ W, int n, int nh,
                                                  uint32_t fsc,
                                                  const StepParams<T>* __restrict__ P,
                                                  int ny = 0, int j0 = 0) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    const T scale = P->scale;
    cplx<T> a[2], b[2], c[2], o[2][6];
    ld2(u0 + idx0, a[0], a[1]);
    ld2(u0 + fsc + idx0, b[0], b[1]);
    ld2(u0 + 2 * fsc + idx0, c[0], c[1]);
    const int ly = ny ? ny : n;
    Walk3 w(idx0, ly, nh, j0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode3<T> m = mode3<T>((int)w.i, w.j(), (int)w.l, n);
        if (!m.keep) a[e] = b[e] = c[e] = mk<T>(0, 0);
        inputs3<T, ROT>(m, scale, a[e], b[e], c[e], o[e]);
        w.next(ly, nh);
    }
    st2(u0 + idx0, a[0], a[1]);
    st2(u0 + fsc + idx0, b[0], b[1]);
    st2(u0 + 2 * fsc + idx0, c[0], c[1]);
#pragma unroll
    for (int f = 0; f < (ROT ? 6 : 3); ++f) st2(W + (size_t)f * fsc + idx0, o[0][f], o[1][f]);
}

// physical space, Basdevant traceless stress: (u, v, w) -> (uu-q, vv-q, uv, uw, vw), q=|u|^2/3
template <typename T>
__global__ void __launch_bounds__(kBlock) k_phys3d_basd(T* __restrict__ R, uint32_t fsr) {
    uint32_t p = 4u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p >= fsr) return;
    Real4<T> u = ld4(R + p), v = ld4(R + fsr + p), w = ld4(R + 2 * (size_t)fsr + p);
    Real4<T> o[5];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        T uu = u.v[e] * u.v[e], vv = v.v[e] * v.v[e], ww = w.v[e] * w.v[e];
        T q = (uu + vv + ww) * ((T)1 / (T)3);
        o[0].v[e] = uu - q;
        o[1].v[e] = vv - q;
        o[2].v[e] = u.v[e] * v.v[e];
        o[3].v[e] = u.v[e] * w.v[e];
        o[4].v[e] = v.v[e] * w.v[e];
    }
#pragma unroll
    for (int f = 0; f < 5; ++f) st4(R + (size_t)f * fsr + p, o[f]);
}

// physical space, rotational form: (u, omega) -> u x omega
template <typename T>
__global__ void __launch_bounds__(kBlock) k_phys3d_rot(T* __restrict__ R, uint32_t fsr) {
    uint32_t p = 4u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (p >= fsr) return;
    Real4<T> u = ld4(R + p), v = ld4(R + fsr + p), w = ld4(R + 2 * (size_t)fsr + p);
    Real4<T> ox = ld4(R + 3 * (size_t)fsr + p), oy = ld4(R + 4 * (size_t)fsr + p),
             oz = ld4(R + 5 * (size_t)fsr + p);
    Real4<T> o[3];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        o[0].v[e] = v.v[e] * oz.v[e] - w.v[e] * oy.v[e];
        o[1].v[e] = w.v[e] * ox.v[e] - u.v[e] * oz.v[e];
        o[2].v[e] = u.v[e] * oy.v[e] - v.v[e] * ox.v[e];
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) st4(R + (size_t)f * fsr + p, o[f]);
}

template <typename T, bool ROT, int STAGE>
__global__ void __launch_bounds__(kBlock) k_post3d(cplx<T>* __restrict__ W,
                                                   cplx<T>* __restrict__ u0,
                                                   cplx<T>* __restrict__ acc,
                                                   const T* __restrict__ tab,
                                                   const StepParams<T>* __restrict__ P, int n,
                                                   int nh, uint32_t fsc, int ny = 0, int j0 = 0) {
    uint32_t idx0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (idx0 >= fsc) return;
    const StepParams<T> p = *P;
    constexpr int NIN = ROT ? 3 : 5;
    cplx<T> F[NIN][2], U[3][2], C[3][2], out[2][6];
#pragma unroll
    for (int f = 0; f < NIN; ++f) ld2(W + (size_t)f * fsc + idx0, F[f][0], F[f][1]);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ld2(u0 + (size_t)c * fsc + idx0, U[c][0], U[c][1]);
        if (STAGE > 0) ld2(acc + (size_t)c * fsc + idx0, C[c][0], C[c][1]);
    }
    const int ly = ny ? ny : n;
    Walk3 w(idx0, ly, nh, j0);
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        Mode3<T> m = mode3<T>((int)w.i, w.j(), (int)w.l, n);
        cplx<T> N0 = mk<T>(0, 0), N1 = mk<T>(0, 0), N2 = mk<T>(0, 0);
        if (m.keep) {
            if (ROT) {
                N0 = F[0][e];
                N1 = F[1][e];
                N2 = F[2][e];
            } else {
                // N_i = -i k_j T_ij with T33 = -(T11 + T22)
                cplx<T> t11 = F[0][e], t22 = F[1][e], t12 = F[2][e], t13 = F[3][e],
                        t23 = F[4][e];
                cplx<T> t33 = mk<T>(-(t11.x + t22.x), -(t11.y + t22.y));
                N0 = mul_mi(add(add(scl(m.kx, t11), scl(m.ky, t12)), scl(m.kz, t13)));
                N1 = mul_mi(add(add(scl(m.kx, t12), scl(m.ky, t22)), scl(m.kz, t23)));
                N2 = mul_mi(add(add(scl(m.kx, t13), scl(m.ky, t23)), scl(m.kz, t33)));
            }
            // Leray projection N <- N - k (k.N) / k^2
            T ik2 = m.k2 > (T)0 ? (T)1 / m.k2 : (T)0;
            cplx<T> d = scl(ik2, add(add(scl(m.kx, N0), scl(m.ky, N1)), scl(m.kz, N2)));
            N0 = axpy(-m.kx, d, N0);
            N1 = axpy(-m.ky, d, N1);
            N2 = axpy(-m.kz, d, N2);
        }
        IFac<T> f = if_factors(tab, nh, m.akx, m.aky, m.kz_i, m.k2, p);
        cplx<T> a = lawson_stage<T, STAGE>(p.dt, f, N0, U[0][e], C[0][e]);
        cplx<T> b = lawson_stage<T, STAGE>(p.dt, f, N1, U[1][e], C[1][e]);
        cplx<T> c = lawson_stage<T, STAGE>(p.dt, f, N2, U[2][e], C[2][e]);
        if (STAGE == 3) {
            U[0][e] = a;
            U[1][e] = b;
            U[2][e] = c;
        }
        inputs3<T, ROT>(m, p.scale, a, b, c, out[e]);
        w.next(ly, nh);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (STAGE == 3) st2(u0 + (size_t)c * fsc + idx0, U[c][0], U[c][1]);
        else st2(acc + (size_t)c * fsc + idx0, C[c][0], C[c][1]);
    }
#pragma unroll
    for (int f = 0; f < (ROT ? 6 : 3); ++f) st2(W + (size_t)f * fsc + idx0, out[0][f], out[1][f]);
}

}  // namespace sp
