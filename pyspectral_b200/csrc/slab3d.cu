// Slab-decomposed 3D IF-RK4 step for runs spread over several GPUs (one process per GPU).
//
// Layout (n divisible by the rank count P, m = n / P):
//   spectral state and RK accumulator: per component (kx: n, ky: m local, kz: n/2+1), rank r
//     holding ky in [r m, (r+1) m) — a ky slab;
//   physical fields: (x: m local, y: n, z: n+2 padded), rank r holding x in [r m, (r+1) m).
// One RK stage = three local parts with an all-to-all exchange after parts 0 and 1 (done by the
// caller, e.g. NCCL all_to_all_single over NVLink/NVSwitch, into this rank's own `recv`
// buffer before part 1 / part 2 reads it):
//   part 0: inverse C2C FFT along kx of the stage inputs (kx is whole in a ky slab), then pack
//           the x blocks: send[p] = fields at x in [p m, (p+1) m);
//   part 1: unpack (x slab, all ky), inverse 2D C2R over (ky, kz) per x plane, the physical
//           products, forward 2D R2C, pack the ky blocks: send[p] = ky in [p m, (p+1) m);
//   part 2: unpack (all x, ky slab), forward C2C FFT along x, then the 3D post kernel on the
//           slab (nonlinear term, Leray projection, Lawson update, next inputs), whose mode
//           wavenumbers use the slab's ky offset.
// The transforms are cuFFT plans (1D strided C2C, 2D batched C2R/R2C in place); the pointwise
// kernels are the single-GPU ones (pointwise.cuh) with a slab offset.  The exchange blocks are
// contiguous per destination, so no collective needs strided data.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "pointwise.cuh"
#include "reduce.cuh"
#include "spectral_b200.h"

using namespace sp;

namespace sp {
void set_thread_error(const char* why);  // spectral_b200.cu
}

struct sp_slab {
    int n = 0, P = 1, rank = 0, m = 0, nh = 0, form = 0, fp64 = 0;
    int ninv = 0, nfwd = 0, nwork = 0;
    uint32_t fsc = 0;       // complex entries of one local field (n m nh)
    size_t csize = 8;       // bytes of one complex
    void *u0 = nullptr, *acc = nullptr, *W = nullptr, *send = nullptr, *recv = nullptr;
    void* aux = nullptr;
    bool bound = false;
    size_t off_params = 0, off_tab = 0, off_partials = 0, off_umax = 0, off_out = 0;
    size_t aux_bytes = 0, ws_bytes = 0;
    cufftHandle px = 0, p2i = 0, p2f = 0;
    bool have_px = false, have_p2i = false, have_p2f = false;
    double nu = 0, alpha = 0, drag_k2 = 1e30, klo = 0, khi = 0, amp = 0;
    // host copies of the last uploaded parameter block and table (kept alive for the async
    // copies; re-sent only when they change)
    std::vector<unsigned char> host_params, host_tab;
    int64_t launches = 0;
    std::string err;

    char* base(size_t off) const { return (char*)aux + off; }
    size_t field_bytes() const { return (size_t)fsc * csize; }
    char* wf(int f) const { return (char*)W + f * field_bytes(); }
    bool rot() const { return form == SP_FORM_ROTATIONAL; }
};

namespace {

int sfail(sp_slab* s, int code, const std::string& why) {
    if (s) s->err = why;
    return code;
}

#define S_CUDA(call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) return sfail(s, SP_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)
#define S_CUFFT(call)                                                                        \
    do {                                                                                     \
        if ((call) != CUFFT_SUCCESS) return sfail(s, SP_ERR_CUFFT, #call);                  \
    } while (0)

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
unsigned blocks_for(uint64_t items, int block) { return (unsigned)((items + block - 1) / block); }

// Row copies between the slab layouts and the exchange blocks.  A "row" is a contiguous run
// of `len` complex values in both source and destination.
//   mode 0  pack x:    W[f][p m + il][q]           -> send[p][f][il][q]        q < m nh
//   mode 1  unpack x:  recv[p][f][il][jl][kz]     -> W[f][il][p m + jl][kz]    len nh
//   mode 2  pack ky:   W[f][il][p m + jl][kz]     -> send[p][f][il][jl][kz]    len nh
//   mode 3  unpack ky: recv[p][f][il][q]          -> W[f][p m + il][q]         q < m nh
template <typename C, int MODE>
__global__ void __launch_bounds__(256) k_slab_rows(const C* __restrict__ src, C* __restrict__ dst,
                                                   int P, int nf, int n, int m, int nh) {
    const size_t row = blockIdx.y + (size_t)gridDim.y * blockIdx.z;
    const size_t fsc = (size_t)n * m * nh;
    const size_t blk = (size_t)nf * m * m * nh;  // complex per exchange block
    if (MODE == 0 || MODE == 3) {
        // rows (p, f, il) of length m nh
        const size_t nrows = (size_t)P * nf * m;
        if (row >= nrows) return;
        const int il = (int)(row % m), f = (int)((row / m) % nf), p = (int)(row / ((size_t)m * nf));
        const size_t len = (size_t)m * nh;
        const size_t a = (size_t)f * fsc + ((size_t)p * m + il) * len;  // slab side
        const size_t b = (size_t)p * blk + ((size_t)f * m + il) * len;  // exchange side
        for (size_t q = blockIdx.x * blockDim.x + threadIdx.x; q < len; q += gridDim.x * blockDim.x) {
            if (MODE == 0) dst[b + q] = src[a + q];
            else dst[a + q] = src[b + q];
        }
    } else {
        // rows (p, f, il, jl) of length nh
        const size_t nrows = (size_t)P * nf * m * m;
        if (row >= nrows) return;
        const int jl = (int)(row % m), il = (int)((row / m) % m);
        const int f = (int)((row / ((size_t)m * m)) % nf), p = (int)(row / ((size_t)m * m * nf));
        const size_t a = (size_t)f * fsc + ((size_t)il * n + (size_t)p * m + jl) * nh;
        const size_t b = (size_t)p * blk + (((size_t)f * m + il) * m + jl) * nh;
        for (size_t q = blockIdx.x * blockDim.x + threadIdx.x; q < (size_t)nh;
             q += gridDim.x * blockDim.x) {
            if (MODE == 2) dst[b + q] = src[a + q];
            else dst[a + q] = src[b + q];
        }
    }
}

template <typename C, int MODE>
int launch_rows(sp_slab* s, const void* src, void* dst, int nf, cudaStream_t st) {
    const bool long_rows = MODE == 0 || MODE == 3;
    const size_t nrows = long_rows ? (size_t)s->P * nf * s->m : (size_t)s->P * nf * s->m * s->m;
    const size_t len = long_rows ? (size_t)s->m * s->nh : (size_t)s->nh;
    const unsigned gx = (unsigned)std::min<size_t>((len + 255) / 256, 64);
    const unsigned gy = (unsigned)std::min<size_t>(nrows, 65535);
    const unsigned gz = (unsigned)((nrows + gy - 1) / gy);
    k_slab_rows<C, MODE><<<dim3(gx, gy, gz), 256, 0, st>>>((const C*)src, (C*)dst, s->P, nf, s->n,
                                                           s->m, s->nh);
    S_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <int MODE>
int rows(sp_slab* s, const void* src, void* dst, int nf, cudaStream_t st) {
    return s->fp64 ? launch_rows<cplx<double>, MODE>(s, src, dst, nf, st)
                   : launch_rows<cplx<float>, MODE>(s, src, dst, nf, st);
}

int exec_x(sp_slab* s, int nf, int dir, cudaStream_t st) {
    S_CUFFT(cufftSetStream(s->px, st));
    for (int f = 0; f < nf; ++f) {
        if (s->fp64) {
            S_CUFFT(cufftExecZ2Z(s->px, (cufftDoubleComplex*)s->wf(f), (cufftDoubleComplex*)s->wf(f), dir));
        } else {
            S_CUFFT(cufftExecC2C(s->px, (cufftComplex*)s->wf(f), (cufftComplex*)s->wf(f), dir));
        }
    }
    return SP_OK;
}

int exec_2d(sp_slab* s, bool inverse, cudaStream_t st) {
    cufftHandle p = inverse ? s->p2i : s->p2f;
    S_CUFFT(cufftSetStream(p, st));
    if (inverse) {
        if (s->fp64) S_CUFFT(cufftExecZ2D(p, (cufftDoubleComplex*)s->W, (cufftDoubleReal*)s->W));
        else S_CUFFT(cufftExecC2R(p, (cufftComplex*)s->W, (cufftReal*)s->W));
    } else {
        if (s->fp64) S_CUFFT(cufftExecD2Z(p, (cufftDoubleReal*)s->W, (cufftDoubleComplex*)s->W));
        else S_CUFFT(cufftExecR2C(p, (cufftReal*)s->W, (cufftComplex*)s->W));
    }
    return SP_OK;
}

template <typename T>
int phys(sp_slab* s, bool record_umax, cudaStream_t st) {
    const uint32_t fsr = 2u * s->fsc;
    auto* R = (T*)s->W;
    if (record_umax) {
        // CFL bound of the stage-0 velocity (the state's), before the products overwrite it
        auto* um = (unsigned long long*)s->base(s->off_umax);
        S_CUDA(cudaMemsetAsync(um, 0, 4 * sizeof(unsigned long long), st));
        const uint32_t rws = (uint32_t)s->m * (uint32_t)s->n;
        unsigned g = blocks_for((uint64_t)rws * (s->n / 2), kRedThreads);
        if (g > (unsigned)kRedBlocks) g = kRedBlocks;
        for (int c = 0; c < 3; ++c) {
            k_max_abs_padded<T><<<g, kRedThreads, 0, st>>>(R + (size_t)c * fsr, s->n, 2 * s->nh,
                                                           rws, um + c);
            S_CUDA(cudaGetLastError());
        }
        s->launches += 3;
    }
    const unsigned g = blocks_for(fsr / 4, kBlock);
    if (s->rot()) k_phys3d_rot<T><<<g, kBlock, 0, st>>>(R, fsr);
    else k_phys3d_basd<T><<<g, kBlock, 0, st>>>(R, fsr);
    S_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <typename T, int STAGE>
void post(sp_slab* s, cudaStream_t st) {
    const unsigned g = blocks_for(s->fsc / 2, kBlock);
    auto* W = (cplx<T>*)s->W;
    auto* u0 = (cplx<T>*)s->u0;
    auto* acc = (cplx<T>*)s->acc;
    auto* tab = (const T*)s->base(s->off_tab);
    auto* P = (const StepParams<T>*)s->base(s->off_params);
    const int j0 = s->rank * s->m;
    if (s->rot())
        k_post3d<T, true, STAGE><<<g, kBlock, 0, st>>>(W, u0, acc, tab, P, s->n, s->nh, s->fsc,
                                                       s->m, j0);
    else
        k_post3d<T, false, STAGE><<<g, kBlock, 0, st>>>(W, u0, acc, tab, P, s->n, s->nh, s->fsc,
                                                        s->m, j0);
}

template <typename T>
int post_stage(sp_slab* s, int stage, cudaStream_t st) {
    switch (stage) {
        case 0: post<T, 0>(s, st); break;
        case 1: post<T, 1>(s, st); break;
        case 2: post<T, 2>(s, st); break;
        default: post<T, 3>(s, st); break;
    }
    S_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <typename T>
int pre(sp_slab* s, cudaStream_t st) {
    const unsigned g = blocks_for(s->fsc / 2, kBlock);
    auto* P = (const StepParams<T>*)s->base(s->off_params);
    if (s->rot())
        k_pre3d<T, true><<<g, kBlock, 0, st>>>((cplx<T>*)s->u0, (cplx<T>*)s->W, s->n, s->nh,
                                              s->fsc, P, s->m, s->rank * s->m);
    else
        k_pre3d<T, false><<<g, kBlock, 0, st>>>((cplx<T>*)s->u0, (cplx<T>*)s->W, s->n, s->nh,
                                               s->fsc, P, s->m, s->rank * s->m);
    S_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <typename T>
int upload(sp_slab* s, double dt, cudaStream_t st) {
    const StepParams<T> p = make_step_params<T>(dt, s->alpha, s->amp, s->klo, s->khi, s->drag_k2,
                                                1.0 / std::pow((double)s->n, 3.0));
    std::vector<unsigned char> pb(sizeof(p));
    std::memcpy(pb.data(), &p, sizeof(p));
    std::vector<T> tab(2 * (size_t)s->nh);
    make_if_table<T>(s->nu, dt, s->nh, tab.data());
    std::vector<unsigned char> tb(tab.size() * sizeof(T));
    std::memcpy(tb.data(), tab.data(), tb.size());
    // pageable sources: the copy returns once the bytes are staged; the members outlive it
    if (pb != s->host_params) {
        s->host_params = pb;
        S_CUDA(cudaMemcpyAsync(s->base(s->off_params), s->host_params.data(), s->host_params.size(),
                               cudaMemcpyHostToDevice, st));
    }
    if (tb != s->host_tab) {
        s->host_tab = tb;
        S_CUDA(cudaMemcpyAsync(s->base(s->off_tab), s->host_tab.data(), s->host_tab.size(),
                               cudaMemcpyHostToDevice, st));
    }
    return SP_OK;
}

int make_plans(sp_slab* s) {
    const int n = s->n, m = s->m, nh = s->nh;
    size_t w1 = 0, w2 = 0, w3 = 0;
    S_CUFFT(cufftCreate(&s->px));
    s->have_px = true;
    S_CUFFT(cufftSetAutoAllocation(s->px, 0));
    long long nx[1] = {n}, emb[1] = {n};
    const long long stride = (long long)m * nh;
    S_CUFFT(cufftMakePlanMany64(s->px, 1, nx, emb, stride, 1, emb, stride, 1,
                                s->fp64 ? CUFFT_Z2Z : CUFFT_C2C, (long long)m * nh, &w1));
    long long shape[2] = {n, n}, cemb[2] = {n, nh}, remb[2] = {n, 2LL * nh};
    const long long cd = (long long)n * nh, rd = 2LL * n * nh;
    S_CUFFT(cufftCreate(&s->p2i));
    s->have_p2i = true;
    S_CUFFT(cufftSetAutoAllocation(s->p2i, 0));
    S_CUFFT(cufftMakePlanMany64(s->p2i, 2, shape, cemb, 1, cd, remb, 1, rd,
                                s->fp64 ? CUFFT_Z2D : CUFFT_C2R, (long long)s->ninv * m, &w2));
    S_CUFFT(cufftCreate(&s->p2f));
    s->have_p2f = true;
    S_CUFFT(cufftSetAutoAllocation(s->p2f, 0));
    S_CUFFT(cufftMakePlanMany64(s->p2f, 2, shape, remb, 1, rd, cemb, 1, cd,
                                s->fp64 ? CUFFT_D2Z : CUFFT_R2C, (long long)s->nfwd * m, &w3));
    s->ws_bytes = std::max(w1, std::max(w2, w3));
    return SP_OK;
}

}  // namespace

extern "C" {

sp_slab* sp_slab_create(int n, int nranks, int rank, int form, int fp64, int* status) {
    auto set = [&](int code, const std::string& why) -> sp_slab* {
        if (status) *status = code;
        sp::set_thread_error(why.c_str());
        return nullptr;
    };
    if (n < 8 || n % 2) return set(SP_ERR_ARG, "n must be even and >= 8");
    if (nranks < 1 || n % nranks || rank < 0 || rank >= nranks)
        return set(SP_ERR_ARG, "ranks must divide n; 0 <= rank < nranks");
    if (form != SP_FORM_BASDEVANT && form != SP_FORM_ROTATIONAL) return set(SP_ERR_ARG, "unknown form");
    auto* s = new sp_slab();
    s->n = n;
    s->P = nranks;
    s->rank = rank;
    s->m = n / nranks;
    s->nh = n / 2 + 1;
    s->form = form;
    s->fp64 = fp64 ? 1 : 0;
    s->csize = fp64 ? 16 : 8;
    const uint64_t fsc = (uint64_t)n * s->m * s->nh;
    if (2 * fsc >= (1ull << 32)) {
        delete s;
        return set(SP_ERR_ARG, "slab too large for 32-bit indexing");
    }
    s->fsc = (uint32_t)fsc;
    if (form == SP_FORM_ROTATIONAL) { s->ninv = 6; s->nfwd = 3; }
    else { s->ninv = 3; s->nfwd = 5; }
    s->nwork = std::max(s->ninv, s->nfwd);
    size_t off = 0;
    s->off_params = off; off += al256(16 * sizeof(double));
    s->off_tab = off; off += al256(2 * (size_t)s->nh * (fp64 ? 8 : 4));
    s->off_partials = off; off += al256((size_t)kRedBlocks * 4 * sizeof(double));
    s->off_umax = off; off += al256(4 * sizeof(unsigned long long));
    s->off_out = off; off += al256(8 * sizeof(double));
    s->aux_bytes = off;
    if (int r = make_plans(s)) {
        std::string why = s->err;
        sp_slab_destroy(s);
        return set(r, why);
    }
    if (status) *status = SP_OK;
    return s;
}

void sp_slab_destroy(sp_slab* s) {
    if (!s) return;
    if (s->have_px) cufftDestroy(s->px);
    if (s->have_p2i) cufftDestroy(s->p2i);
    if (s->have_p2f) cufftDestroy(s->p2f);
    delete s;
}

const char* sp_slab_last_error(const sp_slab* s) { return s ? s->err.c_str() : "null handle"; }

int64_t sp_slab_kernel_launches(const sp_slab* s) { return s ? s->launches : -1; }

int sp_slab_query_sizes(const sp_slab* s, int64_t* out, int count) {
    if (!s || !out || count < 0 || count > 8) return SP_ERR_ARG;
    const int64_t fb = (int64_t)s->fsc * (int64_t)s->csize;
    const int64_t v[8] = {(int64_t)s->fsc, 3 * fb, s->nwork * fb, s->nwork * fb,
                          (int64_t)s->aux_bytes, (int64_t)s->ws_bytes, s->m, s->nwork};
    for (int i = 0; i < count; ++i) out[i] = v[i];
    return SP_OK;
}

int64_t sp_slab_exchange_block_bytes(const sp_slab* s, int part) {
    if (!s || (part != 0 && part != 1)) return -1;
    const int nf = part == 0 ? s->ninv : s->nfwd;
    return (int64_t)nf * s->m * s->m * s->nh * (int64_t)s->csize;
}

int sp_slab_bind(sp_slab* s, void* u0, void* acc, void* work, void* send, void* recv, void* aux,
                 void* fft_workspace) {
    if (!s || !u0 || !acc || !work || !send || !recv || !aux || (s->ws_bytes && !fft_workspace))
        return sfail(s, SP_ERR_ARG, "sp_slab_bind: null buffer");
    if (recv == send && s->P > 1)
        return sfail(s, SP_ERR_ARG, "sp_slab_bind: send and recv must differ with several ranks");
    for (void* p : {u0, acc, work, send, recv, aux})
        if ((uintptr_t)p % 256) return sfail(s, SP_ERR_ARG, "sp_slab_bind: buffer not 256-byte aligned");
    s->u0 = u0;
    s->acc = acc;
    s->W = work;
    s->send = send;
    s->recv = recv;  // one rank: recv may be send itself (no exchange at all)
    s->aux = aux;
    s->host_params.clear();
    s->host_tab.clear();
    if (s->ws_bytes) {
        S_CUFFT(cufftSetWorkArea(s->px, fft_workspace));
        S_CUFFT(cufftSetWorkArea(s->p2i, fft_workspace));
        S_CUFFT(cufftSetWorkArea(s->p2f, fft_workspace));
    }
    s->bound = true;
    return SP_OK;
}

int sp_slab_set_physics(sp_slab* s, double nu, double alpha, double drag_k2, double force_klo,
                        double force_khi) {
    if (!s) return SP_ERR_ARG;
    s->nu = nu;
    s->alpha = alpha;
    s->drag_k2 = drag_k2;
    s->klo = force_klo;
    s->khi = force_khi;
    return SP_OK;
}

int sp_slab_set_forcing_amplitude(sp_slab* s, double amp) {
    if (!s) return SP_ERR_ARG;
    s->amp = amp;
    return SP_OK;
}

int sp_slab_set_dt(sp_slab* s, double dt, void* stream) {
    if (!s || !s->bound) return sfail(s, SP_ERR_STATE, "sp_slab_set_dt: bind first");
    auto st = (cudaStream_t)stream;
    return s->fp64 ? upload<double>(s, dt, st) : upload<float>(s, dt, st);
}

int sp_slab_prepare(sp_slab* s, void* stream) {
    if (!s || !s->bound) return sfail(s, SP_ERR_STATE, "sp_slab_prepare: bind first");
    auto st = (cudaStream_t)stream;
    int r = s->fp64 ? upload<double>(s, 0.0, st) : upload<float>(s, 0.0, st);
    if (r) return r;
    return s->fp64 ? pre<double>(s, st) : pre<float>(s, st);
}

int sp_slab_stage_part(sp_slab* s, int part, int stage, void* stream) {
    if (!s || !s->bound) return sfail(s, SP_ERR_STATE, "sp_slab_stage_part: bind first");
    if (stage < 0 || stage > 3 || part < 0 || part > 2)
        return sfail(s, SP_ERR_ARG, "sp_slab_stage_part: part 0..2, stage 0..3");
    auto st = (cudaStream_t)stream;
    int r;
    if (part == 0) {
        if ((r = exec_x(s, s->ninv, CUFFT_INVERSE, st))) return r;
        return rows<0>(s, s->W, s->send, s->ninv, st);
    }
    if (part == 1) {
        if ((r = rows<1>(s, s->recv, s->W, s->ninv, st))) return r;
        if ((r = exec_2d(s, true, st))) return r;
        if ((r = s->fp64 ? phys<double>(s, stage == 0, st) : phys<float>(s, stage == 0, st))) return r;
        if ((r = exec_2d(s, false, st))) return r;
        return rows<2>(s, s->W, s->send, s->nfwd, st);
    }
    if ((r = rows<3>(s, s->recv, s->W, s->nfwd, st))) return r;
    if ((r = exec_x(s, s->nfwd, CUFFT_FORWARD, st))) return r;
    return s->fp64 ? post_stage<double>(s, stage, st) : post_stage<float>(s, stage, st);
}

int sp_slab_max_velocity(sp_slab* s, double* out3, void* stream) {
    if (!s || !out3) return SP_ERR_ARG;
    auto st = (cudaStream_t)stream;
    unsigned long long bits[4] = {0, 0, 0, 0};
    S_CUDA(cudaMemcpyAsync(bits, s->base(s->off_umax), sizeof(bits), cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaStreamSynchronize(st));
    for (int c = 0; c < 3; ++c) std::memcpy(&out3[c], &bits[c], sizeof(double));
    return SP_OK;
}

int sp_slab_energy(sp_slab* s, const void* state, double* out, void* stream) {
    if (!s || !state || !out) return SP_ERR_ARG;
    auto st = (cudaStream_t)stream;
    const double norm = std::pow((double)s->n, 6.0);
    unsigned g = blocks_for(s->fsc, kRedThreads);
    if (g > (unsigned)kRedBlocks) g = kRedBlocks;
    auto* part = (double*)s->base(s->off_partials);
    // only the energy column is used: its weights depend on kz alone, valid on a ky slab
    if (s->fp64)
        k_reduce_spectral<double><<<g, kRedThreads, 0, st>>>((const cplx<double>*)state, s->n,
                                                             s->nh, 3, s->fsc, 1.0 / norm,
                                                             2.0 / norm, 0.0, -1.0, part);
    else
        k_reduce_spectral<float><<<g, kRedThreads, 0, st>>>((const cplx<float>*)state, s->n, s->nh,
                                                            3, s->fsc, 1.0 / norm, 2.0 / norm,
                                                            0.0, -1.0, part);
    S_CUDA(cudaGetLastError());
    k_finish_sum<4><<<1, kRedThreads, 0, st>>>(part, (int)g, 0.5, (double*)s->base(s->off_out));
    S_CUDA(cudaGetLastError());
    s->launches += 2;
    double o[4];
    S_CUDA(cudaMemcpyAsync(o, s->base(s->off_out), sizeof(o), cudaMemcpyDeviceToHost, st));
    S_CUDA(cudaStreamSynchronize(st));
    *out = o[0];
    return SP_OK;
}

}  // extern "C"
