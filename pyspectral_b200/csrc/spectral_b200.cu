// libspectral_b200: C ABI (include/spectral_b200.h) over the B200 IF-RK4 engine.
//
// One handle = one grid.  The host side of the reference backend (CupyCudaSolver,
// src/pyspectral/backends/cupy_cuda.py) is re-designed here in C++:
//   * cuFFT plans are created from C++ with auto-allocation off; their work area is a caller
//     buffer shared by every plan of the handle (the plans only run one after another).
//   * the per-step scalars (dt, drag and band factors) and the 1D integrating-factor table live
//     in device memory and are refreshed with one small copy only when they change, so a single
//     captured CUDA graph replays every step whatever dt or the forcing amplitude is.
//   * the pointwise phases are the fused kernels of pointwise.cuh; reductions are reduce.cuh.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "spectral_b200.h"
#include "closure.cuh"
#include "fused2d.h"
#include "fused3d.h"
#include "pointwise.cuh"
#include "reduce.cuh"

using namespace sp;

namespace {

thread_local std::string g_create_error;

const char* cufft_name(cufftResult r) {
    switch (r) {
        case CUFFT_SUCCESS: return "CUFFT_SUCCESS";
        case CUFFT_INVALID_PLAN: return "CUFFT_INVALID_PLAN";
        case CUFFT_ALLOC_FAILED: return "CUFFT_ALLOC_FAILED";
        case CUFFT_INVALID_TYPE: return "CUFFT_INVALID_TYPE";
        case CUFFT_INVALID_VALUE: return "CUFFT_INVALID_VALUE";
        case CUFFT_INTERNAL_ERROR: return "CUFFT_INTERNAL_ERROR";
        case CUFFT_EXEC_FAILED: return "CUFFT_EXEC_FAILED";
        case CUFFT_SETUP_FAILED: return "CUFFT_SETUP_FAILED";
        case CUFFT_INVALID_SIZE: return "CUFFT_INVALID_SIZE";
        case CUFFT_UNALIGNED_DATA: return "CUFFT_UNALIGNED_DATA";
        case CUFFT_INVALID_DEVICE: return "CUFFT_INVALID_DEVICE";
        case CUFFT_NO_WORKSPACE: return "CUFFT_NO_WORKSPACE";
        case CUFFT_NOT_IMPLEMENTED: return "CUFFT_NOT_IMPLEMENTED";
        case CUFFT_NOT_SUPPORTED: return "CUFFT_NOT_SUPPORTED";
        default: return "CUFFT_UNKNOWN_ERROR";
    }
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

namespace sp {
// Thread-local message behind sp_create_error(); also set by sp_spectrum_noalloc.
void set_thread_error(const char* why) { g_create_error = why; }
}  // namespace sp

// Device-resident run control (sp_run_to): the simulate.run rules evaluated on the GPU.
struct RunCtl {
    double t, t_end, tol, cfl, dt_max, dx, power, dt_fixed;
    double h_cfl;    // step of the current CFL window
    double dt_last;  // step just taken (t advances by it at the next control)
    double dt_tab;   // step the integrating-factor table was last filled for
    double amp;      // forcing amplitude in use
    long long steps;
    int have_power, pad;
};

struct sp_solver {
    // grid
    int n = 0, dim = 0, form = 0, fp64 = 0, fft_mode = 0;
    int nh = 0, ncomp = 0, nwork = 0, ninv = 0, nfwd = 0, nshell = 0;
    uint32_t fsc = 0, fsr = 0;
    size_t rsize = 0;  // bytes of one real
    // caller buffers
    void *u0 = nullptr, *acc = nullptr, *W = nullptr, *aux = nullptr, *fftws = nullptr;
    bool bound = false;
    // aux sub-blocks
    size_t off_params = 0, off_tab = 0, off_partials = 0, off_umax = 0, off_out = 0, off_spec = 0;
    size_t off_tw = 0;
    size_t aux_bytes = 0;
    // fused 2D mode: kept ky columns, work-array split (X then the transposed state u0t) and
    // whether the NumPy-layout state u0 reflects the transposed state
    int kc = 0;
    size_t work_bytes = 0, off_u0t = 0;
    // fused 3D mode: the work array is B_spec, then (at off_bphys) B_phys, then (at off_u0t) the
    // compact state; the compact accumulator lives at the start of acc
    size_t off_bphys = 0;
    bool u0_fresh = true;
    // cuFFT
    cufftHandle plan_inv = 0, plan_fwd = 0, plan_c2r1 = 0;
    bool have_inv = false, have_fwd = false, have_c2r1 = false;
    // learned closure (coarse 2D runs): work slots [S, u, v, omega, omega_x, omega_y], a batch-5
    // inverse plan over slots 1..5 and a batch-3 forward plan over slots 0..2
    sp_closure* closure = nullptr;
    cufftHandle plan_cl_inv = 0, plan_cl_fwd = 0;
    bool have_cl = false;
    size_t ws_bytes = 0;
    // physics and the host copy of the device parameter block
    double nu = 0, alpha = 0, drag_k2 = 1e30, klo = 0, khi = 0, amp = 0;
    bool tab_valid = false, params_valid = false;
    double tab_dt = 0, tab_nu = 0;
    std::vector<unsigned char> host_params, host_tab;
    // own kernel launches issued so far (graph replays count their captured kernels)
    int64_t launches = 0;
    int64_t graph_kernels = 0;
    // graph
    bool graph_on = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    // device-run chunk graph (sp_run_to): cfl_every steps with their control kernels
    cudaGraphExec_t run_exec = nullptr;
    int run_every = 0, run_flags = -1;
    int64_t run_kernels = 0;        // own kernels per chunk replay
    double run_phys[5] = {0, 0, 0, 0, 0};  // nu, alpha, drag_k2, klo, khi baked into the chunk
    size_t off_ctl = 0;
    RunCtl host_ctl{};
    // last error
    std::string err;

    void* params_dev() const { return (char*)aux + off_params; }
    void* tab_dev() const { return (char*)aux + off_tab; }
    double* partials_dev() const { return (double*)((char*)aux + off_partials); }
    unsigned long long* umax_dev() const { return (unsigned long long*)((char*)aux + off_umax); }
    double* out_dev() const { return (double*)((char*)aux + off_out); }
    double* spec_dev() const { return (double*)((char*)aux + off_spec); }
    void* tw_dev() const { return (char*)aux + off_tw; }
    void* u0t_dev() const { return (char*)W + off_u0t; }
    void* bphys_dev() const { return (char*)W + off_bphys; }
    bool fused() const { return fft_mode == SP_FFT_FUSED; }
    bool fused2() const { return fused() && dim == 2; }
    bool fused3() const { return fused() && dim == 3; }
    int rot() const { return form == SP_FORM_ROTATIONAL ? 1 : 0; }
    bool cl() const { return closure != nullptr; }
};

namespace {

int fail(sp_solver* s, int code, const char* what, const char* why) {
    if (s) {
        s->err = std::string(what) + ": " + why;
    }
    return code;
}

#define SP_CUDA(call)                                                                \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) return fail(s, SP_ERR_CUDA, #call, cudaGetErrorString(e_)); \
    } while (0)
#define SP_CUFFT(call)                                                                \
    do {                                                                              \
        cufftResult r_ = (call);                                                      \
        if (r_ != CUFFT_SUCCESS) return fail(s, SP_ERR_CUFFT, #call, cufft_name(r_)); \
    } while (0)
#define SP_CHECK_BOUND(s)                                                             \
    do {                                                                              \
        if (!(s)) return SP_ERR_ARG;                                                  \
        if (!(s)->bound) return fail((s), SP_ERR_STATE, "engine", "sp_bind was not called"); \
    } while (0)

unsigned grid_for(uint64_t items, int block) { return (unsigned)((items + block - 1) / block); }

// ---------------------------------------------------------------------------- parameters
// Integrating-factor table and step scalars in the real type, computed in fp64 on the host
// exactly like if_table / if_scalars (src/pyspectral/backends/_fused_common.py:10-19) and the
// band on/off rule of cupy_cuda.py:156-159.
template <typename T>
void fill_params(sp_solver* s, double dt, std::vector<unsigned char>& out) {
    const StepParams<T> p = make_step_params<T>(dt, s->alpha, s->amp, s->klo, s->khi, s->drag_k2,
                                                1.0 / std::pow((double)s->n, (double)s->dim));
    out.resize(sizeof(p));
    std::memcpy(out.data(), &p, sizeof(p));
}

template <typename T>
void fill_table(sp_solver* s, double dt, std::vector<unsigned char>& out) {
    std::vector<T> t(2 * (size_t)s->nh);
    make_if_table<T>(s->nu, dt, s->nh, t.data());
    out.resize(t.size() * sizeof(T));
    std::memcpy(out.data(), t.data(), out.size());
}

int upload_params(sp_solver* s, double dt, cudaStream_t st) {
    if (!s->tab_valid || s->tab_dt != dt || s->tab_nu != s->nu) {
        if (s->fp64) fill_table<double>(s, dt, s->host_tab);
        else fill_table<float>(s, dt, s->host_tab);
        // pageable source: the call returns once the bytes are staged, so host_tab may change
        SP_CUDA(cudaMemcpyAsync(s->tab_dev(), s->host_tab.data(), s->host_tab.size(),
                                cudaMemcpyHostToDevice, st));
        s->tab_valid = true;
        s->tab_dt = dt;
        s->tab_nu = s->nu;
    }
    std::vector<unsigned char> p;
    if (s->fp64) fill_params<double>(s, dt, p);
    else fill_params<float>(s, dt, p);
    if (!s->params_valid || p != s->host_params) {
        s->host_params = p;
        SP_CUDA(cudaMemcpyAsync(s->params_dev(), s->host_params.data(), s->host_params.size(),
                                cudaMemcpyHostToDevice, st));
        s->params_valid = true;
    }
    return SP_OK;
}

// ---------------------------------------------------------------------------- FFTs
int make_plan(sp_solver* s, bool inverse, int batch, cufftHandle* plan, size_t* ws) {
    long long shape[3], cemb[3], remb[3];
    for (int i = 0; i < s->dim; ++i) {
        shape[i] = s->n;
        cemb[i] = s->n;
        remb[i] = s->n;
    }
    cemb[s->dim - 1] = s->nh;
    remb[s->dim - 1] = 2LL * s->nh;
    SP_CUFFT(cufftCreate(plan));
    SP_CUFFT(cufftSetAutoAllocation(*plan, 0));
    long long cdist = s->fsc, rdist = 2LL * s->fsc;
    if (inverse) {
        SP_CUFFT(cufftMakePlanMany64(*plan, s->dim, shape, cemb, 1, cdist, remb, 1, rdist,
                                     s->fp64 ? CUFFT_Z2D : CUFFT_C2R, batch, ws));
    } else {
        SP_CUFFT(cufftMakePlanMany64(*plan, s->dim, shape, remb, 1, rdist, cemb, 1, cdist,
                                     s->fp64 ? CUFFT_D2Z : CUFFT_R2C, batch, ws));
    }
    return SP_OK;
}

int exec_c2r(sp_solver* s, cufftHandle plan, void* field, cudaStream_t st) {
    SP_CUFFT(cufftSetStream(plan, st));
    if (s->fp64) {
        SP_CUFFT(cufftExecZ2D(plan, (cufftDoubleComplex*)field, (cufftDoubleReal*)field));
    } else {
        SP_CUFFT(cufftExecC2R(plan, (cufftComplex*)field, (cufftReal*)field));
    }
    return SP_OK;
}

int exec_r2c(sp_solver* s, cufftHandle plan, void* field, cudaStream_t st) {
    SP_CUFFT(cufftSetStream(plan, st));
    if (s->fp64) {
        SP_CUFFT(cufftExecD2Z(plan, (cufftDoubleReal*)field, (cufftDoubleComplex*)field));
    } else {
        SP_CUFFT(cufftExecR2C(plan, (cufftReal*)field, (cufftComplex*)field));
    }
    return SP_OK;
}

size_t field_bytes(const sp_solver* s) { return (size_t)s->fsc * 2 * s->rsize; }

int fft_inverse(sp_solver* s, cudaStream_t st) {
    if (s->cl()) return exec_c2r(s, s->plan_cl_inv, (char*)s->W + field_bytes(s), st);
    if (s->fft_mode == SP_FFT_CUFFT) return exec_c2r(s, s->plan_inv, s->W, st);
    for (int i = 0; i < s->ninv; ++i) {
        int r = exec_c2r(s, s->plan_inv, (char*)s->W + i * field_bytes(s), st);
        if (r) return r;
    }
    return SP_OK;
}

int fft_forward(sp_solver* s, cudaStream_t st) {
    if (s->cl()) return exec_r2c(s, s->plan_cl_fwd, s->W, st);
    if (s->fft_mode == SP_FFT_CUFFT) return exec_r2c(s, s->plan_fwd, s->W, st);
    for (int i = 0; i < s->nfwd; ++i) {
        int r = exec_r2c(s, s->plan_fwd, (char*)s->W + i * field_bytes(s), st);
        if (r) return r;
    }
    return SP_OK;
}

// ---------------------------------------------------------------------------- kernels
template <typename T>
int launch_pre(sp_solver* s, cudaStream_t st) {
    auto* u0 = (cplx<T>*)s->u0;
    auto* W = (cplx<T>*)s->W;
    auto* P = (const StepParams<T>*)s->params_dev();
    unsigned g = grid_for(s->fsc / 2, kBlock);
    if (s->dim == 2 && s->cl())
        k_pre2d<T, true><<<g, kBlock, 0, st>>>(u0, W, s->n, s->nh, s->fsc, P);
    else if (s->dim == 2) k_pre2d<T><<<g, kBlock, 0, st>>>(u0, W, s->n, s->nh, s->fsc, P);
    else if (s->form == SP_FORM_ROTATIONAL)
        k_pre3d<T, true><<<g, kBlock, 0, st>>>(u0, W, s->n, s->nh, s->fsc, P);
    else k_pre3d<T, false><<<g, kBlock, 0, st>>>(u0, W, s->n, s->nh, s->fsc, P);
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <typename T>
int launch_phys(sp_solver* s, cudaStream_t st) {
    auto* R = (T*)s->W;
    unsigned g = grid_for(s->fsr / 4, kBlock);
    if (s->cl()) {
        // products and the closure term in one pass over the coarse field
        SP_CUDA(sp::closure::les_phase(s->closure, (float*)s->W, s->n, s->fsr, st));
        s->launches += 1;
        return SP_OK;
    }
    if (s->dim == 2) k_phys2d<T><<<g, kBlock, 0, st>>>(R, s->fsr);
    else if (s->form == SP_FORM_ROTATIONAL) k_phys3d_rot<T><<<g, kBlock, 0, st>>>(R, s->fsr);
    else k_phys3d_basd<T><<<g, kBlock, 0, st>>>(R, s->fsr);
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

template <typename T, int STAGE>
void post_stage(sp_solver* s, cudaStream_t st) {
    auto* W = (cplx<T>*)s->W;
    auto* u0 = (cplx<T>*)s->u0;
    auto* acc = (cplx<T>*)s->acc;
    auto* tab = (const T*)s->tab_dev();
    auto* P = (const StepParams<T>*)s->params_dev();
    unsigned g = grid_for(s->fsc / 2, kBlock);
    if (s->dim == 2 && s->cl())
        k_post2d<T, STAGE, true><<<g, kBlock, 0, st>>>(
            W, u0, acc, tab, P, s->n, s->nh, s->fsc, sp::closure::shell_gain(s->closure),
            sp::closure::shell_count(s->closure),
            (STAGE == 3 || sp::closure::every_stage(s->closure)) ? 1 : 0);
    else if (s->dim == 2)
        k_post2d<T, STAGE><<<g, kBlock, 0, st>>>(W, u0, acc, tab, P, s->n, s->nh, s->fsc);
    else if (s->form == SP_FORM_ROTATIONAL)
        k_post3d<T, true, STAGE><<<g, kBlock, 0, st>>>(W, u0, acc, tab, P, s->n, s->nh, s->fsc);
    else
        k_post3d<T, false, STAGE><<<g, kBlock, 0, st>>>(W, u0, acc, tab, P, s->n, s->nh, s->fsc);
}

template <typename T>
int launch_post(sp_solver* s, int stage, cudaStream_t st) {
    switch (stage) {
        case 0: post_stage<T, 0>(s, st); break;
        case 1: post_stage<T, 1>(s, st); break;
        case 2: post_stage<T, 2>(s, st); break;
        default: post_stage<T, 3>(s, st); break;
    }
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

int run_pre(sp_solver* s, cudaStream_t st) {
    return s->fp64 ? launch_pre<double>(s, st) : launch_pre<float>(s, st);
}
int run_phys(sp_solver* s, cudaStream_t st) {
    return s->fp64 ? launch_phys<double>(s, st) : launch_phys<float>(s, st);
}
int run_post(sp_solver* s, int stage, cudaStream_t st) {
    return s->fp64 ? launch_post<double>(s, stage, st) : launch_post<float>(s, stage, st);
}

int fused_row(sp_solver* s, cudaStream_t st) {
    SP_CUDA(sp::fused::row_pass(s->n, s->fp64, s->W, s->kc, s->tw_dev(), st));
    s->launches += 1;
    return SP_OK;
}

int fused_col(sp_solver* s, int stage, cudaStream_t st) {
    SP_CUDA(sp::fused::col_pass(s->n, s->fp64, stage, s->W, s->kc, s->u0t_dev(), s->acc,
                                s->tab_dev(), s->params_dev(), s->tw_dev(), st));
    s->launches += 1;
    return SP_OK;
}

// Stage of a closure run whose network term is held from the step's first stage: the plain
// velocity-pair transforms and products on work slots 1-2; slot 0 keeps the transformed term.
// fused 3D: the four passes of a stage (Y inverse, Z, Y forward, X with the Lawson update)
int fused3_phase(sp_solver* s, int phase, int stage, cudaStream_t st) {
    switch (phase) {
        case 0:
            SP_CUDA(sp::fused3::y_inverse(s->n, s->fp64, s->rot(), s->W, s->bphys_dev(), s->ninv,
                                          s->tw_dev(), st));
            break;
        case 1:
            SP_CUDA(sp::fused3::z_pass(s->n, s->fp64, s->rot(), 0, s->bphys_dev(), s->tw_dev(),
                                       s->umax_dev(), 0, st));
            break;
        case 2:
            SP_CUDA(sp::fused3::y_forward(s->n, s->fp64, s->rot(), s->bphys_dev(), s->W, s->nfwd,
                                          s->tw_dev(), st));
            break;
        default:
            SP_CUDA(sp::fused3::x_pass(s->n, s->fp64, s->rot(), stage, s->W, s->u0t_dev(), s->acc,
                                       s->tab_dev(), s->params_dev(), s->tw_dev(), st));
    }
    s->launches += 1;
    return SP_OK;
}

// fused 3D: max |u_i| of the live state into umax_dev()[0..3) (its stage-0 inputs are in B_spec)
int fused3_umax(sp_solver* s, cudaStream_t st) {
    SP_CUDA(sp::fused3::y_inverse(s->n, s->fp64, s->rot(), s->W, s->bphys_dev(), 3, s->tw_dev(),
                                  st));
    SP_CUDA(sp::fused3::z_pass(s->n, s->fp64, s->rot(), 1, s->bphys_dev(), s->tw_dev(),
                               s->umax_dev(), 1, st));
    s->launches += 2;
    return SP_OK;
}

int held_closure_stage(sp_solver* s, cudaStream_t st) {
    char* Wuv = (char*)s->W + field_bytes(s);
    int r;
    if ((r = exec_c2r(s, s->plan_inv, Wuv, st))) return r;
    k_phys2d<float><<<grid_for(s->fsr / 4, kBlock), kBlock, 0, st>>>((float*)Wuv, s->fsr);
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return exec_r2c(s, s->plan_fwd, Wuv, st);
}

// One IF-RK4 step: 4 x (inverse FFT -> phys -> forward FFT -> post), cupy_cuda.py:163-178;
// in the fused mode 4 x (row pass -> column pass).
int run_step(sp_solver* s, cudaStream_t st) {
    if (s->cl() && !sp::closure::every_stage(s->closure)) {
        for (int stage = 0; stage < 4; ++stage) {
            int r;
            if (stage == 0) {
                if ((r = fft_inverse(s, st))) return r;
                if ((r = run_phys(s, st))) return r;
                if ((r = fft_forward(s, st))) return r;
            } else if ((r = held_closure_stage(s, st))) {
                return r;
            }
            if ((r = run_post(s, stage, st))) return r;
        }
        return SP_OK;
    }
    if (s->fused3()) {
        for (int stage = 0; stage < 4; ++stage)
            for (int phase = 0; phase < 4; ++phase) {
                int r = fused3_phase(s, phase, stage, st);
                if (r) return r;
            }
        return SP_OK;
    }
    if (s->fused()) {
        for (int stage = 0; stage < 4; ++stage) {
            int r;
            if ((r = fused_row(s, st))) return r;
            if ((r = fused_col(s, stage, st))) return r;
        }
        return SP_OK;
    }
    for (int stage = 0; stage < 4; ++stage) {
        int r;
        if ((r = fft_inverse(s, st))) return r;
        if ((r = run_phys(s, st))) return r;
        if ((r = fft_forward(s, st))) return r;
        if ((r = run_post(s, stage, st))) return r;
    }
    return SP_OK;
}

int capture_step(sp_solver* s) {
    if (!s->cap_stream) SP_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    SP_CUDA(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    int64_t before = s->launches;
    int r = run_step(s, s->cap_stream);
    s->graph_kernels = s->launches - before;
    s->launches = before;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->cap_stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(s, SP_ERR_CUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&s->exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        s->exec = nullptr;
        return fail(s, SP_ERR_CUDA, "cudaGraphInstantiate", cudaGetErrorString(e));
    }
    return SP_OK;
}

void drop_graph(sp_solver* s) {
    if (s->exec) {
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    if (s->run_exec) {
        cudaGraphExecDestroy(s->run_exec);
        s->run_exec = nullptr;
    }
}

// ---------------------------------------------------------------------------- device runs
// One control per step: t advances by the previous step; at a CFL step (refresh) the CFL bound
// sum_i max|u_i| and the forcing band energy of the live state give h = min(dt_max,
// cfl dx / umax) and A = P / (2 E_band) (simulate.run, simulate.py:45-95); then dt = min(h,
// t_end - t) (0 once t_end is reached: the step leaves the state unchanged) and the step
// scalars and the integrating-factor table are written for it.
template <typename T>
__global__ void __launch_bounds__(256) k_control(RunCtl* __restrict__ c,
                                                 const unsigned long long* __restrict__ umax,
                                                 int ncomp, const double* __restrict__ band,
                                                 int refresh, StepParams<T>* __restrict__ P,
                                                 T* __restrict__ tab, int nh, double nu,
                                                 double alpha, double klo, double khi,
                                                 double drag_k2, double scale) {
    __shared__ double s_dt;
    __shared__ int s_fill;
    if (threadIdx.x == 0) {
        c->t += c->dt_last;
        if (c->dt_last > 0.0) c->steps += 1;
        if (refresh) {
            double h = c->dt_max;
            if (c->dt_fixed > 0.0) {
                h = c->dt_fixed;
            } else {
                double u = 0.0;
                for (int k = 0; k < ncomp; ++k) u += __longlong_as_double((long long)umax[k]);
                if (u > 0.0 && isfinite(u)) h = fmin(c->dt_max, c->cfl * c->dx / u);
            }
            c->h_cfl = h;
            if (c->have_power) {
                const double eb = band[3];
                c->amp = eb > 0.0 ? c->power / (2.0 * eb) : 0.0;
            }
        }
        const double dt = c->t < c->t_end - c->tol ? fmin(c->h_cfl, c->t_end - c->t) : 0.0;
        c->dt_last = dt;
        StepParams<T> p;
        p.dt = (T)dt;
        p.ea1 = (T)exp(-alpha * dt);
        p.eah = (T)exp(-alpha * 0.5 * dt);
        p.eb1 = (T)exp(c->amp * dt);
        p.ebh = (T)exp(c->amp * 0.5 * dt);
        const bool band_on = c->amp != 0.0;
        p.klo2 = band_on ? (T)(klo * klo) : (T)1;
        p.khi2 = band_on ? (T)(khi * khi) : (T)0;
        p.ka2 = (T)drag_k2;
        p.scale = (T)scale;
        *P = p;
        s_fill = dt != c->dt_tab;
        c->dt_tab = dt;
        s_dt = dt;
    }
    __syncthreads();
    if (!s_fill) return;
    const double dt = s_dt;
    for (int m = threadIdx.x; m < nh; m += blockDim.x) {
        const double mm = (double)m;
        tab[m] = (T)exp(-nu * mm * mm * dt);
        tab[nh + m] = (T)exp(-nu * mm * mm * 0.5 * dt);
    }
}

__global__ void k_control_close(RunCtl* __restrict__ c) {
    c->t += c->dt_last;
    if (c->dt_last > 0.0) c->steps += 1;
    c->dt_last = 0.0;
}

}  // namespace

namespace {

// The CFL bound and the band energy of the live state, enqueued without a host read:
// umax_dev()[0..ncomp) and out_dev()[3].
int enqueue_run_diag(sp_solver* s, bool need_umax, bool need_band, cudaStream_t st) {
    if (need_umax) {
        SP_CUDA(cudaMemsetAsync(s->umax_dev(), 0, 4 * sizeof(unsigned long long), st));
        if (s->fused3()) {
            int r = fused3_umax(s, st);
            if (r) return r;
        } else if (s->fused()) {
            SP_CUDA(sp::fused::row_max(s->n, s->fp64, s->W, s->kc, s->tw_dev(), s->umax_dev(), st));
            s->launches += 1;
        } else {
            cufftHandle plan = s->fft_mode == SP_FFT_CUFFT_LEAN ? s->plan_inv : s->plan_c2r1;
            unsigned gv = grid_for(s->fsc, kRedThreads);
            uint32_t rows = s->fsc / (uint32_t)s->nh;
            unsigned gm = grid_for((uint64_t)rows * (s->n / 2), kRedThreads);
            if (gm > (unsigned)kRedBlocks) gm = kRedBlocks;
            double scale = 1.0 / std::pow((double)s->n, (double)s->dim);
            for (int c = 0; c < s->dim; ++c) {
                if (s->fp64)
                    k_velocity_component<double><<<gv, kRedThreads, 0, st>>>(
                        (const cplx<double>*)s->u0, (cplx<double>*)s->acc, s->n, s->nh, s->dim,
                        s->fsc, c, scale);
                else
                    k_velocity_component<float><<<gv, kRedThreads, 0, st>>>(
                        (const cplx<float>*)s->u0, (cplx<float>*)s->acc, s->n, s->nh, s->dim,
                        s->fsc, c, (float)scale);
                SP_CUDA(cudaGetLastError());
                int r = exec_c2r(s, plan, s->acc, st);
                if (r) return r;
                if (s->fp64)
                    k_max_abs_padded<double><<<gm, kRedThreads, 0, st>>>(
                        (const double*)s->acc, s->n, 2 * s->nh, rows, s->umax_dev() + c);
                else
                    k_max_abs_padded<float><<<gm, kRedThreads, 0, st>>>(
                        (const float*)s->acc, s->n, 2 * s->nh, rows, s->umax_dev() + c);
                SP_CUDA(cudaGetLastError());
                s->launches += 2;
            }
        }
    }
    if (need_band) {
        if (s->fused3()) {
            // the live state is the compact copy: refresh the NumPy-layout state it sums over
            SP_CUDA(sp::fused3::state_move(s->fp64, s->u0, s->u0t_dev(), s->n, 0, st));
            s->launches += 1;
        }
        if (s->fused2()) {
            SP_CUDA(sp::fused::reduce_t(s->fp64, s->u0t_dev(), s->n, s->kc, 0, 1, s->klo, s->khi,
                                        s->partials_dev(), kRedBlocks, s->out_dev(), st));
            s->launches += 2;
        } else {
            double norm = std::pow((double)s->n, 2.0 * s->dim);
            unsigned g = grid_for(s->fsc, kRedThreads);
            if (g > (unsigned)kRedBlocks) g = kRedBlocks;
            if (s->fp64)
                k_reduce_spectral<double><<<g, kRedThreads, 0, st>>>(
                    (const cplx<double>*)s->u0, s->n, s->nh, s->dim, s->fsc, 1.0 / norm,
                    2.0 / norm, s->klo * s->klo, s->khi * s->khi, s->partials_dev());
            else
                k_reduce_spectral<float><<<g, kRedThreads, 0, st>>>(
                    (const cplx<float>*)s->u0, s->n, s->nh, s->dim, s->fsc, 1.0 / norm,
                    2.0 / norm, s->klo * s->klo, s->khi * s->khi, s->partials_dev());
            SP_CUDA(cudaGetLastError());
            k_finish_sum<4><<<1, kRedThreads, 0, st>>>(s->partials_dev(), (int)g, 0.5, s->out_dev());
            SP_CUDA(cudaGetLastError());
            s->launches += 2;
        }
    }
    return SP_OK;
}

template <typename T>
int enqueue_control(sp_solver* s, bool refresh, cudaStream_t st) {
    k_control<T><<<1, 256, 0, st>>>((RunCtl*)((char*)s->aux + s->off_ctl), s->umax_dev(), s->dim,
                                    s->out_dev(), refresh ? 1 : 0,
                                    (StepParams<T>*)s->params_dev(), (T*)s->tab_dev(), s->nh,
                                    s->nu, s->alpha, s->klo, s->khi, s->drag_k2,
                                    1.0 / std::pow((double)s->n, (double)s->dim));
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

// One chunk of `every` steps: at its first step the CFL / forcing refresh (when asked for),
// then per step a control and the step; t closed at the end.
int enqueue_run_chunk(sp_solver* s, int every, bool cfl, bool power, cudaStream_t st) {
    int r;
    for (int k = 0; k < every; ++k) {
        const bool refresh = k == 0;
        if (refresh && (r = enqueue_run_diag(s, cfl, power, st))) return r;
        if ((r = s->fp64 ? enqueue_control<double>(s, refresh, st)
                         : enqueue_control<float>(s, refresh, st)))
            return r;
        if ((r = run_step(s, st))) return r;
    }
    k_control_close<<<1, 1, 0, st>>>((RunCtl*)((char*)s->aux + s->off_ctl));
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    return SP_OK;
}

int capture_run_chunk(sp_solver* s, int every, int flags) {
    const double phys[5] = {s->nu, s->alpha, s->drag_k2, s->klo, s->khi};
    if (s->run_exec && s->run_every == every && s->run_flags == flags &&
        std::memcmp(phys, s->run_phys, sizeof(phys)) == 0)
        return SP_OK;
    if (s->run_exec) {
        cudaGraphExecDestroy(s->run_exec);
        s->run_exec = nullptr;
    }
    if (!s->cap_stream) SP_CUDA(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    SP_CUDA(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int64_t before = s->launches;
    int r = enqueue_run_chunk(s, every, flags & 1, flags & 2, s->cap_stream);
    const int64_t per_chunk = s->launches - before;
    s->launches = before;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->cap_stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(s, SP_ERR_CUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&s->run_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        s->run_exec = nullptr;
        return fail(s, SP_ERR_CUDA, "cudaGraphInstantiate", cudaGetErrorString(e));
    }
    s->run_every = every;
    s->run_flags = flags;
    s->run_kernels = per_chunk;
    std::memcpy(s->run_phys, phys, sizeof(phys));
    return SP_OK;
}

}  // namespace

// ============================================================================== C ABI
extern "C" {

int sp_abi_version(void) { return SP_ABI_VERSION; }

const char* sp_create_error(void) { return g_create_error.c_str(); }

const char* sp_last_error(const sp_solver* s) { return s ? s->err.c_str() : "null handle"; }

int64_t sp_kernel_launches(const sp_solver* s) { return s ? s->launches : -1; }

sp_solver* sp_create(int n, int dim, int form, int fp64, int fft_mode, int* status) {
    auto set = [&](int code, const std::string& why) -> sp_solver* {
        if (status) *status = code;
        g_create_error = why;
        return nullptr;
    };
    if (dim != 2 && dim != 3) return set(SP_ERR_ARG, "dim must be 2 or 3");
    if (n < 8 || n % 2) return set(SP_ERR_ARG, "n must be even and >= 8");
    if (form != SP_FORM_BASDEVANT && form != SP_FORM_ROTATIONAL)
        return set(SP_ERR_ARG, "unknown form");
    if (dim == 2 && form != SP_FORM_BASDEVANT)
        return set(SP_ERR_UNSUPPORTED, "2D supports the basdevant form only");
    if (fft_mode != SP_FFT_CUFFT && fft_mode != SP_FFT_CUFFT_LEAN && fft_mode != SP_FFT_FUSED)
        return set(SP_ERR_ARG, "unknown fft_mode");
    if (fft_mode == SP_FFT_FUSED && dim == 3 && !sp::fused3::supported(n, fp64))
        return set(SP_ERR_UNSUPPORTED,
                   "the fused 3D FFT engine needs n a power of two in 16..512");
    if (fft_mode == SP_FFT_FUSED && dim == 2 && !sp::fused::supported(n, fp64))
        return set(SP_ERR_UNSUPPORTED,
                   "the fused FFT engine needs n a power of two in 16..8192 (fp32) or 16..4096 (fp64)");
    int nh = n / 2 + 1;
    uint64_t fsc = (uint64_t)nh * (uint64_t)n * (dim == 3 ? (uint64_t)n : 1ull);
    if (2 * fsc >= (1ull << 32)) return set(SP_ERR_ARG, "grid too large for 32-bit indexing");
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev < 1)
        return set(SP_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(ce));

    auto* s = new sp_solver();
    s->n = n;
    s->dim = dim;
    s->form = form;
    s->fp64 = fp64 ? 1 : 0;
    s->fft_mode = fft_mode;
    s->nh = nh;
    s->fsc = (uint32_t)fsc;
    s->fsr = (uint32_t)(2 * fsc);
    s->rsize = fp64 ? 8 : 4;
    s->ncomp = dim == 2 ? 1 : 3;
    if (dim == 2) { s->ninv = 2; s->nfwd = 2; }
    else if (form == SP_FORM_ROTATIONAL) { s->ninv = 6; s->nfwd = 3; }
    else { s->ninv = 3; s->nfwd = 5; }
    s->nwork = s->ninv > s->nfwd ? s->ninv : s->nfwd;
    s->nshell = (int)std::floor(std::sqrt((double)dim) * (double)(n / 2) + 0.5) + 1;
    // aux layout
    size_t off = 0;
    s->off_params = off; off += align256(16 * sizeof(double));
    s->off_tab = off; off += align256(2 * (size_t)nh * s->rsize);
    s->off_partials = off; off += align256((size_t)kRedBlocks * 4 * sizeof(double));
    s->off_umax = off; off += align256(4 * sizeof(unsigned long long));
    s->off_out = off; off += align256(8 * sizeof(double));
    s->off_spec = off; off += align256((size_t)s->nshell * sizeof(double));
    s->off_ctl = off; off += align256(sizeof(RunCtl));
    s->off_tw = off;
    if (fft_mode == SP_FFT_FUSED && sp::fused::supported(n, fp64))
        off += align256((size_t)sp::fused::twiddle_table_size(n) * 2 * s->rsize);
    s->aux_bytes = off;
    s->work_bytes = (size_t)s->nwork * field_bytes(s);

    if (fft_mode == SP_FFT_FUSED && dim == 3) {
        const int rot = form == SP_FORM_ROTATIONAL ? 1 : 0;
        s->off_bphys = align256(sp::fused3::spec_bytes(n, fp64, rot));
        s->off_u0t = s->off_bphys + align256(sp::fused3::phys_bytes(n, fp64, rot));
        s->work_bytes = s->off_u0t + align256(sp::fused3::compact_bytes(n, fp64));
        cudaError_t e = sp::fused3::set_attributes(n, fp64, rot);
        if (e != cudaSuccess) {
            sp_destroy(s);
            return set(SP_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        }
        if (status) *status = SP_OK;
        return s;
    }
    if (fft_mode == SP_FFT_FUSED) {
        s->kc = sp::fused::kc_of(n);
        size_t csz = 2 * s->rsize;
        s->off_u0t = align256((size_t)n * s->kc * 2 * csz);         // X: n x kc pairs
        s->work_bytes = s->off_u0t + align256((size_t)s->kc * n * csz);  // + u0t: kc x n
        cudaError_t e = sp::fused::set_attributes(n, fp64);
        if (e != cudaSuccess) {
            sp_destroy(s);
            return set(SP_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        }
        if (status) *status = SP_OK;
        return s;
    }

    bool lean = fft_mode == SP_FFT_CUFFT_LEAN;
    size_t ws_inv = 0, ws_fwd = 0, ws_one = 0;
    int r = make_plan(s, true, lean ? 1 : s->ninv, &s->plan_inv, &ws_inv);
    if (!r) { s->have_inv = true; r = make_plan(s, false, lean ? 1 : s->nfwd, &s->plan_fwd, &ws_fwd); }
    if (!r) s->have_fwd = true;
    if (!r && !lean) {
        r = make_plan(s, true, 1, &s->plan_c2r1, &ws_one);
        if (!r) s->have_c2r1 = true;
    }
    if (r) {
        std::string why = s->err;
        sp_destroy(s);
        return set(r, why);
    }
    s->ws_bytes = ws_inv > ws_fwd ? ws_inv : ws_fwd;
    if (ws_one > s->ws_bytes) s->ws_bytes = ws_one;
    if (status) *status = SP_OK;
    return s;
}

void sp_destroy(sp_solver* s) {
    if (!s) return;
    drop_graph(s);
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    if (s->have_inv) cufftDestroy(s->plan_inv);
    if (s->have_fwd) cufftDestroy(s->plan_fwd);
    if (s->have_c2r1) cufftDestroy(s->plan_c2r1);
    if (s->have_cl) {
        cufftDestroy(s->plan_cl_inv);
        cufftDestroy(s->plan_cl_fwd);
    }
    delete s;
}

int sp_query_sizes(const sp_solver* s, int64_t* out, int count) {
    if (!s || !out || count < 0 || count > SP_SZ_COUNT) return SP_ERR_ARG;
    int64_t v[SP_SZ_COUNT];
    v[SP_SZ_MODES] = s->fsc;
    v[SP_SZ_NCOMP] = s->ncomp;
    v[SP_SZ_NWORK] = s->nwork;
    v[SP_SZ_NINV] = s->ninv;
    v[SP_SZ_NFWD] = s->nfwd;
    v[SP_SZ_STATE_BYTES] = (int64_t)s->ncomp * (int64_t)field_bytes(s);
    v[SP_SZ_WORK_BYTES] = (int64_t)s->work_bytes;
    v[SP_SZ_AUX_BYTES] = (int64_t)s->aux_bytes;
    v[SP_SZ_FFTWS_BYTES] = (int64_t)s->ws_bytes;
    v[SP_SZ_NSHELL] = s->nshell;
    for (int i = 0; i < count; ++i) out[i] = v[i];
    return SP_OK;
}

int sp_bind(sp_solver* s, void* u0, void* acc, void* work, void* aux, void* fft_workspace) {
    if (!s) return SP_ERR_ARG;
    if (!u0 || !acc || !work || !aux || (s->ws_bytes && !fft_workspace))
        return fail(s, SP_ERR_ARG, "sp_bind", "null buffer");
    for (void* p : {u0, acc, work, aux})
        if ((uintptr_t)p % 256) return fail(s, SP_ERR_ARG, "sp_bind", "buffer not 256-byte aligned");
    s->u0 = u0;
    s->acc = acc;
    s->W = work;
    s->aux = aux;
    s->fftws = fft_workspace;
    if (s->ws_bytes && !s->fused()) {
        SP_CUFFT(cufftSetWorkArea(s->plan_inv, fft_workspace));
        SP_CUFFT(cufftSetWorkArea(s->plan_fwd, fft_workspace));
        if (s->have_c2r1) SP_CUFFT(cufftSetWorkArea(s->plan_c2r1, fft_workspace));
        if (s->have_cl) {
            SP_CUFFT(cufftSetWorkArea(s->plan_cl_inv, fft_workspace));
            SP_CUFFT(cufftSetWorkArea(s->plan_cl_fwd, fft_workspace));
        }
    }
    s->bound = true;
    s->tab_valid = false;
    s->params_valid = false;
    drop_graph(s);
    if (s->fused()) {
        // per-pass twiddle table, fp64 on the host, rounded to the real type
        std::vector<double> tw(2 * (size_t)sp::fused::twiddle_table_size(s->n));
        sp::fused::fill_twiddles(s->n, tw.data());
        if (s->fp64) {
            SP_CUDA(cudaMemcpy(s->tw_dev(), tw.data(), tw.size() * sizeof(double),
                               cudaMemcpyHostToDevice));
        } else {
            std::vector<float> twf(tw.begin(), tw.end());
            SP_CUDA(cudaMemcpy(s->tw_dev(), twf.data(), twf.size() * sizeof(float),
                               cudaMemcpyHostToDevice));
        }
        s->u0_fresh = true;
    }
    return SP_OK;
}

int sp_set_physics(sp_solver* s, double nu, double alpha, double drag_k2, double force_klo,
                   double force_khi) {
    if (!s) return SP_ERR_ARG;
    s->nu = nu;
    s->alpha = alpha;
    s->drag_k2 = drag_k2;
    s->klo = force_klo;
    s->khi = force_khi;
    return SP_OK;
}

int sp_set_forcing_amplitude(sp_solver* s, double amp) {
    if (!s) return SP_ERR_ARG;
    s->amp = amp;
    return SP_OK;
}

int sp_prepare(sp_solver* s, void* stream) {
    SP_CHECK_BOUND(s);
    auto st = (cudaStream_t)stream;
    // the scale lives in the parameter block: make sure it exists (dt is irrelevant here)
    if (!s->params_valid) {
        int r = upload_params(s, s->tab_valid ? s->tab_dt : 0.0, st);
        if (r) return r;
    }
    if (s->fused3()) {
        SP_CUDA(sp::fused3::mask(s->fp64, s->u0, s->n, st));
        SP_CUDA(sp::fused3::state_move(s->fp64, s->u0, s->u0t_dev(), s->n, 1, st));
        s->launches += 2;
        s->u0_fresh = true;
        return fused3_phase(s, 3, -1, st);
    }
    if (s->fused()) {
        SP_CUDA(sp::fused::mask2d(s->fp64, s->u0, s->n, st));
        SP_CUDA(sp::fused::transpose_in(s->fp64, s->u0, s->u0t_dev(), s->n, s->kc, st));
        s->launches += 2;
        int r = fused_col(s, -1, st);
        s->u0_fresh = true;
        return r;
    }
    return run_pre(s, st);
}

int sp_sync_state(sp_solver* s, void* stream) {
    SP_CHECK_BOUND(s);
    if (!s->fused() || s->u0_fresh) return SP_OK;
    if (s->fused3()) {
        SP_CUDA(sp::fused3::state_move(s->fp64, s->u0, s->u0t_dev(), s->n, 0, (cudaStream_t)stream));
        s->launches += 1;
        s->u0_fresh = true;
        return SP_OK;
    }
    SP_CUDA(sp::fused::transpose_out(s->fp64, s->u0t_dev(), s->u0, s->n, s->kc,
                                     (cudaStream_t)stream));
    s->launches += 1;
    s->u0_fresh = true;
    return SP_OK;
}

int sp_set_column_streaming(int enable) {
    sp::fused::set_streaming(enable != 0);
    return SP_OK;
}
int sp_column_streaming(void) { return sp::fused::streaming() ? 1 : 0; }

int sp_take_device_error(unsigned int* bits) {
    if (!bits) return SP_ERR_ARG;
    cudaError_t e = sp::fused::take_stream_error(bits);
    if (e != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return SP_ERR_CUDA;
    }
    return SP_OK;
}

int sp_wait_probe(unsigned int polls, void* stream) {
    if (polls == 0 || polls > (1u << 20)) {
        set_thread_error("sp_wait_probe: polls must be 1..2^20");
        return SP_ERR_ARG;
    }
    cudaError_t e = sp::fused::wait_probe(polls, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        set_thread_error(cudaGetErrorString(e));
        return SP_ERR_CUDA;
    }
    return SP_OK;
}

int sp_set_graph(sp_solver* s, int enable) {
    if (!s) return SP_ERR_ARG;
    s->graph_on = enable != 0;
    if (!s->graph_on) drop_graph(s);
    return SP_OK;
}

int sp_step(sp_solver* s, double dt, void* stream) {
    SP_CHECK_BOUND(s);
    auto st = (cudaStream_t)stream;
    int r = upload_params(s, dt, st);
    if (r) return r;
    if (s->fused()) s->u0_fresh = false;
    if (!s->graph_on) return run_step(s, st);
    if (!s->exec && (r = capture_step(s))) return r;
    SP_CUDA(cudaGraphLaunch(s->exec, st));
    s->launches += s->graph_kernels;
    return SP_OK;
}

int sp_run_phase(sp_solver* s, int phase, int stage, void* stream) {
    SP_CHECK_BOUND(s);
    auto st = (cudaStream_t)stream;
    if (stage < 0 || stage > 3) return fail(s, SP_ERR_ARG, "sp_run_phase", "stage must be 0..3");
    if (s->fused3()) {
        if (phase < 0 || phase > 3) return fail(s, SP_ERR_ARG, "sp_run_phase", "phase must be 0..3");
        if (phase == 3 && !s->params_valid)
            return fail(s, SP_ERR_STATE, "sp_run_phase", "no step parameters yet");
        if (phase == 3) s->u0_fresh = false;
        return fused3_phase(s, phase, stage, st);
    }
    if (s->fused()) {
        if (phase < 0 || phase > 3) return fail(s, SP_ERR_ARG, "sp_run_phase", "phase must be 0..3");
        if (phase == 0) return fused_row(s, st);
        if (phase == 3) {
            if (!s->params_valid) return fail(s, SP_ERR_STATE, "sp_run_phase", "no step parameters yet");
            s->u0_fresh = false;
            return fused_col(s, stage, st);
        }
        return SP_OK;  // phases 1 and 2 live inside the row pass
    }
    switch (phase) {
        case 0: return fft_inverse(s, st);
        case 1: return run_phys(s, st);
        case 2: return fft_forward(s, st);
        case 3:
            if (!s->params_valid) return fail(s, SP_ERR_STATE, "sp_run_phase", "no step parameters yet");
            return run_post(s, stage, st);
        default: return fail(s, SP_ERR_ARG, "sp_run_phase", "phase must be 0..3");
    }
}

int sp_diagnostics(sp_solver* s, const void* state, double band_klo, double band_khi,
                   double* out, void* stream) {
    SP_CHECK_BOUND(s);
    if (!state || !out) return fail(s, SP_ERR_ARG, "sp_diagnostics", "null pointer");
    auto st = (cudaStream_t)stream;
    if (state == s->u0) {
        int r = sp_sync_state(s, stream);
        if (r) return r;
    }
    double norm = std::pow((double)s->n, 2.0 * s->dim);
    double w_edge = 1.0 / norm, w_mid = 2.0 / norm;
    unsigned g = grid_for(s->fsc, kRedThreads);
    if (g > (unsigned)kRedBlocks) g = kRedBlocks;
    double klo2 = band_klo * band_klo, khi2 = band_khi * band_khi;
    if (s->fp64)
        k_reduce_spectral<double><<<g, kRedThreads, 0, st>>>((const cplx<double>*)state, s->n, s->nh,
                                                             s->dim, s->fsc, w_edge, w_mid, klo2,
                                                             khi2, s->partials_dev());
    else
        k_reduce_spectral<float><<<g, kRedThreads, 0, st>>>((const cplx<float>*)state, s->n, s->nh,
                                                            s->dim, s->fsc, w_edge, w_mid, klo2,
                                                            khi2, s->partials_dev());
    SP_CUDA(cudaGetLastError());
    k_finish_sum<4><<<1, kRedThreads, 0, st>>>(s->partials_dev(), (int)g, 0.5, s->out_dev());
    SP_CUDA(cudaGetLastError());
    s->launches += 2;
    SP_CUDA(cudaMemcpyAsync(out, s->out_dev(), 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    SP_CUDA(cudaStreamSynchronize(st));
    return SP_OK;
}

int sp_max_velocity(sp_solver* s, const void* state, double* out_sum, double* out_per_comp,
                    void* stream) {
    SP_CHECK_BOUND(s);
    if (!state || !out_sum) return fail(s, SP_ERR_ARG, "sp_max_velocity", "null pointer");
    auto st = (cudaStream_t)stream;
    int ncomp = s->dim;  // velocity components
    if (s->fused3()) {
        if (state != s->u0)
            return fail(s, SP_ERR_UNSUPPORTED, "sp_max_velocity",
                        "the fused engine bounds the velocity of its own state only");
        SP_CUDA(cudaMemsetAsync(s->umax_dev(), 0, 4 * sizeof(unsigned long long), st));
        int r = fused3_umax(s, st);
        if (r) return r;
        unsigned long long bits[4] = {0, 0, 0, 0};
        SP_CUDA(cudaMemcpyAsync(bits, s->umax_dev(), sizeof(bits), cudaMemcpyDeviceToHost, st));
        SP_CUDA(cudaStreamSynchronize(st));
        double sum = 0.0;
        for (int c = 0; c < 3; ++c) {
            double v;
            std::memcpy(&v, &bits[c], sizeof(v));
            if (out_per_comp) out_per_comp[c] = v;
            sum += v;
        }
        *out_sum = sum;
        return SP_OK;
    }
    if (s->fused()) {
        // the work array holds the stage-0 inputs of the live state: one inverse row pass
        if (state != s->u0)
            return fail(s, SP_ERR_UNSUPPORTED, "sp_max_velocity",
                        "the fused engine bounds the velocity of its own state only");
        SP_CUDA(cudaMemsetAsync(s->umax_dev(), 0, 4 * sizeof(unsigned long long), st));
        SP_CUDA(sp::fused::row_max(s->n, s->fp64, s->W, s->kc, s->tw_dev(), s->umax_dev(), st));
        s->launches += 1;
        unsigned long long bits[4] = {0, 0, 0, 0};
        SP_CUDA(cudaMemcpyAsync(bits, s->umax_dev(), sizeof(bits), cudaMemcpyDeviceToHost, st));
        SP_CUDA(cudaStreamSynchronize(st));
        double sum = 0.0;
        for (int c = 0; c < 2; ++c) {
            double v;
            std::memcpy(&v, &bits[c], sizeof(v));
            if (out_per_comp) out_per_comp[c] = v;
            sum += v;
        }
        if (out_per_comp) out_per_comp[2] = 0.0;
        *out_sum = sum;
        return SP_OK;
    }
    cufftHandle plan = s->fft_mode == SP_FFT_CUFFT_LEAN ? s->plan_inv : s->plan_c2r1;
    SP_CUDA(cudaMemsetAsync(s->umax_dev(), 0, 4 * sizeof(unsigned long long), st));
    unsigned gv = grid_for(s->fsc, kRedThreads);
    uint32_t rows = s->fsc / (uint32_t)s->nh;
    unsigned gm = grid_for((uint64_t)rows * (s->n / 2), kRedThreads);
    if (gm > (unsigned)kRedBlocks) gm = kRedBlocks;
    double scale = 1.0 / std::pow((double)s->n, (double)s->dim);
    for (int c = 0; c < ncomp; ++c) {
        if (s->fp64) {
            k_velocity_component<double><<<gv, kRedThreads, 0, st>>>(
                (const cplx<double>*)state, (cplx<double>*)s->acc, s->n, s->nh, s->dim, s->fsc, c,
                scale);
        } else {
            k_velocity_component<float><<<gv, kRedThreads, 0, st>>>(
                (const cplx<float>*)state, (cplx<float>*)s->acc, s->n, s->nh, s->dim, s->fsc, c,
                (float)scale);
        }
        SP_CUDA(cudaGetLastError());
        int r = exec_c2r(s, plan, s->acc, st);
        if (r) return r;
        if (s->fp64)
            k_max_abs_padded<double><<<gm, kRedThreads, 0, st>>>((const double*)s->acc, s->n,
                                                                 2 * s->nh, rows, s->umax_dev() + c);
        else
            k_max_abs_padded<float><<<gm, kRedThreads, 0, st>>>((const float*)s->acc, s->n,
                                                                2 * s->nh, rows, s->umax_dev() + c);
        SP_CUDA(cudaGetLastError());
        s->launches += 2;
    }
    unsigned long long bits[4] = {0, 0, 0, 0};
    SP_CUDA(cudaMemcpyAsync(bits, s->umax_dev(), sizeof(bits), cudaMemcpyDeviceToHost, st));
    SP_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (int c = 0; c < ncomp; ++c) {
        double v;
        std::memcpy(&v, &bits[c], sizeof(v));
        if (out_per_comp) out_per_comp[c] = v;
        sum += v;
    }
    if (out_per_comp)
        for (int c = ncomp; c < 3; ++c) out_per_comp[c] = 0.0;
    *out_sum = sum;
    return SP_OK;
}

int sp_spectrum(sp_solver* s, const void* state, double* out, int nshell, void* stream) {
    SP_CHECK_BOUND(s);
    if (!state || !out) return fail(s, SP_ERR_ARG, "sp_spectrum", "null pointer");
    if (nshell != s->nshell) return fail(s, SP_ERR_ARG, "sp_spectrum", "nshell mismatch");
    auto st = (cudaStream_t)stream;
    if (state == s->u0) {
        int r = sp_sync_state(s, stream);
        if (r) return r;
    }
    double norm = std::pow((double)s->n, 2.0 * s->dim);
    SP_CUDA(cudaMemsetAsync(s->spec_dev(), 0, (size_t)nshell * sizeof(double), st));
    unsigned g = grid_for(s->fsc, kRedThreads);
    if (g > (unsigned)kRedBlocks) g = kRedBlocks;
    size_t smem = (size_t)nshell * sizeof(double);
    int use_smem = smem <= 48 * 1024 ? 1 : 0;
    if (!use_smem) smem = 0;
    if (s->fp64)
        k_spectrum<double><<<g, kRedThreads, smem, st>>>((const cplx<double>*)state, s->n, s->nh,
                                                         s->dim, s->fsc, 1.0 / norm, 2.0 / norm,
                                                         nshell, use_smem, s->spec_dev());
    else
        k_spectrum<float><<<g, kRedThreads, smem, st>>>((const cplx<float>*)state, s->n, s->nh,
                                                        s->dim, s->fsc, 1.0 / norm, 2.0 / norm,
                                                        nshell, use_smem, s->spec_dev());
    SP_CUDA(cudaGetLastError());
    s->launches += 1;
    SP_CUDA(cudaMemcpyAsync(out, s->spec_dev(), (size_t)nshell * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    SP_CUDA(cudaStreamSynchronize(st));
    return SP_OK;
}

int sp_attach_closure(sp_solver* s, sp_closure* c) {
    if (!s) return SP_ERR_ARG;
    if (s->bound) return fail(s, SP_ERR_STATE, "sp_attach_closure", "attach before sp_bind");
    if (!c) return fail(s, SP_ERR_ARG, "sp_attach_closure", "null closure");
    if (s->closure) return fail(s, SP_ERR_STATE, "sp_attach_closure", "a closure is attached already");
    if (s->dim != 2 || s->fp64 || s->fft_mode != SP_FFT_CUFFT)
        return fail(s, SP_ERR_UNSUPPORTED, "sp_attach_closure",
                    "the closure runs on 2D fp32 solvers with batched cuFFT plans");
    if (sp::closure::grid_n(c) != s->n)
        return fail(s, SP_ERR_ARG, "sp_attach_closure", "closure and solver grids differ");
    size_t ws_inv = 0, ws_fwd = 0;
    int r = make_plan(s, true, 5, &s->plan_cl_inv, &ws_inv);
    if (r) return r;
    r = make_plan(s, false, 3, &s->plan_cl_fwd, &ws_fwd);
    if (r) {
        cufftDestroy(s->plan_cl_inv);
        return r;
    }
    s->have_cl = true;
    s->closure = c;
    s->ninv = 5;
    s->nfwd = 3;
    s->nwork = 6;
    s->work_bytes = (size_t)s->nwork * field_bytes(s);
    if (ws_inv > s->ws_bytes) s->ws_bytes = ws_inv;
    if (ws_fwd > s->ws_bytes) s->ws_bytes = ws_fwd;
    return SP_OK;
}

int sp_nonlinear(sp_solver* s, const void* state, void* out, void* stream) {
    SP_CHECK_BOUND(s);
    if (!state || !out) return fail(s, SP_ERR_ARG, "sp_nonlinear", "null pointer");
    if (s->dim != 2 || s->fft_mode != SP_FFT_CUFFT)
        return fail(s, SP_ERR_UNSUPPORTED, "sp_nonlinear", "2D solvers with batched cuFFT plans only");
    auto st = (cudaStream_t)stream;
    if (!s->params_valid) {
        int r = upload_params(s, s->tab_valid ? s->tab_dt : 0.0, st);
        if (r) return r;
    }
    unsigned g = grid_for(s->fsc / 2, kBlock);
    int r;
    if (s->fp64) {
        k_nl_pre2d<double><<<g, kBlock, 0, st>>>((const cplx<double>*)state, (cplx<double>*)s->W,
                                                 s->n, s->nh, s->fsc,
                                                 (const StepParams<double>*)s->params_dev());
    } else {
        k_nl_pre2d<float><<<g, kBlock, 0, st>>>((const cplx<float>*)state, (cplx<float>*)s->W, s->n,
                                                s->nh, s->fsc,
                                                (const StepParams<float>*)s->params_dev());
    }
    SP_CUDA(cudaGetLastError());
    if ((r = exec_c2r(s, s->plan_inv, s->W, st))) return r;
    if (s->fp64) k_phys2d<double><<<grid_for(s->fsr / 4, kBlock), kBlock, 0, st>>>((double*)s->W, s->fsr);
    else k_phys2d<float><<<grid_for(s->fsr / 4, kBlock), kBlock, 0, st>>>((float*)s->W, s->fsr);
    SP_CUDA(cudaGetLastError());
    if ((r = exec_r2c(s, s->plan_fwd, s->W, st))) return r;
    if (s->fp64)
        k_nl_post2d<double><<<g, kBlock, 0, st>>>((const cplx<double>*)s->W, (cplx<double>*)out,
                                                  s->n, s->nh, s->fsc);
    else
        k_nl_post2d<float><<<g, kBlock, 0, st>>>((const cplx<float>*)s->W, (cplx<float>*)out, s->n,
                                                 s->nh, s->fsc);
    SP_CUDA(cudaGetLastError());
    s->launches += 3;
    // the work array held the next stage's inputs: rebuild them from the state
    return run_pre(s, st);
}

int sp_run_to(sp_solver* s, double t_end, double cfl, double dt_max, int cfl_every,
              double target_power, double dt_fixed, int64_t max_steps, double* t_io,
              int64_t* steps_out, double* amp_out, void* stream) {
    SP_CHECK_BOUND(s);
    if (!t_io || cfl_every < 1 || cfl_every > 1000 || !(dt_max > 0.0) || max_steps < 0)
        return fail(s, SP_ERR_ARG, "sp_run_to", "bad arguments");
    auto st = (cudaStream_t)stream;
    const bool use_cfl = !(dt_fixed > 0.0);
    const bool use_power = target_power >= 0.0;
    const int flags = (use_cfl ? 1 : 0) | (use_power ? 2 : 0) |
                      ((s->cl() && sp::closure::every_stage(s->closure)) ? 4 : 0);
    // the step graph and the chunk graph share the device parameter block
    int r = capture_run_chunk(s, cfl_every, flags);
    if (r) return r;
    const int64_t per_chunk = s->run_kernels;
    RunCtl& c = s->host_ctl;
    c = RunCtl{};
    c.t = *t_io;
    c.t_end = t_end;
    c.tol = 1e-12 * std::max(1.0, t_end);
    c.cfl = cfl;
    c.dt_max = dt_max;
    c.dx = 2.0 * M_PI / (double)s->n;
    c.power = use_power ? target_power : 0.0;
    c.dt_fixed = use_cfl ? 0.0 : dt_fixed;
    c.dt_tab = -1.0;
    c.amp = s->amp;
    c.have_power = use_power ? 1 : 0;
    RunCtl* dc = (RunCtl*)((char*)s->aux + s->off_ctl);
    SP_CUDA(cudaMemcpyAsync(dc, &c, sizeof(RunCtl), cudaMemcpyHostToDevice, st));
    if (s->fused()) s->u0_fresh = false;
    int64_t chunks = 0;
    while (c.t < t_end - c.tol && c.steps < max_steps) {
        SP_CUDA(cudaGraphLaunch(s->run_exec, st));
        s->launches += per_chunk;
        ++chunks;
        SP_CUDA(cudaMemcpyAsync(&c, dc, sizeof(RunCtl), cudaMemcpyDeviceToHost, st));
        SP_CUDA(cudaStreamSynchronize(st));
    }
    // the host-side caches of the step scalars no longer describe the device block
    s->params_valid = false;
    s->tab_valid = false;
    s->amp = c.amp;
    *t_io = c.t;
    if (steps_out) *steps_out = c.steps;
    if (amp_out) *amp_out = c.amp;
    return SP_OK;
}

}  // extern "C"
