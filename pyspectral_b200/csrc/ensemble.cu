// Batched ensembles of independent 2D runs on the fused-FFT engine.
//
// A batch is `members` runs of one grid size n (a size class): every phase is one launch over
// all members (gridDim.y = member), each member with its own step parameters (dt, drag and band
// factors) and integrating-factor table, so members advance with their own CFL time steps and
// forcing amplitudes.  A group steps several batches (uneven sizes) from one CUDA graph whose
// branches, one per batch, run concurrently.  Reductions (energy, enstrophy, palinstrophy, band
// energy) and the CFL velocity bound are batched too: one launch and one device-to-host copy
// for all members.  No counterpart in the reference, where one solver is one run.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "fused2d.h"
#include "spectral_b200.h"

using namespace sp;

namespace sp {
void set_thread_error(const char* why);  // spectral_b200.cu
}

namespace {
size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

struct sp_batch {
    int n = 0, fp64 = 0, members = 0, nh = 0, kc = 0, nblk = 1;
    int tile = 1;  // sub-block multiplier of the fused passes (autotuner choice)
    size_t rsize = 4, csize = 8, psize = 16;
    // per-member block of the work buffer: [X | u0t | acct]
    size_t off_u0t = 0, off_acct = 0, member_work = 0;
    size_t state_bytes = 0, work_bytes = 0, aux_bytes = 0;
    size_t off_params = 0, off_tab = 0, off_tw = 0, off_partials = 0, off_umax = 0, off_out = 0;
    int tab_stride = 0;
    void *u0 = nullptr, *W = nullptr, *aux = nullptr;
    bool bound = false, fresh = true;
    // physics
    std::vector<double> nu;
    double alpha = 0, drag_k2 = 1e30, klo = 0, khi = 0;
    std::vector<unsigned char> host_params, host_tab, up_params, up_tab;
    bool params_dirty = true;
    // graph of one batch step
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    std::string err;

    char* base(size_t off) const { return (char*)aux + off; }
};

struct sp_group {
    std::vector<sp_batch*> batches;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    // work list (sp_group_bind, sp_group_set_worklist): class descriptors, row items and
    // column items in the caller's device buffer; mt = 0: one launch per class and phase
    void* wl = nullptr;
    int mt = 0, nrow = 0, ncol = 0;
    size_t off_rows = 0, off_cols = 0;
    int64_t launches = 0;
    std::string err;
};

namespace {

int bfail(sp_batch* b, int code, const char* what, const char* why) {
    if (b) b->err = std::string(what) + ": " + why;
    return code;
}

#define B_CUDA(b, call)                                                                 \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return bfail((b), SP_ERR_CUDA, #call, cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
void fill_member(const sp_batch* b, int m, double dt, double amp, unsigned char* params,
                 unsigned char* tab) {
    StepParams<T> p;
    p.dt = (T)dt;
    p.ea1 = (T)std::exp(-b->alpha * dt);
    p.eah = (T)std::exp(-b->alpha * 0.5 * dt);
    p.eb1 = (T)std::exp(amp * dt);
    p.ebh = (T)std::exp(amp * 0.5 * dt);
    const bool band_on = amp != 0.0;
    p.klo2 = band_on ? (T)(b->klo * b->klo) : (T)1;
    p.khi2 = band_on ? (T)(b->khi * b->khi) : (T)0;
    p.ka2 = (T)b->drag_k2;
    p.scale = (T)(1.0 / ((double)b->n * (double)b->n));
    std::memcpy(params + (size_t)m * sizeof(p), &p, sizeof(p));
    T* t = reinterpret_cast<T*>(tab) + (size_t)m * b->tab_stride;
    for (int j = 0; j < b->nh; ++j) {
        const double jj = (double)j;
        t[j] = (T)std::exp(-b->nu[m] * jj * jj * dt);
        t[b->nh + j] = (T)std::exp(-b->nu[m] * jj * jj * 0.5 * dt);
    }
}

int batch_step_kernels(sp_batch* b, cudaStream_t st) {
    const size_t xs = b->member_work / b->psize, us = b->member_work / b->csize;
    void* X = b->W;
    void* u0t = (char*)b->W + b->off_u0t;
    void* acct = (char*)b->W + b->off_acct;
    for (int stage = 0; stage < 4; ++stage) {
        B_CUDA(b, sp::fused::row_pass(b->n, b->fp64, X, b->kc, b->base(b->off_tw), st,
                                      b->members, xs, b->tile));
        B_CUDA(b, sp::fused::col_pass(b->n, b->fp64, stage, X, b->kc, u0t, acct,
                                      b->base(b->off_tab), b->base(b->off_params),
                                      b->base(b->off_tw), st, b->members, xs, us,
                                      b->tab_stride, b->tile));
        b->launches += 2;
    }
    return SP_OK;
}

// The work lists of a group for CTAs of mt threads: per class its descriptor, then per member
// its rows and its kept columns in items of 16 mt / n.
void group_lists(const sp_group* g, int mt, std::vector<sp::fused::MultiClass>& cls,
                 std::vector<sp::fused::MultiItem>& rows, std::vector<sp::fused::MultiItem>& cols) {
    cls.clear();
    rows.clear();
    cols.clear();
    for (size_t ci = 0; ci < g->batches.size(); ++ci) {
        const sp_batch* b = g->batches[ci];
        sp::fused::MultiClass c{};
        c.X = b->W;
        c.u0t = (char*)b->W + b->off_u0t;
        c.acct = (char*)b->W + b->off_acct;
        c.tab = b->base(b->off_tab);
        c.params = b->base(b->off_params);
        c.tw = b->base(b->off_tw);
        c.x_stride = b->member_work / b->psize;
        c.u_stride = b->member_work / b->csize;
        c.tab_stride = b->tab_stride;
        c.n = b->n;
        c.kc = b->kc;
        cls.push_back(c);
        const int per = sp::fused::multi_per_item(b->n, mt);
        for (int m = 0; m < b->members; ++m) {
            for (int r = 0; r < b->n; r += per) rows.push_back({(int)ci, m, r});
            for (int k = 0; k < b->kc; k += per) cols.push_back({(int)ci, m, k});
        }
    }
}

bool group_multi_ok(const sp_group* g, int mt) {
    for (const sp_batch* b : g->batches)
        if (b->fp64 != g->batches[0]->fp64 || !sp::fused::multi_supported(b->n, mt)) return false;
    return true;
}

size_t list_bytes(size_t ncls, size_t nrow, size_t ncol) {
    return al256(ncls * sizeof(sp::fused::MultiClass)) +
           al256(nrow * sizeof(sp::fused::MultiItem)) + ncol * sizeof(sp::fused::MultiItem);
}

int group_step_multi(sp_group* g, cudaStream_t st) {
    const int fp64 = g->batches[0]->fp64;
    const char* base = (const char*)g->wl;
    cudaError_t e;
    for (int stage = 0; stage < 4; ++stage) {
        if ((e = sp::fused::row_multi(fp64, g->mt, base, base + g->off_rows, g->nrow, st)) ||
            (e = sp::fused::col_multi(fp64, g->mt, stage, base, base + g->off_cols, g->ncol, st))) {
            g->err = std::string("work-list pass: ") + cudaGetErrorString(e);
            return SP_ERR_CUDA;
        }
    }
    return SP_OK;
}

}  // namespace

extern "C" {

sp_batch* sp_batch_create(int n, int fp64, int members, int* status) {
    auto set = [&](int code, const char* why) -> sp_batch* {
        if (status) *status = code;
        sp::set_thread_error(why);
        return nullptr;
    };
    if (members < 1 || members > 65535) return set(SP_ERR_ARG, "members must be 1..65535");
    if (!sp::fused::supported(n, fp64))
        return set(SP_ERR_UNSUPPORTED,
                   "batches need n a power of two in 16..8192 (fp32) or 16..4096 (fp64)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return set(SP_ERR_CUDA, "no CUDA device");
    auto* b = new sp_batch();
    b->n = n;
    b->fp64 = fp64 ? 1 : 0;
    b->members = members;
    b->nh = n / 2 + 1;
    b->kc = sp::fused::kc_of(n);
    b->rsize = fp64 ? 8 : 4;
    b->csize = 2 * b->rsize;
    b->psize = 2 * b->csize;
    b->off_u0t = al256((size_t)n * b->kc * b->psize);
    b->off_acct = b->off_u0t + al256((size_t)b->kc * n * b->csize);
    b->member_work = b->off_acct + al256((size_t)b->kc * n * b->csize);
    b->work_bytes = (size_t)members * b->member_work;
    b->state_bytes = (size_t)members * n * b->nh * b->csize;
    b->tab_stride = 2 * b->nh;
    const uint64_t total = (uint64_t)b->kc * n;
    b->nblk = (int)std::min<uint64_t>(64, std::max<uint64_t>(1, total / 2048));
    size_t off = 0;
    b->off_params = off; off += al256((size_t)members * sizeof(StepParams<double>));
    b->off_tab = off; off += al256((size_t)members * b->tab_stride * b->rsize);
    b->off_tw = off; off += al256((size_t)sp::fused::twiddle_table_size(n) * b->csize);
    b->off_partials = off; off += al256((size_t)members * b->nblk * 4 * sizeof(double));
    b->off_umax = off; off += al256((size_t)members * 2 * sizeof(unsigned long long));
    b->off_out = off; off += al256((size_t)members * 4 * sizeof(double));
    b->aux_bytes = off;
    b->nu.assign(members, 0.0);
    cudaError_t e = sp::fused::set_attributes(n, fp64);
    if (e != cudaSuccess) {
        delete b;
        return set(SP_ERR_CUDA, cudaGetErrorString(e));
    }
    if (status) *status = SP_OK;
    return b;
}

void sp_batch_destroy(sp_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
}

int sp_batch_query_sizes(const sp_batch* b, int64_t* out, int count) {
    if (!b || !out || count < 0 || count > 6) return SP_ERR_ARG;
    int64_t v[6] = {b->members, b->kc, (int64_t)b->state_bytes, 0, (int64_t)b->work_bytes,
                    (int64_t)b->aux_bytes};
    for (int i = 0; i < count; ++i) out[i] = v[i];
    return SP_OK;
}

int sp_batch_bind(sp_batch* b, void* u0, void* work, void* aux) {
    if (!b) return SP_ERR_ARG;
    if (!u0 || !work || !aux) return bfail(b, SP_ERR_ARG, "sp_batch_bind", "null buffer");
    for (void* p : {u0, work, aux})
        if ((uintptr_t)p % 256) return bfail(b, SP_ERR_ARG, "sp_batch_bind", "buffer not 256-byte aligned");
    b->u0 = u0;
    b->W = work;
    b->aux = aux;
    std::vector<double> tw(2 * (size_t)sp::fused::twiddle_table_size(b->n));
    sp::fused::fill_twiddles(b->n, tw.data());
    if (b->fp64) {
        B_CUDA(b, cudaMemcpy(b->base(b->off_tw), tw.data(), tw.size() * 8, cudaMemcpyHostToDevice));
    } else {
        std::vector<float> twf(tw.begin(), tw.end());
        B_CUDA(b, cudaMemcpy(b->base(b->off_tw), twf.data(), twf.size() * 4, cudaMemcpyHostToDevice));
    }
    b->bound = true;
    b->params_dirty = true;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    return SP_OK;
}

int sp_batch_set_physics(sp_batch* b, const double* nu, double alpha, double drag_k2,
                         double force_klo, double force_khi) {
    if (!b || !nu) return SP_ERR_ARG;
    for (int m = 0; m < b->members; ++m) b->nu[m] = nu[m];
    b->alpha = alpha;
    b->drag_k2 = drag_k2;
    b->klo = force_klo;
    b->khi = force_khi;
    b->params_dirty = true;
    return SP_OK;
}

int sp_batch_set_step(sp_batch* b, const double* dt, const double* amp, void* stream) {
    if (!b || !dt) return SP_ERR_ARG;
    if (!b->bound) return bfail(b, SP_ERR_STATE, "sp_batch_set_step", "sp_batch_bind was not called");
    const size_t psz = (size_t)b->members * (b->fp64 ? sizeof(StepParams<double>) : sizeof(StepParams<float>));
    const size_t tsz = (size_t)b->members * b->tab_stride * b->rsize;
    b->host_params.assign(psz, 0);
    b->host_tab.assign(tsz, 0);
    for (int m = 0; m < b->members; ++m) {
        const double a = amp ? amp[m] : 0.0;
        if (b->fp64) fill_member<double>(b, m, dt[m], a, b->host_params.data(), b->host_tab.data());
        else fill_member<float>(b, m, dt[m], a, b->host_params.data(), b->host_tab.data());
    }
    auto st = (cudaStream_t)stream;
    // pageable sources: each call returns once the bytes are staged
    if (b->params_dirty || b->host_params != b->up_params) {
        B_CUDA(b, cudaMemcpyAsync(b->base(b->off_params), b->host_params.data(), psz,
                                  cudaMemcpyHostToDevice, st));
        b->up_params = b->host_params;
    }
    if (b->params_dirty || b->host_tab != b->up_tab) {
        B_CUDA(b, cudaMemcpyAsync(b->base(b->off_tab), b->host_tab.data(), tsz,
                                  cudaMemcpyHostToDevice, st));
        b->up_tab = b->host_tab;
    }
    b->params_dirty = false;
    return SP_OK;
}

int sp_batch_prepare(sp_batch* b, void* stream) {
    if (!b) return SP_ERR_ARG;
    if (!b->bound) return bfail(b, SP_ERR_STATE, "sp_batch_prepare", "sp_batch_bind was not called");
    if (b->up_params.empty())
        return bfail(b, SP_ERR_STATE, "sp_batch_prepare", "call sp_batch_set_step first");
    auto st = (cudaStream_t)stream;
    const size_t us = b->member_work / b->csize, u0s = (size_t)b->n * b->nh;
    void* u0t = (char*)b->W + b->off_u0t;
    B_CUDA(b, sp::fused::mask2d(b->fp64, b->u0, b->n, st, b->members));
    B_CUDA(b, sp::fused::transpose_in(b->fp64, b->u0, u0t, b->n, b->kc, st, b->members, u0s, us));
    B_CUDA(b, sp::fused::col_pass(b->n, b->fp64, -1, b->W, b->kc, u0t, (char*)b->W + b->off_acct,
                                  b->base(b->off_tab), b->base(b->off_params), b->base(b->off_tw),
                                  st, b->members, b->member_work / b->psize, us, b->tab_stride,
                                  b->tile));
    b->launches += 3;
    b->fresh = true;
    return SP_OK;
}

int sp_batch_tile_supported(int n, int tile) { return sp::fused::tile_supported(n, tile) ? 1 : 0; }

int sp_batch_set_tile(sp_batch* b, int tile) {
    if (!b) return SP_ERR_ARG;
    if (!sp::fused::tile_supported(b->n, tile))
        return bfail(b, SP_ERR_ARG, "sp_batch_set_tile", "tile not compiled for this grid");
    if (tile != b->tile && b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    b->tile = tile;
    return SP_OK;
}

int sp_batch_tile(const sp_batch* b) { return b ? b->tile : -1; }

int sp_batch_step(sp_batch* b, void* stream) {
    if (!b) return SP_ERR_ARG;
    if (!b->bound || b->up_params.empty())
        return bfail(b, SP_ERR_STATE, "sp_batch_step", "bind, set_step and prepare first");
    auto st = (cudaStream_t)stream;
    if (!b->exec) {
        if (!b->cap) B_CUDA(b, cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
        B_CUDA(b, cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        const int64_t before = b->launches;
        int r = batch_step_kernels(b, b->cap);
        b->launches = before;
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->cap, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess) return bfail(b, SP_ERR_CUDA, "cudaStreamEndCapture", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&b->exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            return bfail(b, SP_ERR_CUDA, "cudaGraphInstantiate", cudaGetErrorString(e));
        }
    }
    B_CUDA(b, cudaGraphLaunch(b->exec, st));
    b->launches += 8;
    b->fresh = false;
    return SP_OK;
}

int sp_batch_sync_state(sp_batch* b, void* stream) {
    if (!b) return SP_ERR_ARG;
    if (!b->bound) return bfail(b, SP_ERR_STATE, "sp_batch_sync_state", "sp_batch_bind was not called");
    if (b->fresh) return SP_OK;
    const size_t us = b->member_work / b->csize, u0s = (size_t)b->n * b->nh;
    B_CUDA(b, sp::fused::transpose_out(b->fp64, (char*)b->W + b->off_u0t, b->u0, b->n, b->kc,
                                       (cudaStream_t)stream, b->members, us, u0s));
    b->launches += 1;
    b->fresh = true;
    return SP_OK;
}

int sp_batch_diagnostics(sp_batch* b, double band_klo, double band_khi, double* out,
                         void* stream) {
    if (!b || !out) return SP_ERR_ARG;
    if (!b->bound) return bfail(b, SP_ERR_STATE, "sp_batch_diagnostics", "sp_batch_bind was not called");
    auto st = (cudaStream_t)stream;
    B_CUDA(b, sp::fused::reduce_t(b->fp64, (char*)b->W + b->off_u0t, b->n, b->kc,
                                  b->member_work / b->csize, b->members, band_klo, band_khi,
                                  (double*)b->base(b->off_partials), b->nblk,
                                  (double*)b->base(b->off_out), st));
    b->launches += 2;
    B_CUDA(b, cudaMemcpyAsync(out, b->base(b->off_out), (size_t)b->members * 4 * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    B_CUDA(b, cudaStreamSynchronize(st));
    return SP_OK;
}

int sp_batch_max_velocity(sp_batch* b, double* out, void* stream) {
    if (!b || !out) return SP_ERR_ARG;
    if (!b->bound) return bfail(b, SP_ERR_STATE, "sp_batch_max_velocity", "sp_batch_bind was not called");
    auto st = (cudaStream_t)stream;
    auto* umax = (unsigned long long*)b->base(b->off_umax);
    B_CUDA(b, cudaMemsetAsync(umax, 0, (size_t)b->members * 2 * sizeof(unsigned long long), st));
    B_CUDA(b, sp::fused::row_max(b->n, b->fp64, b->W, b->kc, b->base(b->off_tw), umax, st,
                                 b->members, b->member_work / b->psize));
    b->launches += 1;
    std::vector<unsigned long long> bits((size_t)b->members * 2);
    B_CUDA(b, cudaMemcpyAsync(bits.data(), umax, bits.size() * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, st));
    B_CUDA(b, cudaStreamSynchronize(st));
    for (int m = 0; m < b->members; ++m) {
        double u, v;
        std::memcpy(&u, &bits[2 * m], 8);
        std::memcpy(&v, &bits[2 * m + 1], 8);
        out[m] = u + v;
    }
    return SP_OK;
}

int64_t sp_batch_kernel_launches(const sp_batch* b) { return b ? b->launches : -1; }

const char* sp_batch_last_error(const sp_batch* b) { return b ? b->err.c_str() : "null handle"; }

sp_group* sp_group_create(sp_batch** batches, int count, int* status) {
    if (!batches || count < 1) {
        if (status) *status = SP_ERR_ARG;
        sp::set_thread_error("sp_group_create: no batches");
        return nullptr;
    }
    auto* g = new sp_group();
    g->batches.assign(batches, batches + count);
    if (status) *status = SP_OK;
    return g;
}

void sp_group_destroy(sp_group* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    for (auto s : g->streams) cudaStreamDestroy(s);
    for (auto e : g->events) cudaEventDestroy(e);
    if (g->cap) cudaStreamDestroy(g->cap);
    delete g;
}

// One step of every batch of the group from one graph: a fork per batch, joined at the end.
int sp_group_step(sp_group* g, void* stream) {
    if (!g) return SP_ERR_ARG;
    for (auto* b : g->batches)
        if (!b->bound || b->up_params.empty()) {
            g->err = "sp_group_step: every batch needs bind, set_step and prepare";
            return SP_ERR_STATE;
        }
    if (!g->exec) {
        auto gfail = [&](const char* what, cudaError_t e) {
            g->err = std::string(what) + ": " + cudaGetErrorString(e);
            return SP_ERR_CUDA;
        };
        cudaError_t e;
        if (!g->cap && (e = cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking)))
            return gfail("cudaStreamCreate", e);
        const size_t nb = g->batches.size();
        while (g->streams.size() < nb) {
            cudaStream_t s;
            if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return gfail("cudaStreamCreate", e);
            g->streams.push_back(s);
        }
        while (g->events.size() < nb + 1) {
            cudaEvent_t ev;
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) return gfail("cudaEventCreate", e);
            g->events.push_back(ev);
        }
        if ((e = cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal)))
            return gfail("cudaStreamBeginCapture", e);
        int r = SP_OK;
        if (g->mt > 0) {
            // one launch per phase over the packed work list of every class
            r = group_step_multi(g, g->cap);
        } else {
            cudaEventRecord(g->events[nb], g->cap);
            for (size_t i = 0; i < nb && !r; ++i) {
                cudaStreamWaitEvent(g->streams[i], g->events[nb], 0);
                const int64_t before = g->batches[i]->launches;
                r = batch_step_kernels(g->batches[i], g->streams[i]);
                g->batches[i]->launches = before;
                cudaEventRecord(g->events[i], g->streams[i]);
                cudaStreamWaitEvent(g->cap, g->events[i], 0);
            }
        }
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(g->cap, &graph);
        if (r) {
            if (graph) cudaGraphDestroy(graph);
            if (g->mt == 0) g->err = "capture failed: " + g->batches[0]->err;
            return r;
        }
        if (e != cudaSuccess) return gfail("cudaStreamEndCapture", e);
        e = cudaGraphInstantiate(&g->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            g->exec = nullptr;
            return gfail("cudaGraphInstantiate", e);
        }
    }
    cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        g->err = std::string("cudaGraphLaunch: ") + cudaGetErrorString(e);
        return SP_ERR_CUDA;
    }
    for (auto* b : g->batches) {
        if (g->mt == 0) b->launches += 8;
        b->fresh = false;
    }
    if (g->mt > 0) g->launches += 8;
    return SP_OK;
}

int sp_group_worklist_bytes(const sp_group* g, int64_t* out) {
    if (!g || !out) return SP_ERR_ARG;
    *out = 0;
    for (int mt : {64, 128}) {  // 64-thread items are the more numerous
        if (!group_multi_ok(g, mt)) continue;
        std::vector<sp::fused::MultiClass> c;
        std::vector<sp::fused::MultiItem> r, k;
        group_lists(g, mt, c, r, k);
        const int64_t b = (int64_t)list_bytes(c.size(), r.size(), k.size());
        if (b > *out) *out = b;
    }
    return SP_OK;
}

int sp_group_bind(sp_group* g, void* buffer) {
    if (!g) return SP_ERR_ARG;
    if (!buffer || ((uintptr_t)buffer % 256)) {
        g->err = "sp_group_bind: null or not 256-byte aligned buffer";
        return SP_ERR_ARG;
    }
    g->wl = buffer;
    return SP_OK;
}

int sp_group_set_worklist(sp_group* g, int mt) {
    if (!g) return SP_ERR_ARG;
    if (mt == g->mt) return SP_OK;
    if (g->exec) {
        cudaGraphExecDestroy(g->exec);
        g->exec = nullptr;
    }
    if (mt == 0) {
        g->mt = 0;
        return SP_OK;
    }
    if (!g->wl) {
        g->err = "sp_group_set_worklist: sp_group_bind first";
        return SP_ERR_STATE;
    }
    for (const sp_batch* b : g->batches)
        if (!b->bound) {
            g->err = "sp_group_set_worklist: every batch must be bound";
            return SP_ERR_STATE;
        }
    if (!group_multi_ok(g, mt)) {
        g->err = "sp_group_set_worklist: classes of one precision, n a power of two with "
                 "n/16 <= mt and 16 mt/n <= n (mt 64: n = 32..1024, 128: 64..1024)";
        return SP_ERR_UNSUPPORTED;
    }
    std::vector<sp::fused::MultiClass> c;
    std::vector<sp::fused::MultiItem> r, k;
    group_lists(g, mt, c, r, k);
    g->off_rows = al256(c.size() * sizeof(sp::fused::MultiClass));
    g->off_cols = g->off_rows + al256(r.size() * sizeof(sp::fused::MultiItem));
    char* base = (char*)g->wl;
    cudaError_t e;
    if ((e = sp::fused::multi_prepare(g->batches[0]->fp64, mt)) ||
        (e = cudaMemcpy(base, c.data(), c.size() * sizeof(c[0]), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(base + g->off_rows, r.data(), r.size() * sizeof(r[0]), cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(base + g->off_cols, k.data(), k.size() * sizeof(k[0]), cudaMemcpyHostToDevice))) {
        g->err = std::string("sp_group_set_worklist: ") + cudaGetErrorString(e);
        return SP_ERR_CUDA;
    }
    g->nrow = (int)r.size();
    g->ncol = (int)k.size();
    g->mt = mt;
    return SP_OK;
}

int sp_group_worklist(const sp_group* g) { return g ? g->mt : -1; }

int64_t sp_group_kernel_launches(const sp_group* g) { return g ? g->launches : -1; }

const char* sp_group_last_error(const sp_group* g) { return g ? g->err.c_str() : "null handle"; }

}  // extern "C"
