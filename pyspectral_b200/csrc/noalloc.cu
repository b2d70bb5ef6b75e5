// sp_spectrum_noalloc: the shell-spectrum reduction without any device allocation.
//
// Who needs this: a caller that cannot allocate device memory — for example a host program
// that hands the whole GPU memory to its own pool allocator up front, or a time-critical loop
// that must not take the implicit device synchronisation of cudaMalloc/cudaFree — and still
// wants the energy spectrum E(k) of a state it already holds on the device.  The regular
// entry point (sp_spectrum) needs an engine handle whose caller-allocated `aux` block holds the
// shell accumulators; this one needs neither a handle nor any buffer beyond the input state
// and the host output array.
//
// Where its scratch lives: the shell accumulators are the file-scope array below, a fixed
// 128 KiB (SP_NOALLOC_MAX_SHELLS doubles) that every GPU which loads this library keeps until
// the process exits.  All calls on a device share it and it keeps the last call's contents,
// so each call zeroes the shells it uses before accumulating.  Two calls whose work overlaps
// on the GPU (different streams, or different host threads without ordering) race on the
// array and give wrong results: order them on one stream or serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "spectral_b200.h"
#include "reduce.cuh"

namespace sp {
void set_thread_error(const char* why);  // defined in spectral_b200.cu
}

using namespace sp;

namespace {

static __device__ __align__(256) double g_noalloc_shells[SP_NOALLOC_MAX_SHELLS];

// Device address of g_noalloc_shells per device.  In host code the array's name is only a
// host-side stand-in, not a device address, so it is looked up with cudaGetSymbolAddress once
// per device (with that device current) and cached.  The cache is never invalidated: a caller
// that resets the device (cudaDeviceReset) must not call this entry point afterwards.
constexpr int kMaxDevices = 64;
std::mutex g_lookup_mutex;
double* g_shells_addr[kMaxDevices] = {};

int shells_address(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SP_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_lookup_mutex);
    if (!g_shells_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_shells);
        if (e != cudaSuccess || !p) return SP_ERR_CUDA;
        g_shells_addr[dev] = (double*)p;
    }
    *out = g_shells_addr[dev];
    return SP_OK;
}

int noalloc_fail(int code, const char* why) {
    sp::set_thread_error(why);  // readable through sp_create_error() in this thread
    return code;
}

}  // namespace

extern "C" {

int sp_spectrum_noalloc(const void* state, int n, int dim, int fp64, double* out, int nshell,
                        void* stream) {
    sp::set_thread_error("");
    if (!state || !out) return noalloc_fail(SP_ERR_ARG, "null state or output pointer");
    if (dim != 2 && dim != 3) return noalloc_fail(SP_ERR_ARG, "dim must be 2 or 3");
    if (n < 8 || n % 2) return noalloc_fail(SP_ERR_ARG, "n must be even and >= 8");
    int want = (int)std::floor(std::sqrt((double)dim) * (double)(n / 2) + 0.5) + 1;
    if (nshell != want) return noalloc_fail(SP_ERR_ARG, "nshell does not match n and dim");
    if (nshell > SP_NOALLOC_MAX_SHELLS)
        return noalloc_fail(SP_ERR_ARG,
                            "grid too large: more shells than SP_NOALLOC_MAX_SHELLS (use sp_spectrum)");
    int nh = n / 2 + 1;
    uint64_t fsc = (uint64_t)nh * (uint64_t)n * (dim == 3 ? (uint64_t)n : 1ull);
    if (2 * fsc >= (1ull << 32)) return noalloc_fail(SP_ERR_ARG, "grid too large for 32-bit indexing");

    double* shells = nullptr;
    if (shells_address(&shells)) return noalloc_fail(SP_ERR_CUDA, "cudaGetSymbolAddress failed");
    auto st = (cudaStream_t)stream;
    // the array keeps the previous call's sums: clear the shells this call accumulates into
    if (cudaMemsetAsync(shells, 0, (size_t)nshell * sizeof(double), st) != cudaSuccess)
        return noalloc_fail(SP_ERR_CUDA, "cudaMemsetAsync failed");
    double norm = std::pow((double)n, 2.0 * dim);
    unsigned g = (unsigned)((fsc + kRedThreads - 1) / kRedThreads);
    if (g > (unsigned)kRedBlocks) g = kRedBlocks;
    size_t smem = (size_t)nshell * sizeof(double);
    int use_smem = smem <= 48 * 1024 ? 1 : 0;
    if (!use_smem) smem = 0;
    if (fp64)
        k_spectrum<double><<<g, kRedThreads, smem, st>>>((const cplx<double>*)state, n, nh, dim,
                                                         (uint32_t)fsc, 1.0 / norm, 2.0 / norm,
                                                         nshell, use_smem, shells);
    else
        k_spectrum<float><<<g, kRedThreads, smem, st>>>((const cplx<float>*)state, n, nh, dim,
                                                        (uint32_t)fsc, 1.0 / norm, 2.0 / norm,
                                                        nshell, use_smem, shells);
    if (cudaGetLastError() != cudaSuccess) return noalloc_fail(SP_ERR_CUDA, "kernel launch failed");
    if (cudaMemcpyAsync(out, shells, (size_t)nshell * sizeof(double), cudaMemcpyDeviceToHost,
                        st) != cudaSuccess)
        return noalloc_fail(SP_ERR_CUDA, "cudaMemcpyAsync failed");
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return noalloc_fail(SP_ERR_CUDA, "cudaStreamSynchronize failed");
    return SP_OK;
}

}  // extern "C"
