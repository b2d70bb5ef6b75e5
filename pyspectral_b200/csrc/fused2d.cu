// Launchers of the fused 2D engine: runtime grid size -> compile-time kernel instantiation.
#include <cuda.h>

#include <atomic>
#include <cmath>

#include "fused2d.h"
#include "fused2d.cuh"

namespace sp {
namespace fused {

// Error bits of the streamed column pass (kStreamTimeout), one word per device context.
__device__ unsigned g_stream_err;

namespace {

std::atomic<bool> g_streaming{true};

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime (no link to
// libcuda); null when the driver does not provide it.
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                 const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                 const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
    static const EncodeTiled fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return (EncodeTiled) nullptr;
        return (EncodeTiled)f;
    }();
    return fn;
}

// Tensor map of the work array X for the streamed column pass: float32 words, row q = row pair
// q (kc * 2 Pairs), box = one column's 2 Pairs x up to 256 row pairs.
template <typename T, int N>
bool x_map(CUtensorMap* map, void* X, int kc) {
    const EncodeTiled enc = encoder();
    if (!enc || ((uintptr_t)X & 15)) return false;
    const cuuint64_t words = (cuuint64_t)kc * 2 * sizeof(Pair<T>) / 4;
    const cuuint64_t dims[2] = {words, (cuuint64_t)(N / 2)};
    const cuuint64_t strides[1] = {words * 4};  // bytes between row pairs
    const cuuint32_t box[2] = {(cuuint32_t)stream_box_w<T>(), (cuuint32_t)stream_box_h<N>()};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, X, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Grids the streamed column pass is built for: 2048..8192 (fp64 up to 4096).
template <typename T, int N>
constexpr bool stream_ok() { return N >= 2048 && (sizeof(T) == 4 ? N <= 8192 : N <= 4096); }

// Launch facts of the streamed pass, gathered by set_attributes (outside any stream capture):
// resident CTAs per SM for each stage, the SM count and this device's error word.
constexpr int kMaxDevices = 64;
unsigned* g_err_addr[kMaxDevices];

template <typename T, int N>
struct StreamLaunch {
    static inline int per_sm[4] = {0, 0, 0, 0};
    static inline int nsm = 0;
};

template <typename T, int N, int STAGE>
cudaError_t stream_prepare(int n_sm) {
    using CS = ColStream<T, N>;
    cudaError_t e = cudaFuncSetAttribute(k_col_stream<T, N, STAGE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)CS::SMEM);
    if (e) return e;
    int occ = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_col_stream<T, N, STAGE>,
                                                           CS::THREADS, CS::SMEM)))
        return e;
    StreamLaunch<T, N>::per_sm[STAGE] = occ;
    StreamLaunch<T, N>::nsm = n_sm;
    return cudaSuccess;
}

template <typename T, int N>
cudaError_t stream_attrs() {
    int dev = 0, n_sm = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) ||
        (e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)))
        return e;
    if (dev < kMaxDevices && !g_err_addr[dev]) {
        if ((e = cudaGetSymbolAddress((void**)&g_err_addr[dev], g_stream_err))) return e;
    }
    encoder();  // resolve the driver entry point now
    if ((e = stream_prepare<T, N, 0>(n_sm)) || (e = stream_prepare<T, N, 1>(n_sm)) ||
        (e = stream_prepare<T, N, 2>(n_sm)) || (e = stream_prepare<T, N, 3>(n_sm)))
        return e;
    return cudaSuccess;
}

// Tile multipliers compiled for a grid: 1, 2, 4 up to n = 1024 (CTAs of at most 256 threads),
// 1 above.
constexpr bool tile_ok(int n, int bx) { return bx == 1 || ((bx == 2 || bx == 4) && n <= 1024); }

template <typename T, int N, int BX>
cudaError_t attrs_tile() {
    if constexpr (!tile_ok(N, BX)) {
        return cudaSuccess;
    } else {
        using F = Fused2D<N, BX>;
        const int row_smem = (int)RowSingle<N, BX>::smem_bytes(sizeof(cplx<T>));
        const int col_smem = (int)F::template smem_bytes<Pair<T>>();
        cudaError_t e;
        if ((e = cudaFuncSetAttribute(k_row_pass<T, N, BX>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, row_smem)))
            return e;
        if ((e = cudaFuncSetAttribute(k_col_pass<T, N, -1, BX>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, col_smem)))
            return e;
        if ((e = cudaFuncSetAttribute(k_col_pass<T, N, 0, BX>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, col_smem)))
            return e;
        if ((e = cudaFuncSetAttribute(k_col_pass<T, N, 1, BX>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, col_smem)))
            return e;
        if ((e = cudaFuncSetAttribute(k_col_pass<T, N, 2, BX>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, col_smem)))
            return e;
        return cudaFuncSetAttribute(k_col_pass<T, N, 3, BX>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, col_smem);
    }
}

template <typename T, int N>
cudaError_t attrs() {
    const int max_smem = (int)RowPairs<N>::smem_bytes(sizeof(Pair<T>));
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_row_max<T, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  max_smem)))
        return e;
    if ((e = attrs_tile<T, N, 1>())) return e;
    if ((e = attrs_tile<T, N, 2>())) return e;
    if ((e = attrs_tile<T, N, 4>())) return e;
    if constexpr (stream_ok<T, N>()) {
        if ((e = stream_attrs<T, N>())) return e;
    }
    return cudaSuccess;
}

template <typename T, int N, int BX>
cudaError_t row_tile(void* X, int kc, const void* tw, cudaStream_t st, int members, size_t xs) {
    if constexpr (!tile_ok(N, BX)) {
        return cudaErrorInvalidValue;
    } else {
        using F = RowSingle<N, BX>;
        k_row_pass<T, N, BX><<<dim3(N / F::B, members), F::THREADS,
                               F::smem_bytes(sizeof(cplx<T>)), st>>>((Pair<T>*)X, kc,
                                                                     (const cplx<T>*)tw, xs);
        return cudaGetLastError();
    }
}

template <typename T, int N>
cudaError_t row(void* X, int kc, const void* tw, cudaStream_t st, int members, size_t xs,
                int tile) {
    switch (tile) {
        case 1: return row_tile<T, N, 1>(X, kc, tw, st, members, xs);
        case 2: return row_tile<T, N, 2>(X, kc, tw, st, members, xs);
        case 4: return row_tile<T, N, 4>(X, kc, tw, st, members, xs);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T, int N>
cudaError_t rmax(const void* X, int kc, const void* tw, unsigned long long* umax,
                 cudaStream_t st, int members, size_t xs) {
    using F = RowPairs<N>;
    k_row_max<T, N><<<dim3((N / 2) / F::B, members), F::THREADS,
                      F::smem_bytes(sizeof(Pair<T>)), st>>>((const Pair<T>*)X, kc,
                                                            (const cplx<T>*)tw, umax, xs);
    return cudaGetLastError();
}

struct ColArgs {
    void* X;
    int kc;
    void* u0t;
    void* acct;
    const void* tab;
    const void* P;
    const void* tw;
    cudaStream_t st;
    int members;
    size_t xs, us;
    int ts;
    int tile;
};

// One persistent CTA per resident slot (SM count x CTAs per SM), at most one per column.
// Returns false (nothing launched) when the pass was not prepared for this device.
template <typename T, int N, int STAGE>
bool col_stream(const ColArgs& a, const CUtensorMap& map, cudaError_t* err_out) {
    using CS = ColStream<T, N>;
    using L = StreamLaunch<T, N>;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevices || !g_err_addr[dev] ||
        L::per_sm[STAGE] < 1 || L::nsm < 1)
        return false;
    const int slots = L::nsm * L::per_sm[STAGE];
    const int grid = a.kc < slots ? a.kc : slots;
    k_col_stream<T, N, STAGE><<<grid, CS::THREADS, CS::SMEM, a.st>>>(
        map, (Pair<T>*)a.X, a.kc, (cplx<T>*)a.u0t, (cplx<T>*)a.acct, (const T*)a.tab,
        (const StepParams<T>*)a.P, (const cplx<T>*)a.tw, g_err_addr[dev]);
    *err_out = cudaGetLastError();
    return true;
}

template <typename T, int N, int STAGE, int BX>
cudaError_t col_stage(const ColArgs& a) {
    if constexpr (!tile_ok(N, BX)) {
        return cudaErrorInvalidValue;
    } else {
        if constexpr (BX == 1 && STAGE >= 0 && stream_ok<T, N>()) {
            CUtensorMap map;
            cudaError_t e = cudaSuccess;
            if (a.members == 1 && g_streaming.load(std::memory_order_relaxed) &&
                x_map<T, N>(&map, a.X, a.kc) && col_stream<T, N, STAGE>(a, map, &e))
                return e;
        }
        using F = Fused2D<N, BX>;
        const int grid = (a.kc + F::B - 1) / F::B;
        k_col_pass<T, N, STAGE, BX><<<dim3(grid, a.members), F::THREADS,
                                      F::template smem_bytes<Pair<T>>(), a.st>>>(
            (Pair<T>*)a.X, a.kc, (cplx<T>*)a.u0t, (cplx<T>*)a.acct, (const T*)a.tab,
            (const StepParams<T>*)a.P, (const cplx<T>*)a.tw, a.xs, a.us, a.ts);
        return cudaGetLastError();
    }
}

template <typename T, int N, int BX>
cudaError_t col_tile(int stage, const ColArgs& a) {
    switch (stage) {
        case -1: return col_stage<T, N, -1, BX>(a);
        case 0: return col_stage<T, N, 0, BX>(a);
        case 1: return col_stage<T, N, 1, BX>(a);
        case 2: return col_stage<T, N, 2, BX>(a);
        case 3: return col_stage<T, N, 3, BX>(a);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T, int N>
cudaError_t col(int stage, const ColArgs& a) {
    switch (a.tile) {
        case 1: return col_tile<T, N, 1>(stage, a);
        case 2: return col_tile<T, N, 2>(stage, a);
        case 4: return col_tile<T, N, 4>(stage, a);
        default: return cudaErrorInvalidValue;
    }
}

// Calls F.operator()<T, N>() for the runtime (n, fp64).
template <typename Fn>
cudaError_t dispatch(int n, int fp64, Fn&& fn) {
    if (fp64) {
        switch (n) {
            case 16: return fn.template operator()<double, 16>();
            case 32: return fn.template operator()<double, 32>();
            case 64: return fn.template operator()<double, 64>();
            case 128: return fn.template operator()<double, 128>();
            case 256: return fn.template operator()<double, 256>();
            case 512: return fn.template operator()<double, 512>();
            case 1024: return fn.template operator()<double, 1024>();
            case 2048: return fn.template operator()<double, 2048>();
            case 4096: return fn.template operator()<double, 4096>();
            default: return cudaErrorInvalidValue;
        }
    }
    switch (n) {
        case 16: return fn.template operator()<float, 16>();
        case 32: return fn.template operator()<float, 32>();
        case 64: return fn.template operator()<float, 64>();
        case 128: return fn.template operator()<float, 128>();
        case 256: return fn.template operator()<float, 256>();
        case 512: return fn.template operator()<float, 512>();
        case 1024: return fn.template operator()<float, 1024>();
        case 2048: return fn.template operator()<float, 2048>();
        case 4096: return fn.template operator()<float, 4096>();
        case 8192: return fn.template operator()<float, 8192>();
        default: return cudaErrorInvalidValue;
    }
}

template <int N>
void fill_table(double* out) {
    using P = FftPlan<N>;
    for (int dir = 0; dir < 2; ++dir) {
        const bool inv = dir == 0;
        for (int p = 1; p < P::NP; ++p) {
            const int S = P::stride(inv, p), R = P::radix(inv, p), o = P::tw_offset(inv, p);
            const int pw[6] = {1, 2, 3, 4, 8, 12};
            for (int k = 0; k < P::npow(R); ++k)
                for (int js = 0; js < S; ++js) {
                    // exp(+2 pi i js q / (S R)); reduce the exponent first for an exact angle
                    const long e = ((long)js * pw[k]) % (S * R);
                    const double a = 2.0 * M_PI * (double)e / (double)(S * R);
                    out[2 * (o + k * S + js)] = std::cos(a);
                    out[2 * (o + k * S + js) + 1] = std::sin(a);
                }
        }
    }
}

template <typename Fn>
auto by_size(int n, Fn&& fn) {
    switch (n) {
        case 16: return fn.template operator()<16>();
        case 32: return fn.template operator()<32>();
        case 64: return fn.template operator()<64>();
        case 128: return fn.template operator()<128>();
        case 256: return fn.template operator()<256>();
        case 512: return fn.template operator()<512>();
        case 1024: return fn.template operator()<1024>();
        case 2048: return fn.template operator()<2048>();
        case 4096: return fn.template operator()<4096>();
        default: return fn.template operator()<8192>();
    }
}

}  // namespace

int twiddle_table_size(int n) {
    return by_size(n, []<int N>() { return FftPlan<N>::TW_SIZE; });
}

void fill_twiddles(int n, double* out) {
    by_size(n, [&]<int N>() {
        fill_table<N>(out);
        return 0;
    });
}

bool tile_supported(int n, int tile) { return tile_ok(n, tile); }

void set_streaming(bool on) { g_streaming.store(on, std::memory_order_relaxed); }
bool streaming() { return g_streaming.load(std::memory_order_relaxed); }

cudaError_t wait_probe(unsigned polls, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    if (dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!g_err_addr[dev] && (e = cudaGetSymbolAddress((void**)&g_err_addr[dev], g_stream_err)))
        return e;
    k_wait_probe<<<1, 32, 0, st>>>(g_err_addr[dev], polls);
    return cudaGetLastError();
}

cudaError_t take_stream_error(unsigned* bits) {
    unsigned h = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&h, g_stream_err, sizeof(h));
    if (e) return e;
    *bits = h;
    const unsigned zero = 0;
    if (h) return cudaMemcpyToSymbol(g_stream_err, &zero, sizeof(zero));
    return cudaSuccess;
}

// ---- work-list passes
namespace {
constexpr int kMaxDevicesMulti = 64;
struct MultiLaunch {
    int grid[2][2][2] = {};  // [fp64][mt == 128][column]
};
MultiLaunch g_multi[kMaxDevicesMulti];

template <typename T, int MT>
cudaError_t multi_prepare_t(int dev) {
    int nsm = 0, occ = 0;
    cudaError_t e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev))) return e;
    const int rs = (int)multi_smem<cplx<T>, MT>(), cs = (int)multi_smem<Pair<T>, MT>();
    if ((e = cudaFuncSetAttribute(k_row_multi<T, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, rs)))
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_row_multi<T, MT>, MT, rs))) return e;
    g_multi[dev].grid[sizeof(T) == 8][MT == 128][0] = nsm * (occ > 0 ? occ : 1);
    auto col = [&](auto kern) -> cudaError_t {
        cudaError_t e2 = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cs);
        if (e2) return e2;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, MT, cs);
    };
    if ((e = col(k_col_multi<T, MT, 0>)) || (e = col(k_col_multi<T, MT, 1>)) ||
        (e = col(k_col_multi<T, MT, 2>)) || (e = col(k_col_multi<T, MT, 3>)))
        return e;
    g_multi[dev].grid[sizeof(T) == 8][MT == 128][1] = nsm * (occ > 0 ? occ : 1);
    return cudaSuccess;
}

template <typename T, int MT>
cudaError_t row_multi_t(const void* cls, const void* items, int nitems, int grid, cudaStream_t st) {
    k_row_multi<T, MT><<<grid, MT, multi_smem<cplx<T>, MT>(), st>>>(
        (const MultiClass*)cls, (const MultiItem*)items, nitems);
    return cudaGetLastError();
}

template <typename T, int MT>
cudaError_t col_multi_t(int stage, const void* cls, const void* items, int nitems, int grid,
                        cudaStream_t st) {
    const size_t sm = multi_smem<Pair<T>, MT>();
    auto c = (const MultiClass*)cls;
    auto it = (const MultiItem*)items;
    switch (stage) {
        case 0: k_col_multi<T, MT, 0><<<grid, MT, sm, st>>>(c, it, nitems); break;
        case 1: k_col_multi<T, MT, 1><<<grid, MT, sm, st>>>(c, it, nitems); break;
        case 2: k_col_multi<T, MT, 2><<<grid, MT, sm, st>>>(c, it, nitems); break;
        case 3: k_col_multi<T, MT, 3><<<grid, MT, sm, st>>>(c, it, nitems); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
}  // namespace

bool multi_supported(int n, int mt) {
    if (mt != 64 && mt != 128) return false;
    if (n < 32 || n > 1024 || (n & (n - 1))) return false;
    return n / 16 <= mt && 16 * mt / n <= n;
}

cudaError_t multi_prepare(int fp64, int mt) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e) return e;
    if (dev >= kMaxDevicesMulti) return cudaErrorInvalidDevice;
    if (mt == 64) return fp64 ? multi_prepare_t<double, 64>(dev) : multi_prepare_t<float, 64>(dev);
    if (mt == 128) return fp64 ? multi_prepare_t<double, 128>(dev) : multi_prepare_t<float, 128>(dev);
    return cudaErrorInvalidValue;
}

int multi_grid(int fp64, int mt, bool column) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= kMaxDevicesMulti) return 0;
    return g_multi[dev].grid[fp64 ? 1 : 0][mt == 128 ? 1 : 0][column ? 1 : 0];
}

cudaError_t row_multi(int fp64, int mt, const void* classes, const void* items, int nitems,
                      cudaStream_t st) {
    const int grid = multi_grid(fp64, mt, false);
    if (grid < 1) return cudaErrorNotReady;  // multi_prepare was not called on this device
    const int g = nitems < grid ? nitems : grid;
    if (mt == 64) return fp64 ? row_multi_t<double, 64>(classes, items, nitems, g, st)
                              : row_multi_t<float, 64>(classes, items, nitems, g, st);
    if (mt == 128) return fp64 ? row_multi_t<double, 128>(classes, items, nitems, g, st)
                               : row_multi_t<float, 128>(classes, items, nitems, g, st);
    return cudaErrorInvalidValue;
}

cudaError_t col_multi(int fp64, int mt, int stage, const void* classes, const void* items,
                      int nitems, cudaStream_t st) {
    const int grid = multi_grid(fp64, mt, true);
    if (grid < 1) return cudaErrorNotReady;
    const int g = nitems < grid ? nitems : grid;
    if (mt == 64) return fp64 ? col_multi_t<double, 64>(stage, classes, items, nitems, g, st)
                              : col_multi_t<float, 64>(stage, classes, items, nitems, g, st);
    if (mt == 128) return fp64 ? col_multi_t<double, 128>(stage, classes, items, nitems, g, st)
                               : col_multi_t<float, 128>(stage, classes, items, nitems, g, st);
    return cudaErrorInvalidValue;
}

bool supported(int n, int fp64) {
    if (n < 16 || (n & (n - 1))) return false;
    return fp64 ? n <= 4096 : n <= 8192;
}

cudaError_t set_attributes(int n, int fp64) {
    return dispatch(n, fp64, [&]<typename T, int N>() { return attrs<T, N>(); });
}

cudaError_t row_pass(int n, int fp64, void* X, int kc, const void* tw, cudaStream_t st,
                     int members, size_t x_stride, int tile) {
    return dispatch(n, fp64, [&]<typename T, int N>() {
        return row<T, N>(X, kc, tw, st, members, x_stride, tile);
    });
}

cudaError_t row_max(int n, int fp64, const void* X, int kc, const void* tw,
                    unsigned long long* umax, cudaStream_t st, int members, size_t x_stride) {
    return dispatch(n, fp64, [&]<typename T, int N>() {
        return rmax<T, N>(X, kc, tw, umax, st, members, x_stride);
    });
}

cudaError_t col_pass(int n, int fp64, int stage, void* X, int kc, void* u0t, void* acct,
                     const void* tab, const void* params, const void* tw, cudaStream_t st,
                     int members, size_t x_stride, size_t u_stride, int tab_stride, int tile) {
    ColArgs a{X, kc, u0t, acct, tab, params, tw, st, members, x_stride, u_stride, tab_stride, tile};
    return dispatch(n, fp64, [&]<typename T, int N>() { return col<T, N>(stage, a); });
}

cudaError_t transpose_in(int fp64, const void* u0, void* u0t, int n, int kc, cudaStream_t st,
                         int members, size_t u0_stride, size_t u_stride) {
    dim3 grid((kc + 31) / 32, (n + 31) / 32, members), block(32, 8);
    const int nh = n / 2 + 1;
    if (fp64)
        k_transpose_in<double><<<grid, block, 0, st>>>((const cplx<double>*)u0,
                                                       (cplx<double>*)u0t, n, nh, kc, u0_stride,
                                                       u_stride);
    else
        k_transpose_in<float><<<grid, block, 0, st>>>((const cplx<float>*)u0, (cplx<float>*)u0t,
                                                      n, nh, kc, u0_stride, u_stride);
    return cudaGetLastError();
}

cudaError_t transpose_out(int fp64, const void* u0t, void* u0, int n, int kc, cudaStream_t st,
                          int members, size_t u_stride, size_t u0_stride) {
    dim3 grid((kc + 31) / 32, (n + 31) / 32, members), block(32, 8);
    const int nh = n / 2 + 1;
    if (fp64)
        k_transpose_out<double><<<grid, block, 0, st>>>((const cplx<double>*)u0t,
                                                        (cplx<double>*)u0, n, nh, kc, u_stride,
                                                        u0_stride);
    else
        k_transpose_out<float><<<grid, block, 0, st>>>((const cplx<float>*)u0t,
                                                       (cplx<float>*)u0, n, nh, kc, u_stride,
                                                       u0_stride);
    return cudaGetLastError();
}

cudaError_t mask2d(int fp64, void* u0, int n, cudaStream_t st, int members) {
    const int nh = n / 2 + 1;
    const uint32_t fsc = (uint32_t)n * (uint32_t)nh;
    const dim3 grid((fsc + 255) / 256, members);
    if (fp64) k_mask2d<double><<<grid, 256, 0, st>>>((cplx<double>*)u0, n, nh, fsc);
    else k_mask2d<float><<<grid, 256, 0, st>>>((cplx<float>*)u0, n, nh, fsc);
    return cudaGetLastError();
}

cudaError_t reduce_t(int fp64, const void* u0t, int n, int kc, size_t u_stride, int members,
                     double klo, double khi, double* partials, int nblk, double* out,
                     cudaStream_t st) {
    const double inv_norm = 1.0 / std::pow((double)n, 4.0);
    const dim3 grid(nblk, members);
    if (fp64)
        k_reduce_t<double><<<grid, 256, 0, st>>>((const cplx<double>*)u0t, n, kc, u_stride,
                                                 inv_norm, klo * klo, khi * khi, partials);
    else
        k_reduce_t<float><<<grid, 256, 0, st>>>((const cplx<float>*)u0t, n, kc, u_stride,
                                                inv_norm, klo * klo, khi * khi, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_reduce_t_finish<<<members, 256, 0, st>>>(partials, nblk, out);
    return cudaGetLastError();
}

}  // namespace fused
}  // namespace sp
