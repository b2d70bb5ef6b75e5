// Host launchers of the fused 2D engine (kernels in fused2d.cuh, compiled in fused2d.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sp {
namespace fused {

// True when the fused 2D engine has kernels for grid n in this precision
// (n a power of two, 16 <= n <= 8192 in fp32, <= 4096 in fp64).
bool supported(int n, int fp64);
// Number of dealiased ky columns kept by the transforms: ky with 3 ky < n.
inline int kc_of(int n) { return (n + 2) / 3; }
// Opt every kernel of this size into its dynamic shared memory; once per process and size.
cudaError_t set_attributes(int n, int fp64);
// Complex entries of the per-pass twiddle table of a length-n transform, and the table itself
// (fp64, interleaved re/im, 2 * twiddle_table_size(n) doubles).
int twiddle_table_size(int n);
void fill_twiddles(int n, double* out);

// Batched forms: `members` independent runs of the same grid, member m's arrays `*_stride`
// elements after member m-1's (X in Pair units, u0/u0t/acct in complex units, tab in reals).
// tile: sub-block multiplier of the row and column passes (1; 2 and 4 for n <= 1024), the
// ensemble autotuner's choice.
bool tile_supported(int n, int tile);
// Process-wide choice of the streamed (persistent, TMA-prefetched) column pass for single runs
// of n = 2048..8192 (fp64 up to 4096); on by default.  Off: the one-column-per-CTA pass.
void set_streaming(bool on);
bool streaming();
// Error bits the streamed pass raised on this device since the last call (then cleared);
// synchronous.
cudaError_t take_stream_error(unsigned* bits);
// One block whose bounded mbarrier wait cannot complete: raises the streamed pass's time-out
// bit after `polls` polls (the failure path, exercised without a fault).
cudaError_t wait_probe(unsigned polls, cudaStream_t st);
cudaError_t row_pass(int n, int fp64, void* X, int kc, const void* tw, cudaStream_t st,
                     int members = 1, size_t x_stride = 0, int tile = 1);
cudaError_t row_max(int n, int fp64, const void* X, int kc, const void* tw,
                    unsigned long long* umax, cudaStream_t st, int members = 1,
                    size_t x_stride = 0);
// stage -1: build the stage-0 inputs from u0t; 0..3: Lawson stage.  params/tab: one
// StepParams and one table (tab_stride reals) per member.
cudaError_t col_pass(int n, int fp64, int stage, void* X, int kc, void* u0t, void* acct,
                     const void* tab, const void* params, const void* tw, cudaStream_t st,
                     int members = 1, size_t x_stride = 0, size_t u_stride = 0,
                     int tab_stride = 0, int tile = 1);
// ---- work-list passes of a batched group: one launch per phase over every size class.
// One size class as the work-list passes see it: member 0's arrays; member m's start m times
// the stride later (X in Pair units, u0t / acct in complex units, tab in reals).
struct MultiClass {
    void* X;
    void* u0t;
    void* acct;
    const void* tab;
    const void* params;  // one StepParams per member
    const void* tw;
    uint64_t x_stride, u_stride;
    int tab_stride, n, kc, pad;
};
// One item: rows (row pass) or columns (column pass) first .. first + 16 mt / n - 1 of member
// `member` of class `cls`, for a CTA of mt threads.
struct MultiItem {
    int cls, member, first;
};
// Sizes the work-list passes run for CTAs of mt (64 or 128) threads: a power of two with
// n / 16 <= mt and 16 mt / n <= n (an item holds whole rows of one member).
bool multi_supported(int n, int mt);
inline int multi_per_item(int n, int mt) { return 16 * mt / n; }
// Dynamic shared memory opt-in and the persistent grids (SMs x resident CTAs) of the passes;
// once per process, outside any stream capture.
cudaError_t multi_prepare(int fp64, int mt);
int multi_grid(int fp64, int mt, bool column);
cudaError_t row_multi(int fp64, int mt, const void* classes, const void* items, int nitems,
                      cudaStream_t st);
cudaError_t col_multi(int fp64, int mt, int stage, const void* classes, const void* items,
                      int nitems, cudaStream_t st);

cudaError_t transpose_in(int fp64, const void* u0, void* u0t, int n, int kc, cudaStream_t st,
                         int members = 1, size_t u0_stride = 0, size_t u_stride = 0);
cudaError_t transpose_out(int fp64, const void* u0t, void* u0, int n, int kc, cudaStream_t st,
                          int members = 1, size_t u_stride = 0, size_t u0_stride = 0);
cudaError_t mask2d(int fp64, void* u0, int n, cudaStream_t st, int members = 1);
// Energy, enstrophy, palinstrophy, band energy of every member's transposed state into
// out[m * 4 + q]; partials: members * nblk * 4 doubles of scratch.
cudaError_t reduce_t(int fp64, const void* u0t, int n, int kc, size_t u_stride, int members,
                     double klo, double khi, double* partials, int nblk, double* out,
                     cudaStream_t st);

}  // namespace fused
}  // namespace sp
