/*
 * spectral_b200.h — C ABI of libspectral_b200.so, the B200 (sm_100a) engine for the Lawson
 * integrating-factor RK4 (IF-RK4) pseudo-spectral Navier-Stokes step on a periodic [0,2pi)^d box.
 *
 * The reference (pyspectral) drives its hot path from Python: the backend class
 * `CupyCudaSolver` (src/pyspectral/backends/cupy_cuda.py) owns CuPy buffers, cuFFT plans and
 * NVRTC kernels.  This header is the boundary that replaces that class's device work: a Python
 * (ctypes) / cgo / JNI caller binds plain device pointers and a stream and calls these entry points.
 *
 * Conventions
 *   - Every function returns an int status: SP_OK (0) or a negative sp_status; the message of
 *     the last failure is returned by sp_last_error(handle) (or sp_create_error() when creation
 *     failed).  No C++ exception crosses this boundary.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).  All device work
 *     is enqueued on it; functions that return host values synchronise that stream.
 *   - Device memory is owned by the caller.  sp_query_sizes() says how many bytes each buffer
 *     needs; sp_bind() hands them over.  The library allocates nothing on the device itself
 *     except what cuFFT plan creation reserves internally (plans run with auto-allocation off
 *     and use the caller's `fft_workspace`).
 *   - Spectral layout (all precisions): r2c layout of numpy.fft.rfftn, shape (n, n/2+1) in 2D and
 *     (n, n, n/2+1) per component in 3D, row-major, unnormalised forward convention.  The state
 *     buffer `u0` is exactly the array the reference's `state_native()` returns.
 */
#ifndef SPECTRAL_B200_H
#define SPECTRAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SP_ABI_VERSION 1

typedef struct sp_solver sp_solver;

enum sp_status {
    SP_OK = 0,
    SP_ERR_ARG = -1,         /* bad argument (size, null pointer, unsupported combination) */
    SP_ERR_CUDA = -2,        /* a CUDA runtime call failed */
    SP_ERR_CUFFT = -3,       /* a cuFFT call failed */
    SP_ERR_STATE = -4,       /* called in the wrong order (e.g. step before bind) */
    SP_ERR_UNSUPPORTED = -5  /* option not built into this engine */
};

/* Nonlinear-term form (src/pyspectral/config.py:7-8).  2D accepts basdevant only, like the
 * reference CUDA backend (src/pyspectral/backends/cupy_cuda.py:42-43). */
enum sp_form { SP_FORM_BASDEVANT = 0, SP_FORM_ROTATIONAL = 1 };

/* How the FFTs of a stage are executed.
 *   SP_FFT_CUFFT       batched in-place cuFFT plans (cupy_cuda.py:100-112, variant fused-inplace)
 *   SP_FFT_CUFFT_LEAN  single-field plans looped over the batch (cupy_cuda.py:114-128,
 *                      variant fused-inplace-lean: cuFFT workspace of one field)
 *   SP_FFT_FUSED       2D only: hand-written transforms fused with the pointwise phases, two
 *                      HBM round trips per RK stage (a row pass: inverse row FFT, products,
 *                      forward row FFT; a column pass: forward column FFT, Lawson update,
 *                      inverse column FFT) over the 2/3-dealiased columns only.  n a power of
 *                      two, 16..8192 (fp32) or 16..4096 (fp64); no cuFFT.  The state is kept
 *                      transposed internally; u0 is refreshed by sp_sync_state (and by the
 *                      diagnostics entry points when given u0). */
enum sp_fft_mode { SP_FFT_CUFFT = 0, SP_FFT_CUFFT_LEAN = 1, SP_FFT_FUSED = 2 };

/* Indices of the array filled by sp_query_sizes(). */
enum sp_size_index {
    SP_SZ_MODES = 0,         /* fsc = n^(d-1) (n/2+1): complex modes per spectral field */
    SP_SZ_NCOMP = 1,         /* state components: 1 (2D vorticity) or 3 (3D velocity) */
    SP_SZ_NWORK = 2,         /* complex work fields W: max(inverse, forward) FFT batch */
    SP_SZ_NINV = 3,          /* inverse FFTs per stage (config.py:84-92) */
    SP_SZ_NFWD = 4,          /* forward FFTs per stage */
    SP_SZ_STATE_BYTES = 5,   /* bytes of u0 (== bytes of acc) */
    SP_SZ_WORK_BYTES = 6,    /* bytes of W */
    SP_SZ_AUX_BYTES = 7,     /* bytes of the aux block: parameters, IF table, reduction scratch */
    SP_SZ_FFTWS_BYTES = 8,   /* bytes of the cuFFT work area */
    SP_SZ_NSHELL = 9,        /* number of spectrum shells (diagnostics.py:39) */
    SP_SZ_COUNT = 10
};

/* Reduction outputs of sp_diagnostics(). */
enum sp_diag_index {
    SP_DIAG_ENERGY = 0,       /* <|u|^2>/2                 diagnostics.py:65-67 */
    SP_DIAG_ENSTROPHY = 1,    /* <|omega|^2>/2             diagnostics.py:69-74 */
    SP_DIAG_PALINSTROPHY = 2, /* <|grad omega|^2>/2 (2D)   diagnostics.py:76-82 */
    SP_DIAG_BAND_ENERGY = 3,  /* energy in klo<=|k|<=khi   diagnostics.py:84-88 */
    SP_DIAG_COUNT = 4
};

/* ABI version of the loaded library (SP_ABI_VERSION at build time). */
int sp_abi_version(void);

/* Create an engine for one grid.  Replaces CupyCudaSolver.__init__'s plan and kernel set-up
 * (src/pyspectral/backends/cupy_cuda.py:40-82, plans :100-112).  Requires a CUDA device;
 * creates the cuFFT plans (auto-allocation off).  Returns NULL on failure with *status set and
 * the reason in sp_create_error(). */
sp_solver* sp_create(int n, int dim, int form, int fp64, int fft_mode, int* status);

/* Release plans, graphs and streams (not the caller's buffers). */
void sp_destroy(sp_solver* s);

/* Fill out[0..count) with the sp_size_index values (count <= SP_SZ_COUNT). */
int sp_query_sizes(const sp_solver* s, int64_t* out, int count);

/* Hand over caller-owned device buffers (sizes from sp_query_sizes, 256-byte aligned):
 * u0 = state, acc = RK accumulator, work = W (FFT work fields), aux = parameter block, IF table
 * and reduction scratch, fft_workspace = cuFFT work area.  Replaces the buffer allocation of
 * cupy_cuda.py:53-66.  Must be called once before any stepping. */
int sp_bind(sp_solver* s, void* u0, void* acc, void* work, void* aux, void* fft_workspace);

/* Physical parameters of the linear operator L(k) (src/pyspectral/backends/base.py:114-123):
 * viscosity nu, drag alpha on k^2 <= drag_k2 (config.py:59-62), forcing band [klo, khi]. */
int sp_set_physics(sp_solver* s, double nu, double alpha, double drag_k2, double force_klo,
                   double force_khi);

/* Band-forcing growth rate A, honoured from the next step on (base.py:98-100). */
int sp_set_forcing_amplitude(sp_solver* s, double amp);

/* Load the state just written into u0 (CupyCudaSolver.set_state + _pre, cupy_cuda.py:134-145,
 * kernels pre2d/pre3d of src/pyspectral/kernels/spectral.cu:93-103,164-173): dealiases u0 in
 * place (the 2/3 mask check_state applies on the host, src/pyspectral/backends/base.py:134-139)
 * and builds the stage-0 FFT inputs. */
int sp_prepare(sp_solver* s, void* stream);

/* Advance one IF-RK4 step of size dt (CupyCudaSolver._step + _stage, cupy_cuda.py:163-195).
 * Parameters live in device memory, so one captured CUDA graph serves every dt and forcing
 * amplitude (no re-capture per (dt, amp) as at cupy_cuda.py:181-195). */
int sp_step(sp_solver* s, double dt, void* stream);

/* Make u0 (the NumPy-layout state) current.  In SP_FFT_FUSED mode the step advances a
 * transposed copy of the state and u0 is written back here, once per change; in the cuFFT
 * modes u0 is always current and this does nothing.  Call before reading u0 directly
 * (state_native(), base.py:65-67). */
int sp_sync_state(sp_solver* s, void* stream);

/* 1 = replay each step from a CUDA graph (variant fused-inplace-graph), 0 = plain launches. */
int sp_set_graph(sp_solver* s, int enable);

/* Column pass of the fused 2D engine (SP_FFT_FUSED), process-wide: 1 (default) = the streamed
 * persistent pass for single runs of n = 2048..8192 (fp64 up to 4096) — each CTA loops over
 * columns and prefetches the next column's work data into shared memory by TMA while it
 * transforms the current one; 0 = one column per CTA.  Both give the same results to round-off.
 * Affects launches made (and graphs captured) after the call.  No reference counterpart. */
int sp_set_column_streaming(int enable);
int sp_column_streaming(void);

/* Error bits raised by this library's kernels on the current device since the last call (then
 * cleared) into *bits: 1 = a streamed column pass gave up waiting for its TMA data and skipped
 * its columns (results invalid).  Synchronous; SP_ERR_CUDA if the read fails.  No reference
 * counterpart. */
int sp_take_device_error(unsigned int* bits);

/* Failure-path check without a fault: launches one block whose mbarrier wait for a copy that is
 * never issued gives up after `polls` polls (1..2^20; a poll suspends for at most a few
 * microseconds), exactly as the streamed passes' waits do, and sets bit 1 of the device error
 * word (read and cleared by sp_take_device_error).  Nothing stays in flight; the context stays
 * usable.  No reference counterpart. */
int sp_wait_probe(unsigned int polls, void* stream);

/* Spectral reductions of a state array (device pointer in the u0 layout, e.g. u0 itself):
 * writes SP_DIAG_COUNT doubles to out (host) — energy, enstrophy, palinstrophy and the energy in
 * band_klo <= |k| <= band_khi — summed in fp64 in a fixed order.  Synchronises `stream`. */
int sp_diagnostics(sp_solver* s, const void* state, double band_klo, double band_khi,
                   double* out, void* stream);

/* sum_i max|u_i| in physical space of a state array (Diagnostics.max_velocity_sum,
 * src/pyspectral/diagnostics.py:99-109); out_per_comp (host, 3 doubles, may be NULL) receives
 * each component's max.  Uses the RK accumulator as scratch (it is dead between steps).
 * In SP_FFT_FUSED mode only `state == u0` is accepted (SP_ERR_UNSUPPORTED otherwise): the
 * bound comes from one inverse row pass over the stage-0 inputs already in the work array.
 * Synchronises `stream`. */
int sp_max_velocity(sp_solver* s, const void* state, double* out_sum, double* out_per_comp,
                    void* stream);

/* Shell-summed energy spectrum E(k), k = 0..nshell-1 (Diagnostics.spectrum,
 * src/pyspectral/diagnostics.py:90-97), written to out (host, nshell doubles). */
int sp_spectrum(sp_solver* s, const void* state, double* out, int nshell, void* stream);

/* Run one phase of one stage by itself (for per-phase timing and profiling):
 * phase 0 = batched inverse FFT, 1 = physical-space kernel, 2 = batched forward FFT,
 * 3 = spectral kernel of RK stage `stage` (0..3) using the parameters of the last step.
 * In SP_FFT_FUSED mode phase 0 is the row pass, 3 the column pass, 1 and 2 do nothing.
 * Phases 0+2 back to back are the standalone "FFT ceiling" of one stage
 * (src/pyspectral/benchmark.py:145-214). */
int sp_run_phase(sp_solver* s, int phase, int stage, void* stream);

/* Number of this library's own kernels launched through the handle so far (a graph replay
 * counts the kernels it contains; cuFFT's kernels are not counted).  -1 for a null handle.
 * No reference counterpart: instrumentation for the benchmark. */
int64_t sp_kernel_launches(const sp_solver* s);

/* Message of the last failure on this handle (never NULL). */
const char* sp_last_error(const sp_solver* s);

/* Message of the last sp_create (or sp_spectrum_noalloc) failure in this thread (never NULL). */
const char* sp_create_error(void);

/* ---------------------------------------------------------------- batched ensembles
 * No counterpart in the reference (one pyspectral solver is one run).  A batch advances
 * `members` independent 2D runs of one grid size on the fused-FFT engine, one launch per phase
 * for all members, each member with its own viscosity, time step and forcing amplitude; a
 * group steps several batches (uneven sizes) from one CUDA graph. */
typedef struct sp_batch sp_batch;
typedef struct sp_group sp_group;

/* n a power of two, 16..8192 (fp32) / 16..4096 (fp64); members 1..65535. */
sp_batch* sp_batch_create(int n, int fp64, int members, int* status);
void sp_batch_destroy(sp_batch* b);
/* out = [members, kc, state bytes (u0: members x n x (n/2+1) complex, NumPy layout each),
 *        0, work bytes, aux bytes] (count <= 6). */
int sp_batch_query_sizes(const sp_batch* b, int64_t* out, int count);
int sp_batch_bind(sp_batch* b, void* u0, void* work, void* aux);
/* nu: one viscosity per member; drag alpha on k^2 <= drag_k2; forcing band [klo, khi]. */
int sp_batch_set_physics(sp_batch* b, const double* nu, double alpha, double drag_k2,
                         double force_klo, double force_khi);
/* Per-member time step and band-forcing rate (host arrays, `amp` may be NULL); uploaded on
 * `stream` when they change; used by the following steps. */
int sp_batch_set_step(sp_batch* b, const double* dt, const double* amp, void* stream);
/* Load the states written into u0 (dealias, transpose, stage-0 inputs). */
int sp_batch_prepare(sp_batch* b, void* stream);
int sp_batch_step(sp_batch* b, void* stream);
/* Tile choice of the batched fused passes: sub-blocks per CTA = tile x the default (tile 1;
 * 2 and 4 are compiled for n <= 1024).  Each sequence is transformed by the same code; the
 * kernels of different tiles are compiled separately and may contract multiply-adds
 * differently, so results agree to round-off (bit-identical for a fixed tile; tile 1 is the
 * single-run engine's).  The ensemble autotuner picks the fastest per size class.
 * Set it before the first sp_group_step of a group that holds the batch (the group's graph is
 * captured then); it drops the batch's own step graph. */
int sp_batch_tile_supported(int n, int tile);
int sp_batch_set_tile(sp_batch* b, int tile);
int sp_batch_tile(const sp_batch* b);
/* Write the members' states back into u0 (NumPy layout) when they changed. */
int sp_batch_sync_state(sp_batch* b, void* stream);
/* out[m * 4 + q]: energy, enstrophy, palinstrophy, energy in band_klo <= |k| <= band_khi. */
int sp_batch_diagnostics(sp_batch* b, double band_klo, double band_khi, double* out,
                         void* stream);
/* out[m] = max|u| + max|v| of member m (CFL). */
int sp_batch_max_velocity(sp_batch* b, double* out, void* stream);
int64_t sp_batch_kernel_launches(const sp_batch* b);
const char* sp_batch_last_error(const sp_batch* b);
/* A group of bound, prepared batches stepped together from one graph: by default one branch
 * per batch (one launch per batch and phase); with a work list, one persistent launch per
 * phase over every batch.  No counterpart in the reference. */
sp_group* sp_group_create(sp_batch** batches, int count, int* status);
void sp_group_destroy(sp_group* g);
int sp_group_step(sp_group* g, void* stream);
const char* sp_group_last_error(const sp_group* g);
/* Work list: the group's row and column passes as two persistent launches per RK stage that
 * take packed items (class, member, 16 mt / n rows or columns) of every batch, CTAs of mt = 64
 * or 128 threads.  Runs batches of one precision with n a power of two, n / 16 <= mt and
 * 16 mt / n <= n (mt 64: n = 32..1024; 128: 64..1024); each item runs the single-run passes'
 * code.  *bytes = the device buffer the lists need (0 when no mt applies); sp_group_bind takes
 * a caller-owned buffer of that size (256-byte aligned); sp_group_set_worklist(g, mt) builds
 * and uploads the lists (synchronous; the batches must be bound; 0 returns to one launch per
 * batch) and drops the group's graph. */
int sp_group_worklist_bytes(const sp_group* g, int64_t* bytes);
int sp_group_bind(sp_group* g, void* buffer);
int sp_group_set_worklist(sp_group* g, int mt);
int sp_group_worklist(const sp_group* g);
/* Kernels the work-list group steps launched (the per-batch counters count the other path). */
int64_t sp_group_kernel_launches(const sp_group* g);

/* ---------------------------------------------------------------- tensor-core tiles
 * Check of the BF16 tcgen05 tile path the closure network uses (no reference counterpart):
 * D[128 x N] (fp32, row-major) = A * B^T with A = [128 x K] (a_mn = 0) or given transposed as
 * [K x 128] (a_mn = 1), B = [N x K] (b_mn = 0) or [K x N] (b_mn = 1), bf16 row-major device
 * arrays; N and K multiples of 16 in 16..256.  Synchronises `stream`. */
int sp_mma_tile_check(const void* A, const void* B, float* D, int N, int K, int a_mn, int b_mn,
                      void* stream);

/* ---------------------------------------------------------------- spectral helpers
 * Dealiased 2D nonlinear term N(state) (Basdevant form, no linear terms) of a spectral state in
 * u0 layout, written to `out` (same layout).  Replaces NumpySolver.nonlinear
 * (src/pyspectral/backends/numpy_ref.py:75-96, 2D branch).  Needs a bound 2D solver created
 * with SP_FFT_CUFFT; uses the work array as scratch and rebuilds the next stage's inputs from u0
 * afterwards, so stepping may continue. */
int sp_nonlinear(sp_solver* s, const void* state, void* out, void* stream);

/* pad_spectrum (src/pyspectral/validation.py:24-35) on the device: zero-pad or truncate an r2c
 * spectrum of grid n_src to grid n_dst (keeping |k| < min(n_src, n_dst)/2, rescaled by
 * (n_dst/n_src)^dim); dealias != 0 also applies n_dst's 2/3 mask, the sharp spectral filter of
 * the learned closure.  dim 2 or 3, fp32 or fp64 complex, src and dst must not overlap. */
int sp_filter_spectrum(const void* src, int n_src, void* dst, int n_dst, int dim, int fp64,
                       int dealias, void* stream);

/* ---------------------------------------------------------------- learned closure
 * No reference counterpart.  A per-point network 75 -> 64 -> 64 -> 64 -> 1 (GELU, tanh form)
 * maps the 5 x 5 stencils of the filtered vorticity and of its x and y derivatives to the
 * subgrid term S = F[N(omega)] - N_c(F[omega]) of a coarse 2D run (F = sp_filter_spectrum with
 * dealiasing, N and N_c the fine and coarse nonlinear terms).  Layers 1-3 are BF16 tcgen05
 * GEMMs with FP32 accumulation; the output layer is FP32.  Parameters (fp32, 15440 values):
 * W1, W2, W3 as [64][80] row-major with the bias in column 75 (W1) or 64 (W2, W3) and zero
 * padding, then w4[80] with the bias at index 64.  Axis x is the first (row) axis of a field,
 * y the contiguous one; feature f * 25 + (dx + 2) * 5 + (dy + 2) is field f at offset (dx, dy). */
typedef struct sp_closure sp_closure;

int sp_closure_param_count(void);
/* n: coarse grid, a power of two in 128..4096; capacity: snapshot-bank entries of 4 n^2 floats
 * (omega, omega_x, omega_y, S in physical space). */
sp_closure* sp_closure_create(int n, int capacity, int* status);
void sp_closure_destroy(sp_closure* c);
const char* sp_closure_last_error(const sp_closure* c);
int64_t sp_closure_kernel_launches(const sp_closure* c);
/* Host fp32 parameters; resets the Adam moments, the step counter and the loss record. */
int sp_closure_set_params(sp_closure* c, const float* host);
int sp_closure_get_params(sp_closure* c, float* host);
/* Gradient of the last sp_closure_grad / training step (15440 floats). */
int sp_closure_get_grad(sp_closure* c, float* host);
/* Network inputs are field * inscale[f]; its output times outscale is S.  clip != 0 zeroes
 * predictions with S * omega > 0 (local enstrophy backscatter) at inference. */
int sp_closure_set_scales(sp_closure* c, const float* inscale3, float outscale, int clip);
int sp_closure_get_scales(const sp_closure* c, float* out5);
/* Per-shell gains g(k) of the closure term in an attached solver's step (N += g(round|k|) S);
 * nshell = floor(sqrt(2) n/2 + 1/2) + 1 entries (sp_closure_shell_count), all 1 at creation. */
int sp_closure_set_shell_gain(sp_closure* c, const float* host, int nshell);
int sp_closure_shell_count(const sp_closure* c);
/* every_stage != 0 (the default): an attached solver evaluates the network at all four RK
 * stages; 0: at the first stage of each step only, its transformed term held for the other
 * three (which then run the plain two-field transforms).  Takes effect at the next step
 * (re-capture the step graph with sp_set_graph after changing it). */
int sp_closure_set_update(sp_closure* c, int every_stage);
/* Adam with linear warm-up over `warmup` steps and cosine decay to lr_min at total_steps. */
int sp_closure_set_adam(sp_closure* c, double lr, double lr_min, double beta1, double beta2,
                        double eps, int total_steps, int warmup);
/* Snapshot bank: load `count` host entries, append one from device spectra (coarse u0 layout,
 * fp32: the filtered vorticity, the filtered fine nonlinear term, the coarse nonlinear term of
 * the filtered vorticity), read one entry back, count, clear. */
int sp_closure_bank_load(sp_closure* c, const float* host, int count);
int sp_closure_add_snapshot(sp_closure* c, const void* wbar_hat, const void* fine_nl_hat,
                            const void* coarse_nl_hat, void* stream);
int sp_closure_bank_read(sp_closure* c, int index, float* host);
int sp_closure_bank_count(const sp_closure* c);
int sp_closure_bank_reset(sp_closure* c);
/* Mean-squared-error gradient over batch_tiles tiles of 128 points (a row segment of one bank
 * entry each, drawn by a counter hash of (seed, step, tile)), without an update. */
int sp_closure_grad(sp_closure* c, int64_t step, int batch_tiles, uint64_t seed, void* stream);
/* `steps` Adam steps at batch_tiles tiles each (graph-replayed in chunks); synchronises. */
int sp_closure_train(sp_closure* c, int steps, int batch_tiles, uint64_t seed, void* stream);
int64_t sp_closure_step_count(const sp_closure* c);
/* One optimiser step split around a gradient exchange (data-parallel training over ranks):
 * _begin runs the forward/backward kernels and leaves this rank's batch gradient (15440 fp32)
 * in the device buffer sp_closure_grad_buffer returns; the caller may replace it there (e.g.
 * by the mean over ranks with an NCCL all-reduce on the same stream); _finish applies Adam.
 * Nothing synchronises; sp_closure_check reports a timed-out wait. */
int sp_closure_train_begin(sp_closure* c, int batch_tiles, uint64_t seed, void* stream);
int sp_closure_train_finish(sp_closure* c, void* stream);
void* sp_closure_grad_buffer(sp_closure* c);
/* Mean loss of steps first .. first+count-1 (the last 65536 steps are kept). */
int sp_closure_losses(sp_closure* c, int64_t first, int count, float* host);
/* S at every point of an n x n field: inputs omega, omega_x, omega_y at fields + f*field_stride
 * (row stride row_stride floats), output rows of out_row_stride floats; synchronises. */
int sp_closure_infer(sp_closure* c, const float* fields, int64_t field_stride, int row_stride,
                     float* out, int out_row_stride, void* stream);
/* The same launch without the check and the synchronisation (sp_closure_check reports a
 * timed-out wait later). */
int sp_closure_infer_async(sp_closure* c, const float* fields, int64_t field_stride,
                           int row_stride, float* out, int out_row_stride, void* stream);
/* Attach a closure to a 2D fp32 SP_FFT_CUFFT solver of the same grid before sp_bind: every
 * stage then adds the network's S to the nonlinear term (the sizes sp_query_sizes reports grow
 * to six work fields).  The closure must outlive the solver. */
int sp_attach_closure(sp_solver* s, sp_closure* c);
/* Reports (and clears) a tensor-core wait that timed out in a closure kernel launched by a
 * solver step; synchronises `stream`. */
int sp_closure_check(sp_closure* c, void* stream);

/* ---------------------------------------------------------------- slab-decomposed 3D runs
 * No reference counterpart (the reference runs on one device).  One run of grid n spread over
 * nranks processes (one GPU each, nranks dividing n, m = n / nranks): rank r holds the ky slab
 * [r m, (r+1) m) of the spectral state (per component (n, m, n/2+1), u0 layout otherwise) and
 * the x slab [r m, (r+1) m) of the physical fields.  An RK stage is sp_slab_stage_part(0, s),
 * an all-to-all of `send` into `recv` (nranks equal contiguous blocks of
 * sp_slab_exchange_block_bytes(part 0) bytes; block p goes to rank p), part 1, the same
 * exchange with part 1's block size, part 2.  Sizes (sp_slab_query_sizes, 8 entries): modes per
 * local field, state bytes (3 fields), work bytes, send bytes (= recv bytes), aux bytes, cuFFT
 * work bytes, m, work fields.  Every call enqueues on `stream`; sp_slab_energy and
 * sp_slab_max_velocity synchronise it. */
typedef struct sp_slab sp_slab;
sp_slab* sp_slab_create(int n, int nranks, int rank, int form, int fp64, int* status);
void sp_slab_destroy(sp_slab* s);
const char* sp_slab_last_error(const sp_slab* s);
int64_t sp_slab_kernel_launches(const sp_slab* s);
int sp_slab_query_sizes(const sp_slab* s, int64_t* out, int count);
int64_t sp_slab_exchange_block_bytes(const sp_slab* s, int part);
/* With one rank `recv` may be `send` itself: the exchange is then nothing. */
int sp_slab_bind(sp_slab* s, void* u0, void* acc, void* work, void* send, void* recv, void* aux,
                 void* fft_workspace);
int sp_slab_set_physics(sp_slab* s, double nu, double alpha, double drag_k2, double force_klo,
                        double force_khi);
int sp_slab_set_forcing_amplitude(sp_slab* s, double amp);
/* Step scalars and integrating-factor table for the next step (as sp_step does). */
int sp_slab_set_dt(sp_slab* s, double dt, void* stream);
/* sp_prepare for the local slab: dealias u0 in place, build the stage-0 inputs. */
int sp_slab_prepare(sp_slab* s, void* stream);
int sp_slab_stage_part(sp_slab* s, int part, int stage, void* stream);
/* max |u_i| of this rank's x slab of the velocity the last stage 0 transformed (the CFL bound of
 * the state that step started from; take the max over ranks). */
int sp_slab_max_velocity(sp_slab* s, double* out3, void* stream);
/* Kinetic energy of this rank's slab of `state` (sum over ranks = the run's energy). */
int sp_slab_energy(sp_slab* s, const void* state, double* out, void* stream);

/* ---------------------------------------------------------------- device-run loop
 * simulate.run's loop (src/pyspectral/simulate.py:45-95, without records or callbacks) with its
 * control on the GPU: every cfl_every steps the CFL bound and, when target_power >= 0, the
 * constant-power amplitude A = P / (2 E_band) come from device reductions of the live state;
 * every step dt = min(h, t_end - t) and the step scalars and integrating-factor table are
 * written by a one-block kernel.  Chunks of cfl_every steps replay one captured graph; the host
 * reads t back once per chunk.  dt_fixed > 0 replaces the CFL rule by a fixed step.  *t_io: the
 * run's start time in, end time out; stops at t_end or after max_steps steps (steps of the last
 * chunk past t_end have dt = 0 and leave the state unchanged). */
int sp_run_to(sp_solver* s, double t_end, double cfl, double dt_max, int cfl_every,
              double target_power, double dt_fixed, int64_t max_steps, double* t_io,
              int64_t* steps_out, double* amp_out, void* stream);

/* Largest number of spectrum shells sp_spectrum_noalloc accepts: its accumulators are a fixed
 * file-scope device array of this many doubles (128 KiB).  2D grids up to n = 23168 fit, and
 * every 3D grid the engine indexes with 32 bits (n <= 1290). */
#define SP_NOALLOC_MAX_SHELLS 16384

/* Shell-summed energy spectrum E(k), k = 0..nshell-1, of a device state (u0 layout, fp32 or
 * fp64 complex) written to the host array `out` — without an engine handle and without
 * allocating any device memory.  No counterpart in the reference: it is for callers that must
 * not allocate device memory (a program whose own pool allocator owns the GPU's memory, or a
 * loop that may not take cudaMalloc's implicit synchronisation) yet need the spectrum of a state
 * they hold.  Same values as sp_spectrum.
 *   - Scratch: a file-scope __device__ array of SP_NOALLOC_MAX_SHELLS doubles, held by every GPU
 *     that loads the library until the process exits.  Each call clears the shells it uses.
 *   - The first call on a device looks the array's device address up (cudaGetSymbolAddress, with
 *     that device current) and caches it; make that first call before any stream capture.  The
 *     cached address belongs to the device's primary context: after cudaDeviceReset (or any
 *     tear-down of that context) this entry point must not be called again in the process.
 *   - Calls share the array: two calls whose work overlaps on the GPU race and give wrong
 *     results; order them on one stream.
 *   - Returns SP_ERR_ARG (message in sp_create_error()) when nshell does not match n and dim, or
 *     exceeds SP_NOALLOC_MAX_SHELLS; synchronises `stream`. */
int sp_spectrum_noalloc(const void* state, int n, int dim, int fp64, double* out, int nshell,
                        void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SPECTRAL_B200_H */
