/*
 * ssam.h -- C ABI of the B200-native register-cache systolic stencil and
 * convolution library (libssam_b200.so).
 *
 * Conventions shared by every entry point
 * ---------------------------------------
 *  - Grids are row-major with x fastest, exactly as the reference lays them
 *    out: 2D index = pitch*y + x (ssai-2dstencil/stencil2D_5pt-v1.cu:29,
 *    ssai-2dconv/conv2D.cu:32), 3D index = nx*ny*z + nx*y + x
 *    (ssai-3dstencil/tmp3d7pt-v2.cu:107).  `pitch` is counted in ELEMENTS, like
 *    the reference's `widthStride` (conv2D.cu:11).
 *  - All grid pointers are DEVICE pointers owned by the caller.  `src` is read
 *    only; `dst` is a separate buffer (no in-place update), as in every
 *    reference kernel (`const T* __restrict__ src, T* dst`).
 *  - Calls are asynchronous on the caller's CUDA stream (`stream` is a
 *    cudaStream_t; NULL = legacy default stream).  The reference is synchronous
 *    on the default stream; callers that want that behaviour synchronise.
 *  - Every function returns an ssam_status.  Nothing throws across the ABI.
 *    ssam_last_error() returns a message for the calling thread's last failure.
 *  - Coefficients are passed as HOST arrays of double and are converted once to
 *    the compute type (float for F32/BF16/F16 storage, double for F64), the
 *    same value the reference obtains from its `T`-typed literals.
 *  - There is no CPU fallback: without a usable sm_100 device every compute
 *    entry point fails with SSAM_ERR_CUDA.
 */
#ifndef SSAM_B200_H
#define SSAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSAM_ABI_VERSION 2

/* Exported symbols (the library is built with hidden visibility). */
#if defined(__GNUC__)
#define SSAM_API __attribute__((visibility("default")))
#else
#define SSAM_API
#endif

typedef enum ssam_status {
  SSAM_OK = 0,
  SSAM_ERR_INVALID = 1,     /* bad argument: null pointer, size, radius, pitch ... */
  SSAM_ERR_UNSUPPORTED = 2, /* valid request that this build has no kernel for */
  SSAM_ERR_CUDA = 3,        /* CUDA runtime error (launch, copy, no device) */
  SSAM_ERR_NOMEM = 4,       /* device scratch allocation failed */
  SSAM_ERR_TIMEOUT = 5      /* a bounded device-side wait gave up */
} ssam_status;

/* Storage type of the grid.  F32 and F64 compute in their own precision, as
 * the reference does; BF16 and F16 are storage-only types that the kernels
 * widen to float and accumulate in float. */
typedef enum ssam_dtype {
  SSAM_F32 = 0,
  SSAM_F64 = 1,
  SSAM_BF16 = 2,
  SSAM_F16 = 3
} ssam_dtype;

/* What a tap that falls outside the grid reads, and what is written near the
 * edge.
 *  ZERO  : out-of-grid taps read 0 and every cell is computed -- the CPU golden
 *          `Convolution` (ssai-2dconv/common.h:186-216) and the conv kernel
 *          (conv2D.cu:36-41).
 *  CLAMP : out-of-grid taps read the nearest edge cell and every cell is
 *          computed -- the 2D/3D stencil kernels' halo load
 *          (stencil2D_5pt-v1.cu:29-46, tmp3d7pt-v2.cu:107-121).  Single step
 *          only.
 *  COPY  : cells closer to the edge than the stencil reach keep their input
 *          value every step (fixed / Dirichlet boundary); all other cells are
 *          computed.  For 3D this is the reference gold with its output
 *          initialised from the input (tmp3d7pt-v2.cu:278-298). */
typedef enum ssam_boundary {
  SSAM_BOUNDARY_ZERO = 0,
  SSAM_BOUNDARY_CLAMP = 1,
  SSAM_BOUNDARY_COPY = 2
} ssam_boundary;

/* Tap pattern of a square 2D stencil of radius r. */
typedef enum ssam_shape2d {
  /* (2r+1)x(2r+1) matrix, non-zero only on the centre row and column: the
   * reference's 5/9/13/17/21/25-pt star stencils (stencil2D_25pt.cu:167-181). */
  SSAM_STAR = 0,
  /* full (2r+1)x(2r+1) box: 9/25/49/81/121-pt (stencil2D_81pt.cu,
   * stencil2D_121pt.cu) and the 64-pt 9x9 with a zero centre cross
   * (stencil2D_64pt.cu:255-266). */
  SSAM_BOX = 1
} ssam_shape2d;

/* Tap pattern of a 3D stencil of radius r (coefficients are always passed as
 * the dense (2r+1)^3 cube, see ssam_stencil3d). */
typedef enum ssam_shape3d {
  /* taps on the three axes: 7-pt (r=1, tmp3d7pt-v2.cu) and 13-pt (r=2,
   * tmp3d13pt.cu) */
  SSAM_STAR3D = 0,
  /* r=1, every tap with at most two non-zero offsets: the reference's 19-point
   * "poisson" operator (tmpPoisson.cu:369-386) */
  SSAM_POISSON19 = 2
} ssam_shape3d;

/* ---------------------------------------------------------------- library */

/* Message for the calling thread's most recent non-OK status ("" if none). */
SSAM_API const char* ssam_last_error(void);

/* SSAM_ABI_VERSION of the loaded library. */
SSAM_API int ssam_abi_version(void);

/* Number of kernels this library has launched in the process so far (all
 * threads, all devices); lets a caller count the launches of a region. */
SSAM_API uint64_t ssam_kernel_launches(void);

/* Device scratch (multi-step ping-pong grids, host-call staging) comes from a
 * library memory pool per device that keeps freed memory mapped for the next
 * call.  This returns all of it that is not in use to the driver. */
SSAM_API int ssam_trim_scratch(void);

/* ------------------------------------------------------------ 2D stencils */

/*
 * One or more time steps of a square 2D stencil of radius r (1..10).
 *
 * Replaces the reference kernels and their host drivers
 *   stencil2d_v1::j2d5pt          ssai-2dstencil/stencil2D_5pt-v1.cu:8-129
 *   j2d9pt .. j2d25pt (star r=2..6)  stencil2D_9pt.cu:9-87 .. stencil2D_25pt.cu:9-126
 *   j2d64pt / j2d81pt / j2d121pt(+v2/v3/v4)  stencil2D_64pt.cu:73-214,
 *                                 stencil2D_81pt.cu:91-249, stencil2D_121pt.cu:131-331
 *   stencil2d_tmp::j2d5pt / j2d9pt (ITERATIVE_COUNT fused steps)
 *                                 stencil2d_temp_5pt.cu:9-82, stencil2d_temp_9pt.cu:13-95
 * and the entry points `int stencil_<N>pt_<float|double>(argc, argv)` and
 * `stencil_tmp_<N>pt_*` that drive them (ssai-2dstencil/main.cpp:29-53).
 *
 * coeffs:
 *   SSAM_STAR: 4r+1 values in the reference's kernel-argument order:
 *              c, then for ring k=1..r: n_k, s_k, w_k, e_k
 *              (stencil2D_25pt.cu:10-16: fc, fn0, fs0, fw0, fe0, fn1, ...).
 *              n = row y-k, s = row y+k, w = column x-k, e = column x+k.
 *   SSAM_BOX : (2r+1)^2 values, row-major, coeffs[(dy+r)*(2r+1) + (dx+r)]
 *              weights in(y+dy, x+dx) -- the reference's `_F<row><col>`
 *              tables (stencil2D_81pt.cu:4-84).
 * steps >= 1: time steps; step k+1 reads step k's result.  Steps are fused in
 * registers (temporal blocking) and chained through a device scratch grid that
 * the library allocates stream-ordered when more than one launch is needed.
 * CLAMP is single-step only.
 */
SSAM_API int ssam_stencil2d(const void* src, void* dst, int64_t width, int64_t height,
                   int64_t pitch, int dtype, int shape, int radius,
                   const double* coeffs, int steps, int boundary, void* stream);

/*
 * ssam_stencil2d on HOST buffers: the grid is copied to the device, stepped
 * and copied back, like the reference Test() drivers (DevBuffer::CopyFromHost
 * -> kernel -> CopyToHost, stencil2D_5pt-v1.cu:164-203).  Device memory is
 * allocated stream-ordered inside the call.  A single step is pipelined over
 * row bands (upload, compute and download overlap).  Returns once the work is
 * queued on `stream`; h_dst is valid after the stream is synchronised.  Use
 * page-locked host memory for full copy bandwidth.
 */
SSAM_API int ssam_stencil2d_host(const void* h_src, void* h_dst, int64_t width,
                                 int64_t height, int64_t pitch, int dtype, int shape,
                                 int radius, const double* coeffs, int steps,
                                 int boundary, void* stream);

/* Largest scratch grid, in bytes (pitch * height * element size), that
 * ssam_stencil2d_noalloc can hold. */
#define SSAM_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)

/*
 * ssam_stencil2d for callers that cannot allocate device memory.  No
 * counterpart in the reference (it has no library interface at all).
 *
 * Callers inside a fixed device-memory budget, or hosts that forbid
 * allocation after start-up, cannot let ssam_stencil2d take its multi-step
 * scratch grid from a memory pool.  This entry point computes the same steps
 * with the same kernels, but keeps that scratch grid in a library-owned
 * device array of SSAM_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until exit; it calls no allocator.  A run that needs scratch
 * (more than one launch in the chain) and a grid larger than the array
 * fails with SSAM_ERR_INVALID.  The array's device address is looked up on
 * every call made outside stream capture (a cudaDeviceReset in between is
 * harmless); a call under capture reuses the last address found on that
 * device, so the first call on each device must come before any capture
 * (under capture it fails with SSAM_ERR_INVALID otherwise).  With lazy module
 * loading (the CUDA 12 default) the array is reserved when the library's
 * module first loads on a device -- possibly during this first call, which
 * can then fail with SSAM_ERR_CUDA (out of memory).  All calls share the
 * array: calls that overlap on the GPU race, so callers serialise them.
 */
SSAM_API int ssam_stencil2d_noalloc(const void* src, void* dst, int64_t width,
                                    int64_t height, int64_t pitch, int dtype, int shape,
                                    int radius, const double* coeffs, int steps,
                                    int boundary, void* stream);

/*
 * Generic 2D correlation with an fw x fh weight matrix (1 <= fw, fh <= 28):
 *   dst(y, x) = sum_{n<fh, m<fw} weight[n*fw + m] * src(y + n - fh/2, x + m - fw/2)
 * Replaces CONV2D::kernel_convolution2D<T,B,P,FW,FH>
 * (ssai-2dconv/conv2D.cu:9-70, weights `smem[n][m]` row n / column m) and its
 * driver Test_conv2D / Test_2D (conv2D.cu:72-230).  The reference always zero
 * pads (boundary = SSAM_BOUNDARY_ZERO); CLAMP and COPY are also accepted.
 * Even and non-square filters follow the same offsets as the reference.
 */
SSAM_API int ssam_conv2d(const void* src, void* dst, int64_t width, int64_t pitch,
                int64_t height, int dtype, const double* weight, int fw, int fh,
                int boundary, void* stream);

/* ------------------------------------------------------- batched 2D grids */

/* One grid of a batch (device pointers, sizes in elements). */
typedef struct ssam_grid2d {
  const void* src;
  void* dst;
  int64_t width, height, pitch;
} ssam_grid2d;

typedef enum ssam_batch_mode {
  /* one cooperative launch steps every grid: warps take tiles from the
   * flattened tile list of all grids, a grid-wide barrier (bounded wait)
   * separates the fused-step phases */
  SSAM_BATCH_PERSISTENT = 0,
  /* ssam_stencil2d on each grid in turn (one launch chain per grid) */
  SSAM_BATCH_PER_GRID = 1
} ssam_batch_mode;

/*
 * `steps` steps of the same stencil on `ngrids` independent grids of
 * arbitrary, unequal sizes (same dtype, shape, coefficients, boundary).  The
 * reference runs one grid per program invocation; this batches them.
 * Persistent mode is compiled for star/box r = 1, 2 (FP32, FP64, BF16) and
 * r = 3 (FP32); other stencils return SSAM_ERR_UNSUPPORTED there and run
 * with SSAM_BATCH_PER_GRID.
 */
SSAM_API int ssam_stencil2d_batched(const ssam_grid2d* grids, int ngrids, int dtype,
                                    int shape, int radius, const double* coeffs, int steps,
                                    int boundary, int mode, void* stream);

/*
 * Test hook for the bounded-wait error path; no counterpart in the reference.
 * Every grid-wide barrier of later persistent ssam_stencil2d_batched launches
 * waits for `extra_arrivals` more CTAs than the launch has (arrivals that
 * never come when > 0), and gives up after `wait_ns` nanoseconds (0 = the
 * normal 2 s).  A barrier that gives up records code 4 in the device error
 * word and its CTA returns (nothing asynchronous is in flight there), so the
 * context stays usable: ssam_device_status then reports SSAM_ERR_TIMEOUT.
 * ssam_debug_batched_barrier(0, 0) restores normal operation.  Process-wide;
 * not for production use.
 */
SSAM_API int ssam_debug_batched_barrier(unsigned extra_arrivals, unsigned long long wait_ns);

/* -------------------------------------------------------------- autotuner */

/* What the autotuner chose for one stencil and grid size. */
typedef struct ssam_tune_report {
  int rows_per_thread;    /* P: output rows a thread keeps in registers */
  int warps_per_block;    /* warps per thread block */
  int columns_per_thread; /* V: columns a thread owns; warp strip = 32*V */
  int fused_steps;        /* temporal depth: steps fused per launch */
  int candidates;         /* kernel configurations timed */
  double ms_per_step;     /* best measured time per step (ms) */
} ssam_tune_report;

/*
 * Times every compiled configuration of this stencil -- outputs per thread,
 * strip width, warps per block and temporal depth -- on the caller's buffers
 * (dst is overwritten) and stores the fastest for the grid's size class
 * (log2 of width and height); later ssam_stencil2d / _host / _noalloc calls
 * on grids of that class use it.  The reference hand-picks these constants
 * per GPU (PROCESS_DATA_COUNT, BLOCK_SIZE, ITERATIVE_COUNT chosen with
 * IsTeslaV100(), tmp3d7pt-v2.cu:341-387); this replaces that choice.
 * Synchronous: returns after the timing runs.  `report` may be NULL.
 */
SSAM_API int ssam_autotune_stencil2d(const void* src, void* dst, int64_t width,
                                     int64_t height, int64_t pitch, int dtype, int shape,
                                     int radius, const double* coeffs, int steps,
                                     int boundary, void* stream, ssam_tune_report* report);

/* What the 3D autotuner chose for one stencil and grid size. */
typedef struct ssam_tune3d_report {
  int rows_per_warp;  /* PY: rows of the column tile each consumer warp computes */
  int consumer_warps; /* NW: consumer warps per CTA; the tile is 32*V x NW*PY cells */
  int ring_slots;     /* S: z-planes of the tile staged in shared memory */
  int registers_z;    /* 1: each thread keeps its own cells of the 2R+1 planes in
                         registers (shared memory carries the halos only) */
  int columns_per_thread; /* V: the tile is 32*V columns wide */
  int candidates;     /* configurations timed */
  double ms_per_step; /* best measured time per step: one launch's time / fused_steps (ms) */
  int fused_steps;    /* time steps one launch of the chosen configuration applies (1 or 2) */
} ssam_tune3d_report;

/*
 * Times every compiled configuration of this 3D stencil (rows per warp,
 * consumer warps, shared-memory ring depth), both the single-step kernels and
 * those that fuse two time steps in one z-march, on the caller's buffers (dst
 * is overwritten), and stores for the grid's size class (log2 of nx, ny, nz)
 * the fastest of each and the temporal depth (1 or 2 steps a launch) with
 * the lower time per step; later ssam_stencil3d / _host calls on grids of
 * that class use them (cached step graphs are re-captured).  The reference
 * fixes these per GPU model (BLOCK_SIZE / PROCESS_DATA_COUNT /
 * ITERATIVE_COUNT chosen with IsTeslaV100(), tmp3d7pt-v2.cu:341-387).
 * Synchronous.  `report` describes the configuration of the chosen depth and
 * may be NULL.
 */
SSAM_API int ssam_autotune_stencil3d(const void* src, void* dst, int64_t nx, int64_t ny,
                                     int64_t nz, int dtype, int shape, int radius,
                                     const double* coeffs, int boundary, void* stream,
                                     ssam_tune3d_report* report);

/*
 * The same for the Jacobi sweep of the Poisson solver (7-point stencil plus
 * right-hand-side term) on `nbatch` stacked n^3 grids stored as sweep_dtype
 * (SSAM_F32 or SSAM_BF16); times on scratch buffers of its own (stream-ordered
 * pool), so it needs no caller data.  Later ssam_poisson_solve* calls of that
 * size use the choice.
 */
SSAM_API int ssam_autotune_jacobi3d(int64_t n, int nbatch, int sweep_dtype, void* stream,
                                    ssam_tune3d_report* report);

/* Persist / restore / forget the measured choices of the 2D and 3D
 * autotuners.  The file is text, one choice a line ('#' starts a comment):
 *   choice   dtype rl rr rt rb star t log2w log2h P warps V
 *   depth    dtype rl rr rt rb star log2w log2h t
 *   choice3d dtype shape radius rhs log2nx log2ny log2(nz*nbatch) PY NW S zreg V t
 *   depth3d  dtype shape radius log2nx log2ny log2nz t
 * (t: time steps fused in one launch; P: rows a thread, or the streaming
 * segment; V: columns a thread; shape: 0 star, 1 19-point)
 * (a choice3d line without its last field means t = 1, without its last two
 * V = 4 and t = 1; with no depth3d line for a size class, multi-step 3D runs
 * take one step a launch).  Writing such lines
 * by hand pins a configuration (one that is not compiled into the library
 * is kept but not used: calls fall back to a compiled default); load fails with SSAM_ERR_INVALID, naming the
 * count of malformed lines, when a line does not parse or a value is out of
 * range, after loading the good ones. */
SSAM_API int ssam_autotune_save(const char* path);
SSAM_API int ssam_autotune_load(const char* path);
SSAM_API int ssam_autotune_clear(void);

/* ------------------------------------------------------------ 3D stencils */

/*
 * `steps` time steps of a 3D stencil on a dense nx*ny*nz grid
 * (index nx*ny*z + nx*y + x).
 *
 * Replaces v2::kernel3d_3d7pt (ssai-3dstencil/tmp3d7pt-v2.cu:62-208),
 * kernel3d_3d13pt (tmp3d13pt.cu:74-230), kernel3d_poisson
 * (tmpPoisson.cu:86-298), their host_code drivers and the entry points
 * stencil_3d7pt_v2 / stencil_3d13pt / stencil_poisson (ssai-3dstencil/
 * main.cpp:5-21).
 *
 * coeffs: the dense (2r+1)^3 cube, coeffs[((dz+r)*(2r+1) + dy+r)*(2r+1) + dx+r]
 * weights in(z+dz, y+dy, x+dx) -- the reference's `_F<z><y><x>` defines with
 * digits = offset + r (tmp3d7pt-v2.cu:9-15).  Entries outside the shape's
 * pattern are ignored.  Supported: SSAM_STAR3D r = 1, 2 and SSAM_POISSON19.
 * boundary: ZERO or COPY (the reference golds' interior with the ring kept).
 * steps > 1: one step a launch, or -- where ssam_autotune_stencil3d measured
 * it faster for the size class, or a depth3d line pins it -- launches that
 * each fuse two time steps in one z-march (temporal blocking, like the
 * reference's ITERATIVE_COUNT, tmp3d7pt-v2.cu:124-170; FP32/BF16 all three
 * shapes, FP64 r = 1) plus a single step for an odd count; they chain
 * through a stream-ordered scratch grid and, unless the stream is already
 * being captured, the whole chain is captured once into a CUDA graph
 * (cached per pointers/sizes/coefficients) and replayed on later calls.
 * Intermediate steps are rounded to the storage type, as a chain of single
 * steps stores them.
 */
SSAM_API int ssam_stencil3d(const void* src, void* dst, int64_t nx, int64_t ny, int64_t nz,
                            int dtype, int shape, int radius, const double* coeffs,
                            int steps, int boundary, void* stream);

/* ssam_stencil3d on HOST buffers (copy in, steps, copy out, on `stream`). */
SSAM_API int ssam_stencil3d_host(const void* h_src, void* h_dst, int64_t nx, int64_t ny,
                                 int64_t nz, int dtype, int shape, int radius,
                                 const double* coeffs, int steps, int boundary,
                                 void* stream);

/* ---------------------------------------------------------------- Poisson */

/*
 * -lap(u) = f on the unit cube with u = 0 on the boundary, discretised with the
 * 7-point operator on n^3 interior points (h = 1/(n+1)); `nbatch` independent
 * right-hand sides stored one after the other (index ((b*n + z)*n + y)*n + x).
 * No counterpart in the reference: its "poisson" program applies a 19-point
 * operator (tmpPoisson.cu); the solver follows its 7-point stencil structure
 * (v2::j3d7pt_gold, tmp3d7pt-v2.cu:281-297).
 */
typedef struct ssam_poisson_options {
  double tol;                /* stop when ||f - A u||_2 / ||f||_2 <= tol for every rhs */
  int sweep_dtype;           /* SSAM_F32 or SSAM_BF16: storage of the Jacobi sweeps */
  int sweeps_per_correction; /* Jacobi sweeps between two FP64 residuals */
  int max_sweeps;            /* give up (converged = 0) after this many sweeps */
  double omega;              /* Jacobi damping: u <- (1-w) u + w (nbrs + h^2 r) / 6;
                                0 is taken as 1 (plain Jacobi) */
  int cnn_smoothing;         /* learned solve: passes of the 7-point average (centre 1/2,
                                neighbours 1/12) applied to the network's input and
                                output; 0 = none */
} ssam_poisson_options;

typedef struct ssam_poisson_stats {
  int converged;               /* every rhs reached tol */
  int sweeps;                  /* Jacobi sweeps run */
  int corrections;             /* FP64 defect-correction steps */
  double initial_rel_residual; /* max over the batch, for the initial guess */
  double rel_residual;         /* max over the batch, final (FP64) */
  int cnn_corrections;         /* network corrections kept (learned solve only) */
  int fell_back;               /* learned solve: the warm start was dropped for u = 0 */
} ssam_poisson_stats;

/*
 * Defect correction: r = f - A u in FP64; e ~= A^-1 r by `sweeps_per_correction`
 * Jacobi sweeps from 0 in sweep_dtype storage with FP32 arithmetic; u += e in
 * FP64; until tol.  `u` (device, FP64) holds the initial guess on entry (zeros
 * for the plain method, a learned warm start otherwise) and the solution on
 * return.  Synchronous: it reads the residual norms on the host.
 */
SSAM_API int ssam_poisson_solve(const double* f, double* u, int n, int nbatch,
                                const ssam_poisson_options* opt, ssam_poisson_stats* stats,
                                void* stream);

/*
 * The learned arm: as ssam_poisson_solve, but each defect-correction step
 * first applies the warm-start network `cnn` (ssam_cnn_create) to the FP64
 * residual, u += CNN(r), and then runs the sweeps on the new residual (with
 * u = 0 on entry the first step is the network's warm start).  A step with
 * the network is kept only when it lowers the residual by 10% or more;
 * otherwise u is restored and the rest of the solve is the plain method.  If
 * the residual of the initial guess exceeds that of u = 0 the guess is
 * replaced by zeros.  Damped sweeps (omega < 1) remove the high-frequency
 * error that the network's BF16 arithmetic leaves.
 * The network must have been created with nbatch_max >= nbatch and the same n.
 * No counterpart in the reference (it has no Poisson solver).
 */
SSAM_API int ssam_poisson_solve_learned(const double* f, double* u, int n, int nbatch,
                                        const ssam_poisson_options* opt, void* cnn,
                                        ssam_poisson_stats* stats, void* stream);

/* ||f - A u||_2 / ||f||_2 per right-hand side, in FP64 (`rel` is host, nbatch);
 * ||f - A u||_2 itself where f = 0. */
SSAM_API int ssam_poisson_residual(const double* f, const double* u, int n, int nbatch,
                                   double* rel, void* stream);

/*
 * `sweeps` plain Jacobi sweeps u <- (sum of the 6 neighbours + h^2 rhs) / 6 in
 * `dtype` storage (F32, BF16 or F64), from u_in into u_out (u_in != u_out).
 */
SSAM_API int ssam_poisson_jacobi(const void* rhs, const void* u_in, void* u_out, int n,
                                 int nbatch, int dtype, int sweeps, void* stream);

/* ------------------------------------------------------- warm-start CNN */

/*
 * Tensor-core (tcgen05) building blocks of the Poisson warm-start network.
 * No counterpart in the reference.  Activations are BF16 with 16 channels in
 * "planar halves": (2, nbatch, n, n, n, 8) -- channels 0-7 of every voxel,
 * then channels 8-15 -- n a power of two (n^3 a multiple of 128); a layer
 * reads one or two 16-channel sources (in1 may be NULL; out may not alias
 * in0 or in1).  Weights are BF16 (16 out, 27 taps, 16 * nsrc in); tap =
 * (kz*3 + ky)*3 + kx reads offset ((kz-1), (ky-1), (kx-1)) * dilation, zero
 * outside the grid.
 */
SSAM_API int ssam_cnn_conv3d(const void* in0, const void* in1, const void* weight, void* out,
                             int nbatch, int n, int dilation, float out_scale, void* stream);

/* fp32 weight gradient (16, 27, 16 * nsrc) of ssam_cnn_conv3d for grad_out
 * (BF16, 16 channels, planar halves). */
SSAM_API int ssam_cnn_conv3d_wgrad(const void* in0, const void* in1, const void* grad_out,
                                   float* dweight, int nbatch, int n, int dilation,
                                   void* stream);

/*
 * The warm-start network for the Poisson solve on n^3 grids (n a power of two
 * >= 32): a 3-level, 16-channel linear U-Net of the convolutions above
 * (levels n, n/2, n/4; dilations 1, 2, 4, 8 at the bottom), trained and run
 * on the GPU.  f and u are FP64 (nbatch, n, n, n) device arrays.
 */
SSAM_API int ssam_cnn_create(int n, int nbatch_max, unsigned long long seed, void** handle);
SSAM_API int ssam_cnn_destroy(void* handle);
SSAM_API int ssam_cnn_num_params(void* handle, int64_t* count);
/* fp32 parameters / last gradient to host arrays of ssam_cnn_num_params (either may be NULL) */
SSAM_API int ssam_cnn_get_params(void* handle, float* host_params, float* host_grads);
SSAM_API int ssam_cnn_set_params(void* handle, const float* host_params);
/* u0 = network(f): the warm start */
SSAM_API int ssam_cnn_forward(void* handle, const double* f, double* u0, int nbatch,
                              void* stream);
/* forward + backward of the loss against `target`: the mean over right-hand
 * sides of ||u0 - target||^2 / ||target||^2; `loss` (host) receives it.
 * Synchronous. */
SSAM_API int ssam_cnn_gradient(void* handle, const double* f, const double* target, int nbatch,
                               double* loss, void* stream);
/* one Adam step (beta 0.9 / 0.999) with the last gradient */
SSAM_API int ssam_cnn_adam_step(void* handle, float lr, void* stream);
/* weights as a one-line JSON header + float32 blob */
SSAM_API int ssam_cnn_save(void* handle, const char* path);
SSAM_API int ssam_cnn_load(void* handle, const char* path);

/*
 * Synchronises `stream` and reports whether a bounded device-side wait of
 * any kernel on the current device gave up since the last call
 * (SSAM_ERR_TIMEOUT, with the code in the message); clears the flag.
 */
SSAM_API int ssam_device_status(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SSAM_B200_H */
