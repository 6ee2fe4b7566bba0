// Many uneven 2D grids in one persistent launch (ssam_stencil2d_batched).
//
// The reference runs one grid per program invocation.  Here a batch of grids
// of different sizes is stepped by a single cooperative launch sized to the
// SMs: every warp takes warp tiles (a 32*V-column strip x P rows of one grid)
// from the flattened list of all grids' tiles with a grid-wide stride, runs
// the same register-cache systolic tile code as ssam_stencil2d
// (stencil2d_warp_tile), and a grid-wide barrier separates the phases of the
// launch chain (each phase fuses up to TMAX steps in registers).  Buffers
// ping-pong per grid between dst and a slice of one scratch allocation so
// that the last phase lands in dst.
//
// The barrier is a monotonically increasing counter in device memory; the
// wait is bounded by %globaltimer and records an error code on expiry (read
// with ssam_device_status), so a lost CTA cannot hang the GPU.
#include <atomic>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "autotune.h"
#include "stencil2d_stream.cuh"

namespace ssam {

int device_error_word(int** out);
int check_grid2d(const void* src, const void* dst, int64_t w, int64_t h, int64_t pitch,
                 int dtype, int boundary);
int stencil_matrix(int shape, int radius, const double* coeffs, int steps, int boundary,
                   std::vector<double>* out);

// One grid of the batch as the kernel sees it.  in/out of a phase: phase 0
// reads `src` (or the previous launch's result), later phases read what the
// phase before wrote; each phase writes `dst` or `scratch` so that the last
// phase of the whole run lands in dst.
struct BatchGrid {
  const void* first_in;    // input of this launch's first phase
  void* dst;
  void* scratch;
  int64_t w, h, pitch;
  int64_t item0;           // first warp tile of this grid in the flat list
  int32_t nwx;             // warp strips across
  int32_t nby;             // row blocks
  int32_t vec_ok;
};

struct BatchWork {
  const BatchGrid* grids;
  int ngrids;
  int64_t items;           // warp tiles of all grids
  int nphases;             // phases in this launch
  int phases_after;        // phases of the run that follow this launch
  int bnd;
  unsigned* barrier;       // zeroed before the launch
  int* err;
  unsigned long long wait_ns;
  unsigned barrier_extra;  // arrivals a phase waits for beyond the grid's own (0)
};

// Test hook (ssam_debug_batched_barrier): arrivals every grid barrier waits
// for beyond the CTAs of the grid, and its time limit (0 = the default).
static std::atomic<unsigned> g_dbg_extra{0};
static std::atomic<unsigned long long> g_dbg_wait_ns{0};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint64_t gclock() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Grid-wide barrier number `k` (0-based); false if it timed out.
__device__ bool batch_barrier(const BatchWork& w, unsigned k) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    __threadfence();
    atomicAdd(w.barrier, 1u);
    const unsigned target = (k + 1) * (gridDim.x + w.barrier_extra);
    const uint64_t t0 = gclock();
    while (ld_acquire(w.barrier) < target) {
      if (gclock() - t0 > w.wait_ns) {
        atomicCAS(w.err, 0, 4);
        ok = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

template <typename TS, int R, bool STAR, int P, int TT, int V>
__global__ void __launch_bounds__(128)
batched_kernel(BatchWork w, CoefBlock<typename Traits<TS>::TA, (2 * R + 1) * (2 * R + 1)> cf) {
  using C = Stencil2DCfg<TS, R, R, R, R, STAR, P, TT, V>;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int ph = 0; ph < w.nphases; ++ph) {
    // phases left in the whole run after this one decide the output buffer
    const bool out_dst = ((w.nphases - 1 - ph + w.phases_after) % 2) == 0;
    int g = 0;
    for (int64_t it = gw; it < w.items; it += nwarps) {
      // grids are in item order and `it` only grows: advance the grid index
      while (g + 1 < w.ngrids && w.grids[g + 1].item0 <= it) ++g;
      const BatchGrid& bg = w.grids[g];
      const int64_t local = it - bg.item0;
      const int64_t wx = local % bg.nwx, by = local / bg.nwx;
      const TS* in = ph == 0 ? (const TS*)bg.first_in
                             : (const TS*)(out_dst ? bg.scratch : bg.dst);
      TS* out = out_dst ? (TS*)bg.dst : (TS*)bg.scratch;
      stencil2d_warp_tile<TS, R, R, R, R, STAR, P, TT, V>(
          in, out, bg.w, bg.h, bg.pitch, wx * C::OUT_COLS, by * P, bg.h, w.bnd, bg.vec_ok,
          cf);
    }
    if (ph + 1 < w.nphases && !batch_barrier(w, (unsigned)ph)) return;
  }
}

// The same with row-streaming warp tiles (stencil2d_stream.cuh): a work item
// is one SEG-row segment of one warp strip of one grid; single steps only.
// Every grid must have 16-byte aligned buffers and a pitch that is a multiple
// of V (checked by the entry point).
template <typename TS, int R, bool STAR, int SEG, int V, int DF>
__global__ void __launch_bounds__(128)
batched_stream_kernel(BatchWork w,
                      CoefBlock<typename Traits<TS>::TA, (2 * R + 1) * (2 * R + 1)> cf) {
  using C = Stream2DCfg<TS, R, R, R, R, STAR, SEG, V, DF>;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int ph = 0; ph < w.nphases; ++ph) {
    const bool out_dst = ((w.nphases - 1 - ph + w.phases_after) % 2) == 0;
    int g = 0;
    for (int64_t it = gw; it < w.items; it += nwarps) {
      while (g + 1 < w.ngrids && w.grids[g + 1].item0 <= it) ++g;
      const BatchGrid& bg = w.grids[g];
      const int64_t local = it - bg.item0;
      const int64_t wx = local % bg.nwx, sgi = local / bg.nwx;
      const TS* in = ph == 0 ? (const TS*)bg.first_in
                             : (const TS*)(out_dst ? bg.scratch : bg.dst);
      TS* out = out_dst ? (TS*)bg.dst : (TS*)bg.scratch;
      stream2d_warp_segments<TS, R, R, R, R, STAR, SEG, V, true, DF>(
          in, out, bg.w, bg.h, bg.pitch, wx * C::OUT_COLS, 0, bg.h, (int)sgi, 1 << 30, w.bnd,
          cf);
    }
    if (ph + 1 < w.nphases && !batch_barrier(w, (unsigned)ph)) return;
  }
}

struct BatchLaunch {
  std::vector<BatchGrid>* grids;  // host copy; item0/nwx/first_in set here
  int nphases;                    // phases of this launch (all of depth TT)
  int phases_after;               // phases of the run after this launch
  const double* coef;
  int bnd;
  cudaStream_t stream;
};

// STREAM: the row-streaming kernel (P = SEG rows per segment, TT = 1, DF
// rows in flight ahead of the reach).
template <typename TS, int R, bool STAR, int P, int TT, int V, bool STREAM = false, int DF = 4>
static int launch_batched(BatchLaunch& a) {
  using TA = typename Traits<TS>::TA;
  using CW = Stencil2DCfg<TS, R, R, R, R, STAR, P, TT, V>;
  using CS = Stream2DCfg<TS, R, R, R, R, STAR, P, V, DF>;
  constexpr int NC = (2 * R + 1) * (2 * R + 1);
  constexpr int OUT_COLS = STREAM ? CS::OUT_COLS : CW::OUT_COLS;
  constexpr int ROWS = STREAM ? CS::SEGL : P;  // rows of one work item
  static_assert(!STREAM || TT == 1, "streaming tiles take single steps");
  auto kern = [] {
    if constexpr (STREAM) return &batched_stream_kernel<TS, R, STAR, P, V, DF>;
    else return &batched_kernel<TS, R, STAR, P, TT, V>;
  }();
  std::vector<BatchGrid>& grids = *a.grids;
  BatchWork w;
  int64_t acc = 0;
  for (BatchGrid& g : grids) {
    g.nwx = (int32_t)((g.w + OUT_COLS - 1) / OUT_COLS);
    g.nby = (int32_t)((g.h + ROWS - 1) / ROWS);
    g.item0 = acc;
    acc += (int64_t)g.nwx * g.nby;
  }
  w.items = acc;

  // device copy of the descriptors plus the barrier counter (zeroed)
  const size_t gbytes = grids.size() * sizeof(BatchGrid);
  const size_t total = gbytes + 256;
  void* meta = nullptr;
  int st = scratch_alloc(&meta, total, a.stream);
  if (st != SSAM_OK) return st;
  std::vector<unsigned char> host(total, 0);
  memcpy(host.data(), grids.data(), gbytes);
  cudaError_t e = cudaMemcpyAsync(meta, host.data(), total, cudaMemcpyHostToDevice, a.stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(a.stream);  // `host` is a local buffer
  if (e != cudaSuccess) {
    scratch_free(meta, a.stream);
    return fail_cuda(e, "batched descriptors");
  }
  w.grids = (const BatchGrid*)meta;
  w.ngrids = (int)grids.size();
  w.nphases = a.nphases;
  w.phases_after = a.phases_after;
  w.bnd = a.bnd;
  w.barrier = (unsigned*)((char*)meta + gbytes + 128);
  w.wait_ns = 2000ull * 1000ull * 1000ull;  // 2 s; a healthy phase takes microseconds
  w.barrier_extra = g_dbg_extra.load();
  if (g_dbg_wait_ns.load() != 0) w.wait_ns = g_dbg_wait_ns.load();
  st = device_error_word(&w.err);
  if (st != SSAM_OK) {
    scratch_free(meta, a.stream);
    return st;
  }
  CoefBlock<TA, NC> cf;
  for (int k = 0; k < NC; ++k) cf.c[k] = (TA)a.coef[k];

  int dev = 0, sms = 0, bps = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  SSAM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SSAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 128, 0));
  if (bps < 1) {
    scratch_free(meta, a.stream);
    return fail(SSAM_ERR_UNSUPPORTED, "batched kernel does not fit on an SM");
  }
  int64_t grid = std::min<int64_t>((int64_t)sms * bps, (w.items + 3) / 4);
  grid = std::max<int64_t>(grid, 1);
  void* args[] = {&w, &cf};
  e = cudaLaunchCooperativeKernel((const void*)kern, dim3((unsigned)grid), dim3(128), args, 0,
                                  a.stream);
  scratch_free(meta, a.stream);
  if (e != cudaSuccess) return fail_cuda(e, "cooperative batched launch");
  count_launch();
  return SSAM_OK;
}

using BatchFn = int (*)(BatchLaunch&);

// (dtype, star, radius, fused depth) -> persistent kernel.  One depth per
// kernel: compiling several depths into one kernel makes the register
// allocation cover all of them (168 instead of 128 registers at r = 1).
static BatchFn find_batched(int dtype, int star, int r, int t) {
#define SSAM_B(TS, R, ST, TT, V)                                                  \
  if (r == R && star == (ST ? 1 : 0) && t == TT) return &launch_batched<TS, R, ST, 8, TT, V>;
  switch (dtype) {
    case SSAM_F32:
      SSAM_B(float, 1, true, 4, 4) SSAM_B(float, 1, false, 4, 4)
      SSAM_B(float, 1, true, 1, 4) SSAM_B(float, 1, false, 1, 4)
      SSAM_B(float, 2, true, 2, 4) SSAM_B(float, 2, false, 2, 4)
      SSAM_B(float, 2, true, 1, 4) SSAM_B(float, 2, false, 1, 4)
      SSAM_B(float, 3, true, 1, 4) SSAM_B(float, 3, false, 1, 4)
      break;
    case SSAM_F64:
      SSAM_B(double, 1, true, 4, 4) SSAM_B(double, 1, false, 4, 4)
      SSAM_B(double, 1, true, 1, 4) SSAM_B(double, 1, false, 1, 4)
      SSAM_B(double, 2, true, 2, 4) SSAM_B(double, 2, false, 2, 4)
      SSAM_B(double, 2, true, 1, 4) SSAM_B(double, 2, false, 1, 4)
      break;
    case SSAM_BF16:
      SSAM_B(__nv_bfloat16, 1, true, 4, 8) SSAM_B(__nv_bfloat16, 1, false, 4, 8)
      SSAM_B(__nv_bfloat16, 1, true, 1, 8) SSAM_B(__nv_bfloat16, 1, false, 1, 8)
      SSAM_B(__nv_bfloat16, 2, true, 2, 8) SSAM_B(__nv_bfloat16, 2, false, 2, 8)
      SSAM_B(__nv_bfloat16, 2, true, 1, 8) SSAM_B(__nv_bfloat16, 2, false, 1, 8)
      break;
  }
#undef SSAM_B
  return nullptr;
}

// Single-step streaming kernels (SEG = 32) for the same stencils, each with
// 4, 6 or 8 rows in flight a warp (`depth`): X(TS, R, STAR, V) per stencil.
#define SSAM_BATCH_STREAM_LIST(X)                                            \
  switch (dtype) {                                                           \
    case SSAM_F32:                                                           \
      X(float, 1, true, 4) X(float, 1, false, 4) X(float, 2, true, 4)        \
      X(float, 2, false, 4) X(float, 3, true, 4) X(float, 3, false, 4)       \
      break;                                                                 \
    case SSAM_F64:                                                           \
      X(double, 1, true, 4) X(double, 1, false, 4) X(double, 2, true, 4)     \
      X(double, 2, false, 4)                                                 \
      break;                                                                 \
    case SSAM_BF16:                                                          \
      X(__nv_bfloat16, 1, true, 8) X(__nv_bfloat16, 1, false, 8)             \
      X(__nv_bfloat16, 2, true, 8) X(__nv_bfloat16, 2, false, 8)             \
      break;                                                                 \
  }

static BatchFn find_batched_stream(int dtype, int star, int r, int depth) {
#define SSAM_BS(TS, R, ST, V)                                                \
  if (r == R && star == (ST ? 1 : 0)) {                                      \
    if (depth == 4) return &launch_batched<TS, R, ST, 32, 1, V, true, 4>;    \
    if (depth == 6) return &launch_batched<TS, R, ST, 32, 1, V, true, 6>;    \
    if (depth == 8) return &launch_batched<TS, R, ST, 32, 1, V, true, 8>;    \
  }
  SSAM_BATCH_STREAM_LIST(SSAM_BS)
#undef SSAM_BS
  return nullptr;
}

#undef SSAM_BATCH_STREAM_LIST

static int stream_width(int dtype) { return dtype == SSAM_BF16 || dtype == SSAM_F16 ? 8 : 4; }

// Rows in flight a warp for the persistent streaming kernel of this stencil.
// A deeper ring keeps more loads in flight a warp but takes registers, and
// the kernel's register count (so its CTAs a SM) does not follow the depth
// monotonically.  Measured on the 256-grid, 50-step benchmark batches (sides
// log-uniform in [64, 2048]) with depths 4 / 6 / 8: FP32 5x5 box 286 / 320 /
// 294 GCells/s, FP32 5-point 539 / 497 / 549, BF16 5-point 623 / 560 / 526,
// BF16 5x5 box 225 / 196 / 181.  SSAM_BATCH_DEPTH=4|6|8 in the environment
// pins one depth.
static int batched_stream_depth(int dtype, int star, int r) {
  if (const char* e = getenv("SSAM_BATCH_DEPTH")) {
    const int d = atoi(e);
    if (d == 4 || d == 6 || d == 8) return d;
  }
  if (dtype == SSAM_F32 && r == 2 && !star) return 6;
  if (dtype == SSAM_F32 && r == 1 && star) return 8;
  return 4;
}

}  // namespace ssam

using namespace ssam;

extern "C" int ssam_debug_batched_barrier(unsigned extra_arrivals,
                                          unsigned long long wait_ns) {
  if (extra_arrivals > 1024)
    return fail(SSAM_ERR_INVALID, "extra_arrivals above 1024");
  if (wait_ns > 60ull * 1000ull * 1000ull * 1000ull)
    return fail(SSAM_ERR_INVALID, "wait_ns above 60 s");
  g_dbg_extra.store(extra_arrivals);
  g_dbg_wait_ns.store(wait_ns);
  return SSAM_OK;
}

extern "C" int ssam_stencil2d_batched(const ssam_grid2d* grids, int ngrids, int dtype,
                                      int shape, int radius, const double* coeffs, int steps,
                                      int boundary, int mode, void* stream) {
  if (!grids || ngrids < 1) return fail(SSAM_ERR_INVALID, "need at least one grid");
  for (int i = 0; i < ngrids; ++i) {
    int st = check_grid2d(grids[i].src, grids[i].dst, grids[i].width, grids[i].height,
                          grids[i].pitch, dtype, boundary);
    if (st != SSAM_OK) return fail(st, "grid " + std::to_string(i) + ": " + ssam_last_error());
  }
  std::vector<double> m;
  int st = stencil_matrix(shape, radius, coeffs, steps, boundary, &m);
  if (st != SSAM_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (mode == SSAM_BATCH_PER_GRID) {
    for (int i = 0; i < ngrids; ++i) {
      st = ssam_stencil2d(grids[i].src, grids[i].dst, grids[i].width, grids[i].height,
                          grids[i].pitch, dtype, shape, radius, coeffs, steps, boundary,
                          stream);
      if (st != SSAM_OK) return st;
    }
    return SSAM_OK;
  }
  if (mode != SSAM_BATCH_PERSISTENT) return fail(SSAM_ERR_INVALID, "unknown batch mode");
  const int star = shape == SSAM_STAR ? 1 : 0;
  // Launch 1: q phases of the deepest compiled depth (4 at r = 1, 2 at r = 2,
  // 1 above, never deeper than the tuned depth); launch 2: the remaining
  // steps as single-step phases.
  int deep = radius == 1 ? 4 : (radius == 2 ? 2 : 1);
  deep = std::min(deep, std::max(1, tune_depth_2d(dtype, radius, radius, radius, radius, star,
                                                  grids[0].width, grids[0].height, steps)));
  // CLAMP is single-step only; with COPY every fused step of an edge tile
  // reloads the fixed ring from the input, which costs more than it saves on
  // grids this small (most warp tiles touch an edge)
  if (boundary == SSAM_BOUNDARY_CLAMP || boundary == SSAM_BOUNDARY_COPY) deep = 1;
  while (deep > 1 && !find_batched(dtype, star, radius, deep)) deep /= 2;
  const int q = steps / deep, rem = steps % deep;
  BatchFn fn_deep = find_batched(dtype, star, radius, deep);
  BatchFn fn_one = find_batched(dtype, star, radius, 1);
  // single-step phases stream rows when every grid's rows are whole 16-byte
  // chunks of V columns (aligned buffers, pitch a multiple of V)
  bool all_aligned = true;
  for (int i = 0; i < ngrids; ++i)
    all_aligned = all_aligned && (uintptr_t)grids[i].src % 16 == 0 &&
                  (uintptr_t)grids[i].dst % 16 == 0 &&
                  grids[i].pitch % stream_width(dtype) == 0 &&
                  (boundary != SSAM_BOUNDARY_CLAMP || grids[i].width % stream_width(dtype) == 0);
  BatchFn fn_stream =
      all_aligned
          ? find_batched_stream(dtype, star, radius, batched_stream_depth(dtype, star, radius))
          : nullptr;
  if (fn_stream) {
    fn_one = fn_stream;
    if (deep == 1) fn_deep = fn_stream;
  }
  if (!fn_deep || (rem && !fn_one))
    return fail(SSAM_ERR_UNSUPPORTED,
                "no persistent batched kernel for this dtype/shape/radius (use "
                "SSAM_BATCH_PER_GRID)");
  const int nphases = q + rem;
  const size_t es = dtype_size(dtype);
  std::vector<BatchGrid> bg(ngrids);
  size_t scratch_bytes = 0;
  std::vector<size_t> offs(ngrids);
  for (int i = 0; i < ngrids; ++i) {
    offs[i] = scratch_bytes;
    scratch_bytes += ((size_t)(grids[i].pitch * grids[i].height) * es + 255) / 256 * 256;
  }
  void* scratch = nullptr;
  if (nphases > 1) {
    st = scratch_alloc(&scratch, scratch_bytes, s);
    if (st != SSAM_OK) return st;
  }
  for (int i = 0; i < ngrids; ++i) {
    BatchGrid& g = bg[i];
    memset(&g, 0, sizeof g);
    g.first_in = grids[i].src;
    g.dst = grids[i].dst;
    g.scratch = scratch ? (char*)scratch + offs[i] : nullptr;
    g.w = grids[i].width;
    g.h = grids[i].height;
    g.pitch = grids[i].pitch;
    g.vec_ok = ((uintptr_t)g.first_in % 16 == 0) && ((uintptr_t)g.dst % 16 == 0) &&
               (!g.scratch || (uintptr_t)g.scratch % 16 == 0) &&
               ((g.pitch * (int64_t)es) % 16 == 0);
  }
  if (q > 0) {
    BatchLaunch a{&bg, q, rem, m.data(), boundary, s};
    st = fn_deep(a);
  }
  if (st == SSAM_OK && rem > 0) {
    // the deep launch's last phase wrote dst or scratch; continue from there
    if (q > 0) {
      const bool deep_out_dst = (rem % 2) == 0;  // phases_after = rem
      for (int i = 0; i < ngrids; ++i) {
        bg[i].first_in = deep_out_dst ? bg[i].dst : bg[i].scratch;
        // first_in may now be dst, whose alignment was checked above
      }
    }
    BatchLaunch a{&bg, rem, 0, m.data(), boundary, s};
    st = fn_one(a);
  }
  scratch_free(scratch, s);
  return st;
}
