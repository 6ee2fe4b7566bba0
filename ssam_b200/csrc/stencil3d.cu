// Host side of the 3D stencils: tensor maps, persistent work split, the
// compiled (dtype, shape, radius) set, multi-step chaining and CUDA-graph
// capture of timestep loops.
#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "stencil3d.cuh"

namespace ssam {

// Device error word written by bounded waits that gave up (0 = ok).
__device__ int g_ssam_device_error;

int device_error_word(int** out) {
  static std::mutex mu;
  static std::map<int, int*> addr;
  int dev = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto it = addr.find(dev);
  if (it == addr.end()) {
    int* p = nullptr;
    SSAM_CUDA_TRY(cudaGetSymbolAddress((void**)&p, g_ssam_device_error));
    it = addr.emplace(dev, p).first;
  }
  *out = it->second;
  return SSAM_OK;
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

// The driver's tensor-map encoder for other translation units (NULL if the
// driver does not provide it).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() { return encode_fn(); }

template <typename TS> CUtensorMapDataType tma_dtype();
template <> CUtensorMapDataType tma_dtype<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> CUtensorMapDataType tma_dtype<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }
template <> CUtensorMapDataType tma_dtype<__nv_bfloat16>() {
  return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}
template <> CUtensorMapDataType tma_dtype<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }

struct Launch3D {
  const void* src;
  void* dst;
  int64_t nx, ny, nz;
  int nb;              // grids stacked along a 4th axis (1 = plain 3D grid)
  const void* rhs;     // NULL, or out += rhs_scale * rhs
  double rhs_scale;
  const double* coef;  // (2R+1)^3, [dz][dy][dx]
  int boundary;
  cudaStream_t stream;
  bool prepare_only;  // resolve attributes/occupancy/symbols, launch nothing
};

template <typename TS, int SH, int R, int PY, int NW, int S, bool RHS = false>
static int launch_3d(const Launch3D& a) {
  using C = Stencil3DCfg<TS, SH, R, PY, NW, S>;
  using TA = typename C::TA;
  auto kern = stencil3d_kernel<TS, SH, R, PY, NW, S, RHS>;
  if ((a.rhs != nullptr) != RHS)
    return fail(SSAM_ERR_INVALID, "3D kernel instance does not match the right-hand side");
  static std::mutex mu;
  static std::map<int, int> ctas_per_sm;  // per device
  int dev = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  int bps, sms;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = ctas_per_sm.find(dev);
    if (it == ctas_per_sm.end()) {
      SSAM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         C::SMEM));
      int b = 0;
      SSAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, C::THREADS,
                                                                  C::SMEM));
      if (b < 1) return fail(SSAM_ERR_UNSUPPORTED, "3D kernel does not fit on an SM");
      it = ctas_per_sm.emplace(dev, b).first;
    }
    bps = it->second;
  }
  SSAM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  const size_t es = sizeof(TS);
  Work3D w;
  w.nx = a.nx;
  w.ny = a.ny;
  w.nz = a.nz;
  w.nb = a.nb;
  w.rhs = a.rhs;
  w.rhs_scale = a.rhs_scale;
  w.ntx = (int)((a.nx + C::TX - 1) / C::TX);
  w.nty = (int)((a.ny + C::TY - 1) / C::TY);
  // z chunk: minimise (rounds of items) x (chunk + 2R prologue planes)
  const int64_t grid_max = (int64_t)sms * bps;
  const int64_t ntiles = (int64_t)w.ntx * w.nty;
  int64_t best = -1;
  for (int zc : {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512}) {
    if (zc > 2 * a.nz && zc > 8) break;
    const int64_t items = ntiles * ((a.nz + zc - 1) / zc) * a.nb;
    const int64_t rounds = (items + grid_max - 1) / grid_max;
    const int64_t cost = rounds * (std::min<int64_t>(zc, a.nz) + 2 * R);
    if (best < 0 || cost < best) {
      best = cost;
      w.zc = zc;
      w.items = items;
    }
  }
  const int64_t grid = std::min(w.items, grid_max);
  w.boundary = a.boundary;
  w.wait_ns = 1000ull * 1000ull * 1000ull;  // 1 s per wait; healthy waits take microseconds
  int st = device_error_word(&w.err);
  if (st != SSAM_OK) return st;
  if (a.prepare_only) return SSAM_OK;

  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  w.use_tma = ((uintptr_t)a.src % 16 == 0) && ((a.nx * (int64_t)es) % 16 == 0) &&
              a.nx <= (int64_t(1) << 32) && encode_fn() != nullptr;
  if (w.use_tma) {
    cuuint64_t dims[4] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz,
                          (cuuint64_t)a.nb};
    cuuint64_t strides[3] = {(cuuint64_t)(a.nx * es), (cuuint64_t)(a.nx * a.ny * es),
                             (cuuint64_t)(a.nx * a.ny * a.nz * es)};
    cuuint32_t box[4] = {(cuuint32_t)C::XW, (cuuint32_t)C::YW, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode_fn()(&map, tma_dtype<TS>(), 4, const_cast<void*>(a.src), dims,
                             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) w.use_tma = 0;  // fall back to plain loads
  }
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  kern<<<(unsigned)grid, C::THREADS, C::SMEM, a.stream>>>(map, (const TS*)a.src, (TS*)a.dst,
                                                          w, cf);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(a.stream, &cap);
  if (cap == cudaStreamCaptureStatusNone) count_launch();  // graphs count at replay
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

using LaunchFn3D = int (*)(const Launch3D&);

// (dtype, shape, radius) -> kernel.  Tile heights and ring depths keep the
// shared-memory ring at <= ~113 KB so that two CTAs fit on an SM.
static LaunchFn3D find_3d(int dtype, int shape, int r) {
  if (shape == SH3_STAR && r == 1) {
    switch (dtype) {
      case SSAM_F32: return &launch_3d<float, SH3_STAR, 1, 4, 8, 6>;
      case SSAM_F64: return &launch_3d<double, SH3_STAR, 1, 4, 4, 5>;
      case SSAM_BF16: return &launch_3d<__nv_bfloat16, SH3_STAR, 1, 4, 8, 6>;
      case SSAM_F16: return &launch_3d<__half, SH3_STAR, 1, 4, 8, 6>;
    }
  }
  if (shape == SH3_STAR && r == 2) {
    switch (dtype) {
      case SSAM_F32: return &launch_3d<float, SH3_STAR, 2, 4, 4, 8>;
      case SSAM_F64: return &launch_3d<double, SH3_STAR, 2, 4, 4, 6>;
      case SSAM_BF16: return &launch_3d<__nv_bfloat16, SH3_STAR, 2, 4, 4, 8>;
      case SSAM_F16: return &launch_3d<__half, SH3_STAR, 2, 4, 4, 8>;
    }
  }
  if (shape == SH3_POISSON19 && r == 1) {
    switch (dtype) {
      case SSAM_F32: return &launch_3d<float, SH3_POISSON19, 1, 4, 8, 6>;
      case SSAM_F64: return &launch_3d<double, SH3_POISSON19, 1, 4, 4, 5>;
      case SSAM_BF16: return &launch_3d<__nv_bfloat16, SH3_POISSON19, 1, 4, 8, 6>;
      case SSAM_F16: return &launch_3d<__half, SH3_POISSON19, 1, 4, 8, 6>;
    }
  }
  return nullptr;
}

// The 7-point instances with the right-hand-side term (the Jacobi sweep).
static LaunchFn3D find_3d_rhs(int dtype) {
  switch (dtype) {
    case SSAM_F32: return &launch_3d<float, SH3_STAR, 1, 4, 8, 6, true>;
    case SSAM_F64: return &launch_3d<double, SH3_STAR, 1, 4, 4, 5, true>;
    case SSAM_BF16: return &launch_3d<__nv_bfloat16, SH3_STAR, 1, 4, 8, 6, true>;
  }
  return nullptr;
}

// ------------------------------------------------------ multi-step + graphs --

struct GraphKey {
  const void* src;
  void* dst;
  int64_t nx, ny, nz;
  int dtype, shape, r, steps, boundary;
  std::vector<double> coef;
  bool operator<(const GraphKey& o) const {
    return std::tie(src, dst, nx, ny, nz, dtype, shape, r, steps, boundary, coef) <
           std::tie(o.src, o.dst, o.nx, o.ny, o.nz, o.dtype, o.shape, o.r, o.steps,
                    o.boundary, o.coef);
  }
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  void* scratch = nullptr;
  int device = 0;
  uint64_t last_use = 0;
  int launches = 0;
};

// Captures run on a private stream: the caller's stream may be the legacy
// default stream, which cannot be captured.  The graph is then launched on
// the caller's stream.
static cudaError_t capture_stream(cudaStream_t* out) {
  thread_local int dev = -1;
  thread_local cudaStream_t s = nullptr;
  int d = 0;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess) return e;
  if (d != dev) {
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    dev = d;
  }
  *out = s;
  return cudaSuccess;
}

static std::mutex g_graph_mu;
static std::map<GraphKey, GraphEntry> g_graphs;
static uint64_t g_graph_clock = 0;
static const size_t kMaxGraphs = 8;

// Enqueues the launch chain src -> (scratch <-> dst) ... -> dst.
static int enqueue_chain_3d(LaunchFn3D fn, const GraphKey& k, void* scratch,
                            cudaStream_t s) {
  const void* in = k.src;
  for (int i = 0; i < k.steps; ++i) {
    void* out = ((k.steps - 1 - i) % 2 == 0) ? k.dst : scratch;
    Launch3D a{in, out, k.nx, k.ny, k.nz, 1, nullptr, 0.0, k.coef.data(), k.boundary, s, false};
    int st = fn(a);
    if (st != SSAM_OK) return st;
    in = out;
  }
  return SSAM_OK;
}

int run_3d(const void* src, void* dst, int64_t nx, int64_t ny, int64_t nz, int dtype,
           int shape, int r, const double* coef, int steps, int boundary, int use_graph,
           cudaStream_t stream) {
  LaunchFn3D fn = find_3d(dtype, shape, r);
  if (!fn)
    return fail(SSAM_ERR_UNSUPPORTED, "no 3D kernel for this dtype/shape/radius (have: "
                                      "star r=1 (7-pt), star r=2 (13-pt), poisson19)");
  const int f = 2 * r + 1;
  GraphKey k{src, dst, nx, ny, nz, dtype, shape, r, steps, boundary,
             std::vector<double>(coef, coef + f * f * f)};
  if (steps == 1) return enqueue_chain_3d(fn, k, nullptr, stream);

  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SSAM_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  const size_t bytes = (size_t)(nx * ny * nz) * dtype_size(dtype);
  if (!use_graph || cap != cudaStreamCaptureStatusNone) {
    // caller is capturing (or asked for plain launches): enqueue directly
    void* scratch = nullptr;
    int st = scratch_alloc(&scratch, bytes, stream);
    if (st != SSAM_OK) return st;
    st = enqueue_chain_3d(fn, k, scratch, stream);
    scratch_free(scratch, stream);
    return st;
  }
  int dev = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(g_graph_mu);
  auto it = g_graphs.find(k);
  if (it == g_graphs.end() || it->second.device != dev) {
    if (it != g_graphs.end()) {
      cudaGraphExecDestroy(it->second.exec);
      scratch_free(it->second.scratch, stream);
      g_graphs.erase(it);
    }
    if (g_graphs.size() >= kMaxGraphs) {  // evict the least recently used
      auto victim = g_graphs.begin();
      for (auto j = g_graphs.begin(); j != g_graphs.end(); ++j)
        if (j->second.last_use < victim->second.last_use) victim = j;
      cudaGraphExecDestroy(victim->second.exec);
      scratch_free(victim->second.scratch, stream);
      g_graphs.erase(victim);
    }
    GraphEntry e;
    e.device = dev;
    // the scratch grid lives as long as the cached graph; make it usable from
    // any stream the graph is later launched on
    int st = scratch_alloc(&e.scratch, bytes, stream);
    if (st != SSAM_OK) return st;
    SSAM_CUDA_TRY(cudaStreamSynchronize(stream));
    Launch3D prep{k.src, k.dst, k.nx, k.ny, k.nz, 1, nullptr, 0.0, k.coef.data(), k.boundary,
                  stream, true};
    st = fn(prep);
    if (st != SSAM_OK) return st;
    cudaStream_t cs = nullptr;
    SSAM_CUDA_TRY(capture_stream(&cs));
    cudaGraph_t graph = nullptr;
    SSAM_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    st = enqueue_chain_3d(fn, k, e.scratch, cs);
    cudaError_t ce = cudaStreamEndCapture(cs, &graph);
    if (st != SSAM_OK || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      scratch_free(e.scratch, stream);
      return st != SSAM_OK ? st : fail_cuda(ce, "cudaStreamEndCapture");
    }
    ce = cudaGraphInstantiate(&e.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
      scratch_free(e.scratch, stream);
      return fail_cuda(ce, "cudaGraphInstantiate");
    }
    e.launches = steps;
    it = g_graphs.emplace(k, e).first;
  }
  it->second.last_use = ++g_graph_clock;
  SSAM_CUDA_TRY(cudaGraphLaunch(it->second.exec, stream));
  for (int i = 0; i < it->second.launches; ++i) count_launch();
  return SSAM_OK;
}

int drop_graphs_3d() {
  std::lock_guard<std::mutex> g(g_graph_mu);
  for (auto& kv : g_graphs) {
    cudaGraphExecDestroy(kv.second.exec);
    if (kv.second.scratch) cudaFree(kv.second.scratch);
  }
  g_graphs.clear();
  return SSAM_OK;
}

}  // namespace ssam

namespace ssam {

// One launch of the 3D star kernel (r = 1) over `nb` stacked n^3 grids with an
// optional right-hand side: out = stencil(in) + rhs_scale * rhs, zero
// (Dirichlet) boundary.  Used by the Poisson Jacobi sweeps.
int sweep_3d(const void* in, void* out, int64_t n, int nb, int dtype, const double* cube,
             const void* rhs, double rhs_scale, cudaStream_t s) {
  LaunchFn3D fn = rhs ? find_3d_rhs(dtype) : find_3d(dtype, SH3_STAR, 1);
  if (!fn) return fail(SSAM_ERR_UNSUPPORTED, "no 3D 7-point kernel for this dtype");
  Launch3D a{in, out, n, n, n, nb, rhs, rhs_scale, cube, SSAM_BOUNDARY_ZERO, s, false};
  return fn(a);
}

}  // namespace ssam
