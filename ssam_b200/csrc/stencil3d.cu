// Host side of the 3D stencils: the table of compiled configurations, the
// measured choice per grid size (ssam_autotune_stencil3d), multi-step
// chaining and CUDA-graph capture of timestep loops.  The launcher template
// is in stencil3d_launch.cuh; the configurations are instantiated in
// generated units (ssam_b200/build.py).
#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "autotune.h"
#include "stencil3d_launch.cuh"

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


// ------------------------------------------------- configuration table --

using Key3D = std::tuple<int, int, int, int, int>;  // dtype, shape, radius, rhs, steps/launch

static std::map<Key3D, std::vector<Cand3D>>& table_3d() {
  static std::map<Key3D, std::vector<Cand3D>> t;
  return t;
}

void register_3d(int dtype, int shape, int r, bool rhs, const Cand3D& c) {
  table_3d()[Key3D{dtype, shape, r, rhs ? 1 : 0, c.t}].push_back(c);
}

static const std::vector<Cand3D>* cands_3d(int dtype, int shape, int r, bool rhs, int t = 1) {
  auto it = table_3d().find(Key3D{dtype, shape, r, rhs ? 1 : 0, t});
  return it == table_3d().end() || it->second.empty() ? nullptr : &it->second;
}

// Measured choices: (dtype, shape, radius, rhs, log2 nx, log2 ny, log2 nz*nb,
// steps per launch) -> (PY, NW, S, zreg, V); and the measured temporal depth
// (1 or 2 steps a launch) of multi-step runs per (dtype, shape, radius,
// log2 nx, log2 ny, log2 nz).
using Tune3DKey = std::tuple<int, int, int, int, int, int, int, int>;
using Tune3DVal = std::tuple<int, int, int, int, int>;
using Depth3DKey = std::tuple<int, int, int, int, int, int>;
static std::mutex g_tune3_mu;
static std::map<Tune3DKey, Tune3DVal> g_tune3;
static std::map<Depth3DKey, int> g_depth3;

static int log2_floor(int64_t v) {
  int b = 0;
  while (v > 1) {
    v >>= 1;
    ++b;
  }
  return b;
}

static Tune3DKey tune3_key(int dtype, int shape, int r, bool rhs, int64_t nx, int64_t ny,
                           int64_t nzb, int t = 1) {
  return Tune3DKey{dtype, shape, r, rhs ? 1 : 0, log2_floor(nx), log2_floor(ny),
                   log2_floor(nzb), t};
}

static Depth3DKey depth3_key(int dtype, int shape, int r, int64_t nx, int64_t ny, int64_t nz) {
  return Depth3DKey{dtype, shape, r, log2_floor(nx), log2_floor(ny), log2_floor(nz)};
}

// The configuration for one launch of `t` steps: the measured one for this
// size class if any, else the default (NULL if none is compiled).
static const Cand3D* pick_3d(int dtype, int shape, int r, bool rhs, int64_t nx, int64_t ny,
                             int64_t nzb, int t = 1) {
  const std::vector<Cand3D>* cs = cands_3d(dtype, shape, r, rhs, t);
  if (!cs) return nullptr;
  {
    std::lock_guard<std::mutex> g(g_tune3_mu);
    auto it = g_tune3.find(tune3_key(dtype, shape, r, rhs, nx, ny, nzb, t));
    if (it != g_tune3.end())
      for (const Cand3D& c : *cs)
        if (Tune3DVal{c.py, c.nw, c.s, c.zreg, c.v} == it->second) return &c;
  }
  for (const Cand3D& c : *cs)
    if (c.dflt) return &c;
  return &cs->front();
}

// Steps per launch of a multi-step run: the measured depth of the size class
// if any, else 1 (the single-step kernels measured faster per step than the
// two-step ones at 512^3 on a B200; the autotuner decides per size class).
static int depth_3d(int dtype, int shape, int r, int64_t nx, int64_t ny, int64_t nz) {
  {
    std::lock_guard<std::mutex> g(g_tune3_mu);
    auto it = g_depth3.find(depth3_key(dtype, shape, r, nx, ny, nz));
    if (it != g_depth3.end()) return it->second;
  }
  return 1;
}

void tune3d_for_each(void (*cb)(const int key[8], const int val[5], void*), void* user) {
  std::lock_guard<std::mutex> g(g_tune3_mu);
  for (auto& kv : g_tune3) {
    const int k[8] = {std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                      std::get<3>(kv.first), std::get<4>(kv.first), std::get<5>(kv.first),
                      std::get<6>(kv.first), std::get<7>(kv.first)};
    const int v[5] = {std::get<0>(kv.second), std::get<1>(kv.second), std::get<2>(kv.second),
                      std::get<3>(kv.second), std::get<4>(kv.second)};
    cb(k, v, user);
  }
}

void depth3d_for_each(void (*cb)(const int key[6], int depth, void*), void* user) {
  std::lock_guard<std::mutex> g(g_tune3_mu);
  for (auto& kv : g_depth3) {
    const int k[6] = {std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first),
                      std::get<3>(kv.first), std::get<4>(kv.first), std::get<5>(kv.first)};
    cb(k, kv.second, user);
  }
}

void tune3d_store(const int key[8], const int val[5]) {
  std::lock_guard<std::mutex> g(g_tune3_mu);
  g_tune3[Tune3DKey{key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7]}] =
      Tune3DVal{val[0], val[1], val[2], val[3], val[4]};
}

void depth3d_store(const int key[6], int depth) {
  std::lock_guard<std::mutex> g(g_tune3_mu);
  g_depth3[Depth3DKey{key[0], key[1], key[2], key[3], key[4], key[5]}] = depth;
}

void tune3d_clear() {
  std::lock_guard<std::mutex> g(g_tune3_mu);
  g_tune3.clear();
  g_depth3.clear();
}

static const char* kNo3D =
    "no 3D kernel for this dtype/shape/radius (have: star r=1 (7-pt), star r=2 (13-pt), "
    "poisson19)";

// ------------------------------------------------------ multi-step + graphs --

struct GraphKey {
  const void* src;
  void* dst;
  int64_t nx, ny, nz;
  int dtype, shape, r, steps, boundary;
  std::vector<double> coef;
  // the configurations captured (a new measured choice recaptures): fn2 runs
  // two steps a launch (NULL: single steps only), fn1 the remaining step
  LaunchFn3D fn1, fn2;
  bool operator<(const GraphKey& o) const {
    return std::tie(src, dst, nx, ny, nz, dtype, shape, r, steps, boundary, coef, fn1, fn2) <
           std::tie(o.src, o.dst, o.nx, o.ny, o.nz, o.dtype, o.shape, o.r, o.steps,
                    o.boundary, o.coef, o.fn1, o.fn2);
  }
  int launches() const { return fn2 ? steps / 2 + steps % 2 : steps; }
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

// Enqueues the launch chain src -> (scratch <-> dst) ... -> dst: steps/2
// two-step launches of fn2 (when set) and the remaining single steps of fn1.
static int enqueue_chain_3d(const GraphKey& k, void* scratch, cudaStream_t s) {
  const int nl = k.launches();
  const int n2 = k.fn2 ? k.steps / 2 : 0;
  const void* in = k.src;
  for (int i = 0; i < nl; ++i) {
    void* out = ((nl - 1 - i) % 2 == 0) ? k.dst : scratch;
    Launch3D a{in, out, k.nx, k.ny, k.nz, 1, nullptr, 0.0, k.coef.data(), k.boundary, s, false};
    int st = (i < n2 ? k.fn2 : k.fn1)(a);
    if (st != SSAM_OK) return st;
    in = out;
  }
  return SSAM_OK;
}

int run_3d(const void* src, void* dst, int64_t nx, int64_t ny, int64_t nz, int dtype,
           int shape, int r, const double* coef, int steps, int boundary, int use_graph,
           cudaStream_t stream) {
  const Cand3D* c = pick_3d(dtype, shape, r, false, nx, ny, nz);
  if (!c) return fail(SSAM_ERR_UNSUPPORTED, kNo3D);
  LaunchFn3D fn2 = nullptr;
  if (steps >= 2 && depth_3d(dtype, shape, r, nx, ny, nz) == 2) {
    const Cand3D* c2 = pick_3d(dtype, shape, r, false, nx, ny, nz, 2);
    if (c2) fn2 = c2->fn;
  }
  const int f = 2 * r + 1;
  GraphKey k{src, dst, nx, ny, nz, dtype, shape, r, steps, boundary,
             std::vector<double>(coef, coef + f * f * f), c->fn, fn2};
  const int nl = k.launches();
  if (nl == 1) return enqueue_chain_3d(k, nullptr, stream);

  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  SSAM_CUDA_TRY(cudaStreamIsCapturing(stream, &cap));
  const size_t bytes = (size_t)(nx * ny * nz) * dtype_size(dtype);
  if (!use_graph || cap != cudaStreamCaptureStatusNone) {
    // caller is capturing (or asked for plain launches): enqueue directly
    void* scratch = nullptr;
    int st = scratch_alloc(&scratch, bytes, stream);
    if (st != SSAM_OK) return st;
    st = enqueue_chain_3d(k, scratch, stream);
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
    for (LaunchFn3D fn : {k.fn1, k.fn2}) {
      if (!fn) continue;
      Launch3D prep{k.src, k.dst, k.nx, k.ny, k.nz, 1, nullptr, 0.0, k.coef.data(), k.boundary,
                    stream, true};
      st = fn(prep);
      if (st != SSAM_OK) return st;
    }
    cudaStream_t cs = nullptr;
    SSAM_CUDA_TRY(capture_stream(&cs));
    cudaGraph_t graph = nullptr;
    SSAM_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    st = enqueue_chain_3d(k, e.scratch, cs);
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
    e.launches = nl;
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
  const Cand3D* c = pick_3d(dtype, SH3_STAR, 1, rhs != nullptr, n, n, n * nb);
  if (!c) return fail(SSAM_ERR_UNSUPPORTED, "no 3D 7-point kernel for this dtype");
  Launch3D a{in, out, n, n, n, nb, rhs, rhs_scale, cube, SSAM_BOUNDARY_ZERO, s, false};
  return c->fn(a);
}

}  // namespace ssam

// ------------------------------------------------------------ autotuner --

namespace ssam {

int check_3d(const void* src, const void* dst, int64_t nx, int64_t ny, int64_t nz,
             int dtype, int shape, int radius, const double* coeffs, int steps,
             int boundary);

// Mean time (ms) of one launch of `c`, after one untimed launch; repetitions
// cover about 3 ms.
static int time_3d(const Cand3D& c, const Launch3D& a, cudaEvent_t e0, cudaEvent_t e1,
                   double* ms_out) {
  int st = c.fn(a);
  if (st != SSAM_OK) return st;
  SSAM_CUDA_TRY(cudaEventRecord(e0, a.stream));
  st = c.fn(a);
  if (st != SSAM_OK) return st;
  SSAM_CUDA_TRY(cudaEventRecord(e1, a.stream));
  SSAM_CUDA_TRY(cudaEventSynchronize(e1));
  float one = 0.f;
  SSAM_CUDA_TRY(cudaEventElapsedTime(&one, e0, e1));
  int reps = one > 0.f ? (int)(3.0f / one) : 20;
  reps = reps < 2 ? 2 : (reps > 20 ? 20 : reps);
  SSAM_CUDA_TRY(cudaEventRecord(e0, a.stream));
  for (int i = 0; i < reps; ++i) {
    st = c.fn(a);
    if (st != SSAM_OK) return st;
  }
  SSAM_CUDA_TRY(cudaEventRecord(e1, a.stream));
  SSAM_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  SSAM_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  *ms_out = ms / reps;
  return SSAM_OK;
}

// Times every configuration in `cs` with launch `a` (its fn ignored) and
// stores the fastest under `key`; *best / *best_ms / *timed describe it.
static int tune_3d(const std::vector<Cand3D>& cs, const Launch3D& a, const Tune3DKey& key,
                   const Cand3D** best_out, double* best_ms_out, int* timed_out) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  SSAM_CUDA_TRY(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail_cuda(ce, "cudaEventCreate");
  }
  int st = SSAM_OK, timed = 0;
  const Cand3D* best = nullptr;
  double best_ms = 0;
  for (const Cand3D& c : cs) {
    double ms = 0;
    st = time_3d(c, a, e0, e1, &ms);
    if (st != SSAM_OK) break;
    ++timed;
    if (!best || ms < best_ms) {
      best = &c;
      best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != SSAM_OK) return st;
  int* err = nullptr;
  st = device_error_word(&err);
  if (st != SSAM_OK) return st;
  int code = 0;
  SSAM_CUDA_TRY(cudaMemcpy(&code, err, sizeof(int), cudaMemcpyDeviceToHost));
  if (code != 0)
    return fail(SSAM_ERR_TIMEOUT, "a 3D kernel gave up waiting while being timed (code " +
                                     std::to_string(code) + ")");
  {
    std::lock_guard<std::mutex> g(g_tune3_mu);
    g_tune3[key] = Tune3DVal{best->py, best->nw, best->s, best->zreg, best->v};
  }
  *best_out = best;
  *best_ms_out = best_ms;
  *timed_out = timed;
  return SSAM_OK;
}

static void fill_report(ssam_tune3d_report* report, const Cand3D* c, double ms_per_step,
                        int timed) {
  if (!report) return;
  report->rows_per_warp = c->py;
  report->consumer_warps = c->nw;
  report->ring_slots = c->s;
  report->registers_z = c->zreg;
  report->columns_per_thread = c->v;
  report->candidates = timed;
  report->ms_per_step = ms_per_step;
  report->fused_steps = c->t;
}

}  // namespace ssam

using namespace ssam;

extern "C" int ssam_autotune_stencil3d(const void* src, void* dst, int64_t nx, int64_t ny,
                                       int64_t nz, int dtype, int shape, int radius,
                                       const double* coeffs, int boundary, void* stream,
                                       ssam_tune3d_report* report) {
  int st = check_3d(src, dst, nx, ny, nz, dtype, shape, radius, coeffs, 1, boundary);
  if (st != SSAM_OK) return st;
  const int sh = shape == SSAM_POISSON19 ? SH3_POISSON19 : SH3_STAR;
  const std::vector<Cand3D>* cs = cands_3d(dtype, sh, radius, false);
  if (!cs) return fail(SSAM_ERR_UNSUPPORTED, kNo3D);
  Launch3D a{src, dst, nx, ny, nz, 1, nullptr, 0.0, coeffs, boundary, (cudaStream_t)stream,
             false};
  const Cand3D* b1 = nullptr;
  double ms1 = 0;
  int n1 = 0;
  st = tune_3d(*cs, a, tune3_key(dtype, sh, radius, false, nx, ny, nz), &b1, &ms1, &n1);
  if (st != SSAM_OK) return st;
  // two steps a launch, kept when its time per step beats one step a launch
  int depth = 1;
  const Cand3D* best = b1;
  double ms = ms1;
  int timed = n1;
  const std::vector<Cand3D>* cs2 = cands_3d(dtype, sh, radius, false, 2);
  if (cs2) {
    const Cand3D* b2 = nullptr;
    double ms2 = 0;
    int n2 = 0;
    st = tune_3d(*cs2, a, tune3_key(dtype, sh, radius, false, nx, ny, nz, 2), &b2, &ms2, &n2);
    if (st != SSAM_OK) return st;
    timed += n2;
    if (ms2 / 2 < ms1) {
      depth = 2;
      best = b2;
      ms = ms2 / 2;
    }
  }
  const Depth3DKey dk = depth3_key(dtype, sh, radius, nx, ny, nz);
  {
    std::lock_guard<std::mutex> g(g_tune3_mu);
    g_depth3[dk] = depth;
  }
  fill_report(report, best, ms, timed);
  return SSAM_OK;
}

extern "C" int ssam_autotune_jacobi3d(int64_t n, int nbatch, int sweep_dtype, void* stream,
                                      ssam_tune3d_report* report) {
  if (n < 1 || nbatch < 1) return fail(SSAM_ERR_INVALID, "n and nbatch must be >= 1");
  if (n > 4096) return fail(SSAM_ERR_INVALID, "n above 4096");
  if (sweep_dtype != SSAM_F32 && sweep_dtype != SSAM_BF16)
    return fail(SSAM_ERR_INVALID, "sweep_dtype must be SSAM_F32 or SSAM_BF16");
  const std::vector<Cand3D>* cs = cands_3d(sweep_dtype, SH3_STAR, 1, true);
  if (!cs) return fail(SSAM_ERR_UNSUPPORTED, "no Jacobi sweep kernel for this dtype");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)(n * n * n) * (size_t)nbatch * dtype_size(sweep_dtype);
  void* buf[3] = {nullptr, nullptr, nullptr};
  int st = SSAM_OK;
  for (int i = 0; i < 3 && st == SSAM_OK; ++i) {
    st = scratch_alloc(&buf[i], bytes, s);
    if (st == SSAM_OK) {
      cudaError_t e = cudaMemsetAsync(buf[i], 0, bytes, s);
      if (e != cudaSuccess) st = fail_cuda(e, "cudaMemsetAsync");
    }
  }
  if (st == SSAM_OK) {
    // the sweep's operator: centre 0, neighbours 1/6 (values do not change the time)
    double cube[27] = {0};
    for (int k : {4, 10, 12, 14, 16, 22}) cube[k] = 1.0 / 6.0;
    Launch3D a{buf[0], buf[1], n, n, n, nbatch, buf[2], 1.0 / 6.0, cube, SSAM_BOUNDARY_ZERO,
               s, false};
    const Cand3D* best = nullptr;
    double ms = 0;
    int timed = 0;
    st = tune_3d(*cs, a, tune3_key(sweep_dtype, SH3_STAR, 1, true, n, n, n * nbatch), &best,
                 &ms, &timed);
    if (st == SSAM_OK) fill_report(report, best, ms, timed);
  }
  for (int i = 0; i < 3; ++i) scratch_free(buf[i], s);
  return st;
}
