// C ABI of libssam_b200.so: argument checking, kernel choice, multi-step
// chaining and error reporting.  Kernels live in the instantiation units.
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "autotune.h"
#include "ssam_internal.cuh"

namespace ssam {

// ------------------------------------------------------------------ status --

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int fail(int st, const std::string& msg) {
  g_last_error = msg;
  return st;
}

int fail_cuda(cudaError_t e, const char* what) {
  cudaGetLastError();  // do not let a non-sticky error leak into the next call
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                 cudaGetErrorString(e) + ")";
  return SSAM_ERR_CUDA;
}

// ----------------------------------------------------------------- scratch --

// Stream-ordered device scratch comes from one memory pool per device that
// keeps freed blocks mapped (release threshold = max), so repeated calls do
// not pay for mapping and unmapping memory.  ssam_trim_scratch() returns it.
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static cudaError_t pool_for_current_device(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(g_pool_mu);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool;
  e = cudaMemPoolCreate(&pool, &props);
  if (e != cudaSuccess) return e;
  uint64_t keep = ~0ull;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  g_pools[dev] = pool;
  *out = pool;
  return cudaSuccess;
}

int scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool;
  cudaError_t e = pool_for_current_device(&pool);
  if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return fail(SSAM_ERR_NOMEM, "cannot allocate " + std::to_string(bytes) +
                                    " bytes of device scratch: " + cudaGetErrorString(e));
  }
  return SSAM_OK;
}

void scratch_free(void* p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

// ---------------------------------------------------------------- registry --

bool Key2D::operator<(const Key2D& o) const {
  const int a[9] = {dtype, rl, rr, rt, rb, star, p, t, v};
  const int b[9] = {o.dtype, o.rl, o.rr, o.rt, o.rb, o.star, o.p, o.t, o.v};
  return std::lexicographical_compare(a, a + 9, b, b + 9);
}
bool Key2D::operator==(const Key2D& o) const { return !(*this < o) && !(o < *this); }

static std::map<Key2D, Kernel2DInfo>& registry_2d() {
  static std::map<Key2D, Kernel2DInfo> m;
  return m;
}

void register_2d(const Key2D& k, const Kernel2DInfo& info) { registry_2d()[k] = info; }

const Kernel2DInfo* find_2d(const Key2D& k) {
  auto& m = registry_2d();
  auto it = m.find(k);
  return it == m.end() ? nullptr : &it->second;
}

void list_2d(int dtype, int rl, int rr, int rt, int rb, int star,
             void (*cb)(const Key2D&, const Kernel2DInfo&, void*), void* user) {
  for (auto& kv : registry_2d()) {
    const Key2D& k = kv.first;
    if (k.dtype == dtype && k.rl == rl && k.rr == rr && k.rt == rt && k.rb == rb &&
        k.star == star)
      cb(k, kv.second, user);
  }
}

// ------------------------------------------------------------ arg checking --

static bool valid_dtype(int dt) { return dt >= SSAM_F32 && dt <= SSAM_F16; }
static bool valid_boundary(int b) {
  return b == SSAM_BOUNDARY_ZERO || b == SSAM_BOUNDARY_CLAMP || b == SSAM_BOUNDARY_COPY;
}

// The byte ranges [p, p + pitch*(h-1) + w) of two grids overlap.
static bool grids_overlap(const void* a, const void* b, int64_t w, int64_t h,
                          int64_t pitch, size_t es) {
  const uintptr_t pa = (uintptr_t)a, pb = (uintptr_t)b;
  const uintptr_t len = (uintptr_t)((pitch * (h - 1) + w) * (int64_t)es);
  return pa < pb + len && pb < pa + len;
}

int check_grid2d(const void* src, const void* dst, int64_t w, int64_t h,
                        int64_t pitch, int dtype, int boundary) {
  if (!src || !dst) return fail(SSAM_ERR_INVALID, "src and dst must be device pointers");
  if (w < 1 || h < 1) return fail(SSAM_ERR_INVALID, "width and height must be >= 1");
  if (pitch < w) return fail(SSAM_ERR_INVALID, "pitch (elements) must be >= width");
  if (w > (int64_t(1) << 31) || h > (int64_t(1) << 31))
    return fail(SSAM_ERR_INVALID, "width/height above 2^31");
  if (!valid_dtype(dtype)) return fail(SSAM_ERR_INVALID, "unknown dtype");
  if (!valid_boundary(boundary)) return fail(SSAM_ERR_INVALID, "unknown boundary");
  // the grid's byte extent must be representable (pitch is otherwise unbounded)
  uint64_t cells = 0, bytes = 0;
  if (__builtin_mul_overflow((uint64_t)pitch, (uint64_t)h, &cells) ||
      __builtin_mul_overflow(cells, (uint64_t)dtype_size(dtype), &bytes) ||
      bytes > (uint64_t(1) << 62))
    return fail(SSAM_ERR_INVALID, "pitch * height * element size overflows");
  if (grids_overlap(src, dst, w, h, pitch, dtype_size(dtype)))
    return fail(SSAM_ERR_INVALID, "src and dst overlap (updates are out of place)");
  return SSAM_OK;
}

// ------------------------------------------------------------- 2D planning --

// Chooses a compiled kernel for one launch of `t` fused steps.
int pick_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t,
                   int64_t w, int64_t h, Plan2D* out) {
  TuneChoice c;
  if (!tune_lookup_2d(dtype, rl, rr, rt, rb, star, t, w, h, &c)) {
    c = tune_default_2d(dtype, rl, rr, rt, rb, star, t);
  }
  Key2D k{dtype, rl, rr, rt, rb, star, c.p, t, c.v};
  const Kernel2DInfo* info = find_2d(k);
  // otherwise any compiled (P, V) for this shape and depth, default width first
  const int vdef = dtype == SSAM_BF16 || dtype == SSAM_F16 ? 8 : 4;
  for (int v : {vdef, 4, 8, 2, 16}) {
    for (int p : {4, 8, 16, 2, 1}) {
      if (info) break;
      k.p = p;
      k.v = v;
      info = find_2d(k);
    }
  }
  if (!info)
    return fail(SSAM_ERR_UNSUPPORTED,
                "no kernel compiled for this dtype/radius/shape/steps (reach " +
                    std::to_string(rl) + "," + std::to_string(rr) + "," +
                    std::to_string(rt) + "," + std::to_string(rb) + ", star=" +
                    std::to_string(star) + ", fused steps=" + std::to_string(t) + ")");
  out->key = k;
  out->info = info;
  out->warps = c.warps;
  return SSAM_OK;
}

// A kernel fusing `t` steps is compiled for this stencil (any P).
bool have_depth_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t) {
  // bit t of the mask: some kernel fuses t steps (computed once per stencil;
  // the registry is complete before the first call)
  static std::mutex mu;
  static std::map<std::vector<int>, unsigned> masks;
  const std::vector<int> key{dtype, rl, rr, rt, rb, star};
  std::lock_guard<std::mutex> g(mu);
  auto it = masks.find(key);
  if (it == masks.end()) {
    unsigned m = 0;
    list_2d(dtype, rl, rr, rt, rb, star,
            [](const Key2D& k, const Kernel2DInfo&, void* u) {
              if (k.t < 32) *(unsigned*)u |= 1u << k.t;
            },
            &m);
    it = masks.emplace(key, m).first;
  }
  return t >= 0 && t < 32 && (it->second >> t) & 1u;
}

// Runs `steps` steps as a chain of launches of <= the tuned temporal depth,
// ping-ponging between dst and a stream-ordered scratch grid.
static int run_2d(const void* src, void* dst, int64_t w, int64_t h, int64_t pitch,
                  int dtype, int rl, int rr, int rt, int rb, int star,
                  const double* coef, int steps, int boundary, cudaStream_t stream) {
  // temporal depths available for this stencil, largest first
  std::vector<int> depths;
  int tuned = tune_depth_2d(dtype, rl, rr, rt, rb, star, w, h, steps);
  for (int t : {8, 4, 2, 1}) {
    if (t > tuned) continue;
    if (t == 1 || have_depth_2d(dtype, rl, rr, rt, rb, star, t)) depths.push_back(t);
  }
  if (boundary == SSAM_BOUNDARY_CLAMP) depths.assign(1, 1);
  std::vector<int> chain;
  for (int left = steps; left > 0;) {
    for (int t : depths)
      if (t <= left) {
        chain.push_back(t);
        left -= t;
        break;
      }
  }
  const size_t es = dtype_size(dtype);
  void* scratch = nullptr;
  if (chain.size() > 1) {
    int st = scratch_alloc(&scratch, (size_t)(pitch * h) * es, stream);
    if (st != SSAM_OK) return st;
  }
  int st = SSAM_OK;
  const void* in = src;
  for (size_t k = 0; k < chain.size() && st == SSAM_OK; ++k) {
    // the last launch lands in dst, earlier ones alternate with scratch
    void* out = ((chain.size() - 1 - k) % 2 == 0) ? dst : scratch;
    Plan2D p;
    st = pick_2d(dtype, rl, rr, rt, rb, star, chain[k], w, h, &p);
    if (st != SSAM_OK) break;
    Launch2D a{in, out, w, h, pitch, 0, h, boundary, coef, p.warps, stream};
    cudaError_t e = p.info->launch(a);
    if (e != cudaSuccess) st = fail_cuda(e, "stencil2d launch");
    in = out;
  }
  scratch_free(scratch, stream);
  return st;
}

// Dense (2r+1)^2 coefficient matrix from the ABI's STAR or BOX layout, with
// the argument checks shared by the device- and host-buffer entry points.
int stencil_matrix(int shape, int radius, const double* coeffs, int steps,
                          int boundary, std::vector<double>* out) {
  if (shape != SSAM_STAR && shape != SSAM_BOX)
    return fail(SSAM_ERR_INVALID, "shape must be SSAM_STAR or SSAM_BOX");
  const int rmax = shape == SSAM_STAR ? 6 : 10;
  if (radius < 1 || radius > rmax)
    return fail(SSAM_ERR_INVALID, "radius must be in 1.." + std::to_string(rmax) +
                                      " for this shape");
  if (!coeffs) return fail(SSAM_ERR_INVALID, "coeffs must not be NULL");
  if (steps < 1) return fail(SSAM_ERR_INVALID, "steps must be >= 1");
  if (boundary == SSAM_BOUNDARY_CLAMP && steps != 1)
    return fail(SSAM_ERR_INVALID, "CLAMP boundary is single-step only");
  const int f = 2 * radius + 1;
  std::vector<double>& m = *out;
  m.assign((size_t)f * f, 0.0);
  if (shape == SSAM_STAR) {
    // c, then per ring k: n, s, w, e  (stencil2D_25pt.cu:10-16)
    m[radius * f + radius] = coeffs[0];
    for (int k = 1; k <= radius; ++k) {
      const double* q = coeffs + 1 + 4 * (k - 1);
      m[(radius - k) * f + radius] = q[0];  // north: row y-k
      m[(radius + k) * f + radius] = q[1];  // south: row y+k
      m[radius * f + radius - k] = q[2];    // west: column x-k
      m[radius * f + radius + k] = q[3];    // east: column x+k
    }
  } else {
    std::copy(coeffs, coeffs + (size_t)f * f, m.begin());
  }
  return SSAM_OK;
}

// Per-thread copy streams and events for the host-buffer path (created once
// per thread and device, reused by every call on that thread).
struct HostPipe {
  int device = -1;
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t event(size_t i) {
    while (ev.size() <= i) {
      cudaEvent_t e;
      if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
      ev.push_back(e);
    }
    return ev[i];
  }
};

static int host_pipe(HostPipe** out) {
  static thread_local HostPipe pipe;
  int dev = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  if (pipe.device != dev) {
    SSAM_CUDA_TRY(cudaStreamCreateWithFlags(&pipe.h2d, cudaStreamNonBlocking));
    SSAM_CUDA_TRY(cudaStreamCreateWithFlags(&pipe.d2h, cudaStreamNonBlocking));
    pipe.ev.clear();
    pipe.device = dev;
  }
  *out = &pipe;
  return SSAM_OK;
}

// Host-buffer run: the grid is copied in, computed and copied back on the
// caller's stream order.  A single step is pipelined over row bands of about
// 8 MiB -- band k+1 uploads while band k computes and band k-1 downloads --
// so that the copy engines in both directions and the SMs work at once.
static int run_2d_host(const void* h_src, void* h_dst, int64_t w, int64_t h,
                       int64_t pitch, int dtype, int r, int star, const double* coef,
                       int steps, int boundary, cudaStream_t stream) {
  const size_t es = dtype_size(dtype);
  const size_t bytes = (size_t)(pitch * h) * es;
  const size_t row_bytes = (size_t)pitch * es;
  void* d_src = nullptr;
  void* d_dst = nullptr;
  int st = scratch_alloc(&d_src, bytes, stream);
  if (st == SSAM_OK) st = scratch_alloc(&d_dst, bytes, stream);
  if (st != SSAM_OK) {
    scratch_free(d_src, stream);
    return st;
  }
  auto copy_rows = [&](void* dst, const void* src, int64_t y0, int64_t y1,
                       cudaMemcpyKind kind, cudaStream_t s) {
    const size_t off = (size_t)y0 * row_bytes;
    return cudaMemcpy2DAsync((char*)dst + off, row_bytes, (const char*)src + off,
                             row_bytes, (size_t)w * es, (size_t)(y1 - y0), kind, s);
  };
  int64_t band = (int64_t)((8u << 20) / row_bytes);
  band = std::max<int64_t>(16, (band + 15) / 16 * 16);
  const int64_t nb = (h + band - 1) / band;
  if (steps > 1 || nb < 3) {
    cudaError_t e = copy_rows(d_src, h_src, 0, h, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) st = fail_cuda(e, "host-to-device copy");
    if (st == SSAM_OK)
      st = run_2d(d_src, d_dst, w, h, pitch, dtype, r, r, r, r, star, coef, steps,
                  boundary, stream);
    if (st == SSAM_OK) {
      e = copy_rows(h_dst, d_dst, 0, h, cudaMemcpyDeviceToHost, stream);
      if (e != cudaSuccess) st = fail_cuda(e, "device-to-host copy");
    }
  } else {
    HostPipe* p = nullptr;
    st = host_pipe(&p);
    Plan2D plan;
    if (st == SSAM_OK) st = pick_2d(dtype, r, r, r, r, star, 1, w, h, &plan);
    // events: [0] caller start, [1..nb] uploads, [nb+1..2nb] computes, [2nb+1] end
    cudaEvent_t e_start = st == SSAM_OK ? p->event(2 * nb + 1) : nullptr;
    if (st == SSAM_OK && !e_start) st = fail(SSAM_ERR_CUDA, "cudaEventCreate failed");
    if (st == SSAM_OK) {
      cudaError_t e = cudaEventRecord(p->event(0), stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(p->h2d, p->event(0), 0);
      for (int64_t k = 0; k < nb && e == cudaSuccess; ++k) {
        e = copy_rows(d_src, h_src, k * band, std::min(h, (k + 1) * band),
                      cudaMemcpyHostToDevice, p->h2d);
        if (e == cudaSuccess) e = cudaEventRecord(p->event(1 + k), p->h2d);
      }
      for (int64_t k = 0; k < nb && e == cudaSuccess; ++k) {
        // band k reads up to r rows of band k+1 (r <= 16 <= band)
        e = cudaStreamWaitEvent(stream, p->event(1 + std::min(k + 1, nb - 1)), 0);
        if (e != cudaSuccess) break;
        Launch2D a{d_src, d_dst, w, h, pitch, k * band, std::min(h, (k + 1) * band),
                   boundary, coef, plan.warps, stream};
        e = plan.info->launch(a);
        if (e == cudaSuccess) e = cudaEventRecord(p->event(1 + nb + k), stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(p->d2h, p->event(1 + nb + k), 0);
        if (e == cudaSuccess)
          e = copy_rows(h_dst, d_dst, k * band, std::min(h, (k + 1) * band),
                        cudaMemcpyDeviceToHost, p->d2h);
      }
      if (e == cudaSuccess) e = cudaEventRecord(p->event(2 * nb + 1), p->d2h);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, p->event(2 * nb + 1), 0);
      if (e != cudaSuccess) st = fail_cuda(e, "host-buffer pipeline");
    }
  }
  scratch_free(d_src, stream);
  scratch_free(d_dst, stream);
  return st;
}

// Argument checks shared by the 3D entry points and the 3D autotuner.
int check_3d(const void* src, const void* dst, int64_t nx, int64_t ny, int64_t nz,
             int dtype, int shape, int radius, const double* coeffs, int steps,
             int boundary) {
  if (!src || !dst) return fail(SSAM_ERR_INVALID, "src and dst must not be NULL");
  if (nx < 1 || ny < 1 || nz < 1) return fail(SSAM_ERR_INVALID, "nx, ny, nz must be >= 1");
  if (nx > (int64_t(1) << 31) || ny > (int64_t(1) << 31) || nz > (int64_t(1) << 31))
    return fail(SSAM_ERR_INVALID, "grid side above 2^31");
  if (!valid_dtype(dtype)) return fail(SSAM_ERR_INVALID, "unknown dtype");
  if (shape != SSAM_STAR3D && shape != SSAM_POISSON19)
    return fail(SSAM_ERR_INVALID, "shape must be SSAM_STAR3D or SSAM_POISSON19");
  if (radius < 1 || radius > 4 || (shape == SSAM_POISSON19 && radius != 1))
    return fail(SSAM_ERR_INVALID, "radius must be 1..4 (POISSON19: 1)");
  if (!coeffs) return fail(SSAM_ERR_INVALID, "coeffs must not be NULL");
  if (steps < 1) return fail(SSAM_ERR_INVALID, "steps must be >= 1");
  if (boundary != SSAM_BOUNDARY_ZERO && boundary != SSAM_BOUNDARY_COPY)
    return fail(boundary == SSAM_BOUNDARY_CLAMP ? SSAM_ERR_UNSUPPORTED : SSAM_ERR_INVALID,
                "3D boundary must be ZERO or COPY");
  const uintptr_t len = (uintptr_t)(nx * ny * nz) * dtype_size(dtype);
  if ((uintptr_t)src < (uintptr_t)dst + len && (uintptr_t)dst < (uintptr_t)src + len)
    return fail(SSAM_ERR_INVALID, "src and dst overlap (updates are out of place)");
  return SSAM_OK;
}

}  // namespace ssam

using namespace ssam;

extern "C" {

const char* ssam_last_error(void) { return g_last_error.c_str(); }

int ssam_abi_version(void) { return SSAM_ABI_VERSION; }

uint64_t ssam_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int ssam_trim_scratch(void) {
  std::lock_guard<std::mutex> g(g_pool_mu);
  for (auto& kv : g_pools) {
    cudaError_t e = cudaMemPoolTrimTo(kv.second, 0);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMemPoolTrimTo");
  }
  return SSAM_OK;
}

int ssam_stencil2d(const void* src, void* dst, int64_t width, int64_t height,
                   int64_t pitch, int dtype, int shape, int radius,
                   const double* coeffs, int steps, int boundary, void* stream) {
  int st = check_grid2d(src, dst, width, height, pitch, dtype, boundary);
  if (st != SSAM_OK) return st;
  std::vector<double> m;
  st = stencil_matrix(shape, radius, coeffs, steps, boundary, &m);
  if (st != SSAM_OK) return st;
  return run_2d(src, dst, width, height, pitch, dtype, radius, radius, radius,
                radius, shape == SSAM_STAR ? 1 : 0, m.data(), steps, boundary,
                (cudaStream_t)stream);
}

int ssam_stencil2d_host(const void* h_src, void* h_dst, int64_t width, int64_t height,
                        int64_t pitch, int dtype, int shape, int radius,
                        const double* coeffs, int steps, int boundary, void* stream) {
  int st = check_grid2d(h_src, h_dst, width, height, pitch, dtype, boundary);
  if (st != SSAM_OK) return st;
  std::vector<double> m;
  st = stencil_matrix(shape, radius, coeffs, steps, boundary, &m);
  if (st != SSAM_OK) return st;
  return run_2d_host(h_src, h_dst, width, height, pitch, dtype, radius,
                     shape == SSAM_STAR ? 1 : 0, m.data(), steps, boundary,
                     (cudaStream_t)stream);
}

int ssam_stencil3d(const void* src, void* dst, int64_t nx, int64_t ny, int64_t nz,
                   int dtype, int shape, int radius, const double* coeffs, int steps,
                   int boundary, void* stream) {
  int st = check_3d(src, dst, nx, ny, nz, dtype, shape, radius, coeffs, steps, boundary);
  if (st != SSAM_OK) return st;
  return run_3d(src, dst, nx, ny, nz, dtype, shape == SSAM_POISSON19 ? 1 : 0, radius,
                coeffs, steps, boundary, 1, (cudaStream_t)stream);
}

int ssam_stencil3d_host(const void* h_src, void* h_dst, int64_t nx, int64_t ny, int64_t nz,
                        int dtype, int shape, int radius, const double* coeffs, int steps,
                        int boundary, void* stream) {
  int st = check_3d(h_src, h_dst, nx, ny, nz, dtype, shape, radius, coeffs, steps, boundary);
  if (st != SSAM_OK) return st;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)(nx * ny * nz) * dtype_size(dtype);
  void* d_src = nullptr;
  void* d_dst = nullptr;
  st = scratch_alloc(&d_src, bytes, s);
  if (st == SSAM_OK) st = scratch_alloc(&d_dst, bytes, s);
  if (st == SSAM_OK) {
    cudaError_t e = cudaMemcpyAsync(d_src, h_src, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) st = fail_cuda(e, "host-to-device copy");
  }
  // plain launches: the device buffers change from call to call
  if (st == SSAM_OK)
    st = run_3d(d_src, d_dst, nx, ny, nz, dtype, shape == SSAM_POISSON19 ? 1 : 0, radius,
                coeffs, steps, boundary, 0, s);
  if (st == SSAM_OK) {
    cudaError_t e = cudaMemcpyAsync(h_dst, d_dst, bytes, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) st = fail_cuda(e, "device-to-host copy");
  }
  scratch_free(d_src, s);
  scratch_free(d_dst, s);
  return st;
}

int ssam_device_status(void* stream) {
  SSAM_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  int* word = nullptr;
  int st = device_error_word(&word);
  if (st != SSAM_OK) return st;
  int v = 0;
  SSAM_CUDA_TRY(cudaMemcpy(&v, word, sizeof(int), cudaMemcpyDeviceToHost));
  if (v != 0) {
    const int zero = 0;
    SSAM_CUDA_TRY(cudaMemcpy(word, &zero, sizeof(int), cudaMemcpyHostToDevice));
    return fail(SSAM_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(v) +
                                      ": 1 producer/empty, 2 drain, 3 consumer/full)");
  }
  return SSAM_OK;
}

int ssam_conv2d(const void* src, void* dst, int64_t width, int64_t pitch,
                int64_t height, int dtype, const double* weight, int fw, int fh,
                int boundary, void* stream) {
  int st = check_grid2d(src, dst, width, height, pitch, dtype, boundary);
  if (st != SSAM_OK) return st;
  if (!weight) return fail(SSAM_ERR_INVALID, "weight must not be NULL");
  if (fw < 1 || fh < 1 || fw > 28 || fh > 28)
    return fail(SSAM_ERR_INVALID, "filter sizes must be in 1..28");
  // Embed fh x fw into the square F = max(fw, fh) matrix so that tap offsets
  // (n - fh/2, m - fw/2) are kept; F's reach covers both sides for any parity.
  const int f = std::max(fw, fh);
  std::vector<double> m((size_t)f * f, 0.0);
  const int oy = f / 2 - fh / 2, ox = f / 2 - fw / 2;
  for (int n = 0; n < fh; ++n)
    for (int c = 0; c < fw; ++c) m[(size_t)(n + oy) * f + (c + ox)] = weight[n * fw + c];
  const int rl = f / 2, rr = f - 1 - f / 2;
  return run_2d(src, dst, width, height, pitch, dtype, rl, rr, rl, rr, 0, m.data(),
                1, boundary, (cudaStream_t)stream);
}

}  // extern "C"
