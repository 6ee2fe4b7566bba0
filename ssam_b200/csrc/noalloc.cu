// ssam_stencil2d_noalloc: multi-step 2D stencils for callers that cannot
// allocate device memory.
//
// ssam_stencil2d chains temporal blocks through a scratch grid that it takes
// from a stream-ordered memory pool.  Some callers cannot let a library
// allocate: code running inside a memory budget that was fixed up front
// (an embedding runtime that owns every device byte, a plugin host that
// forbids cudaMalloc after start-up), or code that must not hit an
// allocation failure in the middle of a time-critical loop.  This entry
// point gives them the same computation with the scratch grid in a
// fixed-size array that is part of the library image instead.
//
// Rules that follow from that design:
//  * The array below is a file-scope __device__ array of
//    SSAM_NOALLOC_SCRATCH_BYTES.  Every GPU that loads the library holds it
//    until the process exits; grids larger than it are rejected.
//  * Host code cannot use the array's name as a device address (in host code
//    the symbol is a host-side stand-in).  Its device address is looked up
//    with cudaGetSymbolAddress, with the device current, on every call made
//    outside stream capture (so a cudaDeviceReset, which unloads the module,
//    never leaves a stale address behind); a call made while the stream is
//    being captured uses the address found by the last uncaptured call on
//    that device, so the first call on a device should come before any
//    capture.  Under lazy module loading (the CUDA 12 default) the array is
//    reserved when the library's module is first loaded on a device, which
//    can be this first call: it can then fail with an out-of-memory error.
//  * Every call shares the one array, and it keeps the last call's contents.
//    Nothing in it has to start at zero: each launch writes every cell of the
//    grid it produces before the next launch reads it.  Calls that overlap on
//    the GPU (other streams, other host threads) race on the array; callers
//    must serialise them.
#include <mutex>
#include <string>
#include <vector>

#include "autotune.h"
#include "ssam_internal.cuh"

namespace ssam {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SSAM_NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch on the current device: looked up
// afresh unless `capturing` (then the last address found on this device).
static int noalloc_scratch(void** out, bool capturing) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(SSAM_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> g(mu);
  if (capturing && !addr[dev])
    return fail(SSAM_ERR_INVALID,
                "ssam_stencil2d_noalloc: first call on this device is under stream capture");
  if (!capturing) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(no-alloc scratch)");
    addr[dev] = p;
  }
  *out = addr[dev];
  return SSAM_OK;
}

// Argument checks and kernel choice shared with ssam_stencil2d (api.cu).
int check_grid2d(const void* src, const void* dst, int64_t w, int64_t h, int64_t pitch,
                 int dtype, int boundary);
int stencil_matrix(int shape, int radius, const double* coeffs, int steps, int boundary,
                   std::vector<double>* out);
bool have_depth_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t);
int pick_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t, int64_t w,
            int64_t h, Plan2D* out);

}  // namespace ssam

using namespace ssam;

extern "C" int ssam_stencil2d_noalloc(const void* src, void* dst, int64_t width,
                                      int64_t height, int64_t pitch, int dtype, int shape,
                                      int radius, const double* coeffs, int steps,
                                      int boundary, void* stream) {
  int st = check_grid2d(src, dst, width, height, pitch, dtype, boundary);
  if (st != SSAM_OK) return st;
  std::vector<double> m;
  st = stencil_matrix(shape, radius, coeffs, steps, boundary, &m);
  if (st != SSAM_OK) return st;
  const int star = shape == SSAM_STAR ? 1 : 0;
  const int r = radius;
  // the same chain of fused-step launches that ssam_stencil2d runs
  std::vector<int> depths;
  const int tuned = tune_depth_2d(dtype, r, r, r, r, star, width, height, steps);
  for (int t : {8, 4, 2, 1})
    if (t <= tuned && (t == 1 || have_depth_2d(dtype, r, r, r, r, star, t)))
      depths.push_back(t);
  if (boundary == SSAM_BOUNDARY_CLAMP) depths.assign(1, 1);
  std::vector<int> chain;
  for (int left = steps; left > 0;)
    for (int t : depths)
      if (t <= left) {
        chain.push_back(t);
        left -= t;
        break;
      }
  void* scratch = nullptr;
  if (chain.size() > 1) {
    // no overflow: check_grid2d bounded pitch * height * element size
    const size_t need = (size_t)(pitch * height) * dtype_size(dtype);
    if (need > (size_t)SSAM_NOALLOC_SCRATCH_BYTES)
      return fail(SSAM_ERR_INVALID,
                  "grid needs " + std::to_string(need) +
                      " bytes of scratch; ssam_stencil2d_noalloc holds at most " +
                      std::to_string((size_t)SSAM_NOALLOC_SCRATCH_BYTES) +
                      " bytes (pitch * height * element size)");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)stream, &cap);
    if (ce != cudaSuccess) return fail_cuda(ce, "cudaStreamIsCapturing");
    st = noalloc_scratch(&scratch, cap != cudaStreamCaptureStatusNone);
    if (st != SSAM_OK) return st;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const void* in = src;
  for (size_t k = 0; k < chain.size(); ++k) {
    // the last launch lands in dst, earlier ones alternate with the array
    void* out = ((chain.size() - 1 - k) % 2 == 0) ? dst : scratch;
    Plan2D p;
    st = pick_2d(dtype, r, r, r, r, star, chain[k], width, height, &p);
    if (st != SSAM_OK) return st;
    Launch2D a{in, out, width, height, pitch, 0, height, boundary, m.data(), p.warps, s};
    cudaError_t e = p.info->launch(a);
    if (e != cudaSuccess) return fail_cuda(e, "stencil2d launch (no-alloc)");
    in = out;
  }
  return SSAM_OK;
}
