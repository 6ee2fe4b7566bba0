// Poisson solver for -lap(u) = f on the unit cube, Dirichlet u = 0, 7-point
// operator on n^3 interior points (h = 1/(n+1)), a batch of right-hand sides.
//
// No reference code exists for this solver (the reference's "poisson" is a
// single 19-point operator sweep, tmpPoisson.cu).  It is built from the
// reference's 7-point stencil structure (v2::j3d7pt_gold,
// tmp3d7pt-v2.cu:281-297) and the mathematics:
//
//   Jacobi sweep:      u <- (sum of the 6 neighbours of u + h^2 f) / 6
//   FP64 residual:     r = f - A u,  A u = (6 u - sum of neighbours) / h^2
//   defect correction: repeat { r = f - A u (FP64, norms per grid);
//                               stop when ||r||/||f|| <= tol for every grid;
//                               e ~= A^-1 r by k low-precision Jacobi sweeps
//                               from e = 0 (FP32 or BF16 storage, FP32
//                               arithmetic, the TMA z-marching stencil kernel);
//                               u += e (FP64) }
//
// The low-precision sweeps are where the time goes; they run on the batch as
// one 4D grid (grids stacked along a 4th axis, zero-filled across grid edges
// by the tensor map).  Each correction's sweep chain is captured once into a
// CUDA graph and replayed.
#include <math.h>

#include <algorithm>
#include <string>
#include <vector>

#include "ssam_internal.cuh"

namespace ssam {

namespace {

constexpr int kResidualThreads = 256;

template <typename TS>
__global__ void __launch_bounds__(kResidualThreads)
residual_kernel(const double* __restrict__ u, const double* __restrict__ f, TS* __restrict__ r_lp,
                double* __restrict__ r64, double* __restrict__ partials, int n, double inv_h2) {
  const int b = blockIdx.y;
  const int64_t n3 = (int64_t)n * n * n, nn = (int64_t)n * n;
  const double* ub = u + b * n3;
  const double* fb = f + b * n3;
  double rr = 0.0, ff = 0.0;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n3;
       c += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(c % n), y = (int)((c / n) % n), z = (int)(c / nn);
    const double uc = ub[c];
    double nb = 0.0;
    if (x > 0) nb += ub[c - 1];
    if (x < n - 1) nb += ub[c + 1];
    if (y > 0) nb += ub[c - n];
    if (y < n - 1) nb += ub[c + n];
    if (z > 0) nb += ub[c - nn];
    if (z < n - 1) nb += ub[c + nn];
    const double fc = fb[c];
    const double r = fc - (6.0 * uc - nb) * inv_h2;
    if (r_lp) r_lp[b * n3 + c] = from_acc<TS>((typename Traits<TS>::TA)r);
    if (r64) r64[b * n3 + c] = r;
    rr += r * r;
    ff += fc * fc;
  }
  // block reduction in double, fixed order (deterministic)
  __shared__ double s_rr[kResidualThreads / 32], s_ff[kResidualThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    rr += __shfl_down_sync(0xffffffffu, rr, o);
    ff += __shfl_down_sync(0xffffffffu, ff, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_rr[threadIdx.x >> 5] = rr;
    s_ff[threadIdx.x >> 5] = ff;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, c = 0.0;
    for (int w = 0; w < kResidualThreads / 32; ++w) {
      a += s_rr[w];
      c += s_ff[w];
    }
    partials[2 * ((int64_t)b * gridDim.x + blockIdx.x)] = a;
    partials[2 * ((int64_t)b * gridDim.x + blockIdx.x) + 1] = c;
  }
}

__global__ void norms_kernel(const double* __restrict__ partials, int blocks, int nb,
                             double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double a = 0.0, c = 0.0;
  for (int k = 0; k < blocks; ++k) {
    a += partials[2 * ((int64_t)b * blocks + k)];
    c += partials[2 * ((int64_t)b * blocks + k) + 1];
  }
  out[2 * b] = a;
  out[2 * b + 1] = c;
}

template <typename TS>
__global__ void add_correction_kernel(double* __restrict__ u, const TS* __restrict__ e,
                                      int64_t count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    u[i] += (double)to_acc(e[i]);
}

__global__ void axpy_kernel(double* __restrict__ u, const double* __restrict__ c, double a,
                            int64_t count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x)
    u[i] += a * c[i];
}

int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

// ||f - A u|| and ||f|| per grid (squared sums written to host `norms2`,
// 2 per grid); optionally r in low precision.  Synchronises the stream.
static int residual(const double* f, const double* u, void* r_lp, int lp_dtype, int n, int nb,
                    double* partials, int blocks, double* d_norms, double* norms2,
                    cudaStream_t s, double* r64 = nullptr) {
  const double h = 1.0 / (n + 1);
  dim3 grid(blocks, nb);
  if (lp_dtype == SSAM_BF16)
    residual_kernel<__nv_bfloat16><<<grid, kResidualThreads, 0, s>>>(
        u, f, (__nv_bfloat16*)r_lp, r64, partials, n, 1.0 / (h * h));
  else
    residual_kernel<float><<<grid, kResidualThreads, 0, s>>>(u, f, (float*)r_lp, r64, partials,
                                                             n, 1.0 / (h * h));
  count_launch();
  norms_kernel<<<(nb + 127) / 128, 128, 0, s>>>(partials, blocks, nb, d_norms);
  count_launch();
  SSAM_CUDA_TRY(cudaGetLastError());
  SSAM_CUDA_TRY(cudaMemcpyAsync(norms2, d_norms, sizeof(double) * 2 * nb,
                                cudaMemcpyDeviceToHost, s));
  SSAM_CUDA_TRY(cudaStreamSynchronize(s));
  return SSAM_OK;
}

// The (damped) Jacobi coefficient cube: neighbours omega/6, centre 1-omega.
static void jacobi_cube(double* cube, double omega = 1.0) {
  for (int i = 0; i < 27; ++i) cube[i] = 0.0;
  cube[13] = 1.0 - omega;
  const double w = omega / 6.0;
  cube[0 * 9 + 1 * 3 + 1] = cube[2 * 9 + 1 * 3 + 1] = w;
  cube[1 * 9 + 0 * 3 + 1] = cube[1 * 9 + 2 * 3 + 1] = w;
  cube[1 * 9 + 1 * 3 + 0] = cube[1 * 9 + 1 * 3 + 2] = w;
}

// `sweeps` Jacobi sweeps u <- (1-omega) u + omega (nbrs(u) + h^2 rhs) / 6
// from u_in; the result is in u_out.  `tmp` is a second grid for the
// ping-pong (may alias nothing).
static int jacobi_chain(const void* rhs, const void* u_in, void* u_out, void* tmp, int n, int nb,
                        int dtype, int sweeps, cudaStream_t s, double omega = 1.0) {
  double cube[27];
  jacobi_cube(cube, omega);
  const double h = 1.0 / (n + 1);
  const void* in = u_in;
  for (int k = 0; k < sweeps; ++k) {
    void* out = ((sweeps - 1 - k) % 2 == 0) ? u_out : tmp;
    int st = sweep_3d(in, out, n, nb, dtype, cube, rhs, omega * h * h / 6.0, s);
    if (st != SSAM_OK) return st;
    in = out;
  }
  return SSAM_OK;
}

}  // namespace ssam

using namespace ssam;

extern "C" int ssam_poisson_jacobi(const void* rhs, const void* u_in, void* u_out, int n,
                                   int nbatch, int dtype, int sweeps, void* stream) {
  if (!rhs || !u_in || !u_out) return fail(SSAM_ERR_INVALID, "NULL grid pointer");
  if (n < 1 || nbatch < 1 || sweeps < 0) return fail(SSAM_ERR_INVALID, "bad n/nbatch/sweeps");
  if (dtype != SSAM_F32 && dtype != SSAM_BF16 && dtype != SSAM_F64)
    return fail(SSAM_ERR_INVALID, "Jacobi sweeps run in F32, BF16 or F64 storage");
  if (u_in == u_out && sweeps > 0) return fail(SSAM_ERR_INVALID, "u_in and u_out must differ");
  cudaStream_t s = (cudaStream_t)stream;
  const size_t bytes = (size_t)n * n * n * nbatch * dtype_size(dtype);
  if (sweeps == 0) {
    SSAM_CUDA_TRY(cudaMemcpyAsync(u_out, u_in, bytes, cudaMemcpyDeviceToDevice, s));
    return SSAM_OK;
  }
  void* tmp = nullptr;
  if (sweeps > 1) {
    int st = scratch_alloc(&tmp, bytes, s);
    if (st != SSAM_OK) return st;
  }
  int st = jacobi_chain(rhs, u_in, u_out, tmp, n, nbatch, dtype, sweeps, s);
  scratch_free(tmp, s);
  return st;
}

extern "C" int ssam_poisson_residual(const double* f, const double* u, int n, int nbatch,
                                     double* rel, void* stream) {
  if (!f || !u || !rel) return fail(SSAM_ERR_INVALID, "NULL pointer");
  if (n < 1 || nbatch < 1) return fail(SSAM_ERR_INVALID, "bad n/nbatch");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = std::max(1, sm_count() * 4 / nbatch);
  void* work = nullptr;
  const size_t pbytes = sizeof(double) * 2 * ((size_t)blocks * nbatch + nbatch);
  int st = scratch_alloc(&work, pbytes, s);
  if (st != SSAM_OK) return st;
  std::vector<double> norms2(2 * nbatch);
  double* partials = (double*)work;
  st = residual(f, u, nullptr, SSAM_F32, n, nbatch, partials, blocks,
                partials + 2 * (size_t)blocks * nbatch, norms2.data(), s);
  scratch_free(work, s);
  if (st != SSAM_OK) return st;
  for (int b = 0; b < nbatch; ++b)
    rel[b] = norms2[2 * b + 1] > 0 ? sqrt(norms2[2 * b] / norms2[2 * b + 1]) : sqrt(norms2[2 * b]);
  return SSAM_OK;
}

namespace ssam {
int cnn_check(void* cnn, int n, int nbatch);
int cnn_apply(void* cnn, const double* r, double* c, int nbatch, cudaStream_t s);
}

// `passes` applications of the 7-point average (centre 1/2, neighbours 1/12,
// zero outside) to buf, ping-ponging with tmp; *out is where the result is.
// It passes the smooth part of a field and removes its highest frequencies
// (the sine mode with eigenvalue lambda of -lap is scaled by 1 - lambda h^2/12).
static int smooth_f64(double* buf, double* tmp, int n, int nb, int passes, const double** out,
                      cudaStream_t s) {
  double cube[27] = {0};
  cube[13] = 0.5;
  for (int k : {4, 10, 12, 14, 16, 22}) cube[k] = 1.0 / 12.0;
  double* in = buf;
  double* o = tmp;
  for (int i = 0; i < passes; ++i) {
    const int st = sweep_3d(in, o, n, nb, SSAM_F64, cube, nullptr, 0.0, s);
    if (st != SSAM_OK) return st;
    std::swap(in, o);
  }
  *out = in;
  return SSAM_OK;
}

// Defect-correction solve; with `cnn`, every correction first adds the
// network's approximate solve of A c = r to u in FP64, then runs the
// low-precision sweeps on the new residual.  A network cycle is kept when the
// next residual is below 0.9 times the one before it; otherwise u is restored
// and the network is not used again in this solve.
static int poisson_solve(const double* f, double* u, int n, int nbatch,
                         const ssam_poisson_options* opt, void* cnn, ssam_poisson_stats* stats,
                         cudaStream_t stream) {
  if (!f || !u || !opt) return fail(SSAM_ERR_INVALID, "NULL pointer");
  if (n < 1 || nbatch < 1) return fail(SSAM_ERR_INVALID, "bad n/nbatch");
  if (opt->sweep_dtype != SSAM_F32 && opt->sweep_dtype != SSAM_BF16)
    return fail(SSAM_ERR_INVALID, "sweep_dtype must be SSAM_F32 or SSAM_BF16");
  if (opt->sweeps_per_correction < 1 || opt->max_sweeps < 0 || !(opt->tol > 0))
    return fail(SSAM_ERR_INVALID, "bad tol / sweeps_per_correction / max_sweeps");
  const double omega = opt->omega == 0.0 ? 1.0 : opt->omega;
  if (!(omega > 0.0 && omega <= 1.0)) return fail(SSAM_ERR_INVALID, "omega must be in (0, 1]");
  if (cnn) {
    const int cs = cnn_check(cnn, n, nbatch);
    if (cs != SSAM_OK) return cs;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int dt = opt->sweep_dtype;
  const size_t cells = (size_t)n * n * n * nbatch;
  const size_t lp = cells * dtype_size(dt);
  const int blocks = std::max(1, sm_count() * 4 / nbatch);
  const size_t pbytes = sizeof(double) * 2 * ((size_t)blocks * nbatch + nbatch);
  // one allocation: r (low precision), e and its ping-pong partner, partial sums
  const size_t lp_al = (lp + 255) / 256 * 256;
  const size_t f64_al = (cells * sizeof(double) + 255) / 256 * 256;
  void* work = nullptr;
  int st = scratch_alloc(&work, 3 * lp_al + pbytes + (cnn ? 4 * f64_al : 0), s);
  if (st != SSAM_OK) return st;
  char* w8 = (char*)work;
  void* r_lp = w8;
  void* e = w8 + lp_al;
  void* e_tmp = w8 + 2 * lp_al;
  double* partials = (double*)(w8 + 3 * lp_al);
  double* d_norms = partials + 2 * (size_t)blocks * nbatch;
  // the learned solve: r in FP64 (network input), the network's correction,
  // and u before the last network cycle (restored if that cycle did not pay)
  double* r64 = cnn ? (double*)(w8 + 3 * lp_al + pbytes) : nullptr;
  double* c64 = cnn ? (double*)(w8 + 3 * lp_al + pbytes + f64_al) : nullptr;
  double* u_save = cnn ? (double*)(w8 + 3 * lp_al + pbytes + 2 * f64_al) : nullptr;
  double* tmp64 = cnn ? (double*)(w8 + 3 * lp_al + pbytes + 3 * f64_al) : nullptr;
  const int passes = std::max(0, opt->cnn_smoothing);
  std::vector<double> norms2(2 * nbatch);
  bool use_cnn = cnn != nullptr;
  bool first = true;
  bool cnn_on_trial = false;  // the last cycle used the network
  double before_cnn = 0.0;

  ssam_poisson_stats local = {};
  ssam_poisson_stats* out = stats ? stats : &local;
  *out = ssam_poisson_stats{};
  double worst = 0.0;
  cudaGraphExec_t chain = nullptr;
  const size_t nthreads = 256;
  const int cblocks = (int)std::min<size_t>((cells + nthreads - 1) / nthreads, 148 * 16);
  auto worst_rel = [&]() {
    double m = 0.0;
    for (int b = 0; b < nbatch; ++b)
      m = std::max(m, norms2[2 * b + 1] > 0 ? sqrt(norms2[2 * b] / norms2[2 * b + 1]) : 0.0);
    return m;
  };
  while (true) {
    st = residual(f, u, r_lp, dt, n, nbatch, partials, blocks, d_norms, norms2.data(), s,
                  use_cnn ? r64 : nullptr);
    if (st != SSAM_OK) break;
    worst = worst_rel();
    if (first) {
      first = false;
      out->initial_rel_residual = worst;
      if (cnn && worst > 1.0) {
        // the initial guess is worse than no guess at all: start from u = 0
        cudaError_t ce = cudaMemsetAsync(u, 0, cells * sizeof(double), s);
        if (ce != cudaSuccess) {
          st = fail_cuda(ce, "cudaMemsetAsync(u)");
          break;
        }
        out->fell_back = 1;
        first = true;
        continue;
      }
    }
    if (cnn_on_trial) {
      cnn_on_trial = false;
      if (worst < 0.9 * before_cnn) {
        out->cnn_corrections += 1;
      } else {
        // the network's cycle did not lower the residual enough: undo it and
        // go on with plain cycles
        use_cnn = false;
        cudaError_t ce =
            cudaMemcpyAsync(u, u_save, cells * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (ce != cudaSuccess) {
          st = fail_cuda(ce, "restoring u");
          break;
        }
        st = residual(f, u, r_lp, dt, n, nbatch, partials, blocks, d_norms, norms2.data(), s);
        if (st != SSAM_OK) break;
        worst = worst_rel();
      }
    }
    out->rel_residual = worst;
    if (worst <= opt->tol) {
      out->converged = 1;
      break;
    }
    if (out->sweeps >= opt->max_sweeps) break;
    if (use_cnn) {
      // u += network(r), then the sweeps below smooth what the network left
      cudaError_t ce =
          cudaMemcpyAsync(u_save, u, cells * sizeof(double), cudaMemcpyDeviceToDevice, s);
      if (ce != cudaSuccess) {
        st = fail_cuda(ce, "saving u");
        break;
      }
      before_cnn = worst;
      cnn_on_trial = true;
      // the network sees the smooth part of r, and its BF16 noise is
      // filtered out of the correction (the sweeps handle the rest)
      const double* cin = r64;
      st = smooth_f64(r64, tmp64, n, nbatch, passes, &cin, s);
      if (st == SSAM_OK) st = cnn_apply(cnn, cin, c64, nbatch, s);
      const double* cout = c64;
      if (st == SSAM_OK) st = smooth_f64(c64, tmp64, n, nbatch, passes, &cout, s);
      if (st != SSAM_OK) break;
      axpy_kernel<<<cblocks, nthreads, 0, s>>>(u, cout, 1.0, (int64_t)cells);
      count_launch();
      st = residual(f, u, r_lp, dt, n, nbatch, partials, blocks, d_norms, norms2.data(), s);
      if (st != SSAM_OK) break;
    }
    const int k = std::min(opt->sweeps_per_correction, opt->max_sweeps - out->sweeps);
    // e = k Jacobi sweeps on A e = r from e = 0; the chain (memset + k sweeps)
    // is captured once and replayed for every correction of this size
    if (!chain || k != opt->sweeps_per_correction) {
      if (chain) {
        cudaGraphExecDestroy(chain);
        chain = nullptr;
      }
      cudaStream_t cs;
      cudaError_t ce = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
      if (ce != cudaSuccess) {
        st = fail_cuda(ce, "cudaStreamCreate");
        break;
      }
      cudaGraph_t g = nullptr;
      // warm the kernel's one-time set-up outside the capture
      double cube[27];
      jacobi_cube(cube);
      ce = cudaMemsetAsync(e, 0, lp, s);
      st = ce == cudaSuccess ? sweep_3d(e, e_tmp, n, nbatch, dt, cube, r_lp, 0.0, s)
                             : fail_cuda(ce, "cudaMemsetAsync");
      if (st == SSAM_OK) {
        ce = cudaStreamSynchronize(s);
        if (ce == cudaSuccess) ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        // the chain's first launch writes e (k odd) or e_tmp (k even); the
        // zero start grid is the other one, so no launch reads what it writes
        void* zero_src = (k % 2 == 1) ? e_tmp : e;
        if (ce == cudaSuccess) ce = cudaMemsetAsync(zero_src, 0, lp, cs);
        if (ce == cudaSuccess)
          st = jacobi_chain(r_lp, zero_src, e, e_tmp, n, nbatch, dt, k, cs, omega);
        cudaError_t ee = cudaStreamEndCapture(cs, &g);
        if (ce == cudaSuccess) ce = ee;
        if (ce == cudaSuccess && st == SSAM_OK) ce = cudaGraphInstantiate(&chain, g, 0);
        if (g) cudaGraphDestroy(g);
        if (ce != cudaSuccess && st == SSAM_OK) st = fail_cuda(ce, "capturing the sweep chain");
      }
      cudaStreamDestroy(cs);
      if (st != SSAM_OK) break;
    }
    cudaError_t ce = cudaGraphLaunch(chain, s);
    if (ce != cudaSuccess) {
      st = fail_cuda(ce, "cudaGraphLaunch(sweeps)");
      break;
    }
    for (int i = 0; i < k + 1; ++i) count_launch();
    if (dt == SSAM_BF16)
      add_correction_kernel<__nv_bfloat16><<<cblocks, nthreads, 0, s>>>(
          u, (const __nv_bfloat16*)e, (int64_t)cells);
    else
      add_correction_kernel<float><<<cblocks, nthreads, 0, s>>>(u, (const float*)e,
                                                                (int64_t)cells);
    count_launch();
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
      st = fail_cuda(ce, "add_correction");
      break;
    }
    out->sweeps += k;
    out->corrections += 1;
  }
  if (chain) cudaGraphExecDestroy(chain);
  scratch_free(work, s);
  return st;
}

extern "C" {

int ssam_poisson_solve(const double* f, double* u, int n, int nbatch,
                       const ssam_poisson_options* opt, ssam_poisson_stats* stats,
                       void* stream) {
  return poisson_solve(f, u, n, nbatch, opt, nullptr, stats, (cudaStream_t)stream);
}

int ssam_poisson_solve_learned(const double* f, double* u, int n, int nbatch,
                               const ssam_poisson_options* opt, void* cnn,
                               ssam_poisson_stats* stats, void* stream) {
  if (!cnn) return fail(SSAM_ERR_INVALID, "cnn handle must not be NULL");
  return poisson_solve(f, u, n, nbatch, opt, cnn, stats, (cudaStream_t)stream);
}

}  // extern "C"
