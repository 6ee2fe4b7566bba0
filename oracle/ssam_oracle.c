/*
 * ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference's CPU golden code for the SSAM stencil
 * and convolution path.  It is the checker that the CUDA library is compared
 * with: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.  The product library (libssam_b200.so) never links or calls it.
 *
 * Each function names the reference code it restates.  Loop order, summation
 * order and accumulation type follow the reference, so that results match it
 * bit for bit (checked against the compiled reference in oracle/_ref and the
 * committed fixtures in tests/golden/).  Build with -ffp-contract=off: the
 * reference's host code multiplies and adds separately.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#define BND_ZERO 0
#define BND_CLAMP 1
#define BND_COPY 2
/* 3D only: interior cells computed, ring cells left as they are in `out`
 * (the reference golds write the interior only, tmp3d7pt-v2.cu:281-297). */
#define BND_GOLD 3

static inline int64_t clampi(int64_t v, int64_t lo, int64_t hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

/* ------------------------------------------------------------------ 2D --- */

/*
 * Convolution<T> (ssai-2dconv/common.h:186-216): zero padding, filter column
 * index n outer, filter row index m inner, weight filter[m*fw + n], sum kept
 * in T.  `pitch` generalises the reference's dense width stride.
 * boundary CLAMP reads the nearest edge cell instead of 0 (the GPU stencil
 * kernels' halo load, stencil2D_5pt-v1.cu:29-46); COPY writes the input value
 * to every cell within the filter's reach of the edge.
 */
#define DEFINE_CONV2D(NAME, T)                                                  \
  void NAME(const T* src, T* dst, int64_t width, int64_t height, int64_t pitch, \
            const T* filter, int fw, int fh, int boundary) {                    \
    const int64_t rl = fw / 2, rr = fw - 1 - fw / 2;                            \
    const int64_t rt = fh / 2, rb = fh - 1 - fh / 2;                            \
    _Pragma("omp parallel for schedule(static)")                                \
    for (int64_t i = 0; i < height; i++) {                                      \
      for (int64_t j = 0; j < width; j++) {                                     \
        if (boundary == BND_COPY &&                                             \
            (j < rl || j >= width - rr || i < rt || i >= height - rb)) {        \
          dst[i * pitch + j] = src[i * pitch + j];                              \
          continue;                                                             \
        }                                                                       \
        T sum = 0;                                                              \
        for (int n = 0; n < fw; n++) {                                          \
          for (int m = 0; m < fh; m++) {                                        \
            int64_t x = j + n - fw / 2;                                         \
            int64_t y = i + m - fh / 2;                                         \
            if (boundary == BND_CLAMP) {                                        \
              x = clampi(x, 0, width - 1);                                      \
              y = clampi(y, 0, height - 1);                                     \
            } else if (!(x >= 0 && x < width && y >= 0 && y < height)) {        \
              continue;                                                         \
            }                                                                   \
            sum += src[y * pitch + x] * filter[m * fw + n];                     \
          }                                                                     \
        }                                                                       \
        dst[i * pitch + j] = sum;                                               \
      }                                                                         \
    }                                                                           \
  }

DEFINE_CONV2D(ssam_oracle_conv2d_f32, float)
DEFINE_CONV2D(ssam_oracle_conv2d_f64, double)

/*
 * `steps` applications of the same filter, each reading the previous result:
 * the reference's temporal-blocking check, which runs Convolution
 * ITERATIVE_COUNT times and copies back between runs
 * (stencil2d_temp_5pt.cu:183-186).  `work` is a caller buffer of the same
 * size as dst (pitch*height elements); it is only used when steps > 1.
 */
#define DEFINE_STEPS2D(NAME, CONV, T)                                           \
  void NAME(const T* src, T* dst, T* work, int64_t width, int64_t height,       \
            int64_t pitch, const T* filter, int fw, int fh, int boundary,       \
            int steps) {                                                        \
    const T* in = src;                                                          \
    for (int s = 0; s < steps; s++) {                                           \
      /* the last step lands in dst; earlier ones alternate with work */        \
      T* out = ((steps - 1 - s) % 2 == 0) ? dst : work;                         \
      CONV(in, out, width, height, pitch, filter, fw, fh, boundary);            \
      in = out;                                                                 \
    }                                                                           \
  }

DEFINE_STEPS2D(ssam_oracle_steps2d_f32, ssam_oracle_conv2d_f32, float)
DEFINE_STEPS2D(ssam_oracle_steps2d_f64, ssam_oracle_conv2d_f64, double)

/* ------------------------------------------------------------------ 3D --- */

/*
 * A 3D stencil given as an ordered tap list, evaluated like the reference
 * golds' single expression `c0*in[..] + c1*in[..] + ...` (left to right, each
 * product and partial sum rounded to T):
 *   v2::j3d7pt_gold  (ssai-3dstencil/tmp3d7pt-v2.cu:278-298)
 *   j3d13pt_gold     (ssai-3dstencil/tmp3d13pt.cu:301-327)
 * Loops are z outer (OpenMP), y, x inner, as in the golds.  `reach` is the
 * largest |offset|; cells closer than `reach` to a face are the ring, treated
 * per `boundary` (GOLD leaves them untouched, COPY copies the input, ZERO and
 * CLAMP compute them with zero / clamped taps).
 */
#define DEFINE_TAPS3D(NAME, T)                                                  \
  void NAME(const T* in, T* out, int64_t nx, int64_t ny, int64_t nz, int ntaps, \
            const int* dz, const int* dy, const int* dx, const T* coef,         \
            int reach, int boundary) {                                          \
    const int64_t nxy = nx * ny;                                                \
    _Pragma("omp parallel for schedule(static)")                                \
    for (int64_t k = 0; k < nz; k++) {                                          \
      for (int64_t j = 0; j < ny; j++) {                                        \
        for (int64_t i = 0; i < nx; i++) {                                      \
          const int ring = k < reach || k >= nz - reach || j < reach ||         \
                           j >= ny - reach || i < reach || i >= nx - reach;     \
          if (ring && boundary == BND_GOLD) continue;                           \
          if (ring && boundary == BND_COPY) {                                   \
            out[k * nxy + j * nx + i] = in[k * nxy + j * nx + i];               \
            continue;                                                           \
          }                                                                     \
          T sum = 0;                                                            \
          for (int t = 0; t < ntaps; t++) {                                     \
            int64_t z = k + dz[t], y = j + dy[t], x = i + dx[t];                \
            T v;                                                                \
            if (boundary == BND_CLAMP) {                                        \
              z = clampi(z, 0, nz - 1);                                         \
              y = clampi(y, 0, ny - 1);                                         \
              x = clampi(x, 0, nx - 1);                                         \
              v = in[z * nxy + y * nx + x];                                     \
            } else if (z < 0 || z >= nz || y < 0 || y >= ny || x < 0 ||         \
                       x >= nx) {                                               \
              v = 0;                                                            \
            } else {                                                            \
              v = in[z * nxy + y * nx + x];                                     \
            }                                                                   \
            T prod = coef[t] * v;                                               \
            sum = (t == 0) ? prod : sum + prod;                                 \
          }                                                                     \
          out[k * nxy + j * nx + i] = sum;                                      \
        }                                                                       \
      }                                                                         \
    }                                                                           \
  }

DEFINE_TAPS3D(ssam_oracle_taps3d_f32, float)
DEFINE_TAPS3D(ssam_oracle_taps3d_f64, double)

/*
 * poisson_gold (ssai-3dstencil/tmpPoisson.cu:369-386): the 19-point operator
 * written with double literals, so the expression is evaluated in double and
 * rounded to T once at the store, whatever T is:
 *   2.666*c - 0.166*(6 face neighbours) + 0.0833*(12 edge neighbours, the
 *   four y-z edges negated).
 * Interior only (ring per `boundary`: GOLD or COPY).
 */
#define DEFINE_POISSON19(NAME, T)                                                \
  void NAME(const T* in_, T* out_, int64_t n_x, int64_t n_y, int64_t n_z,        \
            int boundary) {                                                      \
    const int64_t nxy = n_x * n_y;                                               \
    _Pragma("omp parallel for schedule(static)")                                 \
    for (int64_t k = 0; k < n_z; k++) {                                          \
      for (int64_t j = 0; j < n_y; j++) {                                        \
        for (int64_t i = 0; i < n_x; i++) {                                      \
          const int64_t c = k * nxy + j * n_x + i;                               \
          if (k < 1 || k >= n_z - 1 || j < 1 || j >= n_y - 1 || i < 1 ||         \
              i >= n_x - 1) {                                                    \
            if (boundary == BND_COPY) out_[c] = in_[c];                          \
            continue;                                                            \
          }                                                                      \
          const T* in = in_;                                                     \
          const int64_t zm = -nxy, zp = nxy, ym = -n_x, yp = n_x;                \
          out_[c] = 2.666 * in[c] -                                              \
                    0.166 * (in[c + zm] + in[c + zp] + in[c + ym] + in[c + yp] + \
                             in[c + 1] + in[c - 1]) +                            \
                    0.0833 * (-in[c + zm + ym] - in[c + zp + ym] -               \
                              in[c + zm + yp] - in[c + zp + yp] +                \
                              in[c + zm - 1] + in[c + zp - 1] +                  \
                              in[c + ym - 1] + in[c + yp - 1] +                  \
                              in[c + zm + 1] + in[c + zp + 1] +                  \
                              in[c + ym + 1] + in[c + yp + 1]);                  \
        }                                                                        \
      }                                                                          \
    }                                                                            \
  }

DEFINE_POISSON19(ssam_oracle_poisson19_f32, float)
DEFINE_POISSON19(ssam_oracle_poisson19_f64, double)

/*
 * checkError3D (ssai-3dstencil/common.hpp:84-127): RMS and max of |out - ref|
 * over the box [z_lb,z_ub) x [y_lb,y_ub) x [x_lb,x_ub), accumulated in double.
 */
void ssam_oracle_check_error3d_f64(const double* out, const double* ref,
                                   int64_t nx, int64_t ny, int64_t z_lb,
                                   int64_t z_ub, int64_t y_lb, int64_t y_ub,
                                   int64_t x_lb, int64_t x_ub, double* rms,
                                   double* max_err) {
  double err = 0.0, mx = 0.0;
  for (int64_t i = z_lb; i < z_ub; i++)
    for (int64_t j = y_lb; j < y_ub; j++)
      for (int64_t k = x_lb; k < x_ub; k++) {
        double d = out[(i * ny + j) * nx + k] - ref[(i * ny + j) * nx + k];
        d = d < 0 ? -d : d;
        err += d * d;
        if (d > mx) mx = d;
      }
  *rms = sqrt(err / (double)((z_ub - z_lb) * (y_ub - y_lb) * (x_ub - x_lb)));
  *max_err = mx;
}

/* ------------------------------------------------------------- Poisson --- */

/*
 * No reference code exists for the Poisson solver; these restate the
 * mathematics in FP64 with the loop structure of v2::j3d7pt_gold
 * (ssai-3dstencil/tmp3d7pt-v2.cu:281-297): z outer (OpenMP), y, x inner.
 * Grids: `nb` stacked n^3 interior grids, u = 0 outside (Dirichlet),
 * h = 1/(n+1).
 *
 * One Jacobi sweep: out = (sum of the 6 neighbours of in + h^2 rhs) / 6,
 * neighbours summed in the order z-1, y-1, x-1, x+1, y+1, z+1.
 */
void ssam_oracle_jacobi7_f64(const double* rhs, const double* in, double* out, int64_t n,
                             int64_t nb, int sweeps, double* work) {
  const double h2 = 1.0 / (double)((n + 1) * (n + 1));
  const int64_t nn = n * n, n3 = n * n * n;
  const double* src = in;
  for (int s = 0; s < sweeps; s++) {
    double* dst = ((sweeps - 1 - s) % 2 == 0) ? out : work;
    for (int64_t b = 0; b < nb; b++) {
      const double* u = src + b * n3;
      const double* f = rhs + b * n3;
      double* o = dst + b * n3;
      _Pragma("omp parallel for schedule(static)")
      for (int64_t k = 0; k < n; k++)
        for (int64_t j = 0; j < n; j++)
          for (int64_t i = 0; i < n; i++) {
            const int64_t c = k * nn + j * n + i;
            double sum = 0.0;
            if (k > 0) sum += u[c - nn];
            if (j > 0) sum += u[c - n];
            if (i > 0) sum += u[c - 1];
            if (i < n - 1) sum += u[c + 1];
            if (j < n - 1) sum += u[c + n];
            if (k < n - 1) sum += u[c + nn];
            o[c] = (sum + h2 * f[c]) / 6.0;
          }
    }
    src = dst;
  }
}

/* r = f - A u with A u = (6 u - sum of neighbours) / h^2; per-grid
 * sum r^2 and sum f^2 into norms2[2*b], norms2[2*b+1]. */
void ssam_oracle_residual7_f64(const double* f, const double* u, double* r, int64_t n,
                               int64_t nb, double* norms2) {
  const double inv_h2 = (double)((n + 1) * (n + 1));
  const int64_t nn = n * n, n3 = n * n * n;
  for (int64_t b = 0; b < nb; b++) {
    const double* ub = u + b * n3;
    const double* fb = f + b * n3;
    double rr = 0.0, ff = 0.0;
    _Pragma("omp parallel for schedule(static) reduction(+:rr,ff)")
    for (int64_t k = 0; k < n; k++)
      for (int64_t j = 0; j < n; j++)
        for (int64_t i = 0; i < n; i++) {
          const int64_t c = k * nn + j * n + i;
          double sum = 0.0;
          if (k > 0) sum += ub[c - nn];
          if (j > 0) sum += ub[c - n];
          if (i > 0) sum += ub[c - 1];
          if (i < n - 1) sum += ub[c + 1];
          if (j < n - 1) sum += ub[c + n];
          if (k < n - 1) sum += ub[c + nn];
          const double rc = fb[c] - (6.0 * ub[c] - sum) * inv_h2;
          if (r) r[b * n3 + c] = rc;
          rr += rc * rc;
          ff += fb[c] * fb[c];
        }
    norms2[2 * b] = rr;
    norms2[2 * b + 1] = ff;
  }
}
