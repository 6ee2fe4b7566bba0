// ssai-3dstencil <7pt|13pt|poisson> <float|double> [N] [IT]
//
// Drop-in for the reference's 3D program (ssai-3dstencil/main.cpp:5-21: the
// stencil picked by a substring of argv[1], precision by argv[2]; entries
// stencil_3d7pt_v2 / stencil_3d13pt / stencil_poisson) that runs the
// computation of the reference's tests:
//  * N = GRID_SIZE = 512 (common.hpp:10) unless argv[3] gives it;
//  * the reference's sequence of ITERATIVE_COUNT runs on GPUs other than
//    the V100 -- 7pt: 2, 3, 3, 4 (tmp3d7pt-v2.cu:364-385), 13pt: 2
//    (tmp3d13pt.cu:404-408), poisson: 2, 3, 3 (tmpPoisson.cu:440-462) --
//    or one run of argv[4] steps;
//  * its input, getRandom3DArray: rand() / (RAND_MAX - 1) + 0.02121 per cell
//    from the C library's unseeded rand() (common.hpp:57-74), each run
//    drawing a fresh grid from the same sequence (SSAM_SEED reseeds it);
//  * its coefficients, the _F3d7PT / _F3d13PT / poisson defines
//    (ref_tables.h);
//  * its check: the gold applied IT times to the interior (the ring of the
//    grid left as it is) and checkError3D (common.hpp:84-127) over the band
//    [IT, N - IT) of every axis -- match / unmatch counts, max error and the
//    RMS error against TOLERANCE = 1e-5 (common.hpp:31), printed in its
//    format.
// The GPU runs IT steps of ssam_stencil3d with the ring copied unchanged.
#include <omp.h>

#include "ref_tables.h"
#include "ssai_cli.h"

namespace {

struct Spec {
  int shape, radius;
  const ssai_ref::Tap3D* taps;
  int ntaps;
  std::vector<int> its;  // the reference's ITERATIVE_COUNT sequence
};

template <typename T>
int run_one(const Spec& sp, int64_t n, int IT) {
  const int r = sp.radius, F = 2 * r + 1;
  std::vector<double> cube(F * F * F, 0.0);
  for (int k = 0; k < sp.ntaps; ++k) {
    const auto& t = sp.taps[k];
    cube[((t.dz + r) * F + t.dy + r) * F + t.dx + r] = t.c;
  }
  auto idx = [&](int64_t z, int64_t y, int64_t x) { return (size_t)((z * n + y) * n + x); };
  // getRandom3DArray: z, y, x order, one rand() per cell
  std::vector<T> in((size_t)(n * n * n));
  for (auto& v : in) v = (T)((T)rand() / (T)(RAND_MAX - 1) + 0.02121);
  ssai::DeviceRun<T> dev(in);
  auto call = [&] {
    ssai::check(ssam_stencil3d(dev.src, dev.dst, n, n, n, ssai::dtype<T>(), sp.shape, r,
                               cube.data(), IT, SSAM_BOUNDARY_COPY, nullptr),
                "ssam_stencil3d");
  };
  const double ms = dev.time_ms(call, 5);
  const std::vector<T> out = dev.result();
  printf("N=%d, ITERATIVE_COUNT=%d: %.4f ms, %.2f GCells/s\n", (int)n, IT, ms,
         (double)n * n * n * IT / (ms * 1e-3) / 1e9);
  // the gold, in T, on the interior; the ring keeps its input values
  std::vector<T> g = in, h = in;
  std::vector<T> c(sp.ntaps);
  for (int k = 0; k < sp.ntaps; ++k) c[k] = (T)sp.taps[k].c;
  for (int s = 0; s < IT; ++s) {
#pragma omp parallel for schedule(static)
    for (int64_t z = r; z < n - r; ++z)
      for (int64_t y = r; y < n - r; ++y)
        for (int64_t x = r; x < n - r; ++x) {
          T sum = 0;
          for (int k = 0; k < sp.ntaps; ++k) {
            const auto& t = sp.taps[k];
            sum += c[k] * g[idx(z + t.dz, y + t.dy, x + t.dx)];
          }
          h[idx(z, y, x)] = sum;
        }
    g.swap(h);
  }
  // checkError3D over [IT, N - IT)^3
  const int64_t lo = IT, hi = n - IT;
  if (hi <= lo) {
    printf("check: empty band\n");
    return 0;
  }
  double err = 0, max_err = 1e-5, sum = 0;
  int64_t match = 0, unmatch = 0, mi = 0, mj = 0, mk = 0;
  for (int64_t i = lo; i < hi; ++i)
    for (int64_t j = lo; j < hi; ++j)
      for (int64_t k = lo; k < hi; ++k) {
        const size_t q = idx(i, j, k);
        sum += out[q];
        const double d = fabs((double)out[q] - (double)g[q]);
        (d == 0 ? match : unmatch) += 1;
        err += d * d;
        if (d > max_err) {
          max_err = d;
          mi = i;
          mj = j;
          mk = k;
        }
      }
  printf("sum = %e, match = %lld, unmatch = %lld\n", sum, (long long)match, (long long)unmatch);
  printf("[Test] Max Error : %e @ (%lld,%lld,%lld)\n", max_err, (long long)mi, (long long)mj,
         (long long)mk);
  const double rms = sqrt(err / ((double)(hi - lo) * (hi - lo) * (hi - lo)));
  printf("N=%d, [Test] RMS Error : %e\n", (int)n, rms);
  return rms > 1e-5 ? -1 : 0;  // the reference's TOLERANCE (common.hpp:31)
}

template <typename T>
int run(int argc, char** argv, const Spec& sp) {
  int N = 512;
  if (argc > 3) N = atoi(argv[3]);
  std::vector<int> its = sp.its;
  if (argc > 4) its.assign(1, atoi(argv[4]));
  if (N < 1) {
    fprintf(stderr, "bad N\n");
    return 1;
  }
  for (int it : its)
    if (it < 1) {
      fprintf(stderr, "bad IT\n");
      return 1;
    }
  const char* env = getenv("SSAM_SEED");
  if (env) srand((unsigned)atoi(env));
  int rc = 0;
  for (int it : its)
    if (run_one<T>(sp, N, it) != 0) rc = -1;
  return rc;
}

Spec spec7() { return {SSAM_STAR3D, 1, ssai_ref::k_j3d7pt, 7, {2, 3, 3, 4}}; }
Spec spec13() { return {SSAM_STAR3D, 2, ssai_ref::k_j3d13pt, 13, {2}}; }
Spec spec19() { return {SSAM_POISSON19, 1, ssai_ref::k_poisson, 19, {2, 3, 3}}; }

}  // namespace

int stencil_3d7pt_v2(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, spec7()) : run<float>(argc, argv, spec7());
}
int stencil_3d13pt(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, spec13()) : run<float>(argc, argv, spec13());
}
int stencil_poisson(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, spec19()) : run<float>(argc, argv, spec19());
}

int main(int argc, char** argv) {
  ssai::echo_args(argc, argv);
  if (argc < 3) {
    printf("error, argc = %d\n", argc);
    return 1;
  }
  const char* f = argv[1];
  if (strstr(f, "7pt")) return stencil_3d7pt_v2(argc, argv);
  if (strstr(f, "13pt")) return stencil_3d13pt(argc, argv);
  if (strstr(f, "poisson")) return stencil_poisson(argc, argv);
  printf("invalid function name!\n");
  return 1;
}
