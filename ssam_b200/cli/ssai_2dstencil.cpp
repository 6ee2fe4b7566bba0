// ssai-2dstencil <size> <pts> <float|double> [steps]
//
// Drop-in for the reference's 2D stencil program: the same argv spelling
// (ssai-2dstencil/main.cpp:17-53: pts = 5, 9, 13, 17, 21, 25 (star r = 1..6),
// 64 (9x9 box without its centre row and column), 81 / 121 (9x9 / 11x11
// box), tmp_5 / tmp_9 (the temporal-blocked 5- and 9-point stars)), and the
// same entry functions stencil_<pts>pt_<float|double>(argc, argv) with the
// grid size in argv[1] (default 8192, stencil2D_5pt-v1.cu:254-269).  Each
// entry seeds a size x size grid, runs ssam_stencil2d on the GPU (clamped
// halo like the reference's kernels; zero padding for multi-step runs),
// prints the kernel time and GCells/s,
// and checks 4096 sampled cells (every cell of multi-step runs up to 1024^2)
// against a direct evaluation in double on the host.
#include "ssai_cli.h"

namespace {

struct Spec {
  int shape, radius, steps;
  bool cross_free;  // the 64-point stencil: a 9x9 box whose centre row/column is zero
};

template <typename T>
int run(int argc, char** argv, Spec sp) {
  int size = 8192;
  if (argc > 1) size = atoi(argv[1]);
  if (argc > 4) sp.steps = atoi(argv[4]);
  if (size < 1 || sp.steps < 1) {
    fprintf(stderr, "bad size / steps\n");
    return 1;
  }
  const int r = sp.radius, F = 2 * r + 1;
  std::vector<double> c;
  if (sp.shape == SSAM_STAR) {
    c = ssai::coefficients(4 * r + 1, 11);
  } else {
    c = ssai::coefficients(F * F, 11);
    if (sp.cross_free) {
      double s = 0;
      for (int i = 0; i < F * F; ++i) {
        if (i / F == r || i % F == r) c[i] = 0;
        s += c[i];
      }
      for (auto& v : c) v /= s;
    }
  }
  // the equivalent dense (2r+1)^2 matrix for the host check
  std::vector<double> m(F * F, 0.0);
  if (sp.shape == SSAM_STAR) {
    m[r * F + r] = c[0];
    for (int k = 1; k <= r; ++k) {
      m[(r - k) * F + r] = c[1 + 4 * (k - 1)];
      m[(r + k) * F + r] = c[2 + 4 * (k - 1)];
      m[r * F + r - k] = c[3 + 4 * (k - 1)];
      m[r * F + r + k] = c[4 + 4 * (k - 1)];
    }
  } else {
    m = c;
  }
  const int64_t W = size, H = size;
  const std::vector<T> in = ssai::uniform<T>((size_t)W * H, 7);
  ssai::DeviceRun<T> dev(in);
  // one step: the clamped halo of the reference's kernels; several steps:
  // zero padding (the reference checks temporal runs on the interior band only)
  const int bnd = sp.steps == 1 ? SSAM_BOUNDARY_CLAMP : SSAM_BOUNDARY_ZERO;
  auto call = [&] {
    ssai::check(ssam_stencil2d(dev.src, dev.dst, W, H, W, ssai::dtype<T>(), sp.shape, r,
                               c.data(), sp.steps, bnd, nullptr),
                "ssam_stencil2d");
  };
  const double ms = dev.time_ms(call, 10);
  const std::vector<T> out = dev.result();
  printf("%dx%d, %s, radius %d, %d step(s): %.4f ms, %.2f GCells/s\n", size, size,
         sp.shape == SSAM_STAR ? "star" : "box", r, sp.steps, ms,
         (double)W * H * sp.steps / (ms * 1e-3) / 1e9);

  // host check: the same boundary, `steps` applications, in double
  auto at = [&](const std::vector<double>& g, int64_t y, int64_t x) {
    if (bnd == SSAM_BOUNDARY_ZERO && (y < 0 || y >= H || x < 0 || x >= W)) return 0.0;
    y = y < 0 ? 0 : (y >= H ? H - 1 : y);
    x = x < 0 ? 0 : (x >= W ? W - 1 : x);
    return g[(size_t)y * W + x];
  };
  auto apply = [&](const std::vector<double>& g, int64_t y, int64_t x) {
    double s = 0;
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) s += m[(dy + r) * F + dx + r] * at(g, y + dy, x + dx);
    return s;
  };
  double worst = 0;
  if (sp.steps == 1) {
    std::vector<double> g(in.begin(), in.end());
    std::mt19937_64 rng(3);
    for (int k = 0; k < 4096; ++k) {
      const int64_t y = rng() % H, x = rng() % W;
      const double want = apply(g, y, x);
      worst = fmax(worst, fabs((double)out[(size_t)y * W + x] - want) / fmax(fabs(want), 1e-30));
    }
    printf("check: 4096 sampled cells, max relative error %.3e\n", worst);
  } else if (W * H <= 1024 * 1024) {
    std::vector<double> g(in.begin(), in.end()), h(g.size());
    for (int s = 0; s < sp.steps; ++s) {
      for (int64_t y = 0; y < H; ++y)
        for (int64_t x = 0; x < W; ++x) h[(size_t)y * W + x] = apply(g, y, x);
      g.swap(h);
    }
    for (size_t i = 0; i < g.size(); ++i)
      worst = fmax(worst, fabs((double)out[i] - g[i]) / fmax(fabs(g[i]), 1e-30));
    printf("check: every cell, max relative error %.3e\n", worst);
  } else {
    printf("check: skipped for multi-step runs above 1024^2 (the test suite covers them)\n");
    return 0;
  }
  const double tol = (sizeof(T) == 8 ? 1e-12 : 1e-5) * sp.steps;
  if (worst > tol) {
    printf("FAILED (tolerance %.1e)\n", tol);
    return -1;
  }
  return 0;
}

}  // namespace

#define SSAI_ENTRY(name, shape, r, steps, cross)                              \
  int stencil_##name##pt_float(int argc, char** argv) {                       \
    return run<float>(argc, argv, Spec{shape, r, steps, cross});              \
  }                                                                           \
  int stencil_##name##pt_double(int argc, char** argv) {                      \
    return run<double>(argc, argv, Spec{shape, r, steps, cross});             \
  }

SSAI_ENTRY(5, SSAM_STAR, 1, 1, false)
SSAI_ENTRY(9, SSAM_STAR, 2, 1, false)
SSAI_ENTRY(13, SSAM_STAR, 3, 1, false)
SSAI_ENTRY(17, SSAM_STAR, 4, 1, false)
SSAI_ENTRY(21, SSAM_STAR, 5, 1, false)
SSAI_ENTRY(25, SSAM_STAR, 6, 1, false)
SSAI_ENTRY(64, SSAM_BOX, 4, 1, true)
SSAI_ENTRY(81, SSAM_BOX, 4, 1, false)
SSAI_ENTRY(121, SSAM_BOX, 5, 1, false)
SSAI_ENTRY(tmp_5, SSAM_STAR, 1, 4, false)
SSAI_ENTRY(tmp_9, SSAM_STAR, 2, 4, false)

int main(int argc, char** argv) {
  ssai::echo_args(argc, argv);
  if (argc < 4) {
    printf("usage: %s <size> <5|9|13|17|21|25|64|81|121|tmp_5|tmp_9> <float|double> [steps]\n",
           argv[0]);
    return 1;
  }
  const char* pts = argv[2];
  const bool dbl = strcmp(argv[3], "double") == 0;
  if (!dbl && strcmp(argv[3], "float") != 0) {
    printf("error!\n");
    return 1;
  }
#define SSAI_DISPATCH(name)                                                            \
  if (strcmp(pts, #name) == 0)                                                         \
    return dbl ? stencil_##name##pt_double(argc, argv) : stencil_##name##pt_float(argc, argv);
  SSAI_DISPATCH(5)
  SSAI_DISPATCH(9)
  SSAI_DISPATCH(13)
  SSAI_DISPATCH(17)
  SSAI_DISPATCH(21)
  SSAI_DISPATCH(25)
  SSAI_DISPATCH(64)
  SSAI_DISPATCH(81)
  SSAI_DISPATCH(121)
  SSAI_DISPATCH(tmp_5)
  SSAI_DISPATCH(tmp_9)
  printf("error, do not call functions\n");
  return 1;
}
