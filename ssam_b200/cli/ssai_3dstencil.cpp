// ssai-3dstencil <7pt|13pt|poisson> <float|double> [N] [IT]
//
// Drop-in for the reference's 3D program (ssai-3dstencil/main.cpp:5-21: the
// stencil picked by a substring of argv[1], precision by argv[2]; entries
// stencil_3d7pt_v2 / stencil_3d13pt / stencil_poisson).  The grid side N
// (default 512, the reference's GRID_SIZE) and the fused step count IT
// (default 2) are optional extra arguments where the reference fixes them at
// compile time.  Seeds an N^3 grid, runs IT steps of ssam_stencil3d on the GPU
// (the ring of the grid copied unchanged, like the reference golds leave it),
// prints the time and GCells/s, and reports the RMS error against a direct
// evaluation in double over a 4096-cell sample of the band the reference
// checks ([IT*r, N - IT*r) in every axis) for IT = 1, or over the whole band
// for N <= 128.
#include "ssai_cli.h"

namespace {

struct Spec {
  int shape, radius;
};

template <typename T>
int run(int argc, char** argv, Spec sp) {
  int N = 512, IT = 2;
  if (argc > 3) N = atoi(argv[3]);
  if (argc > 4) IT = atoi(argv[4]);
  if (N < 1 || IT < 1) {
    fprintf(stderr, "bad N / IT\n");
    return 1;
  }
  const int r = sp.radius, F = 2 * r + 1;
  // coefficient cube: the stencil's taps get seeded weights summing to 1
  std::vector<double> cube(F * F * F, 0.0);
  std::vector<int> taps;
  for (int dz = -r; dz <= r; ++dz)
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) {
        const int nz = (dz != 0) + (dy != 0) + (dx != 0);
        const bool on = sp.shape == SSAM_POISSON19 ? nz <= 2 : nz <= 1;
        if (on) taps.push_back(((dz + r) * F + dy + r) * F + dx + r);
      }
  const std::vector<double> w = ssai::coefficients(taps.size(), 17);
  for (size_t i = 0; i < taps.size(); ++i) cube[taps[i]] = w[i];
  const int64_t n = N;
  const std::vector<T> in = ssai::uniform<T>((size_t)(n * n * n), 7);
  ssai::DeviceRun<T> dev(in);
  auto call = [&] {
    ssai::check(ssam_stencil3d(dev.src, dev.dst, n, n, n, ssai::dtype<T>(), sp.shape, r,
                               cube.data(), IT, SSAM_BOUNDARY_COPY, nullptr),
                "ssam_stencil3d");
  };
  const double ms = dev.time_ms(call, 5);
  const std::vector<T> out = dev.result();
  printf("N=%d, %d step(s): %.4f ms, %.2f GCells/s\n", N, IT, ms,
         (double)n * n * n * IT / (ms * 1e-3) / 1e9);
  auto idx = [&](int64_t z, int64_t y, int64_t x) { return (size_t)((z * n + y) * n + x); };
  auto apply = [&](const std::vector<double>& g, int64_t z, int64_t y, int64_t x) {
    double s = 0;
    for (int t : taps) {
      const int dz = t / (F * F) - r, dy = (t / F) % F - r, dx = t % F - r;
      s += cube[t] * g[idx(z + dz, y + dy, x + dx)];
    }
    return s;
  };
  const int64_t lo = (int64_t)IT * r, hi = n - lo;
  if (hi <= lo) {
    printf("check: empty band\n");
    return 0;
  }
  double se = 0;
  int64_t cnt = 0;
  std::vector<double> g(in.begin(), in.end());
  if (IT == 1) {
    std::mt19937_64 rng(3);
    for (int k = 0; k < 4096; ++k) {
      const int64_t z = lo + rng() % (hi - lo), y = lo + rng() % (hi - lo),
                    x = lo + rng() % (hi - lo);
      const double d = out[idx(z, y, x)] - apply(g, z, y, x);
      se += d * d;
      ++cnt;
    }
  } else if (N <= 128) {
    std::vector<double> h = g;
    for (int s = 0; s < IT; ++s) {
      for (int64_t z = r; z < n - r; ++z)
        for (int64_t y = r; y < n - r; ++y)
          for (int64_t x = r; x < n - r; ++x) h[idx(z, y, x)] = apply(g, z, y, x);
      g.swap(h);
    }
    for (int64_t z = lo; z < hi; ++z)
      for (int64_t y = lo; y < hi; ++y)
        for (int64_t x = lo; x < hi; ++x) {
          const double d = out[idx(z, y, x)] - g[idx(z, y, x)];
          se += d * d;
          ++cnt;
        }
  } else {
    printf("check: skipped for IT > 1 above N = 128 (the test suite covers it)\n");
    return 0;
  }
  const double rms = sqrt(se / (double)cnt);
  printf("N=%d, [Test] RMS Error : %e\n", N, rms);
  return rms > 1e-5 ? -1 : 0;  // the reference's TOLERANCE (common.hpp:31)
}

}  // namespace

int stencil_3d7pt_v2(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, {SSAM_STAR3D, 1}) : run<float>(argc, argv, {SSAM_STAR3D, 1});
}
int stencil_3d13pt(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, {SSAM_STAR3D, 2}) : run<float>(argc, argv, {SSAM_STAR3D, 2});
}
int stencil_poisson(int argc, char** argv) {
  const bool dbl = argc > 2 && strstr(argv[2], "double");
  return dbl ? run<double>(argc, argv, {SSAM_POISSON19, 1})
             : run<float>(argc, argv, {SSAM_POISSON19, 1});
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
