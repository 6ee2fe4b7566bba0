// ssai-2dstencil <size> <pts> <float|double> [steps]
//
// Drop-in for the reference's 2D stencil program: the same argv spelling
// (ssai-2dstencil/main.cpp:17-53: pts = 5, 9, 13, 17, 21, 25 (star r = 1..6),
// 64 (9x9 box without its centre row and column), 81 / 121 (9x9 / 11x11
// box), tmp_5 / tmp_9 (the temporal-blocked 5- and 9-point stars)), and the
// same entry functions stencil_<pts>pt_<float|double>(argc, argv) with the
// grid size in argv[1] (default 8192, stencil2D_5pt-v1.cu:254-269).
//
// Each entry runs the computation of the reference test it replaces:
//  * the reference's own coefficient table (ref_tables.h); the 5-point test
//    redraws its five taps as rand() % 20 - 10 (stencil2D_5pt-v1.cu:180-184)
//    and does so here too;
//  * the reference's input: ../data/Lena<N>x<N>.raw when present, else its
//    generated data -- the row index for the 5-point test
//    (stencil2D_5pt-v1.cu:157-161), rand() % 256 for the other single-step
//    tests (e.g. stencil2D_25pt.cu:151), rand() / (RAND_MAX - 1) + 0.02121
//    for the temporal ones (stencil2d_temp_5pt.cu:111), from the C library's
//    rand() in the reference's call order.  The reference seeds rand() with
//    the time in the 5-point test only (stencil2D_5pt-v1.cu:133); here every
//    test uses srand(SSAM_SEED) (default 1, the unseeded sequence the other
//    tests draw from), so runs repeat;
//  * the reference's step count: 1, or ITERATIVE_COUNT = 5 (tmp_5) / 3
//    (tmp_9) (stencil2d_temp_5pt.cu:221-226, stencil2d_temp_9pt.cu:223-225);
//    an optional argv[4] overrides it;
//  * its check: Convolution<T> (ssai-2dconv/common.h:186-216) applied `steps`
//    times on the host, and the sum of |gold - gpu| over the band the
//    reference sums ("verify dif", stencil2D_5pt-v1.cu:229-236,
//    stencil2d_temp_5pt.cu:181-191), printed in its format; the program
//    fails when a cell of that band differs from the gold by more than
//    1e-5 (FP32) / 1e-12 (FP64) per step of sum |c||x|.
// The GPU runs ssam_stencil2d with the reference kernels' clamped halo for a
// single step and zero padding for several (the band excludes the edges).
#include <omp.h>
#include <time.h>

#include "ref_tables.h"
#include "ssai_cli.h"

namespace {

enum Input { ROW_INDEX, RAND_256, RAND_UNIT };

struct Spec {
  const char* table;  // name in ssai_ref::kTables2D
  int shape;          // SSAM_STAR (the ABI's star argument order) or SSAM_BOX
  int steps;          // the reference's ITERATIVE_COUNT (1 for single-step tests)
  Input input;
  bool redraw;        // the 5-point test redraws its five taps
};

const ssai_ref::Table2D* find_table(const char* name) {
  for (const auto& t : ssai_ref::kTables2D)
    if (strcmp(t.name, name) == 0) return &t;
  return nullptr;
}

// Convolution<T> of the reference: zero outside the grid, x offset in the
// outer loop and y offset in the inner one, the sum kept in T.
template <typename T>
void convolution(const std::vector<T>& src, std::vector<T>& dst, int64_t W, int64_t H,
                 const std::vector<T>& f, int F) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < H; ++i)
    for (int64_t j = 0; j < W; ++j) {
      T sum = 0;
      for (int n = 0; n < F; ++n)
        for (int m = 0; m < F; ++m) {
          const int64_t x = j + n - F / 2, y = i + m - F / 2;
          if (x >= 0 && x < W && y >= 0 && y < H) sum += src[y * W + x] * f[m * F + n];
        }
      dst[i * W + j] = sum;
    }
}

template <typename T>
int run(int argc, char** argv, Spec sp) {
  int size = 8192;
  if (argc > 1) size = atoi(argv[1]);
  if (argc > 4) sp.steps = atoi(argv[4]);
  if (size < 1 || sp.steps < 1) {
    fprintf(stderr, "bad size / steps\n");
    return 1;
  }
  const ssai_ref::Table2D* tab = find_table(sp.table);
  const int r = tab->radius, F = 2 * r + 1;
  const int64_t W = size, H = size;
  const char* env = getenv("SSAM_SEED");
  srand(env ? (unsigned)atoi(env) : 1u);
  // input: the reference's image if present, else its generated data
  std::vector<T> in;
  char path[256];
  snprintf(path, sizeof path, "../data/Lena%dx%d.raw", size, size);
  if (ssai::load_raw_uchar(path, (size_t)(W * H), &in)) {
    printf("Load success : %s\n", path);
  } else {
    printf("Load failed : %s, generate random data\n", path);
    in.resize((size_t)(W * H));
    for (size_t i = 0; i < in.size(); ++i) {
      if (sp.input == RAND_UNIT) {
        in[i] = (T)((T)rand() / (T)(RAND_MAX - 1) + 0.02121);
      } else {
        in[i] = (T)(rand() % 256);
        if (sp.input == ROW_INDEX) in[i] = (T)(i / W);
      }
    }
  }
  // coefficients: the reference's table, in T (its filter is a T array)
  std::vector<T> f(tab->m, tab->m + F * F);
  if (sp.redraw) {  // [1][1], [0][1], [2][1], [1][0], [1][2]
    const int cells[5][2] = {{1, 1}, {0, 1}, {2, 1}, {1, 0}, {1, 2}};
    for (auto& c : cells) f[c[0] * F + c[1]] = (T)(rand() % 20 - 10);
  }
  // the ABI's arguments: c, then n, s, w, e per ring for stars; the matrix for boxes
  std::vector<double> c;
  if (sp.shape == SSAM_STAR) {
    c.push_back(f[r * F + r]);
    for (int k = 1; k <= r; ++k) {
      c.push_back(f[(r - k) * F + r]);
      c.push_back(f[(r + k) * F + r]);
      c.push_back(f[r * F + r - k]);
      c.push_back(f[r * F + r + k]);
    }
  } else {
    c.assign(f.begin(), f.end());
  }
  ssai::DeviceRun<T> dev(in);
  const int bnd = sp.steps == 1 ? SSAM_BOUNDARY_CLAMP : SSAM_BOUNDARY_ZERO;
  auto call = [&] {
    ssai::check(ssam_stencil2d(dev.src, dev.dst, W, H, W, ssai::dtype<T>(), sp.shape, r,
                               c.data(), sp.steps, bnd, nullptr),
                "ssam_stencil2d");
  };
  const double ms = dev.time_ms(call, 10);
  const std::vector<T> out = dev.result();
  printf("%dx%d , %dx%d , Iterative=%d, %f ms , %f fps, %.2f GCells/s\n", size, size, F, F,
         sp.steps, ms, 1000.0 / ms, (double)W * H * sp.steps / (ms * 1e-3) / 1e9);

  // the reference's check: Convolution<T> `steps` times, |gold - gpu| summed
  // over the band it sums; plus sum |c||x| for the per-cell bound
  std::vector<T> gold = in, tmp(in.size());
  std::vector<T> mag(in.size()), fa(f.size());
  for (size_t i = 0; i < in.size(); ++i) mag[i] = (T)fabs((double)in[i]);
  for (size_t i = 0; i < f.size(); ++i) fa[i] = (T)fabs((double)f[i]);
  for (int s = 0; s < sp.steps; ++s) {
    convolution(gold, tmp, W, H, f, F);
    gold.swap(tmp);
    convolution(mag, tmp, W, H, fa, F);
    mag.swap(tmp);
  }
  const int64_t e = (int64_t)(F / 2) * sp.steps;
  double dif = 0, worst = 0;
  for (int64_t y = e + 1; y < H - e; ++y)
    for (int64_t x = e + 1; x < W - e; ++x) {
      const size_t i = (size_t)(y * W + x);
      const double d = fabs((double)gold[i] - (double)out[i]);
      dif += d;
      worst = fmax(worst, d / fmax((double)mag[i], 1e-300));
    }
  if (sp.steps == 1) {
    printf("verify dif =%f\n", dif);
  } else {
    const double avg = dif / ((double)(W - F + 1) * (double)(H - F + 1));
    printf("verify dif =%e, precision=%e\n", dif, avg);
  }
  const double tol = (sizeof(T) == 8 ? 1e-12 : 1e-5) * sp.steps;
  printf("check: band of %lld x %lld cells, max relative error %.3e (bound %.1e)\n",
         (long long)(W - 2 * e - 1 > 0 ? W - 2 * e - 1 : 0),
         (long long)(H - 2 * e - 1 > 0 ? H - 2 * e - 1 : 0), worst, tol);
  if (worst > tol) {
    printf("FAILED\n");
    return -1;
  }
  return 0;
}

}  // namespace

#define SSAI_ENTRY(name, table, shape, steps, input, redraw)                   \
  int stencil_##name##pt_float(int argc, char** argv) {                       \
    return run<float>(argc, argv, Spec{table, shape, steps, input, redraw});  \
  }                                                                           \
  int stencil_##name##pt_double(int argc, char** argv) {                      \
    return run<double>(argc, argv, Spec{table, shape, steps, input, redraw}); \
  }

SSAI_ENTRY(5, "star1", SSAM_STAR, 1, ROW_INDEX, true)
SSAI_ENTRY(9, "star2", SSAM_STAR, 1, RAND_256, false)
SSAI_ENTRY(13, "star3", SSAM_STAR, 1, RAND_256, false)
SSAI_ENTRY(17, "star4", SSAM_STAR, 1, RAND_256, false)
SSAI_ENTRY(21, "star5", SSAM_STAR, 1, RAND_256, false)
SSAI_ENTRY(25, "star6", SSAM_STAR, 1, RAND_256, false)
SSAI_ENTRY(64, "box64", SSAM_BOX, 1, RAND_256, false)
SSAI_ENTRY(81, "box81", SSAM_BOX, 1, RAND_256, false)
SSAI_ENTRY(121, "box121", SSAM_BOX, 1, RAND_256, false)
SSAI_ENTRY(tmp_5, "tmp5", SSAM_STAR, 5, RAND_UNIT, false)
SSAI_ENTRY(tmp_9, "tmp9", SSAM_STAR, 3, RAND_UNIT, false)

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
