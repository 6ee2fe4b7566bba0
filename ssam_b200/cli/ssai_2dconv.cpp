// ssai-2dconv <float|double> <size> <fsize>
//
// Drop-in for the reference's convolution program (ssai-2dconv/conv2D.cu:
// 175-246: data type in argv[1], square grid size in argv[2] (default 8192),
// square filter size 2..28 in argv[3] (default 3)).  Reads the reference's
// 8-bit input image ../data/Lena<size>x<size>.raw when it exists (else seeds
// the grid), seeds the filter, runs ssam_conv2d on the GPU (zero padding,
// offsets x + m - fw/2 and y + n - fh/2 like the reference), prints the kernel
// time and GCells/s, and checks 4096 sampled cells against a direct
// evaluation in double.
#include "ssai_cli.h"

namespace {

template <typename T>
int run(int argc, char** argv) {
  int size = 8192, fsize = 3;
  if (argc >= 3) size = atoi(argv[2]);
  if (argc >= 4) fsize = atoi(argv[3]);
  if (size < 1 || fsize < 1 || fsize > 28) {
    fprintf(stderr, "bad size / fsize\n");
    return 1;
  }
  const int64_t W = size, H = size;
  const std::vector<double> w = ssai::coefficients((size_t)fsize * fsize, 13);
  // the reference's input image when it is there (conv2D.cu:88-104), else
  // seeded data
  std::vector<T> in;
  char path[256];
  snprintf(path, sizeof path, "../data/Lena%dx%d.raw", size, size);
  if (ssai::load_raw_uchar<T>(path, (size_t)W * H, &in)) {
    printf("Load success : %s\n", path);
  } else {
    printf("Load failed : %s, generate random data\n", path);
    in = ssai::uniform<T>((size_t)W * H, 7);
  }
  ssai::DeviceRun<T> dev(in);
  auto call = [&] {
    ssai::check(ssam_conv2d(dev.src, dev.dst, W, W, H, ssai::dtype<T>(), w.data(), fsize, fsize,
                            SSAM_BOUNDARY_ZERO, nullptr),
                "ssam_conv2d");
  };
  const double ms = dev.time_ms(call, 10);
  const std::vector<T> out = dev.result();
  printf("%dx%d, %dx%d filter: %.4f ms, %.2f GCells/s\n", size, size, fsize, fsize, ms,
         (double)W * H / (ms * 1e-3) / 1e9);
  std::mt19937_64 rng(3);
  double worst = 0;
  for (int k = 0; k < 4096; ++k) {
    const int64_t y = rng() % H, x = rng() % W;
    double want = 0;
    for (int n = 0; n < fsize; ++n)
      for (int m = 0; m < fsize; ++m) {
        const int64_t yy = y + n - fsize / 2, xx = x + m - fsize / 2;
        if (yy >= 0 && yy < H && xx >= 0 && xx < W) want += w[n * fsize + m] * in[yy * W + xx];
      }
    worst = fmax(worst, fabs((double)out[(size_t)y * W + x] - want) / fmax(fabs(want), 1e-30));
  }
  printf("check: 4096 sampled cells, max relative error %.3e\n", worst);
  const double tol = sizeof(T) == 8 ? 1e-12 : 1e-5;
  if (worst > tol) {
    printf("FAILED (tolerance %.1e)\n", tol);
    return -1;
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  ssai::echo_args(argc, argv);
  if (argc < 2) {
    printf("usage: %s <float|double> [size] [fsize]\n", argv[0]);
    return 1;
  }
  return strcmp(argv[1], "float") == 0 ? run<float>(argc, argv) : run<double>(argc, argv);
}
