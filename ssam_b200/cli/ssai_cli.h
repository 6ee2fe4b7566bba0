// Shared pieces of the command-line drop-ins for the reference's three
// programs (ssai-2dstencil, ssai-2dconv, ssai-3dstencil): argument echo,
// seeded inputs, device buffers, CUDA-event timing and a sampled host check.
// The programs keep the reference's argv spelling; every stencil runs through
// the C ABI in include/ssam.h (no kernel lives here).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <random>
#include <vector>

#include "ssam.h"

namespace ssai {

inline void echo_args(int argc, char** argv) {
  for (int i = 0; i < argc; ++i) printf("%s%s", argv[i], i == argc - 1 ? "\n" : " ");
}

inline int check(int st, const char* what) {
  if (st != SSAM_OK) {
    fprintf(stderr, "%s failed: %s\n", what, ssam_last_error());
    exit(2);
  }
  return st;
}

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
    exit(2);
  }
}

// Coefficients uniform[0,1) normalised to sum 1, seeded.
inline std::vector<double> coefficients(size_t count, uint64_t seed) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::vector<double> c(count);
  double s = 0;
  for (auto& v : c) s += (v = u(g));
  for (auto& v : c) v /= s;
  return c;
}

template <typename T>
std::vector<T> uniform(size_t count, uint64_t seed) {
  std::mt19937_64 g(seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  std::vector<T> v(count);
  for (auto& x : v) x = (T)u(g);
  return v;
}

// A raw 8-bit image of `count` pixels (the reference conv driver's
// ../data/Lena<W>x<H>.raw, read by DataT::Load_uchar, ssai-2dconv/common.h:
// 151-178) as values of T; false when the file is missing or short.
template <typename T>
bool load_raw_uchar(const char* path, size_t count, std::vector<T>* out) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  std::vector<unsigned char> px(count);
  const size_t got = fread(px.data(), 1, count, f);
  fclose(f);
  if (got != count) return false;
  out->resize(count);
  for (size_t i = 0; i < count; ++i) (*out)[i] = (T)px[i];
  return true;
}

// Device copy of a host vector, the result buffer and a timed launch.
template <typename T>
struct DeviceRun {
  T* src = nullptr;
  T* dst = nullptr;
  size_t count;
  explicit DeviceRun(const std::vector<T>& in) : count(in.size()) {
    cuda_check(cudaMalloc(&src, count * sizeof(T)), "cudaMalloc");
    cuda_check(cudaMalloc(&dst, count * sizeof(T)), "cudaMalloc");
    cuda_check(cudaMemcpy(src, in.data(), count * sizeof(T), cudaMemcpyHostToDevice),
               "cudaMemcpy");
  }
  ~DeviceRun() {
    cudaFree(src);
    cudaFree(dst);
  }
  // mean milliseconds of `reps` calls of f() after one warm-up call
  template <typename F>
  double time_ms(F f, int reps) {
    f();
    cuda_check(cudaDeviceSynchronize(), "warm-up");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    for (int i = 0; i < reps; ++i) f();
    cudaEventRecord(b);
    cuda_check(cudaEventSynchronize(b), "timed calls");
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / reps;
  }
  std::vector<T> result() const {
    std::vector<T> out(count);
    cuda_check(cudaMemcpy(out.data(), dst, count * sizeof(T), cudaMemcpyDeviceToHost),
               "cudaMemcpy");
    return out;
  }
};

template <typename T>
constexpr int dtype() {
  return sizeof(T) == 8 ? SSAM_F64 : SSAM_F32;
}

}  // namespace ssai
