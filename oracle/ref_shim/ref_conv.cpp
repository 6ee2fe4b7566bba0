// ORACLE BUILD SHIM -- test infrastructure only.
// Compiles the reference's own CPU golden `Convolution<T>`
// (ssai-2dconv/common.h:186-216), included in place from the read-only
// reference tree, and exports it with C linkage for the parity tests and the
// CPU baseline.  Output goes to oracle/_ref/ only.
#include <cmath>
#include <cstring>
#include "ssai-2dconv/common.h"

extern "C" {
void ssam_ref_convolution_f32(const float* src, float* dst, int w, int h,
                              const float* filter, int fw, int fh) {
  Convolution<float>(src, dst, w, h, filter, fw, fh);
}
void ssam_ref_convolution_f64(const double* src, double* dst, int w, int h,
                              const double* filter, int fw, int fh) {
  Convolution<double>(src, dst, w, h, filter, fw, fh);
}
}
