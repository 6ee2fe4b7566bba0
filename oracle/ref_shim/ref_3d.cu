// ORACLE BUILD SHIM -- test infrastructure only.
// Compiles one of the reference's 3D programs (chosen by REF_3D_FILE) as a
// host translation unit and exports its CPU golden for the grid sizes listed
// below (the golds take the size as a template argument _N).  Standard headers
// come first because the reference files #define max/min/ceil.  Nothing from
// the file runs on a GPU.
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>
#include REF_3D_FILE

#define SSAM_REF_SIZES(X) X(8) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(96) X(128) X(256) X(512)

#define SSAM_CASE(NN) case NN: GOLD<T, NN>(in, out, NN); return 0;
template <typename T>
static int run_gold(const T* in, T* out, int n) {
  switch (n) { SSAM_REF_SIZES(SSAM_CASE) default: return -1; }
}

extern "C" {
int REF_EXPORT_F32(const float* in, float* out, int n) { return run_gold<float>(in, out, n); }
int REF_EXPORT_F64(const double* in, double* out, int n) { return run_gold<double>(in, out, n); }
}
