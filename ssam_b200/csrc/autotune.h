// Launch-parameter choice for the 2D kernels: built-in defaults, plus a
// cache of measured choices filled by the autotuner (ssam_autotune_* in the C
// ABI) and optionally persisted to a text file.
#pragma once

#include <stdint.h>

namespace ssam {

struct TuneChoice {
  int p;      // output rows per thread (template P)
  int warps;  // warps per block
  int v;      // columns per thread (template V; warp strip = 32*V columns)
};

// Measured choice for this stencil, fused depth and grid size, if any.
bool tune_lookup_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t,
                    int64_t w, int64_t h, TuneChoice* out);
// Static choice used when nothing was measured.
TuneChoice tune_default_2d(int dtype, int rl, int rr, int rt, int rb, int star, int t);
// Largest number of steps to fuse in one launch for a `steps`-step run.
int tune_depth_2d(int dtype, int rl, int rr, int rt, int rb, int star, int64_t w,
                  int64_t h, int steps);

// The 3D autotuner's measured choices (stencil3d.cu): key = (dtype, shape,
// radius, rhs, log2 nx, log2 ny, log2 nz*nbatch, steps per launch), value =
// (PY, NW, S, zreg, V); and the temporal depth of multi-step runs, key =
// (dtype, shape, radius, log2 nx, log2 ny, log2 nz), value = steps per launch.
void tune3d_for_each(void (*cb)(const int key[8], const int val[5], void*), void* user);
void tune3d_store(const int key[8], const int val[5]);
void depth3d_for_each(void (*cb)(const int key[6], int depth, void*), void* user);
void depth3d_store(const int key[6], int depth);
void tune3d_clear();

}  // namespace ssam
