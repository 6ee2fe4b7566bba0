// Internal declarations shared by the CUDA translation units of
// libssam_b200.so: status plumbing, storage-type traits, 128-bit row
// loads/stores, and the kernel registry that the C ABI dispatches through.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <string>
#include <type_traits>

#include "../../include/ssam.h"

namespace ssam {

// ------------------------------------------------------------------ status --

// Records `msg` as the calling thread's last error and returns `st`.
int fail(int st, const std::string& msg);
// Maps a CUDA error to SSAM_ERR_CUDA with the runtime's message.
int fail_cuda(cudaError_t e, const char* what);

// Process-wide count of kernel launches (ssam_kernel_launches).
void count_launch();

// 3D path (stencil3d.cu).  shape: 0 = star, 1 = 19-point.
int run_3d(const void* src, void* dst, int64_t nx, int64_t ny, int64_t nz, int dtype,
           int shape, int r, const double* coef, int steps, int boundary, int use_graph,
           cudaStream_t stream);
int device_error_word(int** out);
int sweep_3d(const void* in, void* out, int64_t n, int nb, int dtype, const double* cube,
             const void* rhs, double rhs_scale, cudaStream_t s);

// Stream-ordered device scratch from the library's per-device pool.
int scratch_alloc(void** p, size_t bytes, cudaStream_t s);
void scratch_free(void* p, cudaStream_t s);

#define SSAM_CUDA_TRY(expr)                                \
  do {                                                       \
    cudaError_t _e = (expr);                                 \
    if (_e != cudaSuccess) return ::ssam::fail_cuda(_e, #expr); \
  } while (0)

// ------------------------------------------------------------ dtype traits --

// TA = accumulation type, V = default number of columns a thread owns along
// x (16 or 32 bytes); the 2D kernels are also compiled for other widths.
template <typename TS> struct Traits;
template <> struct Traits<float> {
  using TA = float;
  static constexpr int V = 4;
  static constexpr int DT = SSAM_F32;
};
template <> struct Traits<double> {
  using TA = double;
  static constexpr int V = 4;
  static constexpr int DT = SSAM_F64;
};
template <> struct Traits<__nv_bfloat16> {
  using TA = float;
  static constexpr int V = 8;
  static constexpr int DT = SSAM_BF16;
};
template <> struct Traits<__half> {
  using TA = float;
  static constexpr int V = 8;
  static constexpr int DT = SSAM_F16;
};

inline size_t dtype_size(int dt) {
  return dt == SSAM_F64 ? 8 : (dt == SSAM_F32 ? 4 : 2);
}

__device__ __forceinline__ float to_acc(float v) { return v; }
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ float to_acc(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_acc(__half v) { return __half2float(v); }

template <typename TS> __device__ __forceinline__ TS from_acc(float v);
template <> __device__ __forceinline__ float from_acc<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_acc<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <> __device__ __forceinline__ __half from_acc<__half>(float v) {
  return __float2half_rn(v);
}
template <typename TS> __device__ __forceinline__ TS from_acc(double v);
template <> __device__ __forceinline__ double from_acc<double>(double v) { return v; }

// N elements of storage held as N * sizeof(TS) / 4 whole 32-bit words, to
// accumulator values and back.  A 16-bit word pair holds the element of the
// lower address in its low half.  Widening BF16 is exact bit placement (a
// bf16 is the upper half of the fp32 of the same value: one shift or one mask
// an element); narrowing rounds both halves to nearest even in one paired
// conversion.  The values are those of the per-element conversions.
template <typename TS, int N, typename TA>
__device__ __forceinline__ void words_to_acc(TA* d, const uint32_t* w) {
  if constexpr (std::is_same<TS, __nv_bfloat16>::value) {
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      d[2 * k] = __uint_as_float(w[k] << 16);
      d[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
    }
  } else if constexpr (std::is_same<TS, __half>::value) {
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      __half2 h;
      memcpy(&h, &w[k], 4);
      const float2 f = __half22float2(h);
      d[2 * k] = f.x;
      d[2 * k + 1] = f.y;
    }
  } else {
    TS e[N];
    memcpy(e, w, sizeof(e));
#pragma unroll
    for (int k = 0; k < N; ++k) d[k] = to_acc(e[k]);
  }
}

template <typename TS, int N, typename TA>
__device__ __forceinline__ void acc_to_words(uint32_t* w, const TA* d) {
  if constexpr (std::is_same<TS, __nv_bfloat16>::value) {
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(d[2 * k], d[2 * k + 1]);
      memcpy(&w[k], &h, 4);
    }
  } else if constexpr (std::is_same<TS, __half>::value) {
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const __half2 h = __floats2half2_rn(d[2 * k], d[2 * k + 1]);
      memcpy(&w[k], &h, 4);
    }
  } else {
    TS e[N];
#pragma unroll
    for (int k = 0; k < N; ++k) e[k] = from_acc<TS>(d[k]);
    memcpy(w, e, sizeof(e));
  }
}

// V consecutive elements starting at a 16-byte aligned address, as 16-byte
// (128-bit) transactions.
template <typename TS, int V, typename TA>
__device__ __forceinline__ void load_vec(TA (&r)[V], const TS* __restrict__ p) {
  static_assert((V * sizeof(TS)) % 16 == 0, "whole 16-byte chunks");
  constexpr int CH = V * sizeof(TS) / 16;
  constexpr int PER = 16 / sizeof(TS);
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    const uint4 u = __ldg(reinterpret_cast<const uint4*>(p) + c);
    const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
    words_to_acc<TS, PER>(r + c * PER, wd);
  }
}

template <typename TS, int V, typename TA>
__device__ __forceinline__ void store_vec(TS* __restrict__ p, const TA (&r)[V]) {
  constexpr int CH = V * sizeof(TS) / 16;
  constexpr int PER = 16 / sizeof(TS);
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    uint32_t wd[4];
    acc_to_words<TS, PER>(wd, r + c * PER);
    reinterpret_cast<uint4*>(p)[c] = make_uint4(wd[0], wd[1], wd[2], wd[3]);
  }
}

// Programmatic dependent launch.  The 2D and 3D stencil kernels are
// launched with cudaLaunchAttributeProgrammaticStreamSerialization
// (launch_pdl), so that a launch may begin while the launch before it in the
// stream is finishing.  Every thread of such a kernel calls this before its
// first global memory access (the 3D kernels after their shared-memory
// set-up): the wait returns once the previous grid has completed and its
// writes are visible (at once when there is none), and the release then lets
// the next launch of the stream start on SMs this grid frees.
__device__ __forceinline__ void pdl_wait_then_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t stream, Args&&... args) {
  cudaLaunchConfig_t lc;
  memset(&lc, 0, sizeof(lc));
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = stream;
  cudaLaunchAttribute la[1];
  la[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  la[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = la;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, kern, static_cast<Args&&>(args)...);
}

// Coefficients passed by value as a kernel parameter (constant bank), indexed
// with compile-time offsets by the unrolled kernels.
template <typename TA, int N>
struct CoefBlock {
  TA c[N];
};

// One tap of the own-column part of a 2D stencil row: acc[j] += w * row[j+dx]
// for every j with 0 <= j + dx < V (dx is a constant once the caller's tap
// loop is unrolled).  For a float accumulator and an even dx the columns go
// in pairs through the packed two-lane FP32 FMA (FFMA2): each lane is rounded
// like a scalar fma, so every sum keeps its bits and its order, with half the
// FMA instructions.  An odd dx would pair registers across a pair boundary,
// which costs a move per lane, so it stays scalar.  PAIR = false keeps every
// tap scalar: the paired form holds more registers, which costs the
// row-streaming tiles of bandwidth-bound stencils more occupancy than the
// saved instructions are worth (see pair_taps).
template <int V, bool PAIR = true, typename TA>
__device__ __forceinline__ void tap_row(TA (&acc)[V], TA w, const TA* row, int dx) {
  if constexpr (PAIR && std::is_same<TA, float>::value && V % 2 == 0) {
    if ((dx & 1) == 0) {
      const float2 w2 = make_float2(w, w);
#pragma unroll
      for (int j = 0; j < V; j += 2) {
        if (j + dx < 0 || j + dx >= V) continue;  // both lanes of the pair leave together
        float2 a = make_float2(acc[j], acc[j + 1]);
        a = __ffma2_rn(w2, make_float2(row[j + dx], row[j + dx + 1]), a);
        acc[j] = a.x;
        acc[j + 1] = a.y;
      }
      return;
    }
  }
#pragma unroll
  for (int j = 0; j < V; ++j) {
    if (j + dx < 0 || j + dx >= V) continue;
    acc[j] = fma(w, row[j + dx], acc[j]);
  }
}

// Whether the row-streaming tiles pair their taps: only where the stencil
// does at least 8 flop per byte of HBM traffic (2*taps-1 flop per cell
// against a read and a write of the storage type), i.e. where the FMA pipe
// and not HBM bounds the tile.  Measured on 8192^2 grids: BF16 5x5 box
// 637 -> 724 GCells/s paired; the FP32 5x5 box and 13-point star lost 15 %
// paired (more registers, fewer warps in flight).
template <typename TS, int TAPS>
__host__ __device__ constexpr bool pair_taps() {
  return 2 * TAPS - 1 >= 16 * (int)sizeof(TS);
}

// ---------------------------------------------------------- kernel registry --

// One compiled 2D stencil kernel: radii left/right/top/bottom, tap pattern,
// outputs per thread along y (P), fused time steps (T), columns per thread (V).
struct Key2D {
  int dtype, rl, rr, rt, rb, star, p, t, v;
  bool operator<(const Key2D& o) const;
  bool operator==(const Key2D& o) const;
};

struct Launch2D {
  const void* src;
  void* dst;
  int64_t width, height, pitch;
  int64_t y_begin, y_end;  // rows of the grid this launch writes
  int boundary;
  const double* coef;  // (rt+rb+1) x (rl+rr+1) row-major, host
  int warps_per_block;
  cudaStream_t stream;
};

using LaunchFn2D = cudaError_t (*)(const Launch2D&);

struct Kernel2DInfo {
  LaunchFn2D launch;
  const void* func;  // the __global__ symbol, for occupancy queries
  int vec;           // elements per thread along x
};

// A chosen kernel and block size for one launch.
struct Plan2D {
  Key2D key;
  const Kernel2DInfo* info;
  int warps;
};

void register_2d(const Key2D& k, const Kernel2DInfo& info);
const Kernel2DInfo* find_2d(const Key2D& k);
// All registered kernels matching dtype/radii/shape (any P, T).
void list_2d(int dtype, int rl, int rr, int rt, int rb, int star,
             void (*cb)(const Key2D&, const Kernel2DInfo&, void*), void* user);

}  // namespace ssam
