// Host-side launcher of the 3D z-marching kernel, one template instance per
// compiled configuration, and the registrar through which the generated
// instantiation units add configurations to the library's 3D table.
#pragma once

#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "stencil3d_t2.cuh"

namespace ssam {

// The driver's tensor-map encoder (NULL if the driver does not provide it).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

template <typename TS> CUtensorMapDataType tma_dtype();
template <> inline CUtensorMapDataType tma_dtype<float>() {
  return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
}
template <> inline CUtensorMapDataType tma_dtype<double>() {
  return CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
}
template <> inline CUtensorMapDataType tma_dtype<__nv_bfloat16>() {
  return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}
template <> inline CUtensorMapDataType tma_dtype<__half>() {
  return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
}

struct Launch3D {
  const void* src;
  void* dst;
  int64_t nx, ny, nz;
  int nb;              // grids stacked along a 4th axis (1 = plain 3D grid)
  const void* rhs;     // NULL, or out += rhs_scale * rhs
  double rhs_scale;
  const double* coef;  // (2R+1)^3, [dz][dy][dx]
  int boundary;
  cudaStream_t stream;
  bool prepare_only;  // resolve attributes/occupancy/symbols, launch nothing
};

// Dynamic shared memory of a 3D CTA and the rows a column tile stores: those
// of Stencil3DCfg for single-step launches, of Stencil3DT2Cfg (tiles that
// overlap by 2R rows) for two-step ones.
template <int T_, typename TS, int SH, int R, int PY, int NW, int S, int V_>
struct Geom3D {
  static constexpr int SMEM = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::SMEM;
  static constexpr int TYS = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::TY;
};
template <typename TS, int SH, int R, int PY, int NW, int S, int V_>
struct Geom3D<2, TS, SH, R, PY, NW, S, V_> {
  static constexpr int SMEM = Stencil3DT2Cfg<TS, SH, R, PY, NW, S, V_>::SMEM;
  static constexpr int TYS = Stencil3DT2Cfg<TS, SH, R, PY, NW, S, V_>::OY;
};

// ZREG: the kernel of stencil3d_zreg.cuh (own cells in a register ring
// along z) instead of stencil3d_kernel.  T_ = 2: the kernel of
// stencil3d_t2.cuh, two time steps per launch (no right-hand side).
template <typename TS, int SH, int R, int PY, int NW, int S, bool RHS = false,
          bool ZREG = false, int V_ = 4, int T_ = 1>
int launch_3d(const Launch3D& a) {
  static_assert(T_ == 1 || (T_ == 2 && !RHS && !ZREG), "fused launches: two steps, no rhs");
  using C = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>;
  using TA = typename C::TA;
  auto kern = [] {
    if constexpr (T_ == 2) return &stencil3d_t2_kernel<TS, SH, R, PY, NW, S, V_>;
    else if constexpr (ZREG) return &stencil3d_zreg_kernel<TS, SH, R, PY, NW, S, RHS, V_>;
    else return &stencil3d_kernel<TS, SH, R, PY, NW, S, RHS, V_>;
  }();
  // dynamic shared memory, rows stored per column tile, input planes staged
  // beyond each end of a z chunk
  constexpr int SMEM = Geom3D<T_, TS, SH, R, PY, NW, S, V_>::SMEM;
  constexpr int TYS = Geom3D<T_, TS, SH, R, PY, NW, S, V_>::TYS;
  constexpr int ZR = T_ * R;
  if ((a.rhs != nullptr) != RHS)
    return fail(SSAM_ERR_INVALID, "3D kernel instance does not match the right-hand side");
  static std::mutex mu;
  static std::map<int, int> ctas_per_sm;  // per device
  int dev = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  int bps, sms;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = ctas_per_sm.find(dev);
    if (it == ctas_per_sm.end()) {
      SSAM_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         SMEM));
      int b = 0;
      SSAM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, C::THREADS,
                                                                  SMEM));
      if (b < 1) return fail(SSAM_ERR_UNSUPPORTED, "3D kernel does not fit on an SM");
      it = ctas_per_sm.emplace(dev, b).first;
    }
    bps = it->second;
  }
  SSAM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  const size_t es = sizeof(TS);
  Work3D w;
  w.nx = a.nx;
  w.ny = a.ny;
  w.nz = a.nz;
  w.nb = a.nb;
  w.rhs = a.rhs;
  w.rhs_scale = a.rhs_scale;
  w.ntx = (int)((a.nx + C::TX - 1) / C::TX);
  w.nty = (int)((a.ny + TYS - 1) / TYS);
  // z chunk: minimise (rounds of items) x (chunk + the 2*T*R planes staged
  // beyond its ends; a fused launch also forms 2R extra level-1 planes)
  const int64_t grid_max = (int64_t)sms * bps;
  const int64_t ntiles = (int64_t)w.ntx * w.nty;
  int64_t best = -1;
  for (int zc : {8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 384, 512}) {
    if (zc > 2 * a.nz && zc > 8) break;
    const int64_t items = ntiles * ((a.nz + zc - 1) / zc) * a.nb;
    const int64_t rounds = (items + grid_max - 1) / grid_max;
    const int64_t cost = rounds * (T_ * std::min<int64_t>(zc, a.nz) + 2 * ZR);
    if (best < 0 || cost < best) {
      best = cost;
      w.zc = zc;
      w.items = items;
    }
  }
  const int64_t grid = std::min(w.items, grid_max);
  w.boundary = a.boundary;
  w.wait_ns = 1000ull * 1000ull * 1000ull;  // 1 s per wait; healthy waits take microseconds
  int st = device_error_word(&w.err);
  if (st != SSAM_OK) return st;
  if (a.prepare_only) return SSAM_OK;

  CUtensorMap map;
  memset(&map, 0, sizeof(map));
  w.use_tma = ((uintptr_t)a.src % 16 == 0) && ((a.nx * (int64_t)es) % 16 == 0) &&
              a.nx <= (int64_t(1) << 32) && tensor_map_encoder() != nullptr;
  if (w.use_tma) {
    cuuint64_t dims[4] = {(cuuint64_t)a.nx, (cuuint64_t)a.ny, (cuuint64_t)a.nz,
                          (cuuint64_t)a.nb};
    cuuint64_t strides[3] = {(cuuint64_t)(a.nx * es), (cuuint64_t)(a.nx * a.ny * es),
                             (cuuint64_t)(a.nx * a.ny * a.nz * es)};
    cuuint32_t box[4] = {(cuuint32_t)C::BW, (cuuint32_t)C::YW, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = tensor_map_encoder()(&map, tma_dtype<TS>(), 4, const_cast<void*>(a.src), dims,
                             strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) w.use_tma = 0;  // fall back to plain loads
  }
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  // programmatic dependent launch: this grid's set-up may overlap the tail
  // of the launch before it (pdl_wait_then_release in the kernel)
  SSAM_CUDA_TRY(launch_pdl(kern, dim3((unsigned)grid), dim3(C::THREADS), SMEM, a.stream, map,
                           (const TS*)a.src, (TS*)a.dst, w, cf));
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(a.stream, &cap);
  if (cap == cudaStreamCaptureStatusNone) count_launch();  // graphs count at replay
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

using LaunchFn3D = int (*)(const Launch3D&);

// One compiled configuration of a 3D stencil: rows per consumer warp (PY),
// consumer warps per CTA (NW; the column tile is 32*V x NW*PY), ring slots
// (S planes of the tile in shared memory), the kernel variant, the columns a
// thread (V) and the time steps one launch applies (t).  `dflt` marks the
// configuration used when nothing was measured for the grid's size class.
struct Cand3D {
  LaunchFn3D fn;
  int py, nw, s;
  int zreg;  // 1: own cells in a register ring along z (stencil3d_zreg.cuh)
  int v;     // columns a thread (the tile is 32*v columns)
  bool dflt;
  int t;     // time steps per launch (2: stencil3d_t2.cuh)
};

// Adds a configuration to the table of (dtype, shape, radius, rhs term,
// steps per launch).
void register_3d(int dtype, int shape, int r, bool rhs, const Cand3D& c);

template <typename TS, int SH, int R, int PY, int NW, int S, bool RHS, bool DEFAULT,
          bool ZREG = false, int V_ = 4, int T_ = 1>
struct Register3D {
  Register3D() {
    register_3d(Traits<TS>::DT, SH, R, RHS,
                Cand3D{&launch_3d<TS, SH, R, PY, NW, S, RHS, ZREG, V_, T_>, PY, NW, S,
                       ZREG ? 1 : 0, V_, DEFAULT, T_});
  }
};

}  // namespace ssam
