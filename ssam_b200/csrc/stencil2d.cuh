// Register-cache systolic 2D stencil / correlation kernel for sm_100a.
//
// The method is SSAM's (Chen et al., SC19; reference kernels
// ssai-2dstencil/stencil2D_*.cu and ssai-2dconv/conv2D.cu:9-70):
//   * every warp loads a strip of the grid plus a redundant halo into
//     thread-private registers (the "register cache");
//   * partial sums are formed where the data lives and moved to the
//     downstream lane with __shfl_*_sync, where they are accumulated;
//   * shared memory is not used.
//
// What is laid out for Blackwell instead of P100/V100:
//   * a thread owns V consecutive columns (V*sizeof(T) = 16 or 32 bytes) and
//     moves them with 128-bit loads/stores; a warp strip is 32*V columns and
//     its tiles start on 16-byte boundaries (the reference strip is one
//     column per lane, 4- or 8-byte accesses);
//   * because a lane holds V columns, partial sums only cross lanes for taps
//     that leave the thread's own columns: per output row the warp exchanges
//     rl + rr partial sums per thread (a systolic chain when a radius exceeds
//     V), for V outputs;
//   * halo lanes: ceil(rl*T/V) on the left, ceil(rr*T/V) on the right, so a
//     warp writes (32 - halo lanes) * V columns;
//   * T time steps are fused in registers (temporal blocking, as
//     stencil2d_temp_5pt.cu:48-65): the register window holds P + (rt+rb)*T
//     rows, each step recomputes it in place and shrinks it by rt+rb rows, and
//     the boundary rule is re-applied to the window after every step;
//   * y blocks are grid-strided, so any height runs with a bounded grid, and
//     a launch may write only the rows [y_begin, y_end) of the grid (the
//     host-buffer entry point pipelines row bands this way).
//
// Template parameters: TS storage type, RL/RR/RT/RB reach to the left, right,
// top (smaller y) and bottom, STAR (only the centre row and column are
// non-zero), P output rows per thread, T fused steps, V columns per thread
// (the warp strip is 32*V columns wide).
#pragma once

#include "ssam_internal.cuh"

namespace ssam {

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int P, int T, int V_>
struct Stencil2DCfg {
  using TA = typename Traits<TS>::TA;
  static constexpr int V = V_;
  static constexpr int FW = RL + RR + 1;
  static constexpr int FH = RT + RB + 1;
  static constexpr int NC = FW * FH;
  static constexpr int HL = (RL * T + V - 1) / V;  // halo lanes, left
  static constexpr int HR = (RR * T + V - 1) / V;  // halo lanes, right
  static constexpr int OUT_LANES = 32 - HL - HR;
  static constexpr int OUT_COLS = OUT_LANES * V;
  static constexpr int ROWS = P + (RT + RB) * T;
  static_assert(OUT_LANES >= 2, "radius too large for one warp strip");
  static_assert((V * sizeof(TS)) % 16 == 0, "a thread owns whole 16-byte chunks");
};

// Boundary rule applied to a value of the register window that sits at
// (y, x): ZERO forces cells outside the grid to 0; COPY restores cells within
// the reach of the edge to the launch input.  (CLAMP is single-step and is
// handled at load time.)
template <typename TS, typename TA>
__device__ __forceinline__ TA fix_cell(TA v, int64_t y, int64_t x, int64_t W,
                                       int64_t H, int64_t pitch, int bnd, int rl,
                                       int rr, int rt, int rb,
                                       const TS* __restrict__ src) {
  const bool outside = (x < 0) | (x >= W) | (y < 0) | (y >= H);
  if (bnd == SSAM_BOUNDARY_ZERO) return outside ? TA(0) : v;
  if (bnd == SSAM_BOUNDARY_COPY && !outside &&
      ((x < rl) | (x >= W - rr) | (y < rt) | (y >= H - rb)))
    return to_acc(src[y * pitch + x]);
  return v;
}

// Row load/store for a lane whose V columns are not all inside [0, W) or not
// 16-byte aligned: per element, with the boundary rule for columns outside.
template <typename TS, int V, typename TA>
__device__ __forceinline__ void load_row_edge(TA (&d)[V], const TS* __restrict__ row,
                                              int64_t x0, int64_t W, int bnd) {
#pragma unroll
  for (int j = 0; j < V; ++j) {
    int64_t x = x0 + j;
    if ((x < 0 || x >= W) && bnd == SSAM_BOUNDARY_ZERO) {
      d[j] = TA(0);
    } else {
      x = x < 0 ? 0 : (x >= W ? W - 1 : x);
      d[j] = to_acc(row[x]);
    }
  }
}
template <typename TS, int V, typename TA>
__device__ __forceinline__ void store_row_edge(TS* __restrict__ row, int64_t x0, int64_t W,
                                               const TA (&d)[V]) {
#pragma unroll
  for (int j = 0; j < V; ++j)
    if (x0 + j < W) row[x0 + j] = from_acc<TS>(d[j]);
}

// One warp's work: the P output rows starting at row y_out0 of the strip
// whose first output column is x_out0, T fused steps, rows >= y_end not
// written.  Shared by the grid kernel below and the persistent batched kernel.
template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int P, int T, int V_>
__device__ __forceinline__ void stencil2d_warp_tile(
    const TS* __restrict__ src, TS* __restrict__ dst, int64_t W, int64_t H, int64_t pitch,
    int64_t x_out0, int64_t y_out0, int64_t y_end, int bnd, int vec_ok,
    const CoefBlock<typename Traits<TS>::TA, Stencil2DCfg<TS, RL, RR, RT, RB, STAR, P, T, V_>::NC>& cf) {
  using C = Stencil2DCfg<TS, RL, RR, RT, RB, STAR, P, T, V_>;
  using TA = typename C::TA;
  constexpr int V = C::V;
  constexpr int FW = C::FW;
  constexpr int ROWS = C::ROWS;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t x0 = x_out0 + (int64_t)(lane - C::HL) * V;
  const bool lane_stores = lane >= C::HL && lane < 32 - C::HR;
  // Does this thread's window touch cells that the boundary rule rewrites?
  const bool x_edge = bnd == SSAM_BOUNDARY_ZERO
                          ? (x0 < 0 || x0 + V > W)
                          : (x0 < RL || x0 + V > W - RR);
  const int64_t y0 = y_out0 - (int64_t)RT * T;
  const bool y_edge = bnd == SSAM_BOUNDARY_ZERO
                          ? (y0 < 0 || y0 + ROWS > H)
                          : (y0 < RT || y0 + ROWS > H - RB);
  const bool edge = x_edge || y_edge;

  // ---- register cache: ROWS rows x V columns, 16-byte loads ----------
  TA d[ROWS][V];
  // Columns of this thread inside the grid?  Then rows are read whole: with
  // 16-byte loads when the grid is 16-byte aligned (vec_ok), else with one
  // load per element.  Separate loops per case: a branch inside one unrolled
  // loop makes the compiler keep every path's loads live (2-4x registers).
  const bool cols_in = x0 >= 0 && x0 + V <= W;
  const bool row_vec = vec_ok && cols_in;
  const bool rows_in = y0 >= 0 && y0 + ROWS <= H;
  if (cols_in && rows_in) {
    const TS* p = src + y0 * pitch + x0;
    if (vec_ok) {
#pragma unroll
      for (int k = 0; k < ROWS; ++k) {
        load_vec<TS, V>(d[k], p);
        p += pitch;
      }
    } else {
#pragma unroll
      for (int k = 0; k < ROWS; ++k) {
#pragma unroll
        for (int j = 0; j < V; ++j) d[k][j] = to_acc(__ldg(p + j));
        p += pitch;
      }
    }
  } else if (cols_in) {
    // rows beyond the top/bottom edge: zero or clamped row
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
      int64_t y = y0 + k;
      if ((y < 0 || y >= H) && bnd == SSAM_BOUNDARY_ZERO) {
#pragma unroll
        for (int j = 0; j < V; ++j) d[k][j] = TA(0);
      } else {
        y = y < 0 ? 0 : (y >= H ? H - 1 : y);
        const TS* p = src + y * pitch + x0;
        if (vec_ok) {
          load_vec<TS, V>(d[k], p);
        } else {
#pragma unroll
          for (int j = 0; j < V; ++j) d[k][j] = to_acc(__ldg(p + j));
        }
      }
    }
  } else if constexpr (T == 1) {
    // columns beyond the left/right edge (edge lanes only): per element from
    // clamped coordinates, zeros outside the grid for ZERO; no branches, so
    // every load can be in flight at once (single-step windows are short
    // enough to keep all of them in registers)
#pragma unroll
    for (int k = 0; k < ROWS; ++k) {
      const int64_t y = y0 + k;
      const bool y_out = y < 0 || y >= H;
      const TS* row = src + (y < 0 ? 0 : (y >= H ? H - 1 : y)) * pitch;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        const int64_t x = x0 + j;
        const bool out = y_out || x < 0 || x >= W;
        const TA v = to_acc(__ldg(row + (x < 0 ? 0 : (x >= W ? W - 1 : x))));
        d[k][j] = (out && bnd == SSAM_BOUNDARY_ZERO) ? TA(0) : v;
      }
    }
  } else {
    // the same for fused multi-step windows, one row at a time (rotated into
    // its static slot), which keeps the register count of the deep windows
#pragma unroll 1
    for (int k = 0; k < ROWS; ++k) {
      int64_t y = y0 + k;
      TA v[V];
      if ((y < 0 || y >= H) && bnd == SSAM_BOUNDARY_ZERO) {
#pragma unroll
        for (int j = 0; j < V; ++j) v[j] = TA(0);
      } else {
        y = y < 0 ? 0 : (y >= H ? H - 1 : y);
        load_row_edge<TS, V>(v, src + y * pitch, x0, W, bnd);
      }
#pragma unroll
      for (int r = 0; r < ROWS - 1; ++r)
#pragma unroll
        for (int j = 0; j < V; ++j) d[r][j] = d[r + 1][j];
#pragma unroll
      for (int j = 0; j < V; ++j) d[ROWS - 1][j] = v[j];
    }
  }

  // ---- T fused steps; step s rewrites rows [0, ROWS-(RT+RB)(s+1)) ----
#pragma unroll
  for (int s = 0; s < T; ++s) {
    constexpr int FH = RT + RB + 1;
    const int n_rows = ROWS - (RT + RB) * (s + 1);
#pragma unroll
    for (int i = 0; i < ROWS - (RT + RB); ++i) {
      if (i >= n_rows) break;
      TA acc[V];
#pragma unroll
      for (int j = 0; j < V; ++j) acc[j] = TA(0);
      // own columns
#pragma unroll
      for (int dy = -RT; dy <= RB; ++dy) {
#pragma unroll
        for (int dx = -RL; dx <= RR; ++dx) {
          if (STAR && dy != 0 && dx != 0) continue;
          tap_row<V>(acc, cf.c[(dy + RT) * FW + (dx + RL)], d[i + RT + dy], dx);
        }
      }
      // partial sums travelling right: virtual column V+q, q < RL
      if constexpr (RL > 0) {
        TA pr[RL];
#pragma unroll
        for (int q = 0; q < RL; ++q) {
          pr[q] = TA(0);
#pragma unroll
          for (int dy = -RT; dy <= RB; ++dy) {
            if (STAR && dy != 0) continue;
#pragma unroll
            for (int j = 0; j < V; ++j) {
              const int dx = j - V - q;  // source column minus destination
              if (dx < -RL || dx > -1) continue;
              pr[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], d[i + RT + dy][j], pr[q]);
            }
          }
        }
        constexpr int K = (RL + V - 1) / V;
#pragma unroll
        for (int st = K - 1; st >= 0; --st) {
#pragma unroll
          for (int q = st * V; q < (st + 1) * V && q < RL; ++q) {
            const TA v = __shfl_up_sync(FULL, pr[q], 1);
            if (st == 0) acc[q] += v;
            else pr[q - V] += v;
          }
        }
      }
      // partial sums travelling left: virtual column -1-q, q < RR
      if constexpr (RR > 0) {
        TA pl[RR];
#pragma unroll
        for (int q = 0; q < RR; ++q) {
          pl[q] = TA(0);
#pragma unroll
          for (int dy = -RT; dy <= RB; ++dy) {
            if (STAR && dy != 0) continue;
#pragma unroll
            for (int j = 0; j < V; ++j) {
              const int dx = j + 1 + q;
              if (dx < 1 || dx > RR) continue;
              pl[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], d[i + RT + dy][j], pl[q]);
            }
          }
        }
        constexpr int K = (RR + V - 1) / V;
#pragma unroll
        for (int st = K - 1; st >= 0; --st) {
#pragma unroll
          for (int q = st * V; q < (st + 1) * V && q < RR; ++q) {
            const TA v = __shfl_down_sync(FULL, pl[q], 1);
            if (st == 0) acc[V - 1 - q] += v;
            else pl[q - V] += v;
          }
        }
      }
      (void)FH;
      if (T > 1) {
        // the window row i now holds grid row y0 + RT*(s+1) + i
        if (edge) {
          const int64_t y = y0 + (int64_t)RT * (s + 1) + i;
#pragma unroll
          for (int j = 0; j < V; ++j)
            acc[j] = fix_cell<TS, TA>(acc[j], y, x0 + j, W, H, pitch, bnd, RL,
                                      RR, RT, RB, src);
        }
#pragma unroll
        for (int j = 0; j < V; ++j) d[i][j] = acc[j];
      } else {
        // single step: keep the result in place of row i (row i is not
        // read again), centre value d[i+RT] is still intact for COPY.
        if (bnd == SSAM_BOUNDARY_COPY && edge) {
          const int64_t y = y_out0 + i;
#pragma unroll
          for (int j = 0; j < V; ++j) {
            const int64_t x = x0 + j;
            if ((x < RL) | (x >= W - RR) | (y < RT) | (y >= H - RB))
              acc[j] = d[i + RT][j];
          }
        }
#pragma unroll
        for (int j = 0; j < V; ++j) d[i][j] = acc[j];
      }
    }
  }

  // ---- store P rows from the strip's interior lanes ------------------
  if (lane_stores) {
    TS* p = dst + y_out0 * pitch;
#pragma unroll
    for (int i = 0; i < P; ++i) {
      if (y_out0 + i < y_end) {
        if (row_vec) {
          store_vec<TS, V>(p + x0, d[i]);
        } else if (cols_in) {
#pragma unroll
          for (int j = 0; j < V; ++j) p[x0 + j] = from_acc<TS>(d[i][j]);
        } else {
          store_row_edge<TS, V>(p, x0, W, d[i]);
        }
      }
      p += pitch;
    }
  }
}

// The FP32 25-point star (4-column tiles) is bounded to 128 registers (two
// 256-thread blocks' worth a SM): 16 warps a SM instead of 12 hide more of
// its latency -- 8192^2, 417-427 -> 468 GCells/s -- for 24 bytes of spill.
template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int P, int T, int V_>
__global__ void __launch_bounds__(256, (STAR && RL >= 6 && sizeof(TS) == 4 && V_ == 4) ? 2 : 1)
stencil2d_kernel(const TS* __restrict__ src, TS* __restrict__ dst, int64_t W,
                 int64_t H, int64_t pitch, int64_t y_begin, int64_t y_end, int bnd,
                 int vec_ok,
                 CoefBlock<typename Traits<TS>::TA,
                           Stencil2DCfg<TS, RL, RR, RT, RB, STAR, P, T, V_>::NC> cf) {
  using C = Stencil2DCfg<TS, RL, RR, RT, RB, STAR, P, T, V_>;
  pdl_wait_then_release();
  const int64_t warp_x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t x_out0 = warp_x * C::OUT_COLS;
  if (x_out0 >= W) return;  // whole warp leaves together
  const int64_t nby = (y_end - y_begin + P - 1) / P;
  for (int64_t by = blockIdx.y; by < nby; by += gridDim.y)
    stencil2d_warp_tile<TS, RL, RR, RT, RB, STAR, P, T, V_>(
        src, dst, W, H, pitch, x_out0, y_begin + by * P, y_end, bnd, vec_ok, cf);
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int P, int T, int V_>
cudaError_t launch_stencil2d(const Launch2D& a) {
  using C = Stencil2DCfg<TS, RL, RR, RT, RB, STAR, P, T, V_>;
  using TA = typename C::TA;
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  const int nw = a.warps_per_block;
  const int64_t warps_x = (a.width + C::OUT_COLS - 1) / C::OUT_COLS;
  const int64_t nby = (a.y_end - a.y_begin + P - 1) / P;
  dim3 grid((unsigned)((warps_x + nw - 1) / nw), (unsigned)(nby < 65535 ? nby : 65535));
  const int vec_ok = ((uintptr_t)a.src % 16 == 0) && ((uintptr_t)a.dst % 16 == 0) &&
                     (a.pitch % C::V == 0);
  const cudaError_t e =
      launch_pdl(&stencil2d_kernel<TS, RL, RR, RT, RB, STAR, P, T, V_>, grid, dim3(32 * nw), 0,
                 a.stream, (const TS*)a.src, (TS*)a.dst, a.width, a.height, a.pitch,
                 a.y_begin, a.y_end, a.boundary, vec_ok, cf);
  count_launch();
  return e;
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int P, int T, int V_>
struct Register2D {
  Register2D() {
    Kernel2DInfo info;
    info.launch = &launch_stencil2d<TS, RL, RR, RT, RB, STAR, P, T, V_>;
    info.func = (const void*)&stencil2d_kernel<TS, RL, RR, RT, RB, STAR, P, T, V_>;
    info.vec = V_;
    register_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, STAR ? 1 : 0, P, T, V_}, info);
  }
};

}  // namespace ssam
