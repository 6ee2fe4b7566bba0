// Row-loop variant of the register-cache systolic 2D kernel for wide square
// filters (one time step per launch).
//
// The windowed tile (stencil2d.cuh) unrolls every filter row of every output
// row it keeps: for a 21 x 21 correlation and 4 rows a thread that is over
// ten thousand FMAs of straight-line code, far more than the instruction
// cache holds, and the kernel stalls on instruction fetch.  Here a warp keeps
// one output row at a time and walks the filter rows in a loop unrolled only
// by two: per filter row it loads the input row for its strip (V columns a
// lane, halo lanes beyond both sides, 16-byte loads; the next row's load is
// issued before this row's products), reads that filter row's coefficients,
// and forms the own-column products and the partial sums for the lanes
// downstream -- the same products in the same order as the windowed tile.
// The partial sums travel by shuffle once per output row, after the last
// filter row (SSAM's systolic exchange).  The input rows of neighbouring
// output rows are re-read from L1/L2, not DRAM.  Registered in the kernel
// table with P = 1, which the autotuner times against the other tiles.
#pragma once

#include "stencil2d.cuh"

namespace ssam {

template <typename TS, int RL, int RR, int RT, int RB, int V_>
struct RowLoop2DCfg {
  using TA = typename Traits<TS>::TA;
  static constexpr int V = V_;
  static constexpr int FW = RL + RR + 1;
  static constexpr int FH = RT + RB + 1;
  static constexpr int NC = FW * FH;
  static constexpr int HL = (RL + V - 1) / V;
  static constexpr int HR = (RR + V - 1) / V;
  static constexpr int OUT_LANES = 32 - HL - HR;
  static constexpr int OUT_COLS = OUT_LANES * V;
  static constexpr int ROWS = 8;  // output rows a warp walks per work item
  static_assert(OUT_LANES >= 2, "radius too large for one warp strip");
  static_assert((V * sizeof(TS)) % 16 == 0, "a thread owns whole 16-byte chunks");
};

template <typename TS, int RL, int RR, int RT, int RB, int V_>
__global__ void __launch_bounds__(256)
stencil2d_rowloop_kernel(const TS* __restrict__ src, TS* __restrict__ dst, int64_t W,
                         int64_t H, int64_t pitch, int64_t y_begin, int64_t y_end, int bnd,
                         int vec_ok,
                         CoefBlock<typename Traits<TS>::TA,
                                   RowLoop2DCfg<TS, RL, RR, RT, RB, V_>::NC> cf) {
  using C = RowLoop2DCfg<TS, RL, RR, RT, RB, V_>;
  using TA = typename C::TA;
  constexpr int V = C::V, FW = C::FW, ROWS = C::ROWS;
  constexpr unsigned FULL = 0xffffffffu;
  pdl_wait_then_release();
  const int64_t warp_x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t x_out0 = warp_x * C::OUT_COLS;
  if (x_out0 >= W) return;  // whole warp leaves together
  const int lane = threadIdx.x & 31;
  const int64_t x0 = x_out0 + (int64_t)(lane - C::HL) * V;
  const bool lane_stores = lane >= C::HL && lane < 32 - C::HR;
  const bool cols_in = x0 >= 0 && x0 + V <= W;
  const bool row_vec = vec_ok && cols_in;
  const bool x_ring = bnd == SSAM_BOUNDARY_COPY && (x0 < RL || x0 + V > W - RR);
  const int64_t nby = (y_end - y_begin + ROWS - 1) / ROWS;

  for (int64_t by = blockIdx.y; by < nby; by += gridDim.y) {
    const int64_t ya = y_begin + by * ROWS;
    const int64_t yb = ya + ROWS < y_end ? ya + ROWS : y_end;
#pragma unroll 1
    for (int64_t y = ya; y < yb; ++y) {
      TA acc[V], pr[RL > 0 ? RL : 1], pl[RR > 0 ? RR : 1];
#pragma unroll
      for (int j = 0; j < V; ++j) acc[j] = TA(0);
#pragma unroll
      for (int q = 0; q < (RL > 0 ? RL : 1); ++q) pr[q] = TA(0);
#pragma unroll
      for (int q = 0; q < (RR > 0 ? RR : 1); ++q) pl[q] = TA(0);

      // input row y + fy - RT with the boundary rule (ZERO: zeros outside)
      auto load = [&](int fy, TA (&d)[V]) {
        int64_t yy = y + fy - RT;
        const bool y_out = yy < 0 || yy >= H;
        yy = yy < 0 ? 0 : (yy >= H ? H - 1 : yy);
        const TS* row = src + yy * pitch;
        if (y_out && bnd == SSAM_BOUNDARY_ZERO) {
#pragma unroll
          for (int j = 0; j < V; ++j) d[j] = TA(0);
        } else if (row_vec) {
          load_vec<TS, V>(d, row + x0);
        } else {
          load_row_edge<TS, V>(d, row, x0, W, bnd);
        }
      };
      // one filter row's products: own columns, then the partial sums for
      // the lanes to the right (virtual column V+q) and left (-1-q)
      auto compute = [&](int fy, const TA (&d)[V]) {
        TA w[FW];
#pragma unroll
        for (int dx = 0; dx < FW; ++dx) w[dx] = cf.c[fy * FW + dx];
#pragma unroll
        for (int dx = -RL; dx <= RR; ++dx) tap_row<V>(acc, w[dx + RL], d, dx);
        if constexpr (RL > 0) {
#pragma unroll
          for (int q = 0; q < RL; ++q) {
#pragma unroll
            for (int j = 0; j < V; ++j) {
              const int dx = j - V - q;
              if (dx < -RL || dx > -1) continue;
              pr[q] = fma(w[dx + RL], d[j], pr[q]);
            }
          }
        }
        if constexpr (RR > 0) {
#pragma unroll
          for (int q = 0; q < RR; ++q) {
#pragma unroll
            for (int j = 0; j < V; ++j) {
              const int dx = j + 1 + q;
              if (dx < 1 || dx > RR) continue;
              pl[q] = fma(w[dx + RL], d[j], pl[q]);
            }
          }
        }
      };
      // two rows in flight: the next row's load is issued before the
      // current row's products (ping-pong between two register rows)
      TA da[V], db[V];
      load(0, da);
#pragma unroll 1
      for (int fy = 0; fy < C::FH; fy += 2) {
        if (fy + 1 < C::FH) load(fy + 1, db);
        compute(fy, da);
        if (fy + 2 < C::FH) load(fy + 2, da);
        if (fy + 1 < C::FH) compute(fy + 1, db);
      }
      // systolic exchange of the partial sums (a chain when a reach exceeds V)
      if constexpr (RL > 0) {
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
      if constexpr (RR > 0) {
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
      // COPY keeps the cells within the reach of an edge at their input value
      if (bnd == SSAM_BOUNDARY_COPY && (x_ring || y < RT || y >= H - RB)) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
          const int64_t x = x0 + j;
          if (x >= 0 && x < W && ((x < RL) | (x >= W - RR) | (y < RT) | (y >= H - RB)))
            acc[j] = to_acc(src[y * pitch + x]);
        }
      }
      if (lane_stores) {
        TS* p = dst + y * pitch;
        if (row_vec) {
          store_vec<TS, V>(p + x0, acc);
        } else {
          store_row_edge<TS, V>(p, x0, W, acc);
        }
      }
    }
  }
}

template <typename TS, int RL, int RR, int RT, int RB, int V_>
cudaError_t launch_stencil2d_rowloop(const Launch2D& a) {
  using C = RowLoop2DCfg<TS, RL, RR, RT, RB, V_>;
  using TA = typename C::TA;
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  const int nw = a.warps_per_block;
  const int64_t warps_x = (a.width + C::OUT_COLS - 1) / C::OUT_COLS;
  const int64_t nby = (a.y_end - a.y_begin + C::ROWS - 1) / C::ROWS;
  dim3 grid((unsigned)((warps_x + nw - 1) / nw), (unsigned)(nby < 65535 ? nby : 65535));
  const int vec_ok = ((uintptr_t)a.src % 16 == 0) && ((uintptr_t)a.dst % 16 == 0) &&
                     (a.pitch % C::V == 0);
  const cudaError_t e =
      launch_pdl(&stencil2d_rowloop_kernel<TS, RL, RR, RT, RB, V_>, grid, dim3(32 * nw), 0,
                 a.stream, (const TS*)a.src, (TS*)a.dst, a.width, a.height, a.pitch,
                 a.y_begin, a.y_end, a.boundary, vec_ok, cf);
  count_launch();
  return e;
}

template <typename TS, int RL, int RR, int RT, int RB, int V_>
struct RegisterRowLoop2D {
  RegisterRowLoop2D() {
    Kernel2DInfo info;
    info.launch = &launch_stencil2d_rowloop<TS, RL, RR, RT, RB, V_>;
    info.func = (const void*)&stencil2d_rowloop_kernel<TS, RL, RR, RT, RB, V_>;
    info.vec = V_;
    register_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, 0, 1, 1, V_}, info);
  }
};

}  // namespace ssam
