// Row-streaming 2D kernel with T time steps fused in registers.
//
// The single-step streaming tile (stencil2d_stream.cuh) keeps a ring of input
// rows per warp and emits one output row per iteration.  Here the same
// pipeline has T levels: every iteration loads one input row (D rows ahead),
// forms one row of step 1 from the input ring, one row of step 2 from the
// ring of step-1 rows, ..., and stores one row of step T.  Level s lags level
// s-1 by RB rows; each level keeps the last RT+RB+1 of its rows in registers
// (a ring indexed by the iteration, unrolled over its length).  So a fused
// launch reads and writes every cell once, like one step, without the
// windowed tile's vertical redundancy (its window shrinks by RT+RB rows per
// fused step); the halo lanes (RL*T / V on the left, RR*T / V on the right)
// absorb the lanes that each step's one-hop exchange leaves wrong.  Each
// segment starts (T-1)*(RT+RB) rows early to fill the levels.
//
// Boundary rules between the fused steps, as the chain of single steps
// would apply them: ZERO makes the intermediate grids zero outside the grid
// (rows and columns), COPY resets the cells within the reach of an edge to
// their input values.  (CLAMP is single-step only.)
#pragma once

#include "stencil2d_stream.cuh"

namespace ssam {

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_, int T>
struct StreamT2DCfg {
  using TA = typename Traits<TS>::TA;
  static constexpr int V = V_;
  static constexpr int FW = RL + RR + 1;
  static constexpr int FH = RT + RB + 1;
  static constexpr int NC = FW * FH;
  static constexpr int HL = (RL * T + V - 1) / V;  // halo lanes, left
  static constexpr int HR = (RR * T + V - 1) / V;  // halo lanes, right
  static constexpr int OUT_LANES = 32 - HL - HR;
  static constexpr int OUT_COLS = OUT_LANES * V;
  static constexpr int CH = V * (int)sizeof(TS) / 16;
  static constexpr int D = FH;      // input rows in flight ahead of the reach
  static constexpr int L = FH + D;  // input ring; a multiple of the level rings' FH
  static constexpr int W0 = (T - 1) * (FH - 1);  // iterations that fill the levels
  static constexpr int PF = 8;
  static constexpr int SEGL = SEG;  // output rows a warp walks
  static_assert(T >= 2, "the single-step kernel is stencil2d_stream.cuh");
  static_assert(OUT_LANES >= 2, "radius too large for one warp strip");
  static_assert((V * sizeof(TS)) % 16 == 0, "a thread owns whole 16-byte chunks");
};

// One row of a step: sums of the row whose reach sits in ring slots
// (o + RT + dy) % NR, dy = -RT .. RB (o >= 0): own columns, then the partial
// sums for the neighbouring lanes' columns moved one lane downstream by
// shuffle (a chain when a reach exceeds V) -- the products and their order
// are those of the other 2D tiles.
template <int RL, int RR, int RT, int RB, bool STAR, int V, int NR, bool PAIR, typename TA,
          int NC>
__device__ __forceinline__ void stream_row_sum(TA (&acc)[V], const TA (&ring)[NR][V], int o,
                                               const CoefBlock<TA, NC>& cf) {
  constexpr int FW = RL + RR + 1;
  constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int j = 0; j < V; ++j) acc[j] = TA(0);
#pragma unroll
  for (int dy = -RT; dy <= RB; ++dy) {
#pragma unroll
    for (int dx = -RL; dx <= RR; ++dx) {
      if (STAR && dy != 0 && dx != 0) continue;
      tap_row<V, PAIR>(acc, cf.c[(dy + RT) * FW + (dx + RL)], ring[(o + RT + dy) % NR], dx);
    }
  }
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
          const int dx = j - V - q;
          if (dx < -RL || dx > -1) continue;
          pr[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], ring[(o + RT + dy) % NR][j], pr[q]);
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
          pl[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], ring[(o + RT + dy) % NR][j], pl[q]);
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
}

// Requirements as for the single-step streaming kernel without partial
// chunks (checked by the launcher): 16-byte aligned buffers, pitch and width
// multiples of V.
template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_, int T>
__global__ void __launch_bounds__(256)
stencil2d_stream_t_kernel(const TS* __restrict__ src, TS* __restrict__ dst, int64_t W,
                          int64_t H, int64_t pitch, int64_t y_begin, int64_t y_end, int bnd,
                          CoefBlock<typename Traits<TS>::TA,
                                    StreamT2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_, T>::NC> cf) {
  using C = StreamT2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_, T>;
  using TA = typename C::TA;
  constexpr int V = C::V, FH = C::FH, CH = C::CH, D = C::D, L = C::L, W0 = C::W0,
                PF = C::PF, SEGL = C::SEGL;
  constexpr bool PAIR = pair_taps<TS, STAR ? RL + RR + FH : (RL + RR + 1) * FH>();
  pdl_wait_then_release();
  const int64_t warp_x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t x_out0 = warp_x * C::OUT_COLS;
  if (x_out0 >= W) return;  // whole warp leaves together
  const int lane = threadIdx.x & 31;
  const int64_t x0 = x_out0 + (int64_t)(lane - C::HL) * V;
  const bool lane_stores = lane >= C::HL && lane < 32 - C::HR && x0 < W;
  const int where = x0 < 0 ? kLaneLeft : (x0 >= W ? kLaneRight : kLaneIn);
  const int64_t xc = x0 < 0 ? 0 : (x0 >= W ? W - V : x0);
  const bool edge_warp = x_out0 - (int64_t)C::HL * V < 0 || x_out0 + (32 - C::HL) * V > W;
  const bool fix_lane = edge_warp && where != kLaneIn;
  const bool x_copy = bnd == SSAM_BOUNDARY_COPY && (x0 < RL || x0 + V > W - RR);
  const int h = (int)H;
  const unsigned y_inner = h > RT + RB ? (unsigned)(h - RT - RB) : 0u;
  const TS* const row_top =
      bnd == SSAM_BOUNDARY_ZERO ? reinterpret_cast<const TS*>(g_stream_zero) : src + xc;
  const TS* const row_bot = bnd == SSAM_BOUNDARY_ZERO
                                ? reinterpret_cast<const TS*>(g_stream_zero)
                                : src + (H - 1) * pitch + xc;
  const int nseg = (int)((y_end - y_begin + SEGL - 1) / SEGL);

  // the boundary rule on a computed row of an intermediate step (or, COPY
  // only, of the last step): the chain of single steps would apply it here
  auto fix_row = [&](TA (&acc)[V], int ys) {
    if (bnd == SSAM_BOUNDARY_ZERO) {
      if ((unsigned)ys >= (unsigned)h) {
#pragma unroll
        for (int j = 0; j < V; ++j) acc[j] = TA(0);
      } else if (fix_lane) {
        stream_fix_lane<V>(acc, where, V, bnd);
      }
    } else if (bnd == SSAM_BOUNDARY_COPY && (unsigned)ys < (unsigned)h &&
               (x_copy || (unsigned)(ys - RT) >= y_inner)) {
      const bool y_ring = (unsigned)(ys - RT) >= y_inner;
#pragma unroll
      for (int j = 0; j < V; ++j) {
        const int64_t x = x0 + j;
        if (x >= 0 && x < W && (y_ring | (x < RL) | (x >= W - RR)))
          acc[j] = to_acc(src[(int64_t)ys * pitch + x]);
      }
    }
  };

  for (int sg = blockIdx.y; sg < nseg; sg += gridDim.y) {
    const int ya = (int)y_begin + sg * SEGL;  // first output row of the segment
    const int nrows = (int)(y_end - ya) < SEGL ? (int)(y_end - ya) : SEGL;
    const int nit = (nrows + W0 + L - 1) / L * L;  // iterations, whole rings
    // level-1 row at iteration ii: y1f + ii; level s: y1f + ii - (s-1)*RB
    const int y1f = ya + (T - 1) * RB - W0;
    uint4 raw[L][CH];
    TA val[L][V];
    TA lev[T - 1][FH][V];
#pragma unroll
    for (int s = 0; s < T - 1; ++s)
#pragma unroll
      for (int k = 0; k < FH; ++k)
#pragma unroll
        for (int j = 0; j < V; ++j) lev[s][k][j] = TA(0);
    // prologue: input rows y1f-RT .. y1f+RB+D-1 in flight, the first FH-1 converted
#pragma unroll
    for (int k = 0; k < FH - 1 + D; ++k) {
      const int y = y1f - RT + k;
      stream_load<CH>(raw[k],
                      (unsigned)y < (unsigned)h ? src + (int64_t)y * pitch + xc
                                                : (y < 0 ? row_top : row_bot),
                      CH);
    }
#pragma unroll
    for (int k = 0; k < FH - 1; ++k) {
      stream_unpack<TS, V, CH>(val[k], raw[k]);
      if (fix_lane) stream_fix_lane<V>(val[k], where, V, bnd);
    }
    const int y_rows_end = (h < y1f + nit + RB) ? h : y1f + nit + RB;  // rows read, < h
    const TS* ldp = src + (int64_t)(y1f + RB + D) * pitch + xc;
    const TS* pfp = ldp + (int64_t)PF * pitch;
    TS* stp = dst + (int64_t)(ya - W0) * pitch + x0;  // row of the last step, iteration 0
    for (int base = 0; base < nit; base += L) {
#pragma unroll
      for (int u = 0; u < L; ++u) {
        const int ii = base + u;
        const int y1 = y1f + ii;
        {
          const int y = y1 + RB + D;
          stream_load<CH>(raw[(u + FH - 1 + D) % L],
                          (unsigned)y < (unsigned)h ? ldp : (y < 0 ? row_top : row_bot), CH);
          ldp += pitch;
        }
        asm volatile(
            "{ .reg .pred q; setp.lt.u32 q, %1, %2; @q prefetch.global.L2 [%0]; }" ::"l"(pfp),
            "r"(y1 + RB + D + PF), "r"(y_rows_end));  // rows 0 .. y_rows_end-1 only
        pfp += pitch;
        stream_unpack<TS, V, CH>(val[(u + FH - 1) % L], raw[(u + FH - 1) % L]);
        if (fix_lane) stream_fix_lane<V>(val[(u + FH - 1) % L], where, V, bnd);

        // step 1 from the input ring
        TA acc[V];
        stream_row_sum<RL, RR, RT, RB, STAR, V, L, PAIR>(acc, val, u, cf);
        fix_row(acc, y1);
#pragma unroll
        for (int j = 0; j < V; ++j) lev[0][u % FH][j] = acc[j];
        // steps 2 .. T from the ring of the step before (its row of this
        // iteration is the newest of the reach)
#pragma unroll
        for (int s = 2; s <= T; ++s) {
          const int ys = y1 - (s - 1) * RB;
          stream_row_sum<RL, RR, RT, RB, STAR, V, FH, PAIR>(acc, lev[s - 2],
                                                     (u + 2 * FH - RB - RT) % FH, cf);
          fix_row(acc, ys);
          if (s < T) {
#pragma unroll
            for (int j = 0; j < V; ++j) lev[s - 1][u % FH][j] = acc[j];
          }
        }
        // the last step's row ya - W0 + ii
        const int yt = ya - W0 + ii;
        if (lane_stores && ii >= W0 && yt < (int)y_end) store_vec<TS, V>(stp, acc);
        stp += pitch;
      }
    }
  }
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_, int T>
cudaError_t launch_stencil2d_stream_t(const Launch2D& a) {
  using C = StreamT2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_, T>;
  using TA = typename C::TA;
  const bool aligned = ((uintptr_t)a.src % 16 == 0) && ((uintptr_t)a.dst % 16 == 0) &&
                       (a.pitch % C::V == 0) && (a.width % C::V == 0) &&
                       a.boundary != SSAM_BOUNDARY_CLAMP;
  if (!aligned) {
    // other grids: the windowed kernel of the same stencil and depth
    const Kernel2DInfo* w =
        find_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, STAR ? 1 : 0, 8, T, V_});
    if (!w) return cudaErrorInvalidValue;
    return w->launch(a);
  }
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  const int nw = a.warps_per_block;
  const int64_t warps_x = (a.width + C::OUT_COLS - 1) / C::OUT_COLS;
  const int64_t nseg = (a.y_end - a.y_begin + C::SEGL - 1) / C::SEGL;
  dim3 grid((unsigned)((warps_x + nw - 1) / nw), (unsigned)(nseg < 65535 ? nseg : 65535));
  const cudaError_t e =
      launch_pdl(&stencil2d_stream_t_kernel<TS, RL, RR, RT, RB, STAR, SEG, V_, T>, grid,
                 dim3(32 * nw), 0, a.stream, (const TS*)a.src, (TS*)a.dst, a.width, a.height,
                 a.pitch, a.y_begin, a.y_end, a.boundary, cf);
  count_launch();
  return e;
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_, int T>
struct RegisterStreamT2D {
  static_assert(SEG >= 32, "P >= 32 marks a streaming kernel in the table");
  RegisterStreamT2D() {
    Kernel2DInfo info;
    info.launch = &launch_stencil2d_stream_t<TS, RL, RR, RT, RB, STAR, SEG, V_, T>;
    info.func = (const void*)&stencil2d_stream_t_kernel<TS, RL, RR, RT, RB, STAR, SEG, V_, T>;
    info.vec = V_;
    register_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, STAR ? 1 : 0, SEG, T, V_}, info);
  }
};

}  // namespace ssam
