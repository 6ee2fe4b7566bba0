// Row-streaming variant of the register-cache systolic 2D kernel (one time
// step per launch).
//
// The warp tile of stencil2d.cuh loads its whole window (P + rt + rb rows)
// up front, computes P rows and stores them: the halo rows are read again by
// the tile below, and a warp has loads in flight only between two compute
// phases.  Here a warp walks SEG consecutive output rows of its 32*V-column
// strip instead, keeping a ring of rows in registers:
//   * the rows of the stencil's reach (rt + rb + 1 of them, converted to the
//     accumulation type) plus D rows still in flight as raw 16-byte words;
//   * every output row issues the load of the row D rows ahead of the reach,
//     converts the row that has just come into reach, forms the row's sums
//     with the same own-column / shuffled partial-sum scheme (SSAM's systolic
//     exchange, reference ssai-2dstencil/stencil2D_*.cu), and stores it;
//   * the ring is unrolled over its length, so every slot is a fixed set of
//     registers (no local memory, no data movement between slots).
// Each row of the strip is read once per segment (plus rt + rb + D rows at
// the segment's ends), and every warp keeps D rows of loads in flight while it
// computes.  Registered in the kernel table with P = SEG >= 32, which the
// autotuner times against the windowed tiles.
#pragma once

#include "stencil2d.cuh"

namespace ssam {

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_, int DF = 0>
struct Stream2DCfg {
  using TA = typename Traits<TS>::TA;
  static constexpr int V = V_;
  static constexpr int FW = RL + RR + 1;
  static constexpr int FH = RT + RB + 1;
  static constexpr int NC = FW * FH;
  static constexpr int HL = (RL + V - 1) / V;  // halo lanes, left
  static constexpr int HR = (RR + V - 1) / V;  // halo lanes, right
  static constexpr int OUT_LANES = 32 - HL - HR;
  static constexpr int OUT_COLS = OUT_LANES * V;
  static constexpr int CH = V * (int)sizeof(TS) / 16;  // 16-byte words per row
  // rows in flight ahead of the reach: 2 KB (FP32/16-bit) or 4 KB (FP64) a
  // warp, or DF rows when given.  (The 13-row reach of the 25-point star
  // takes 4 too: with 1 its ring needed 128 registers and spilled, with 4 it
  // holds 68 -- 110 / 80 for BF16, 178 / 128 for FP64.)
  static constexpr int D = DF > 0 ? DF : 4;
  static constexpr int L = FH + D;  // ring length = unroll factor
  // rows beyond the ones in flight that are prefetched into L2 (no registers
  // held), so that the loads D rows ahead find their lines on chip
  static constexpr int PF = 8;
  // rows a warp walks: SEG rounded up to whole ring lengths
  static constexpr int SEGL = (SEG + L - 1) / L * L;
  static_assert(OUT_LANES >= 2, "radius too large for one warp strip");
  static_assert((V * sizeof(TS)) % 16 == 0, "a thread owns whole 16-byte chunks");
};

// Where a lane's V columns lie: all inside the grid, all outside it (left or
// right), or -- the last chunk of a row whose width is not a multiple of V --
// partly inside.
enum StreamLane { kLaneIn = 0, kLaneLeft = 1, kLaneRight = 2, kLanePartial = 3 };

template <typename TS, int V, int CH, typename TA>
__device__ __forceinline__ void stream_unpack(TA (&d)[V], const uint4 (&w)[CH]) {
  constexpr int PER = 16 / sizeof(TS);
#pragma unroll
  for (int c = 0; c < CH; ++c) {
    const uint32_t wd[4] = {w[c].x, w[c].y, w[c].z, w[c].w};
    words_to_acc<TS, PER>(d + c * PER, wd);
  }
}

// 16 zero bytes per 16-byte word of a row chunk (up to 32-byte chunks): rows
// outside the grid under the ZERO rule are loaded from here, so that every
// row of the ring is one plain load from a selected pointer.
__device__ __align__(16) const uint4 g_stream_zero[2] = {};

// `chv` = 16-byte words of the chunk that hold a column inside the grid (the
// others of a row's last, partial chunk are not read: they may lie past the
// end of the buffer's last row).
template <int CH>
__device__ __forceinline__ void stream_load(uint4 (&w)[CH], const void* p, int chv) {
#pragma unroll
  for (int c = 0; c < CH; ++c)
    w[c] = (c == 0 || c < chv) ? __ldg(reinterpret_cast<const uint4*>(p) + c)
                               : make_uint4(0u, 0u, 0u, 0u);
}

// Values of a lane's columns outside the grid after unpacking its (clamped)
// chunk: 0 under ZERO, the edge column under CLAMP; under COPY they never
// reach an output that is kept, so they stay as loaded.  `nin` = columns of a
// partial chunk inside the grid.  (Grids with a partial last chunk run the
// streaming kernel only under ZERO and COPY; under CLAMP every outside lane
// is wholly outside, and its edge column is element 0 or V-1.)
template <int V, typename TA>
__device__ __forceinline__ void stream_fix_lane(TA (&d)[V], int where, int nin, int bnd) {
  if (bnd == SSAM_BOUNDARY_COPY) return;
  if (where == kLanePartial) {
#pragma unroll
    for (int j = 1; j < V; ++j)
      if (j >= nin) d[j] = TA(0);
  } else if (bnd == SSAM_BOUNDARY_ZERO) {
#pragma unroll
    for (int j = 0; j < V; ++j) d[j] = TA(0);
  } else {
    const TA e = where == kLaneLeft ? d[0] : d[V - 1];
#pragma unroll
    for (int j = 0; j < V; ++j) d[j] = e;
  }
}

// One warp's work: segments sg0, sg0 + sstride, ... (of SEGL rows from
// y_begin; rows >= y_end are not written) of the strip whose first output
// column is x_out0.  Shared by the grid kernel below and the persistent
// batched kernel.  Requirements (checked by the launchers, which hand other
// grids to the windowed kernel): src/dst 16-byte aligned, pitch a multiple
// of V, and under CLAMP a width that is a multiple of V too.  Then every
// lane's columns are one 16-byte-aligned chunk inside the grid, outside it,
// or (width not a multiple of V) the row's last chunk, partly inside; all
// loads are 16-byte loads of a clamped chunk (a partial chunk never leaves
// its row's pitch, nor the 16-byte block of its last valid element).
// PARTIAL: widths need not be a multiple of V (the batched kernel); without
// it the launcher guarantees whole chunks and the partial-chunk code is left
// out of the unrolled ring (it costs registers and instruction fetch).
template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_,
          bool PARTIAL = false, int DF = 0>
__device__ __forceinline__ void stream2d_warp_segments(
    const TS* __restrict__ src, TS* __restrict__ dst, int64_t W, int64_t H, int64_t pitch,
    int64_t x_out0, int64_t y_begin, int64_t y_end, int sg0, int sstride, int bnd,
    const CoefBlock<typename Traits<TS>::TA,
                    Stream2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_>::NC>& cf) {
  using C = Stream2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_, DF>;
  using TA = typename C::TA;
  constexpr int V = C::V, FW = C::FW, FH = C::FH, CH = C::CH, D = C::D, L = C::L,
                PF = C::PF;
  constexpr int SEGL = C::SEGL;
  constexpr unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int64_t x0 = x_out0 + (int64_t)(lane - C::HL) * V;
  const bool lane_stores = lane >= C::HL && lane < 32 - C::HR && x0 < W;
  const int where =
      x0 < 0 ? kLaneLeft
             : (x0 >= W ? kLaneRight : (PARTIAL && x0 + V > W ? kLanePartial : kLaneIn));
  // this lane's chunk, clamped into the grid (the last chunk of a row)
  const int64_t wlast = (W - 1) / V * V;
  const int64_t xc = x0 < 0 ? 0 : (x0 > wlast ? wlast : x0);
  // columns of that chunk inside the grid, and its 16-byte words holding any
  const int nin = PARTIAL ? (int)(W - xc < V ? W - xc : V) : V;
  const int chv = PARTIAL ? (nin * (int)sizeof(TS) + 15) / 16 : CH;
  // warp-uniform: some lane of this warp lies outside the grid, or partly
  const bool edge_warp = x_out0 - (int64_t)C::HL * V < 0 || x_out0 + (32 - C::HL) * V > W;
  // columns of this lane that the COPY rule keeps at their input value
  const bool x_copy = bnd == SSAM_BOUNDARY_COPY && (x0 < RL || x0 + V > W - RR);
  const int nseg = (int)((y_end - y_begin + SEGL - 1) / SEGL);
  // rows outside the grid: the clamped edge row of this lane's chunk (CLAMP,
  // COPY) or zeros (ZERO)
  const TS* const row_top =
      bnd == SSAM_BOUNDARY_ZERO ? reinterpret_cast<const TS*>(g_stream_zero) : src + xc;
  const TS* const row_bot = bnd == SSAM_BOUNDARY_ZERO
                                ? reinterpret_cast<const TS*>(g_stream_zero)
                                : src + (H - 1) * pitch + xc;
  const int h = (int)H;  // H, W < 2^31 (checked by the entry points)
  const bool fix_lane = edge_warp && where != kLaneIn;
  const bool copy = bnd == SSAM_BOUNDARY_COPY;
  // rows RT .. h-RB-1 are not in the ring COPY keeps (none when h <= RT+RB)
  const unsigned y_inner = h > RT + RB ? (unsigned)(h - RT - RB) : 0u;

  for (int sg = sg0; sg < nseg; sg += sstride) {
    const int ya = (int)y_begin + sg * SEGL;  // first output row of the segment
    // ring slot of grid row ya + k (k >= -RT) is (k + RT) % L
    uint4 raw[L][CH];
    TA val[L][V];
    // prologue: rows ya-RT .. ya+RB+D-1 in flight, ya-RT .. ya+RB-1 converted
#pragma unroll
    for (int k = 0; k < FH - 1 + D; ++k) {
      const int y = ya - RT + k;
      stream_load<CH>(raw[k],
                      (unsigned)y < (unsigned)h ? src + (int64_t)y * pitch + xc
                                                : (y < 0 ? row_top : row_bot),
                      chv);
    }
#pragma unroll
    for (int k = 0; k < FH - 1; ++k) {
      stream_unpack<TS, V, CH>(val[k], raw[k]);
      if (fix_lane) stream_fix_lane<V>(val[k], where, nin, bnd);
    }

    // whole groups of L rows (rows past y_end are computed, not stored)
    const int left = (int)y_end - ya;
    const int nrows = left < SEGL ? left : SEGL;
    // rows ya + k, k < pf_rows, are read by this segment and inside the grid
    const int pf_rows = (h - ya) < nrows + RB ? (h - ya) : nrows + RB;
    const TS* ldp = src + (int64_t)(ya + RB + D) * pitch + xc;  // next ring load
    const TS* pfp = ldp + (int64_t)PF * pitch;                   // next L2 prefetch
    TS* stp = dst + (int64_t)ya * pitch + x0;                    // next store
    for (int base = 0; base < nrows; base += L) {
#pragma unroll
      for (int u = 0; u < L; ++u) {
        const int i = base + u;  // output row ya + i
        // the row D ahead of the reach; its slot held row ya+i-RT-1, now done
        {
          const int y = ya + i + RB + D;
          stream_load<CH>(raw[(u + FH - 1 + D) % L],
                          (unsigned)y < (unsigned)h ? ldp : (y < 0 ? row_top : row_bot), chv);
          ldp += pitch;
        }
        // L2 prefetch PF rows further on, within the rows this segment reads
        asm volatile(
            "{ .reg .pred q; setp.lt.s32 q, %1, %2; @q prefetch.global.L2 [%0]; }" ::"l"(pfp),
            "r"(i + RB + D + PF), "r"(pf_rows));
        pfp += pitch;
        // the row entering the reach
        stream_unpack<TS, V, CH>(val[(u + FH - 1) % L], raw[(u + FH - 1) % L]);
        if (fix_lane) stream_fix_lane<V>(val[(u + FH - 1) % L], where, nin, bnd);

        TA acc[V];
#pragma unroll
        for (int j = 0; j < V; ++j) acc[j] = TA(0);
        // own columns
#pragma unroll
        for (int dy = -RT; dy <= RB; ++dy) {
#pragma unroll
          for (int dx = -RL; dx <= RR; ++dx) {
            if (STAR && dy != 0 && dx != 0) continue;
            tap_row<V, pair_taps<TS, STAR ? FW + FH - 1 : FW * FH>()>(
                acc, cf.c[(dy + RT) * FW + (dx + RL)], val[(u + RT + dy) % L], dx);
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
                const int dx = j - V - q;
                if (dx < -RL || dx > -1) continue;
                pr[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], val[(u + RT + dy) % L][j],
                            pr[q]);
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
                pl[q] = fma(cf.c[(dy + RT) * FW + (dx + RL)], val[(u + RT + dy) % L][j],
                            pl[q]);
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
        const int y = ya + i;
        if (copy && (x_copy || (unsigned)(y - RT) >= y_inner)) {
          const bool y_ring = (unsigned)(y - RT) >= y_inner;
#pragma unroll
          for (int j = 0; j < V; ++j) {
            const int64_t x = x0 + j;
            if (y_ring | (x < RL) | (x >= W - RR)) acc[j] = val[(u + RT) % L][j];
          }
        }
        if (lane_stores && y < (int)y_end) {
          if (!PARTIAL || where == kLaneIn) store_vec<TS, V>(stp, acc);
          else store_row_edge<TS, V>(stp - x0, x0, W, acc);  // the row's partial chunk
        }
        stp += pitch;
      }
    }
  }
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_>
__global__ void __launch_bounds__(256)
stencil2d_stream_kernel(const TS* __restrict__ src, TS* __restrict__ dst, int64_t W,
                        int64_t H, int64_t pitch, int64_t y_begin, int64_t y_end, int bnd,
                        CoefBlock<typename Traits<TS>::TA,
                                  Stream2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_>::NC> cf) {
  using C = Stream2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_>;
  pdl_wait_then_release();
  const int64_t warp_x = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int64_t x_out0 = warp_x * C::OUT_COLS;
  if (x_out0 >= W) return;  // whole warp leaves together
  stream2d_warp_segments<TS, RL, RR, RT, RB, STAR, SEG, V_>(
      src, dst, W, H, pitch, x_out0, y_begin, y_end, (int)blockIdx.y, (int)gridDim.y, bnd, cf);
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_>
cudaError_t launch_stencil2d_stream(const Launch2D& a) {
  using C = Stream2DCfg<TS, RL, RR, RT, RB, STAR, SEG, V_>;
  using TA = typename C::TA;
  CoefBlock<TA, C::NC> cf;
  for (int k = 0; k < C::NC; ++k) cf.c[k] = (TA)a.coef[k];
  const int nw = a.warps_per_block;
  const int64_t warps_x = (a.width + C::OUT_COLS - 1) / C::OUT_COLS;
  const int64_t nseg = (a.y_end - a.y_begin + C::SEGL - 1) / C::SEGL;
  dim3 grid((unsigned)((warps_x + nw - 1) / nw), (unsigned)(nseg < 65535 ? nseg : 65535));
  const bool aligned = ((uintptr_t)a.src % 16 == 0) && ((uintptr_t)a.dst % 16 == 0) &&
                       (a.pitch % C::V == 0) && (a.width % C::V == 0);
  if (!aligned) {
    // unaligned grids: the windowed kernel of the same stencil
    const Kernel2DInfo* w =
        find_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, STAR ? 1 : 0, 8, 1, V_});
    if (!w) return cudaErrorInvalidValue;
    return w->launch(a);
  }
  const cudaError_t e =
      launch_pdl(&stencil2d_stream_kernel<TS, RL, RR, RT, RB, STAR, SEG, V_>, grid,
                 dim3(32 * nw), 0, a.stream, (const TS*)a.src, (TS*)a.dst, a.width, a.height,
                 a.pitch, a.y_begin, a.y_end, a.boundary, cf);
  count_launch();
  return e;
}

template <typename TS, int RL, int RR, int RT, int RB, bool STAR, int SEG, int V_>
struct RegisterStream2D {
  static_assert(SEG >= 32, "P >= 32 marks a streaming kernel in the table");
  RegisterStream2D() {
    Kernel2DInfo info;
    info.launch = &launch_stencil2d_stream<TS, RL, RR, RT, RB, STAR, SEG, V_>;
    info.func = (const void*)&stencil2d_stream_kernel<TS, RL, RR, RT, RB, STAR, SEG, V_>;
    info.vec = V_;
    register_2d(Key2D{Traits<TS>::DT, RL, RR, RT, RB, STAR ? 1 : 0, SEG, 1, V_}, info);
  }
};

}  // namespace ssam
