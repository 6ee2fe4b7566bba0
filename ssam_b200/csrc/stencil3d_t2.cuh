// 3D z-marching kernel with two time steps fused per launch (temporal
// blocking).
//
// A single-step launch reads and writes every cell once per step, so a chain
// of steps is bound by 2 * sizeof(T) bytes of HBM traffic per cell and step.
// Here one launch applies the stencil twice: step 1 ("level 1") is formed for
// the planes of the column tile as they arrive from the TMA ring, kept in
// registers and shared memory, and step 2 is formed from those values a few
// planes behind; only step 2 is written.  The reference fuses ITERATIVE_COUNT
// steps the same way inside one z-march, shrinking the valid window by 2r per
// step (ssai-3dstencil/tmp3d7pt-v2.cu:124-170; IT = 2..4 at :370-387,
// tmp3d13pt.cu:404-408, tmpPoisson.cu:498-512).
//
// Layout of one work item (z chunk za..zb-1 of one column tile of 32*V x TY
// cells, NW consumer warps of PY rows stacked along y):
//   * input: the producer warp stages planes za-2R .. zb+2R-1 (halo columns
//     HX and rows R included) into the shared-memory ring, as for one step;
//   * level 1 (iteration i, plane i-R): every thread forms its PY x V cells
//     from the staged planes i-2R .. i (the register-cache window of the
//     single-step kernel: y-strip in registers, x partial sums moved one lane
//     by __shfl, z-neighbours from the adjacent slots), applies the boundary
//     rule, rounds to the storage type, and keeps them in a register ring of
//     RL planes; the top R and bottom R rows of each warp's strip also go to
//     a small shared-memory buffer, from which the neighbouring warps read
//     their y halo for step 2;
//   * the x halo of step 2 -- R level-1 columns left and right of the tile --
//     is computed directly from the staged input by spare lanes (one value a
//     lane: NE = 2 * R * (PY + 2*EY) values per warp and plane) and handed to
//     lanes 0 and 31 by __shfl, so column tiles need no overlap and stay
//     32*V wide and 16-byte aligned;
//   * level 2 (plane i-2R-L): own rows from the register ring, y-halo rows
//     from the buffer, x halo from the spare lanes; the same tap loop and
//     one-hop exchange as level 1; written to HBM.  Rows R .. TY-R-1 of the
//     tile are stored (the outer R rows lack their level-1 y halo), so tiles
//     overlap by 2R rows: tile ty stores rows ty*(TY-2R) .. +TY-2R-1;
//   * the consumer warps meet at one named barrier per iteration, which
//     orders the halo-row buffer (D slots, written before the barrier, read
//     after it).  L = 1 extra plane of lag for the 19-point operator, whose
//     step 2 reads the y halo of planes z-1..z+1 (the newest one is written
//     one iteration earlier); stars read it of plane z only.
//
// Boundary rules inside the fused launch are those of the chain of single
// steps: ZERO gives level-1 cells outside the grid the value 0 (the padding
// the next step reads), COPY keeps ring cells at their input value at both
// levels.  Every wait is bounded; whether any consumer warp's wait gave up
// is reduced over the consumer warps by the iteration's barrier itself
// (bar.red.or), so they all leave after the same barrier and none waits at
// a barrier for a warp that left.
#pragma once

#include <utility>

#include "stencil3d_zreg.cuh"

namespace ssam {

// Extra planes of lag of level 2 behind level 1 (0 for stars, 1 for the
// 19-point operator): level 2 must read the y halo of level-1 planes written
// in an earlier iteration.
template <int SH, int R>
__host__ __device__ constexpr int t2_lag() {
  return halo_reach_z<SH, R>() + 1 - R > 0 ? halo_reach_z<SH, R>() + 1 - R : 0;
}

// Largest |dy| of a tap with dx != 0: the rows beyond a warp's strip whose x
// halo step 2 reads (0 for stars, 1 for the 19-point operator).
template <int SH, int R>
__host__ __device__ constexpr int xhalo_reach_y() {
  int m = 0;
  for (int dz = -R; dz <= R; ++dz)
    for (int dy = -R; dy <= R; ++dy)
      for (int dx = -R; dx <= R; ++dx)
        if (tap3<SH, R>(dz, dy, dx) && dx != 0 && iabs_(dy) > m) m = iabs_(dy);
  return m;
}

// Does row k (relative to the warp's strip) of plane dz need its x halo in a
// step over PY rows?
template <int SH, int R, int PY>
__host__ __device__ constexpr bool needs_xhalo(int dz, int k) {
  for (int i = 0; i < PY; ++i)
    for (int dx = -R; dx <= R; ++dx)
      if (dx != 0 && iabs_(k - i) <= R && tap3<SH, R>(dz, k - i, dx)) return true;
  return false;
}

template <typename TS, int SH, int R, int PY, int NW, int S, int V_>
struct Stencil3DT2Cfg {
  using B = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>;
  static constexpr int RH = halo_reach_z<SH, R>();
  static constexpr int L = t2_lag<SH, R>();
  static constexpr int RL = 2 * R + 1 + L;     // level-1 planes kept in registers
  static constexpr int D = R + L + RH + 1;     // level-1 halo-row slots
  static constexpr int H = R;                  // tile rows computed but not stored, each side
  static constexpr int OY = B::TY - 2 * H;     // rows stored per tile
  static constexpr int EY = xhalo_reach_y<SH, R>();
  static constexpr int NR = PY + 2 * EY;       // rows of the x halo per warp
  static constexpr int NE = 2 * R * NR;        // x-halo values per warp and plane
  static constexpr int HB_ELEMS = D * NW * 2 * R * B::TX;
  static constexpr int HB_BYTES = (HB_ELEMS * (int)sizeof(TS) + 127) / 128 * 128;
  static constexpr int SMEM = S * B::SLOT_BYTES + HB_BYTES + 2 * S * 8 + 128 + 128;
  static constexpr int THREADS = B::THREADS;
  static_assert(NE <= 32, "one x-halo value a lane");
  static_assert(2 * R <= B::HX, "the x halo of step 2 needs 2R staged halo columns");
  static_assert(PY >= R, "a warp's strip holds the R halo rows its neighbours read");
  static_assert(OY > 0, "tile taller than its two overlaps");
  static_assert(S >= 2 * R + 2, "ring holds the 2R+1 input planes of level 1 plus one in flight");
};

// Named barrier 1 over the consumer warps (the producer warp never joins it)
// that also returns, to every thread, whether any thread passed `failed`.
__device__ __forceinline__ bool consumer_bar_any(int nthreads, bool failed) {
  uint32_t r;
  asm volatile(
      "{ .reg .pred p, q; setp.ne.u32 p, %1, 0; bar.red.or.pred q, 1, %2, p; "
      "selp.u32 %0, 1, 0, q; }"
      : "=r"(r)
      : "r"((uint32_t)failed), "r"(nthreads)
      : "memory");
  return r != 0;
}

// fn(std::integral_constant<int, 0>{}) .. fn(std::integral_constant<int, N-1>{}):
// a loop body unrolled with a compile-time index (register-ring slots).
template <typename Fn, int... I>
__device__ __forceinline__ void static_for_impl(Fn& fn, std::integer_sequence<int, I...>) {
  (fn(std::integral_constant<int, I>{}), ...);
}
template <int N, typename Fn>
__device__ __forceinline__ void static_for(Fn& fn) {
  static_for_impl(fn, std::make_integer_sequence<int, N>{});
}

template <typename TS, int SH, int R, int PY, int NW, int S, int V_ = 4>
__global__ void __launch_bounds__(32 * (NW + 1), 1)
stencil3d_t2_kernel(const __grid_constant__ CUtensorMap map, const TS* __restrict__ src,
                    TS* __restrict__ dst, Work3D w,
                    CoefBlock<typename Traits<TS>::TA,
                              Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::NC> cf) {
  using C = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>;
  using T2 = Stencil3DT2Cfg<TS, SH, R, PY, NW, S, V_>;
  using TA = typename C::TA;
  constexpr int V = C::V, XW = C::XW, HX = C::HX, RYM = C::RYM, TY = C::TY, TX = C::TX;
  constexpr int F = 2 * R + 1;
  constexpr int L = T2::L, RL = T2::RL, D = T2::D, H = T2::H, OY = T2::OY;
  constexpr int EY = T2::EY, NR = T2::NR, NE = T2::NE;
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int SLOT_ELEMS = C::SLOT_BYTES / (int)sizeof(TS);

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  TS* slots = (TS*)base;
  TS* hbuf = (TS*)(base + S * C::SLOT_BYTES);
  uint64_t* full = (uint64_t*)(base + S * C::SLOT_BYTES + T2::HB_BYTES);
  uint64_t* empty = full + S;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], w.use_tma ? 1u : 32u);
      mbar_init(&empty[s], (unsigned)NW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  pdl_wait_then_release();

  const int64_t nx = w.nx, ny = w.ny, nz = w.nz, nxy = nx * ny;

  if (warp == NW) {
    produce_planes<TS, R, S, C, 2 * R, OY, H>(map, src, w, slots, full, empty, lane);
    return;
  }

  // ---------------------------------------------------------- consumer warps
  // this lane's x-halo value: side es (0 left, 1 right), column offset eh,
  // strip row ek (-EY .. PY+EY-1)
  const int e = lane < NE ? lane : NE - 1;
  const int es = e / (R * NR);
  const int eh = (e / NR) % R;
  const int ek = e % NR - EY;
  const int xe = es == 0 ? -1 - eh : TX + eh;  // tile column of the value
  // slot offset of tile column xe + dx (the value's box: the left one for the
  // left side, the right one for the right side when a plane is two boxes)
  const int ebox = C::NBOX == 2 ? es : 0;
  const int ecol0 = ebox * C::BOXS + (ebox == 0 ? HX + xe : xe - TX / 2);

  uint32_t n = 0;  // ring position of the segment's first staged plane (za - 2R)
  for (int64_t it = blockIdx.x; it < w.items; it += gridDim.x) {
    const Seg3D sg = item_seg(it, w);
    const int tx = (int)(sg.tile % w.ntx), ty = (int)(sg.tile / w.ntx);
    const int64_t cx0 = (int64_t)tx * TX;                 // tile's first column
    const int64_t cy0 = (int64_t)ty * OY - H;             // tile's first computed row
    const int64_t x0 = cx0 + lane * V;                    // my first column
    const int64_t y0 = cy0 + warp * PY;                   // my first row
    const int col = C::col_off(lane);
    const int row0 = RYM + warp * PY;
    const int nzc = (int)(sg.zb - sg.za);
    const int nit = nzc + 2 * R + L;                      // iterations of the segment
    const bool copy = w.boundary == SSAM_BOUNDARY_COPY;
    // rows of my strip inside the grid; rows stored (tile rows H .. TY-H-1)
    unsigned row_in = 0, row_st = 0;
#pragma unroll
    for (int i = 0; i < PY; ++i) {
      const int64_t y = y0 + i;
      if (y >= 0 && y < ny) row_in |= 1u << i;
      const int trow = warp * PY + i;
      if (y >= 0 && y < ny && trow >= H && trow < TY - H && x0 < nx) row_st |= 1u << i;
    }
    // where the boundary rule acts on level 1 (ZERO: cells outside the grid;
    // COPY: the ring of width R): rows -- warp-uniform, handled cell by cell
    // -- and columns -- a per-lane mask, non-zero only for lanes at the grid's
    // x faces, so that those lanes do not send their warp down the per-cell
    // path
    const bool edge_y = copy ? (y0 < R || y0 + PY > ny - R) : (y0 < 0 || y0 + PY > ny);
    unsigned xmask1 = 0;
#pragma unroll
    for (int j = 0; j < V; ++j)
      if (copy ? (x0 + j < R || x0 + j >= nx - R) : (x0 + j >= nx)) xmask1 |= 1u << j;
    // the x-halo value's cell
    const int64_t egx = cx0 + xe, egy = y0 + ek;
    const bool e_out = egx < 0 || egx >= nx || egy < 0 || egy >= ny;
    const bool e_ring = egx < R || egx >= nx - R || egy < R || egy >= ny - R;
    constexpr int VB = V * (int)sizeof(TS);
    constexpr int AL = VB >= 16 ? 16 : 8;
    const int64_t ybase = y0 >= 0 ? y0 : 0;
    const bool vec_seg = x0 + V <= nx &&
                         (uintptr_t)(dst + (sg.b * nz + sg.za) * nxy + ybase * nx + x0) % AL == 0 &&
                         (nx * (int64_t)sizeof(TS)) % AL == 0 &&
                         (nxy * (int64_t)sizeof(TS)) % AL == 0;
    // level 2's store: a lane that stores rows needs whole vector stores for
    // the warp to take the fast path (rows not stored are skipped by row_st)
    const StripEdges edges = strip_edges<R, PY, V>(x0, y0, nx, ny, w.boundary, (1u << PY) - 1u,
                                                   vec_seg || row_st == 0);

    TA ring[RL][PY][V];  // level-1 own cells: plane q in slot (q - za + R) % RL
    TA ext[RL];          // level-1 x-halo value of this lane, same slots

    bool stop = false;  // a bounded wait of some consumer warp gave up
    int qb = 0;
    // iteration qb + u of the segment, u a compile-time register-ring slot
    auto iteration = [&](auto uc) {
      constexpr int u = decltype(uc)::value;
      {
        const int qi = qb + u;
        if (stop || qi >= nit) return;
        const bool lvl1 = qi < nzc + 2 * R;   // level-1 plane za+qi-R is needed
        const bool lvl2 = qi >= 2 * R + L;    // level-2 plane za+qi-2R-L is in the chunk
        bool ok = true;
        if (lvl1) {
          // input planes za+qi-2R .. za+qi at ring positions n+qi .. n+qi+2R
          for (int k = qi == 0 ? 0 : 2 * R; k <= 2 * R; ++k) {
            const uint32_t q = n + (uint32_t)(qi + k);
            if (!mbar_wait(&full[q % S], (q / S) & 1, w.wait_ns)) ok = false;
          }
          if (!ok && lane == 0) atomicCAS(w.err, 0, 3);
        }
        if (lvl1 && ok) {
          // ------------------------------------------------- level 1
          const int64_t q = sg.za + qi - R;  // level-1 plane
          const bool zout = q < 0 || q >= nz;
          const bool zring = q < R || q >= nz - R;
          TA acc[PY][V];
          TA pr[PY][R], pl[PY][R], inl[PY][R], inr[PY][R];
          TA center[PY][V];
#pragma unroll
          for (int i = 0; i < PY; ++i) {
#pragma unroll
            for (int j = 0; j < V; ++j) acc[i][j] = center[i][j] = TA(0);
#pragma unroll
            for (int h = 0; h < R; ++h) pr[i][h] = pl[i][h] = inl[i][h] = inr[i][h] = TA(0);
          }
          TA ev = TA(0), ec = TA(0);  // this lane's x-halo value and its centre
#pragma unroll
          for (int dz = -R; dz <= R; ++dz) {
            const int ry = ry3<SH, R>(dz);
            if (ry < 0) continue;
            const uint32_t qp = n + (uint32_t)(qi + R + dz);
            const TS* sl = slots + (size_t)(qp % S) * SLOT_ELEMS;
            TA d[PY + 2 * RYM][V];
            TA hv[PY + 2 * RYM][R];
#pragma unroll
            for (int k = -RYM; k < PY + RYM; ++k) {
              if (k < -ry || k >= PY + ry) continue;
              load_slot_row<TS, V>(d[k + ry], sl + (row0 + k) * XW + col);
              const TS* hrow = sl + (row0 + k) * XW;
#pragma unroll
              for (int h = 0; h < R; ++h)
                hv[k + ry][h] =
                    to_acc(hrow[lane == 0 ? C::col_off(0) - 1 - h : C::col_off(31) + V + h]);
            }
            if (dz == 0) {
#pragma unroll
              for (int i = 0; i < PY; ++i)
#pragma unroll
                for (int j = 0; j < V; ++j) center[i][j] = d[i + ry][j];
            }
#pragma unroll
            for (int i = 0; i < PY; ++i) {
#pragma unroll
              for (int dy = -RYM; dy <= RYM; ++dy) {
                if (dy < -ry || dy > ry || rx3<SH, R>(dz, dy) < 0) continue;
#pragma unroll
                for (int dx = -R; dx <= R; ++dx) {
                  if (!tap3<SH, R>(dz, dy, dx)) continue;
                  const TA c = cf.c[((dz + R) * F + (dy + R)) * F + (dx + R)];
                  const TA* src_row = d[i + dy + ry];
                  if (dx == 0) {
                    fma_row<V>(acc[i], c, src_row);
                  } else
#pragma unroll
                  for (int j = 0; j < V; ++j) {
                    const int t = j - dx;
                    if (t >= 0 && t < V) acc[i][t] = fma(c, src_row[j], acc[i][t]);
                    else if (t >= V) pr[i][t - V] = fma(c, src_row[j], pr[i][t - V]);
                    else pl[i][-1 - t] = fma(c, src_row[j], pl[i][-1 - t]);
                  }
#pragma unroll
                  for (int h = 0; h < R; ++h) {
                    const TA v = hv[i + dy + ry][h];
                    const int tl = -1 - h - dx;
                    const int tr = V + h - dx;
                    if (tl >= 0 && tl < V) inl[i][tl] = fma(c, v, inl[i][tl]);
                    if (tr >= 0 && tr < V) inr[i][V - 1 - tr] = fma(c, v, inr[i][V - 1 - tr]);
                  }
                }
              }
            }
            // this lane's x-halo value: taps of plane dz at tile column xe,
            // strip row ek (rows beyond the staged tile are clamped: they
            // only feed tile rows that are not stored)
#pragma unroll
            for (int dy = -R; dy <= R; ++dy) {
              if (rx3<SH, R>(dz, dy) < 0) continue;
              int rr = row0 + ek + dy;
              rr = rr < 0 ? 0 : (rr >= C::YW ? C::YW - 1 : rr);
              const TS* er = sl + rr * XW + ecol0;
#pragma unroll
              for (int dx = -R; dx <= R; ++dx) {
                if (!tap3<SH, R>(dz, dy, dx)) continue;
                const TA c = cf.c[((dz + R) * F + (dy + R)) * F + (dx + R)];
                const TA v = to_acc(er[dx]);
                ev = fma(c, v, ev);
                if (dz == 0 && dy == 0 && dx == 0) ec = v;
              }
            }
          }
          // systolic exchange: one hop right, one hop left
#pragma unroll
          for (int i = 0; i < PY; ++i) {
#pragma unroll
            for (int h = 0; h < R; ++h) {
              TA v = __shfl_up_sync(FULL, pr[i][h], 1);
              if (lane == 0) v = inl[i][h];
              acc[i][h] += v;
              TA uu = __shfl_down_sync(FULL, pl[i][h], 1);
              if (lane == 31) uu = inr[i][h];
              acc[i][V - 1 - h] += uu;
            }
          }
          // the staged plane za+qi-2R has been read for the last time
          __syncwarp();
          if (lane == 0) mbar_arrive(&empty[(n + (uint32_t)qi) % S]);
          // boundary rule, rounding to the storage type, into the register ring
          if (edge_y || (copy ? zring : zout)) {
#pragma unroll
            for (int i = 0; i < PY; ++i) {
#pragma unroll
              for (int j = 0; j < V; ++j) {
                TA o = acc[i][j];
                const int64_t x = x0 + j, y = y0 + i;
                if (copy) {
                  if (zring || y < R || y >= ny - R || x < R || x >= nx - R) o = center[i][j];
                } else if (zout || !((row_in >> i) & 1u) || x >= nx) {
                  o = TA(0);
                }
                ring[u][i][j] = to_acc(from_acc<TS>(o));
              }
            }
          } else {
            if (xmask1) {
#pragma unroll
              for (int i = 0; i < PY; ++i)
#pragma unroll
                for (int j = 0; j < V; ++j)
                  if ((xmask1 >> j) & 1u) acc[i][j] = copy ? center[i][j] : TA(0);
            }
#pragma unroll
            for (int i = 0; i < PY; ++i)
#pragma unroll
              for (int j = 0; j < V; ++j) ring[u][i][j] = to_acc(from_acc<TS>(acc[i][j]));
          }
          if (copy ? (e_ring || zring) : (e_out || zout)) ev = copy ? ec : TA(0);
          ext[u] = to_acc(from_acc<TS>(ev));
          // the top and bottom R rows of my strip, for the warps above and below
          TS* hb = hbuf + ((size_t)((qi % D) * NW + warp) * 2 * R) * TX + lane * V;
#pragma unroll
          for (int r = 0; r < 2 * R; ++r) {
            const int row = r < R ? r : PY - 2 * R + r;
            store_row<TS, V>(hb + r * TX, ring[u][row]);
          }
        }
        if (lvl2 && ok) {
          // ------------------------------------------------- level 2
          const int64_t p2 = sg.za + qi - 2 * R - L;
          TA acc[PY][V];
          TA pr[PY][R], pl[PY][R], inl[PY][R], inr[PY][R];
#pragma unroll
          for (int i = 0; i < PY; ++i) {
#pragma unroll
            for (int j = 0; j < V; ++j) acc[i][j] = TA(0);
#pragma unroll
            for (int h = 0; h < R; ++h) pr[i][h] = pl[i][h] = inl[i][h] = inr[i][h] = TA(0);
          }
          const int wup = warp > 0 ? warp - 1 : 0;
          const int wdn = warp < NW - 1 ? warp + 1 : NW - 1;
#pragma unroll
          for (int dz = -R; dz <= R; ++dz) {
            const int ry = ry3<SH, R>(dz);
            if (ry < 0) continue;
            const int zs = (u + 2 * RL - R - L + dz) % RL;  // ring slot of plane p2+dz
            const int hs = (qi - R - L + dz) % D;           // halo-row slot of plane p2+dz
            const TS* hb = hbuf + (size_t)hs * NW * 2 * R * TX + lane * V;
            TA d[PY + 2 * RYM][V];
            TA hv[PY + 2 * RYM][R];
#pragma unroll
            for (int k = -RYM; k < PY + RYM; ++k) {
              if (k < -ry || k >= PY + ry) continue;
              if (k >= 0 && k < PY) {
#pragma unroll
                for (int j = 0; j < V; ++j) d[k + ry][j] = ring[zs][k][j];
              } else if (k < 0) {
                load_slot_row<TS, V>(d[k + ry], hb + (wup * 2 * R + 2 * R + k) * TX);
              } else {
                load_slot_row<TS, V>(d[k + ry], hb + (wdn * 2 * R + (k - PY)) * TX);
              }
              if (needs_xhalo<SH, R, PY>(dz, k)) {
#pragma unroll
                for (int h = 0; h < R; ++h) {
                  const int el = h * NR + k + EY, er = (R + h) * NR + k + EY;
                  hv[k + ry][h] = __shfl_sync(FULL, ext[zs], lane == 0 ? el : er);
                }
              } else {
#pragma unroll
                for (int h = 0; h < R; ++h) hv[k + ry][h] = TA(0);
              }
            }
#pragma unroll
            for (int i = 0; i < PY; ++i) {
#pragma unroll
              for (int dy = -RYM; dy <= RYM; ++dy) {
                if (dy < -ry || dy > ry || rx3<SH, R>(dz, dy) < 0) continue;
#pragma unroll
                for (int dx = -R; dx <= R; ++dx) {
                  if (!tap3<SH, R>(dz, dy, dx)) continue;
                  const TA c = cf.c[((dz + R) * F + (dy + R)) * F + (dx + R)];
                  const TA* src_row = d[i + dy + ry];
                  if (dx == 0) {
                    fma_row<V>(acc[i], c, src_row);
                  } else
#pragma unroll
                  for (int j = 0; j < V; ++j) {
                    const int t = j - dx;
                    if (t >= 0 && t < V) acc[i][t] = fma(c, src_row[j], acc[i][t]);
                    else if (t >= V) pr[i][t - V] = fma(c, src_row[j], pr[i][t - V]);
                    else pl[i][-1 - t] = fma(c, src_row[j], pl[i][-1 - t]);
                  }
#pragma unroll
                  for (int h = 0; h < R; ++h) {
                    const TA v = hv[i + dy + ry][h];
                    const int tl = -1 - h - dx;
                    const int tr = V + h - dx;
                    if (tl >= 0 && tl < V) inl[i][tl] = fma(c, v, inl[i][tl]);
                    if (tr >= 0 && tr < V) inr[i][V - 1 - tr] = fma(c, v, inr[i][V - 1 - tr]);
                  }
                }
              }
            }
          }
#pragma unroll
          for (int i = 0; i < PY; ++i) {
#pragma unroll
            for (int h = 0; h < R; ++h) {
              TA v = __shfl_up_sync(FULL, pr[i][h], 1);
              if (lane == 0) v = inl[i][h];
              acc[i][h] += v;
              TA uu = __shfl_down_sync(FULL, pl[i][h], 1);
              if (lane == 31) uu = inr[i][h];
              acc[i][V - 1 - h] += uu;
            }
          }
          // store the tile's rows H .. TY-H-1 that lie in the grid
          const int zc = (u + 2 * RL - R - L) % RL;  // ring slot of plane p2 (centre values)
          const bool zring2 = copy && (p2 < R || p2 >= nz - R);
          const bool ring_xy = copy && (x0 < R || x0 + V > nx - R || y0 < R || y0 + PY > ny - R);
          TS* outz = dst + (sg.b * nz + p2) * nxy + y0 * nx + x0;
          if (edges.fast && !zring2) {
            // whole vector stores of the rows the tile keeps (the x ring by a
            // per-lane column mask)
#pragma unroll
            for (int i = 0; i < PY; ++i) {
              if (edges.xring) {
#pragma unroll
                for (int j = 0; j < V; ++j)
                  if ((edges.xring >> j) & 1u) acc[i][j] = ring[zc][i][j];
              }
              if ((row_st >> i) & 1u) store_row<TS, V>(outz + i * nx, acc[i]);
            }
          } else {
#pragma unroll
          for (int i = 0; i < PY; ++i) {
            if (!((row_st >> i) & 1u)) continue;
            const int64_t y = y0 + i;
            TA o[V];
#pragma unroll
            for (int j = 0; j < V; ++j) o[j] = acc[i][j];
            if (ring_xy || zring2) {
#pragma unroll
              for (int j = 0; j < V; ++j) {
                const int64_t x = x0 + j;
                if (zring2 || y < R || y >= ny - R || x < R || x >= nx - R) o[j] = ring[zc][i][j];
              }
            }
            TS* outp = outz + i * nx;
            if (vec_seg) {
              store_row<TS, V>(outp, o);
            } else {
#pragma unroll
              for (int j = 0; j < V; ++j)
                if (x0 + j < nx) outp[j] = from_acc<TS>(o[j]);
            }
          }
          }
        }
        stop = consumer_bar_any(32 * NW, !ok);
      }
    };
    for (; qb < nit && !stop; qb += RL) static_for<RL>(iteration);
    if (stop) return;
    // the last 2R staged planes (zb .. zb+2R-1) were only read as the upper
    // z halo of level 1
    __syncwarp();
    if (lane == 0)
      for (int k = 0; k < 2 * R; ++k) mbar_arrive(&empty[(n + (uint32_t)(nzc + 2 * R + k)) % S]);
    n += (uint32_t)(nzc + 4 * R);
  }
}

}  // namespace ssam
