// 3D z-marching kernel with the thread's own cells kept in a register ring
// along z.
//
// The kernel of stencil3d.cuh reads, for every output plane z, the thread's
// rows of all 2R+1 planes z-R .. z+R from the shared-memory ring.  Here every
// plane's own rows (the thread's PY rows x V columns) are read from shared
// memory once, when the plane enters the window as plane z+R, and stay in a
// register ring of 2R+1 planes (unrolled over its length, so every slot is a
// fixed set of registers).  Shared memory still carries what other warps'
// data the thread needs -- the y-halo rows above and below its strip and the
// x-halo columns of lanes 0 and 31 -- and only for the planes whose taps leave
// the thread's own column (plane z for star stencils; z-1 .. z+1 for the
// 19-point operator).  Per output row and thread that is 1 + 2*ry/PY row reads
// instead of (2R+1) + 2*ry/PY, one full-barrier wait per plane instead of
// 2R+1, and a ring that only has to cover planes z-RH .. z+R plus the ones in
// flight.
//
// The producer warp, work split, boundary rules and bounded waits are those
// of stencil3d_kernel (produce_planes); the x exchange is the same one-hop
// systolic shuffle.
#pragma once

#include "stencil3d.cuh"

namespace ssam {

// Largest |dz| of a plane with taps off the centre column (0 for stars, 1
// for the 19-point operator): planes z-RH .. z+RH are read for halos.
template <int SH, int R>
__host__ __device__ constexpr int halo_reach_z() {
  int m = 0;
  for (int dz = -R; dz <= R; ++dz)
    for (int dy = -R; dy <= R; ++dy)
      for (int dx = -R; dx <= R; ++dx)
        if (tap3<SH, R>(dz, dy, dx) && (dy != 0 || dx != 0) && iabs_(dz) > m) m = iabs_(dz);
  return m;
}

template <typename TS, int SH, int R, int PY, int NW, int S, bool RHS = false, int V_ = 4>
__global__ void __launch_bounds__(32 * (NW + 1), (Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::MINB))
stencil3d_zreg_kernel(const __grid_constant__ CUtensorMap map, const TS* __restrict__ src,
                      TS* __restrict__ dst, Work3D w,
                      CoefBlock<typename Traits<TS>::TA,
                                Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::NC> cf) {
  using C = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>;
  using TA = typename C::TA;
  constexpr int V = C::V, XW = C::XW, HX = C::HX, RYM = C::RYM, TY = C::TY;
  constexpr int F = 2 * R + 1;
  constexpr int RH = halo_reach_z<SH, R>();
  constexpr unsigned FULL = 0xffffffffu;
  static_assert(S >= R + RH + 2, "ring must hold planes z-RH .. z+R plus one in flight");

  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* base =
      (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  TS* slots = (TS*)base;
  uint64_t* full = (uint64_t*)(base + S * C::SLOT_BYTES);
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
    produce_planes<TS, R, S, C>(map, src, w, slots, full, empty, lane);
    return;
  }

  // --------------------------------------------------------- consumer warps
  constexpr int SLOT_ELEMS = C::SLOT_BYTES / (int)sizeof(TS);
  uint32_t n = 0;  // ring position of the segment's first plane (za - R)
  for (int64_t it = blockIdx.x; it < w.items; it += gridDim.x) {
    const Seg3D sg = item_seg(it, w);
    const int tx = (int)(sg.tile % w.ntx), ty = (int)(sg.tile / w.ntx);
    const int64_t x0 = (int64_t)tx * C::TX + lane * V;  // my first column
    const int64_t y0 = (int64_t)ty * TY + warp * PY;    // my first row
    const int col = C::col_off(lane);                   // my first column in a slot
    const int row0 = RYM + warp * PY;                   // my first row in a slot
    const int nzc = (int)(sg.zb - sg.za);
    // does my strip touch the x/y ring that COPY keeps?
    const bool ring_xy = w.boundary == SSAM_BOUNDARY_COPY &&
                         (x0 < R || x0 + V > nx - R || y0 < R || y0 + PY > ny - R);
    // this thread's output rows at plane za (advanced by one plane per z), the
    // rows inside the grid, and whether every row of the segment takes whole
    // vector stores (alignment is the same for all of them when rows and
    // planes are vector multiples)
    constexpr int VB = V * (int)sizeof(TS);
    constexpr int AL = VB >= 16 ? 16 : 8;
    TS* outz = dst + (sg.b * nz + sg.za) * nxy + y0 * nx + x0;
    unsigned row_ok = 0;
#pragma unroll
    for (int i = 0; i < PY; ++i)
      if (y0 + i < ny && x0 < nx) row_ok |= 1u << i;
    const bool vec_seg = x0 + V <= nx && (uintptr_t)outz % AL == 0 &&
                         (nx * (int64_t)sizeof(TS)) % AL == 0 &&
                         (nxy * (int64_t)sizeof(TS)) % AL == 0;
    const StripEdges edges = strip_edges<R, PY, V>(x0, y0, nx, ny, w.boundary, row_ok, vec_seg);
    // right-hand side rows as raw 32-bit words (as in stencil3d_kernel)
    constexpr int RW = V * (int)sizeof(TS) / 4;
    constexpr bool PIPE = sizeof(TS) == 2;
    uint32_t rawc[RHS ? PY : 1][RW];
    uint32_t rawn[(RHS && PIPE) ? PY : 1][RW];
    const TS* rhz =
        RHS ? (const TS*)w.rhs + (sg.b * nz + sg.za) * nxy + y0 * nx + x0 : nullptr;
    const bool vec_rhs = RHS && x0 + V <= nx && (uintptr_t)rhz % AL == 0 &&
                         (nx * (int64_t)sizeof(TS)) % AL == 0 &&
                         (nxy * (int64_t)sizeof(TS)) % AL == 0;
    // rows of plane za + zi
    auto load_rhs = [&](int zi, uint32_t (&dstw)[RHS ? PY : 1][RW]) {
#pragma unroll
      for (int i = 0; i < (RHS ? PY : 1); ++i) {
        const TS* fp = rhz + (int64_t)zi * nxy + i * nx;
        const bool in_row = (row_ok >> i) & 1u;
        if (vec_rhs && in_row) {
          if constexpr (RW == 2) {
            const uint2 v = __ldg(reinterpret_cast<const uint2*>(fp));
            dstw[i][0] = v.x;
            dstw[i][1] = v.y;
          } else {
#pragma unroll
            for (int c = 0; c < RW / 4; ++c) {
              const uint4 v = __ldg(reinterpret_cast<const uint4*>(fp) + c);
              dstw[i][4 * c] = v.x;
              dstw[i][4 * c + 1] = v.y;
              dstw[i][4 * c + 2] = v.z;
              dstw[i][4 * c + 3] = v.w;
            }
          }
        } else {
          TS tmp[V];
#pragma unroll
          for (int j = 0; j < V; ++j)
            tmp[j] = (in_row && x0 + j < nx) ? fp[j] : from_acc<TS>(TA(0));
          memcpy(dstw[i], tmp, sizeof(tmp));
        }
      }
    };
    if constexpr (RHS && PIPE) load_rhs(0, rawc);

    // register ring: plane p = za - R + k sits in zr[k % F]
    TA zr[F][PY][V];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 2 * R; ++k) {
      const uint32_t q = n + (uint32_t)k;
      if (!mbar_wait(&full[q % S], (q / S) & 1, w.wait_ns)) ok = false;
      const TS* sl = slots + (size_t)(q % S) * SLOT_ELEMS;
#pragma unroll
      for (int i = 0; i < PY; ++i) load_slot_row<TS, V>(zr[k][i], sl + (row0 + i) * XW + col);
    }
    if (!ok) {
      if (lane == 0) atomicCAS(w.err, 0, 3);
      return;
    }
    // planes za-R .. za-RH-1 are not read again (no halos needed from them)
    if constexpr (R - RH > 0) {
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < R - RH; ++k) mbar_arrive(&empty[(n + (uint32_t)k) % S]);
    }

    for (int zz = 0; zz < nzc; zz += F) {
#pragma unroll
      for (int u = 0; u < F; ++u) {
        const int zi = zz + u;
        if (zi >= nzc) break;
        const int64_t z = sg.za + zi;
        const uint32_t q0 = n + (uint32_t)zi;  // ring position of plane z-R
        if constexpr (RHS) {
          if constexpr (PIPE) {
            if (zi + 1 < nzc) load_rhs(zi + 1, rawn);
          } else {
            load_rhs(zi, rawc);
          }
        }
        // the plane entering the register ring: z+R
        {
          const uint32_t q = q0 + 2 * R;
          if (!mbar_wait(&full[q % S], (q / S) & 1, w.wait_ns)) {
            if (lane == 0) atomicCAS(w.err, 0, 3);
            return;
          }
          const TS* sl = slots + (size_t)(q % S) * SLOT_ELEMS;
#pragma unroll
          for (int i = 0; i < PY; ++i)
            load_slot_row<TS, V>(zr[(u + 2 * R) % F][i], sl + (row0 + i) * XW + col);
        }
        TA acc[PY][V];
        TA pr[PY][R];   // partial sums for the lane to the right
        TA pl[PY][R];   // partial sums for the lane to the left
        TA inl[PY][R];  // lane 0: contributions of the left halo columns
        TA inr[PY][R];  // lane 31: contributions of the right halo columns
#pragma unroll
        for (int i = 0; i < PY; ++i) {
#pragma unroll
          for (int j = 0; j < V; ++j) acc[i][j] = TA(0);
#pragma unroll
          for (int q = 0; q < R; ++q) pr[i][q] = pl[i][q] = inl[i][q] = inr[i][q] = TA(0);
        }
#pragma unroll
        for (int dz = -R; dz <= R; ++dz) {
          const int ry = ry3<SH, R>(dz);  // folds to a constant once unrolled
          if (ry < 0) continue;
          const int zs = (u + R + dz) % F;  // register slot of plane z+dz
          const TS* sl = slots + (size_t)((q0 + (uint32_t)(R + dz)) % S) * SLOT_ELEMS;
          // rows -ry .. PY+ry-1 of plane z+dz: own rows from the ring, the
          // y halo from the plane's slot
          TA d[PY + 2 * RYM][V];
          TA hv[PY + 2 * RYM][R];
#pragma unroll
          for (int k = -RYM; k < PY + RYM; ++k) {
            if (k < -ry || k >= PY + ry) continue;
            const TS* rowp = sl + (row0 + k) * XW + col;
            if (k >= 0 && k < PY) {
#pragma unroll
              for (int j = 0; j < V; ++j) d[k + ry][j] = zr[zs][k][j];
            } else {
              load_slot_row<TS, V>(d[k + ry], rowp);
            }
            // x halo for lanes 0 / 31 (the loads whose values no tap uses are
            // dropped by the compiler): lane 0 reads left of its strip, every
            // other lane lane 31's right halo column -- two addresses a warp,
            // a broadcast without bank conflicts
            const TS* hrow = sl + (row0 + k) * XW;
#pragma unroll
            for (int h = 0; h < R; ++h)
              hv[k + ry][h] =
                  to_acc(hrow[lane == 0 ? C::col_off(0) - 1 - h : C::col_off(31) + V + h]);
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
                  const int t = j - dx;  // column that source column j feeds
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
        // systolic exchange: one hop right, one hop left (R <= V)
#pragma unroll
        for (int i = 0; i < PY; ++i) {
#pragma unroll
          for (int qq = 0; qq < R; ++qq) {
            TA v = __shfl_up_sync(FULL, pr[i][qq], 1);
            if (lane == 0) v = inl[i][qq];
            acc[i][qq] += v;
            TA uu = __shfl_down_sync(FULL, pl[i][qq], 1);
            if (lane == 31) uu = inr[i][qq];
            acc[i][V - 1 - qq] += uu;
          }
        }
        // plane z-RH has been read for the last time (at the segment's end,
        // every plane still held)
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(&empty[(q0 + (uint32_t)(R - RH)) % S]);
          if (zi == nzc - 1)
            for (int k = R - RH + 1; k <= 2 * R; ++k) mbar_arrive(&empty[(q0 + (uint32_t)k) % S]);
        }
        // store PY rows x V columns
        const bool zring = w.boundary == SSAM_BOUNDARY_COPY && (z < R || z >= nz - R);
        const int zc = (u + R) % F;  // register slot of plane z (the centre values)
        // (the 8-column 4- and 8-byte tiles measured faster without the
        // separate fast store: 512^3 FP32 7-point 0.174 against 0.206 ms)
        constexpr bool kFastStore = sizeof(TS) == 2 || V == 4;
        if (kFastStore && edges.fast && !zring) {
#pragma unroll
          for (int i = 0; i < PY; ++i) {
            TA o[V];
#pragma unroll
            for (int j = 0; j < V; ++j) o[j] = acc[i][j];
            if constexpr (RHS) {
              TA fv[V];
              words_to_acc<TS, V>(fv, rawc[i]);
#pragma unroll
              for (int j = 0; j < V; ++j) o[j] = fma((TA)w.rhs_scale, fv[j], o[j]);
            }
            if (edges.xring) {
#pragma unroll
              for (int j = 0; j < V; ++j)
                if ((edges.xring >> j) & 1u) o[j] = zr[zc][i][j];
            }
            if (x0 < nx) store_row<TS, V>(outz + i * nx, o);
          }
        } else {
        const bool any_ring = ring_xy || zring;
#pragma unroll
        for (int i = 0; i < PY; ++i) {
          const int64_t y = y0 + i;
          if (!((row_ok >> i) & 1u)) continue;
          TA o[V];
#pragma unroll
          for (int j = 0; j < V; ++j) o[j] = acc[i][j];
          if constexpr (RHS) {
            TA fv[V];
            words_to_acc<TS, V>(fv, rawc[i]);
#pragma unroll
            for (int j = 0; j < V; ++j) o[j] = fma((TA)w.rhs_scale, fv[j], o[j]);
          }
          if (any_ring) {
#pragma unroll
            for (int j = 0; j < V; ++j) {
              const int64_t x = x0 + j;
              if (zring || y < R || y >= ny - R || x < R || x >= nx - R) o[j] = zr[zc][i][j];
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
        outz += nxy;
        if constexpr (RHS && PIPE) {
#pragma unroll
          for (int i = 0; i < PY; ++i)
#pragma unroll
            for (int c = 0; c < RW; ++c) rawc[i][c] = rawn[i][c];
        }
      }
    }
    n += (uint32_t)(nzc + 2 * R);
  }
}

}  // namespace ssam
