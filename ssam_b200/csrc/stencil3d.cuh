// 3D stencils for sm_100a: persistent z-marching CTAs fed by TMA.
//
// Method (the reference's 3D scheme, ssai-3dstencil/tmp3d7pt-v2.cu:62-208:
// "y-strip in registers, x by shuffles, z through shared memory"), laid out
// for Blackwell:
//   * a CTA owns column tiles of 32*V x TY cells and walks them along z.  A
//     producer warp stages each z-plane of the tile -- 32*V + 2*HX columns by
//     TY + 2*RY rows, halos included -- into a ring of S shared-memory slots
//     with one cp.async.bulk.tensor (TMA, no multicast) per plane, or two
//     when the row is wider than a TMA box (256 elements; V = 8: the left
//     half with the left halo, the right half with the right one, stored one
//     after the other in the slot), signalled through mbarriers (full: bytes
//     landed; empty: consumers are done);
//   * NW consumer warps each own a 32*V x PY strip.  A thread owns V (4 or 8)
//     consecutive columns; for every plane of the stencil it reads its rows
//     (plus the y reach) from the slot into registers, forms its own
//     contributions and the partial sums destined for the neighbouring
//     lanes' columns, and the partial sums move one lane downstream with
//     __shfl_up/down_sync (lanes 0 and 31 take theirs from the slot's halo
//     columns instead);
//   * z-neighbours are read from the slots of the adjacent planes (shared
//     memory between warps, as in the reference);
//   * work items are (z chunk, column tile) pairs taken chunk-major with a
//     stride of the grid size by a persistent grid sized to the SMs, so that
//     neighbouring tiles of the same z chunk run at the same time and share
//     their halos through L2;
//   * every mbarrier wait is bounded (%globaltimer): on expiry the kernel
//     records an error code, the producer drains its own copies in flight
//     (again bounded), and the CTA returns.
//
// Shapes: STAR (7-pt r=1, 13-pt r=2, ...: taps on the three axes) and
// POISSON19 (all taps with |d|_inf <= 1 and |d|_1 <= 2: the reference's
// 19-point operator, tmpPoisson.cu:369-386).
#pragma once

#include <cuda.h>

#include <type_traits>

#include "ssam_internal.cuh"

namespace ssam {

enum { SH3_STAR = 0, SH3_POISSON19 = 1 };

__host__ __device__ constexpr int iabs_(int v) { return v < 0 ? -v : v; }

template <int SH, int R>
__host__ __device__ constexpr bool tap3(int dz, int dy, int dx) {
  return SH == SH3_STAR
             ? ((dy == 0 && dx == 0) || (dz == 0 && dx == 0) || (dz == 0 && dy == 0))
             : (iabs_(dz) <= 1 && iabs_(dy) <= 1 && iabs_(dx) <= 1 &&
                iabs_(dz) + iabs_(dy) + iabs_(dx) <= 2);
}

// y reach needed in plane dz; x reach needed in row (dz, dy).
template <int SH, int R>
__host__ __device__ constexpr int ry3(int dz) {
  int m = -1;
  for (int dy = -R; dy <= R; ++dy)
    for (int dx = -R; dx <= R; ++dx)
      if (tap3<SH, R>(dz, dy, dx) && iabs_(dy) > m) m = iabs_(dy);
  return m;  // -1: plane unused
}
template <int SH, int R>
__host__ __device__ constexpr int rx3(int dz, int dy) {
  int m = -1;
  for (int dx = -R; dx <= R; ++dx)
    if (tap3<SH, R>(dz, dy, dx) && iabs_(dx) > m) m = iabs_(dx);
  return m;
}

// V columns a thread (4, or 8: a 256-column tile).  A plane of the tile with
// its halo columns is staged as NBOX boxes side by side (one TMA copy each:
// a box is at most 256 elements wide), box b holding columns b*BW .. of the
// staged row; a lane reads only its own box (lanes 0..15 the first, 16..31 the
// second when NBOX = 2, and the halo columns lanes 0 / 31 need are in theirs).
template <typename TS, int SH, int R, int PY, int NW, int S, int V_ = 4>
struct Stencil3DCfg {
  using TA = typename Traits<TS>::TA;
  static constexpr int V = V_;                      // columns per thread
  static constexpr int TX = 32 * V;                 // tile columns
  static constexpr int HX = 16 / (int)sizeof(TS);   // halo columns (16 bytes)
  static constexpr int TY = NW * PY;                // tile rows
  static constexpr int RYM = ry3<SH, R>(0) > 0 ? ry3<SH, R>(0) : 1;  // max y reach
  static constexpr int NBOX = TX + 2 * HX > 256 ? 2 : 1;  // staged boxes per plane
  static constexpr int BW = (TX + 2 * HX) / NBOX;   // box width (elements)
  static constexpr int XW = BW;                     // slot row length (within a box)
  static constexpr int YW = TY + 2 * RYM;           // slot rows
  static constexpr int BOXE = BW * YW;              // elements of one box
  // element stride between the boxes of a slot: a TMA copy's shared-memory
  // destination must be 128-byte aligned
  static constexpr int BOXS = (BOXE * (int)sizeof(TS) + 127) / 128 * 128 / (int)sizeof(TS);
  static constexpr int LPB = 32 / NBOX;             // lanes reading one box
  static constexpr int SLOT_BYTES = NBOX * BOXS * (int)sizeof(TS);
  // element offset, within a slot, of row 0 / a lane's first column
  __host__ __device__ static constexpr int col_off(int lane) {
    return (lane / LPB) * BOXS + (lane / LPB == 0 ? HX : 0) + (lane % LPB) * V;
  }
  static_assert(NBOX == 1 || (TX / 2 + HX) * (int)sizeof(TS) % 16 == 0,
                "the second box must start on a 16-byte column");
  static_assert((BOXS * (int)sizeof(TS)) % 128 == 0 && SLOT_BYTES % 128 == 0,
                "every box of every slot starts on a 128-byte boundary");
  static constexpr int SMEM = S * SLOT_BYTES + 2 * S * 8 + 128;
  static constexpr int NC = (2 * R + 1) * (2 * R + 1) * (2 * R + 1);
  static constexpr int THREADS = 32 * (NW + 1);
  // CTAs per SM the register budget is cut for: two when two rings fit in
  // shared memory and the CTA is at most 12 warps of 4-column threads, else
  // one (8-column threads hold twice the cells and would spill at half)
  static constexpr int MINB = (V == 4 && NW < 12 && 2 * (SMEM + 1024) <= 233472) ? 2 : 1;
  static_assert(R <= HX && R <= V, "x reach must fit in the halo and one lane hop");
};

struct Work3D {
  int64_t nx, ny, nz;
  int nb;                // independent grids stacked along a 4th axis
  int ntx, nty;          // column tiles
  int zc;                // planes per work item (z chunk)
  int64_t items;         // nb*ntx*nty*ceil(nz/zc) (grid, chunk, tile) work items
  const void* rhs;       // optional: out += rhs_scale * rhs (same layout), else NULL
  double rhs_scale;
  int boundary;
  int use_tma;
  unsigned long long wait_ns;
  int* err;              // device error word (0 = ok)
};

// ------------------------------------------------------------ PTX helpers --

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)),
               "r"(bytes)
               : "memory");
}
// Waits for the phase with parity `par` to complete; false after `ns`.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned par, unsigned long long ns) {
  const uint32_t a = smem_u32(b);
  uint32_t ok = 0;
  asm volatile(
      "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
      "selp.u32 %0, 1, 0, p; }"
      : "=r"(ok)
      : "r"(a), "r"(par)
      : "memory");
  if (ok) return true;
  const uint64_t t0 = gtimer();
  while (true) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; "
        "selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(a), "r"(par)
        : "memory");
    if (ok) return true;
    if (gtimer() - t0 > ns) return false;
  }
}
// One z-plane tile of grid b: a 4D tiled TMA load (x, y, z, b), no multicast.
// Coordinates outside the tensor (halo beyond a face, z beyond a grid of the
// batch) are filled with zeros by the copy engine.
__device__ __forceinline__ void tma_load_plane(void* dst, const CUtensorMap* map, int x, int y,
                                               int z, int b, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(b), "r"(smem_u32(bar))
      : "memory");
}

// V elements of a staged plane row (16-byte aligned for 4- and 8-byte types,
// 8-byte aligned for 2-byte types).
template <typename TS, int V, typename TA>
__device__ __forceinline__ void load_slot_row(TA (&d)[V], const TS* p) {
  constexpr int B = V * (int)sizeof(TS);
  if constexpr (B % 16 == 0) {
#pragma unroll
    for (int c = 0; c < B / 16; ++c) {
      const uint4 u = reinterpret_cast<const uint4*>(p)[c];
      const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
      words_to_acc<TS, 16 / (int)sizeof(TS)>(d + c * (16 / sizeof(TS)), wd);
    }
  } else if constexpr (B == 8) {
    const uint2 u = *reinterpret_cast<const uint2*>(p);
    const uint32_t wd[2] = {u.x, u.y};
    words_to_acc<TS, V>(d, wd);
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) d[k] = to_acc(p[k]);
  }
}

template <typename TS, int V, typename TA>
__device__ __forceinline__ void store_row(TS* p, const TA (&o)[V]) {
  constexpr int B = V * (int)sizeof(TS);
  if constexpr (B % 16 == 0) {
    store_vec<TS, V>(p, o);
  } else if constexpr (B == 8) {
    uint32_t wd[2];
    acc_to_words<TS, V>(wd, o);
    *reinterpret_cast<uint2*>(p) = make_uint2(wd[0], wd[1]);
  } else {
#pragma unroll
    for (int k = 0; k < V; ++k) p[k] = from_acc<TS>(o[k]);
  }
}

// acc[t] += c * src[t] over a thread's V columns (a tap with dx = 0).  For a
// float accumulator the columns go in pairs through the packed two-lane FP32
// FMA (FFMA2): each lane is rounded like a scalar fma, so the sums are the
// same bits, with half the FMA instructions of the scalar loop.
template <int V, typename TA>
__device__ __forceinline__ void fma_row(TA (&acc)[V], TA c, const TA* src) {
  if constexpr (std::is_same<TA, float>::value && V % 2 == 0) {
    const float2 c2 = make_float2(c, c);
#pragma unroll
    for (int j = 0; j < V; j += 2) {
      float2 a = make_float2(acc[j], acc[j + 1]);
      a = __ffma2_rn(c2, make_float2(src[j], src[j + 1]), a);
      acc[j] = a.x;
      acc[j + 1] = a.y;
    }
  } else {
#pragma unroll
    for (int j = 0; j < V; ++j) acc[j] = fma(c, src[j], acc[j]);
  }
}

// Boundary bookkeeping of one thread's PY x V strip for the store paths.
// xring: the columns of this lane inside the COPY ring along x (only lanes at
// the grid's x faces have any); fast: warp-uniform -- every lane that stores
// has all its rows in the grid and whole vector stores, and no row of the
// warp's strip lies in the COPY ring along y.  A fast warp stores each plane
// without per-row checks (the x ring by a per-lane column mask), so the rare
// edge lanes do not send their whole warp down the general path.
struct StripEdges {
  unsigned xring;
  bool fast;
};
template <int R, int PY, int V>
__device__ __forceinline__ StripEdges strip_edges(int64_t x0, int64_t y0, int64_t nx,
                                                  int64_t ny, int boundary, unsigned rows_ok,
                                                  bool vec_seg) {
  StripEdges e;
  e.xring = 0;
  const bool copy = boundary == SSAM_BOUNDARY_COPY;
  if (copy) {
#pragma unroll
    for (int j = 0; j < V; ++j)
      if (x0 + j < R || x0 + j >= nx - R) e.xring |= 1u << j;
  }
  const bool yring = copy && (y0 < R || y0 + PY > ny - R);
  const bool lane_ok = x0 >= nx || (vec_seg && rows_ok == (1u << PY) - 1u);
  e.fast = __all_sync(0xffffffffu, lane_ok) && !yring;
  return e;
}

// Work item `it` = (z chunk, column tile), chunk-major.  CTAs take items
// it = blockIdx.x + k*gridDim.x, so at any moment the grid works on a band
// of consecutive items -- the same z chunk of neighbouring tiles -- and the
// halo rows and columns that neighbouring tiles share are served by L2.
struct Seg3D {
  int64_t tile, za, zb, b;
};
__device__ __forceinline__ Seg3D item_seg(int64_t it, const Work3D& w) {
  const int64_t ntiles = (int64_t)w.ntx * w.nty;
  const int64_t nchunks = (w.nz + w.zc - 1) / w.zc;
  Seg3D s;
  s.tile = it % ntiles;
  const int64_t rest = it / ntiles;
  s.za = (rest % nchunks) * w.zc;
  s.b = rest / nchunks;
  s.zb = s.za + w.zc < w.nz ? s.za + w.zc : w.nz;
  return s;
}

// The producer warp of a 3D CTA: stages every plane of every work item of
// this CTA -- planes za-ZR .. zb+ZR-1 of the item's column tile, halos
// included -- into the ring of S slots, in order.  A slot is reused once the
// consumer warps have released its previous plane (empty barrier); a TMA copy
// signals `full` by bytes, the plain-load path by 32 arrivals.  Every wait is
// bounded: on expiry the error word is set and staging stops.  Before
// returning, the last use of every slot must have landed.  Column tiles are
// C::TX wide; tile row ty starts at grid row ty*YSTRIDE - YOFF (the kernels
// with fused steps overlap their tiles by YOFF rows on each side).
template <typename TS, int R, int S, typename C, int ZR = R, int YSTRIDE = C::TY,
          int YOFF = 0>
__device__ __forceinline__ void produce_planes(const CUtensorMap& map, const TS* __restrict__ src,
                                               const Work3D& w, TS* slots, uint64_t* full,
                                               uint64_t* empty, int lane) {
  using TA = typename C::TA;
  constexpr int XW = C::XW, HX = C::HX, RYM = C::RYM;
  const int64_t nx = w.nx, ny = w.ny, nz = w.nz, nxy = nx * ny;
  uint32_t n = 0;  // planes issued so far (ring position)
  bool ok = true;
  for (int64_t it = blockIdx.x; ok && it < w.items; it += gridDim.x) {
    const Seg3D sg = item_seg(it, w);
    const int tx = (int)(sg.tile % w.ntx), ty = (int)(sg.tile / w.ntx);
    const int gx = tx * C::TX - HX, gy = ty * YSTRIDE - YOFF - RYM;
    for (int64_t p = sg.za - ZR; p < sg.zb + ZR; ++p, ++n) {
      const int s = n % S;
      const unsigned use = n / S;
      if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1, w.wait_ns)) {
        if (lane == 0) atomicCAS(w.err, 0, 1);
        ok = false;
        break;
      }
      TS* slot = slots + (size_t)s * (C::SLOT_BYTES / sizeof(TS));
      if (w.use_tma) {
        if (lane == 0) {
          mbar_expect_tx(&full[s], (unsigned)(C::NBOX * C::BOXE * sizeof(TS)));
#pragma unroll
          for (int b = 0; b < C::NBOX; ++b)
            tma_load_plane(slot + b * C::BOXS, &map, gx + b * XW, gy, (int)p, (int)sg.b,
                           &full[s]);
        }
      } else {
        // plain loads for grids whose rows are not 16-byte multiples
        for (int i = lane; i < C::NBOX * C::BOXE; i += 32) {
          const int b = i / C::BOXE, e = i % C::BOXE;
          const int r = e / XW, c = e % XW;
          const int64_t x = gx + b * XW + c, y = gy + r;
          TS v = from_acc<TS>(TA(0));
          if (x >= 0 && x < nx && y >= 0 && y < ny && p >= 0 && p < nz)
            v = src[(sg.b * nz + p) * nxy + y * nx + x];
          slot[b * C::BOXS + e] = v;
        }
        mbar_arrive(&full[s]);
      }
      __syncwarp();
    }
  }
  // drain: the last use of every slot must have landed before exit
  if (w.use_tma && lane == 0) {
    const uint32_t first = n > (uint32_t)S ? n - S : 0;
    for (uint32_t k = first; k < n; ++k)
      if (!mbar_wait(&full[k % S], (k / S) & 1, w.wait_ns)) atomicCAS(w.err, 0, 2);
  }
}

// RHS: the Jacobi form out = stencil(in) + rhs_scale * rhs.  Its rows are
// loaded at the top of every plane, so their latency overlaps the plane's
// barrier waits and arithmetic (instances without it carry no rhs code).
template <typename TS, int SH, int R, int PY, int NW, int S, bool RHS = false, int V_ = 4>
__global__ void __launch_bounds__(32 * (NW + 1), (Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::MINB))
stencil3d_kernel(const __grid_constant__ CUtensorMap map, const TS* __restrict__ src,
                 TS* __restrict__ dst, Work3D w,
                 CoefBlock<typename Traits<TS>::TA,
                           Stencil3DCfg<TS, SH, R, PY, NW, S, V_>::NC> cf) {
  using C = Stencil3DCfg<TS, SH, R, PY, NW, S, V_>;
  using TA = typename C::TA;
  constexpr int V = C::V, XW = C::XW, HX = C::HX, RYM = C::RYM, TY = C::TY;
  constexpr int F = 2 * R + 1;
  constexpr unsigned FULL = 0xffffffffu;
  static_assert(S >= 2 * R + 2, "ring must hold the stencil window plus one plane");

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
  uint32_t n = 0;  // ring position of the segment's first plane
  for (int64_t it = blockIdx.x; it < w.items; it += gridDim.x) {
    const Seg3D sg = item_seg(it, w);
    const int tx = (int)(sg.tile % w.ntx), ty = (int)(sg.tile / w.ntx);
    const int64_t x0 = (int64_t)tx * C::TX + lane * V;  // my first column
    const int64_t y0 = (int64_t)ty * TY + warp * PY;    // my first row
    const int col = C::col_off(lane);                   // my first column in a slot
    const int row0 = RYM + warp * PY;                   // my first row in a slot
    const int64_t seg_planes = sg.zb - sg.za + 2 * R;
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
    // right-hand side rows, kept as raw 32-bit words: 2-byte types load plane
    // z+1 while plane z is computed (software pipelined across the z loop);
    // wider types load plane z at the top of its iteration (registers)
    constexpr int RW = V * (int)sizeof(TS) / 4;  // words per rhs row
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
    for (int64_t z = sg.za; z < sg.zb; ++z) {
      // planes z-R .. z+R sit at ring positions n + (z - za) .. + 2R
      const uint32_t q0 = n + (uint32_t)(z - sg.za);
      if constexpr (RHS) {
        if constexpr (PIPE) {
          if (z + 1 < sg.zb) load_rhs((int)(z + 1 - sg.za), rawn);
        } else {
          load_rhs((int)(z - sg.za), rawc);
        }
      }
      bool ok = true;
#pragma unroll
      for (int k = 0; k < F; ++k) {
        const uint32_t q = q0 + k;
        if (!mbar_wait(&full[q % S], (q / S) & 1, w.wait_ns)) ok = false;
      }
      if (!ok) {
        if (lane == 0) atomicCAS(w.err, 0, 3);
        return;
      }
      TA acc[PY][V];
      TA pr[PY][R];   // partial sums for the lane to the right
      TA pl[PY][R];   // partial sums for the lane to the left
      TA inl[PY][R];  // lane 0: contributions of the left halo columns
      TA inr[PY][R];  // lane 31: contributions of the right halo columns
      TA center[PY][V];
#pragma unroll
      for (int i = 0; i < PY; ++i) {
#pragma unroll
        for (int j = 0; j < V; ++j) acc[i][j] = center[i][j] = TA(0);
#pragma unroll
        for (int q = 0; q < R; ++q) pr[i][q] = pl[i][q] = inl[i][q] = inr[i][q] = TA(0);
      }
#pragma unroll
      for (int dz = -R; dz <= R; ++dz) {
        const int ry = ry3<SH, R>(dz);  // folds to a constant once unrolled
        if (ry < 0) continue;
        const uint32_t q = q0 + (uint32_t)(dz + R);
        const TS* slot = slots + (size_t)(q % S) * (C::SLOT_BYTES / sizeof(TS));
        // y-strip register cache of this plane: rows -ry .. PY+ry-1
        TA d[PY + 2 * RYM][V];
        TA hv[PY + 2 * RYM][R];
#pragma unroll
        for (int k = -RYM; k < PY + RYM; ++k) {
          if (k < -ry || k >= PY + ry) continue;
          const TS* rowp = slot + (row0 + k) * XW + col;
          load_slot_row<TS, V>(d[k + ry], rowp);
          // the x-halo columns, used by lanes 0 and 31 only: lane 0 reads
          // left of its strip and every other lane reads lane 31's right halo
          // column, so the warp touches two addresses (a broadcast, no bank
          // conflict) and issues the load once
          const TS* hrow = slot + (row0 + k) * XW;
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
                const int t = j - dx;  // column that source column j feeds
                if (t >= 0 && t < V) acc[i][t] = fma(c, src_row[j], acc[i][t]);
                else if (t >= V) pr[i][t - V] = fma(c, src_row[j], pr[i][t - V]);
                else pl[i][-1 - t] = fma(c, src_row[j], pl[i][-1 - t]);
              }
#pragma unroll
              for (int h = 0; h < R; ++h) {
                const TA v = hv[i + dy + ry][h];
                const int tl = -1 - h - dx;  // as lane 0: halo column -1-h feeds tl
                const int tr = V + h - dx;   // as lane 31: halo column V+h feeds tr
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
          TA u = __shfl_down_sync(FULL, pl[i][qq], 1);
          if (lane == 31) u = inr[i][qq];
          acc[i][V - 1 - qq] += u;
        }
      }
      // planes whose last use this was: z - R (and the rest at segment end)
      __syncwarp();
      if (lane == 0) {
        const uint32_t q = q0;
        mbar_arrive(&empty[q % S]);
        if (z == sg.zb - 1)
          for (uint32_t k = 1; k < (uint32_t)F; ++k) mbar_arrive(&empty[(q0 + k) % S]);
      }
      // store PY rows x V columns
      const bool zring = w.boundary == SSAM_BOUNDARY_COPY && (z < R || z >= nz - R);
      if (edges.fast && !zring) {
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
              if ((edges.xring >> j) & 1u) o[j] = center[i][j];
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
            if (zring || y < R || y >= ny - R || x < R || x >= nx - R) o[j] = center[i][j];
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
    n += (uint32_t)seg_planes;
  }
}

}  // namespace ssam
