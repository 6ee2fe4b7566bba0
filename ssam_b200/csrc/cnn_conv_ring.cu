// Persistent, bulk-copy-fed implicit-GEMM 3D convolution for the warm-start
// CNN (forward, and the data gradient with mirrored / transposed weights).
//
// Activations are "planar halves": [2][nb][n][n][n][8] BF16 -- channels 0-7
// of every voxel in one plane, channels 8-15 in the next -- so a grid row of
// one half is n * 16 contiguous bytes and moves as one cp.async.bulk copy.
//
// Shared-memory operand trick: the 27 taps of a 3x3x3 convolution read the
// same input shifted by (dz, dy, dx) * d (d = dilation).  Each input plane a
// work item needs is staged as a "slab" per half: TY + 2d rows of XP = n + d
// voxels, row r at voxel r * XP + d (the d voxels before it stay zero).  In
// that padded, row-major layout a shift by (dy, dx) is a constant offset of
// (dy * XP + dx) * d voxels, and the zeros between rows are the x-halo of
// both neighbouring rows.  So the A operand of every tap is a slab seen from
// another start address: a K-major, no-swizzle UMMA descriptor whose 8-row
// core matrices are 8 consecutive voxels (SBO = 128 B) and whose two K halves
// (channels 0-7 / 8-15) are the two half-slabs (LBO).  Rows outside the grid
// are copied from a row of zeros, so every copy has the same size.
//
// A work item is (grid b, TY output rows from y0, a chunk of output planes
// z0 ..).  With d = 1 it marches in z: planes z0-1 .. z0+ZC are staged once
// each into a ring of plane slots and every output plane uses three
// consecutive slots; with d > 1 each output plane stages its own three
// planes z-d, z, z+d.  Output positions are enumerated in the padded layout,
// 128 per MMA tile; positions in the gaps or past the last row are computed
// and discarded.
//
// Warp roles of the 27-MMA kernel (one CTA per SM, persistent over items):
//   warp 0      producer: 2 * (TY + 2d) row copies per plane into the ring
//               (mbarrier full / empty per slot)
//   warp 1      MMA issuer: TILES x 27 tcgen05.mma (128 x 16 x 16, BF16 in,
//               FP32 in TMEM) per output plane; two accumulator buffers
//   warps 2-5   epilogue: tcgen05.ld of each tile's accumulators, scale,
//               add the optional addend, round to BF16, store valid voxels
// Dilation 1 runs the z-stacked kernel further down instead (three z taps
// on the MMA's N side; by default two CTAs a SM, three MMA-issuing warps
// and two groups of epilogue warps a CTA).
// Every wait is bounded by %globaltimer; on expiry the kernel records error
// code 8 and winds down (drains its copies and MMAs, frees tensor memory).
#include <stdlib.h>
#include <string.h>

#include <algorithm>

#include "cnn_tc.cuh"

namespace ssam {

int device_error_word(int** out);

namespace {

constexpr int kFrontGuard = 8;   // voxels (16 B each) before every slab
constexpr int kMaxTiles = 16;    // 2 accumulator buffers x 16 tiles x 16 columns
constexpr int kMaxSlots = 8;
constexpr int kThreads = 192;
constexpr int kSmemLimit = 227 * 1024;
constexpr int kMaxRow = 1024;    // voxels per grid row (the zero row's length)

__device__ __align__(16) uint4 g_zero_row[kMaxRow];  // zero-initialised, never written

struct ConvArgs {
  const __nv_bfloat16* in;      // planar halves
  const __nv_bfloat16* addend;  // NULL or planar halves, added after scaling
  const __nv_bfloat16* w;       // [16][27][ci_total]
  __nv_bfloat16* out;           // planar halves
  float out_scale;
  int ci_total, ci_off;         // this pass uses input channels ci_off .. +15
  int n, dil, ty, xp, tiles, nyb, nzc, zc, box_rows, slab, slots;
  int tmem_cols;                // TMEM columns a CTA allocates (512, or 256 at 2 CTAs a SM)
  int64_t half;                 // elements per half-plane: nb * n^3 * 8
  int64_t items;
  int* err;
  unsigned long long wait_ns;
};

struct Plan {
  int ty, xp, tiles, box_rows, slab, slots, smem;
  int ctas_per_sm = 1;
};

// Largest TY (rows per item) with at most kMaxTiles MMA tiles per output
// plane and a ring of at least 4 plane slots in shared memory.
bool make_plan(int n, int dil, Plan* p) {
  const int xp = n + dil;
  if (n > kMaxRow) return false;
  for (int ty = std::min(n, 16); ty >= 1; ty /= 2) {
    const int box_rows = ty + 2 * dil;
    const int tiles = (ty * xp + 127) / 128;
    if (tiles > kMaxTiles) continue;
    const int tail = tiles * 128 - ty * xp + dil;  // reach past the last row of the last tile
    const int slab = ((kFrontGuard + box_rows * xp + tail) * 16 + 127) / 128 * 128;
    const int avail = kSmemLimit - 1024 - 27 * 512 - 256;
    const int slots = std::min(kMaxSlots, avail / (2 * slab));
    if (slots < 4) continue;
    // (at least 120 KB, so that one CTA -- and its 512 TMEM columns -- is
    // alone on its SM)
    const int smem = std::max(1024 + 27 * 512 + slots * 2 * slab + 256, 120 * 1024);
    *p = Plan{ty, xp, tiles, box_rows, slab, slots, smem};
    return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_addr(b)) : "memory");
}
// Contiguous global -> shared copy (16-byte aligned, size a multiple of 16),
// completion counted on `bar`.  No multicast.
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

struct Item {
  int b, y0, z0, nout, len;  // len: plane positions the item streams
};

__device__ __forceinline__ Item decode(const ConvArgs& a, int64_t it) {
  Item m;
  m.y0 = (int)(it % a.nyb) * a.ty;
  const int64_t r = it / a.nyb;
  const int zci = (int)(r % a.nzc);
  m.b = (int)(r / a.nzc);
  m.z0 = zci * a.zc;
  m.nout = min(a.zc, a.n - m.z0);
  m.len = a.dil == 1 ? m.nout + 2 : 3 * m.nout;
  return m;
}

// The grid plane staged at stream position p of an item.
__device__ __forceinline__ int plane_at(const ConvArgs& a, const Item& m, int p) {
  return a.dil == 1 ? m.z0 - 1 + p : m.z0 + p / 3 + (p % 3 - 1) * a.dil;
}

__global__ void __launch_bounds__(kThreads, 1) conv3d_ring_kernel(ConvArgs a) {
  constexpr uint32_t IDESC = tc::idesc_bf16(128, 16, 0, 0);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* Ws = base;
  unsigned char* Ring = Ws + 27 * 512;
  const int slot_bytes = 2 * a.slab;
  const int S = a.slots;
  uint64_t* full = (uint64_t*)(Ring + S * slot_bytes);
  uint64_t* empty = full + kMaxSlots;
  uint64_t* accf = empty + kMaxSlots;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = a.n, dil = a.dil, xp = a.xp;
  // weights -> canonical K-major B tiles (one per tap)
  for (int idx = threadIdx.x; idx < 27 * 32; idx += kThreads) {
    const int tap = idx >> 5, co = (idx >> 1) & 15, c = idx & 1;
    const uint4 v = *reinterpret_cast<const uint4*>(
        a.w + ((size_t)co * 27 + tap) * a.ci_total + a.ci_off + c * 8);
    *reinterpret_cast<uint4*>(Ws + tap * 512 + (co >> 3) * 256 + c * 128 + (co & 7) * 16) = v;
  }
  // zero the ring once: the gaps between rows and the guards are never copied to
  for (int idx = threadIdx.x; idx < S * slot_bytes / 16; idx += kThreads)
    reinterpret_cast<uint4*>(Ring)[idx] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&accf[i], 1);
      tc::mbar_init(&acce[i], 128);
    }
    tc::mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tc::tmem_alloc(tmem_slot, 512);
  tc::fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (warp == 0) {
    // ---------------------------------------------------------- producer
    const uint32_t row_bytes = (uint32_t)n * 16;
    const uint32_t plane_bytes = 2u * a.box_rows * row_bytes;
    uint32_t gp = 0;  // stream position over all items
    for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
      const Item m = decode(a, it);
      for (int p = 0; p < m.len; ++p, ++gp) {
        const int s = (int)(gp % S);
        const uint32_t use = gp / S;
        int good = 1;
        if (lane == 0) {
          if (use > 0 && !tc::mbar_wait(&empty[s], (use - 1) & 1, a.wait_ns)) good = 0;
          if (good) mbar_expect_tx(&full[s], plane_bytes);
        }
        good = __shfl_sync(0xffffffffu, good, 0);
        if (!good) {
          ok = false;
          break;
        }
        const int z = plane_at(a, m, p);
        const uint32_t bar = tc::smem_addr(&full[s]);
        unsigned char* slot = Ring + s * slot_bytes;
        for (int k = lane; k < 2 * a.box_rows; k += 32) {
          const int h = k / a.box_rows, r = k % a.box_rows;
          const int y = m.y0 - dil + r;
          const void* src = g_zero_row;
          if (z >= 0 && z < n && y >= 0 && y < n)
            src = a.in + h * a.half + ((((int64_t)m.b * n + z) * n + y) * n) * 8;
          bulk_copy(tc::smem_addr(slot + h * a.slab + (kFrontGuard + r * xp + dil) * 16), src,
                    row_bytes, bar);
        }
        __syncwarp();
      }
    }
    // the last copies must land before the CTA exits
    if (lane == 0)
      for (uint32_t k = gp > (uint32_t)S ? gp - S : 0; k < gp; ++k)
        if (!tc::mbar_wait(&full[k % S], (k / S) & 1, a.wait_ns)) ok = false;
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      // A descriptor of a tap = the slot's base descriptor + a constant
      // offset (16-byte units; the address field stays below 2^14)
      int toff[9];
#pragma unroll
      for (int t9 = 0; t9 < 9; ++t9) {
        const int dy = t9 / 3 - 1, dx = t9 % 3 - 1;
        toff[t9] = kFrontGuard + dil * xp + (dy * xp + dx) * dil;
      }
      const uint64_t abase0 = tc::smem_desc(Ring, (uint32_t)a.slab, 128);
      const uint64_t wbase = tc::smem_desc(Ws, 128, 256);
      uint32_t gbase = 0, outs = 0;
      bool issued = false;
      for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
        const Item m = decode(a, it);
        for (int j = 0; j < m.nout; ++j, ++outs) {
          const int ab = outs & 1;
          const uint32_t ause = outs >> 1;
          if (ause > 0 && !tc::mbar_wait(&acce[ab], (ause - 1) & 1, a.wait_ns)) {
            ok = false;
            break;
          }
          // stream positions of planes z-d, z, z+d
          const uint32_t q0 = gbase + (dil == 1 ? j : 3 * j);
          for (int k = 0; k < 3; ++k) {
            const uint32_t q = q0 + k;
            if (dil == 1 && j > 0 && k < 2) continue;  // waited for by an earlier plane
            if (!tc::mbar_wait(&full[q % S], (q / S) & 1, a.wait_ns)) ok = false;
          }
          if (!ok) break;
          tc::tc_fence_after();
          for (int t = 0; t < a.tiles; ++t) {
            const uint32_t d = tmem + (uint32_t)(ab * 256 + t * 16);
#pragma unroll
            for (int dz = 0; dz < 3; ++dz) {
              const uint64_t at =
                  abase0 + (uint64_t)(((q0 + dz) % S) * (slot_bytes >> 4) + 128 * t);
#pragma unroll
              for (int t9 = 0; t9 < 9; ++t9)
                tc::mma_bf16(d, at + (uint64_t)toff[t9], wbase + (uint64_t)((dz * 9 + t9) * 32),
                             IDESC, dz > 0 || t9 > 0);
            }
          }
          issued = true;
          tc::mma_commit(&accf[ab]);
          // release the planes no later output of this item reads
          if (dil == 1) {
            tc::mma_commit(&empty[q0 % S]);
            if (j == m.nout - 1) {
              tc::mma_commit(&empty[(q0 + 1) % S]);
              tc::mma_commit(&empty[(q0 + 2) % S]);
            }
          } else {
            for (int k = 0; k < 3; ++k) tc::mma_commit(&empty[(q0 + k) % S]);
          }
        }
        gbase += m.len;
      }
      // every MMA issued must finish before tensor memory is released
      if (issued) {
        tc::mma_commit(drain);
        if (!tc::mbar_wait(drain, 0, a.wait_ns)) ok = false;
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;  // TMEM lane quarter this warp may read
    const int row = q * 32 + lane;
    uint32_t outs = 0;
    for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
      const Item m = decode(a, it);
      for (int j = 0; j < m.nout; ++j, ++outs) {
        const int ab = outs & 1;
        if (!tc::mbar_wait(&accf[ab], (outs >> 1) & 1, a.wait_ns)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const int64_t zrow = ((int64_t)m.b * n + m.z0 + j) * n;
        for (int t = 0; t < a.tiles; ++t) {
          float v[16];
          tc::tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * 256 + t * 16), v);
          const int p = 128 * t + row;
          const int r = p / xp, x = p % xp - dil;
          if (r < a.ty && x >= 0 && m.y0 + r < n) {
            const int64_t e = ((zrow + m.y0 + r) * n + x) * 8;
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] *= a.out_scale;
            if (a.addend) {
              const uint4 u0 = *reinterpret_cast<const uint4*>(a.addend + e);
              const uint4 u1 = *reinterpret_cast<const uint4*>(a.addend + a.half + e);
              const __nv_bfloat16* b0 = reinterpret_cast<const __nv_bfloat16*>(&u0);
              const __nv_bfloat16* b1 = reinterpret_cast<const __nv_bfloat16*>(&u1);
#pragma unroll
              for (int i = 0; i < 8; ++i) {
                v[i] += __bfloat162float(b0[i]);
                v[8 + i] += __bfloat162float(b1[i]);
              }
            }
            uint4 o[2];
            __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(o);
#pragma unroll
            for (int i = 0; i < 16; ++i) ob[i] = __float2bfloat16_rn(v[i]);
            *reinterpret_cast<uint4*>(a.out + e) = o[0];
            *reinterpret_cast<uint4*>(a.out + a.half + e) = o[1];
          }
        }
        tc::tc_fence_before();
        mbar_arrive(&acce[ab]);
      }
    }
  }
  if (!ok) atomicCAS(a.err, 0, 8);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 1) tc::tmem_free(tmem, 512);
}

// ---------------------------------------------------------------------------
// Dilation 1 with the three z taps stacked on the MMA's N side.
//
// An input plane z feeds output planes z-1, z and z+1 (through the weights of
// tap dz = +1, 0, -1).  Instead of 27 MMAs of N = 16 per output plane and
// tile, every input plane gets 9 MMAs of N = 48 per tile (one per (dy, dx)
// tap): the 48 accumulator columns of a tile are three 16-column slots, and
// output plane zo accumulates in slot zo mod 3.  The B operand of input plane
// z is the weight block permuted for z mod 3 (three copies in shared memory),
// so that each slot receives its own output plane's tap.  After input plane
// z, slot (z-1) mod 3 holds the finished output plane z-1: the epilogue reads
// it, stores it, and zeroes the slot, which input plane z+1 then starts as
// output plane z+2.  Each output plane still sums its taps in the order of
// the 27-MMA kernel (dz = -1, 0, +1, each over the 9 (dy, dx) taps).
//
// Per tile one mbarrier pair hands the tile between the MMA issuer (accf:
// input plane done) and the epilogue (acce: slot drained and zeroed), so the
// epilogue of one tile overlaps the MMAs of the others.  The first MMA of
// every work item does not accumulate, which clears all three slots.
// ---------------------------------------------------------------------------
constexpr int kZsMaxTiles = 10;  // 10 tiles x 48 columns <= 512
constexpr int kZsWBytes = 3 * 9 * 1536;  // 3 rotations x 9 taps x (48 x 16 BF16)

bool make_plan_zs(int n, Plan* p) {
  const int xp = n + 1;
  if (n > kMaxRow) return false;
  for (int ty = std::min(n, 16); ty >= 1; ty /= 2) {
    const int box_rows = ty + 2;
    const int tiles = (ty * xp + 127) / 128;
    if (tiles > kZsMaxTiles) continue;
    const int tail = tiles * 128 - ty * xp + 1;
    const int slab = ((kFrontGuard + box_rows * xp + tail) * 16 + 127) / 128 * 128;
    const int avail = kSmemLimit - 1024 - kZsWBytes - 512;
    const int slots = std::min(kMaxSlots, avail / (2 * slab));
    if (slots < 3) continue;
    const int smem = std::max(1024 + kZsWBytes + slots * 2 * slab + 512, 120 * 1024);
    *p = Plan{ty, xp, tiles, box_rows, slab, slots, smem};
    return true;
  }
  return false;
}

// Two CTAs a SM: fewer rows a work item (at most 5 tiles = 240 of 256 TMEM
// columns, at most 113 KB of shared memory), so that two MMA-issuing CTAs
// share each SM's tensor pipe.
bool make_plan_zs2(int n, Plan* p) {
  const int xp = n + 1;
  if (n > kMaxRow) return false;
  for (int ty = std::min(n, 16); ty >= 1; ty /= 2) {
    const int box_rows = ty + 2;
    const int tiles = (ty * xp + 127) / 128;
    if (tiles > 5) continue;
    const int tail = tiles * 128 - ty * xp + 1;
    const int slab = ((kFrontGuard + box_rows * xp + tail) * 16 + 127) / 128 * 128;
    const int avail = 113 * 1024 - 1024 - kZsWBytes - 512;
    const int slots = std::min(kMaxSlots, avail / (2 * slab));
    if (slots < 2) continue;
    const int smem = 1024 + kZsWBytes + slots * 2 * slab + 512;
    *p = Plan{ty, xp, tiles, box_rows, slab, slots, smem, 2};
    return true;
  }
  return false;
}

// NI MMA-issuing warps (1 .. 4): warp 0 producer, warps 1 .. NI issue the
// MMAs of tiles t = i, i + NI, ... (each tile's handshake stays with one
// issuer; a plane's slot and the final drain wait for all NI), warps NI+1 ..
// NI+4 the epilogue.
// NE epilogue groups of 4 warps (one a TMEM lane quarter); group g drains
// the tiles t = g, g + NE, ...
template <int NI, int NE = 1>
__global__ void __launch_bounds__(32 * (1 + NI + 4 * NE), 1) conv3d_zstack_kernel(ConvArgs a) {
  constexpr int NT = 32 * (1 + NI + 4 * NE);
  constexpr uint32_t IDESC = tc::idesc_bf16(128, 48, 0, 0);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* Ws = base;
  unsigned char* Ring = Ws + kZsWBytes;
  const int slot_bytes = 2 * a.slab;
  const int S = a.slots;
  const int T = a.tiles;
  uint64_t* full = (uint64_t*)(Ring + S * slot_bytes);
  uint64_t* empty = full + kMaxSlots;
  uint64_t* accf = empty + kMaxSlots;
  uint64_t* acce = accf + kZsMaxTiles;
  uint64_t* drain = acce + kZsMaxTiles;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = a.n, xp = a.xp;
  // weights -> B tiles: rotation rot (= input plane mod 3), tap t9 = (dy, dx);
  // row 16k + co is output channel co of slot k, whose output plane is the
  // one of z-1, z, z+1 that is k mod 3, so its z tap is
  // dz = +1, 0, -1 for (rot - k) mod 3 = 1, 0, 2 (tap index dz + 1).
  for (int idx = threadIdx.x; idx < 3 * 9 * 48 * 2; idx += NT) {
    const int c = idx & 1, row = (idx >> 1) % 48, rt = (idx >> 1) / 48;
    const int rot = rt / 9, t9 = rt % 9, k = row >> 4, co = row & 15;
    const int m = ((rot - k) % 3 + 3) % 3;
    const int tz = m == 0 ? 1 : (m == 1 ? 2 : 0);
    const uint4 v = *reinterpret_cast<const uint4*>(
        a.w + ((size_t)co * 27 + tz * 9 + t9) * a.ci_total + a.ci_off + c * 8);
    *reinterpret_cast<uint4*>(Ws + rt * 1536 + (row >> 3) * 256 + c * 128 + (row & 7) * 16) = v;
  }
  for (int idx = threadIdx.x; idx < S * slot_bytes / 16; idx += NT)
    reinterpret_cast<uint4*>(Ring)[idx] = make_uint4(0, 0, 0, 0);
  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], NI);
    }
    for (int i = 0; i < kZsMaxTiles; ++i) {
      tc::mbar_init(&accf[i], 1);
      tc::mbar_init(&acce[i], 128);
    }
    tc::mbar_init(drain, NI);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tc::tmem_alloc(tmem_slot, (uint32_t)a.tmem_cols);
  tc::fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  if (warp == 0) {
    // ---------------------------------------------------------- producer
    const uint32_t row_bytes = (uint32_t)n * 16;
    const uint32_t plane_bytes = 2u * a.box_rows * row_bytes;
    uint32_t gp = 0;
    for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
      const Item m = decode(a, it);
      for (int p = 0; p < m.len; ++p, ++gp) {
        const int s = (int)(gp % S);
        const uint32_t use = gp / S;
        int good = 1;
        if (lane == 0) {
          if (use > 0 && !tc::mbar_wait(&empty[s], (use - 1) & 1, a.wait_ns)) good = 0;
          if (good) mbar_expect_tx(&full[s], plane_bytes);
        }
        good = __shfl_sync(0xffffffffu, good, 0);
        if (!good) {
          ok = false;
          break;
        }
        const int z = m.z0 - 1 + p;
        const uint32_t bar = tc::smem_addr(&full[s]);
        unsigned char* slot = Ring + s * slot_bytes;
        for (int k = lane; k < 2 * a.box_rows; k += 32) {
          const int h = k / a.box_rows, r = k % a.box_rows;
          const int y = m.y0 - 1 + r;
          const void* src = g_zero_row;
          if (z >= 0 && z < n && y >= 0 && y < n)
            src = a.in + h * a.half + ((((int64_t)m.b * n + z) * n + y) * n) * 8;
          bulk_copy(tc::smem_addr(slot + h * a.slab + (kFrontGuard + r * xp + 1) * 16), src,
                    row_bytes, bar);
        }
        __syncwarp();
      }
    }
    if (lane == 0)
      for (uint32_t k = gp > (uint32_t)S ? gp - S : 0; k < gp; ++k)
        if (!tc::mbar_wait(&full[k % S], (k / S) & 1, a.wait_ns)) ok = false;
  } else if (warp <= NI) {
    // ---------------------------------------------------------- MMA issuers
    const int me = warp - 1;
    if (lane == 0) {
      int toff[9];
#pragma unroll
      for (int t9 = 0; t9 < 9; ++t9) {
        const int dy = t9 / 3 - 1, dx = t9 % 3 - 1;
        toff[t9] = kFrontGuard + xp + dy * xp + dx;
      }
      const uint64_t abase0 = tc::smem_desc(Ring, (uint32_t)a.slab, 128);
      const uint64_t wbase = tc::smem_desc(Ws, 128, 256);
      uint32_t gp = 0, pc = 0;
      bool issued = false;
      for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
        const Item m = decode(a, it);
        for (int p = 0; p < m.len; ++p, ++gp, ++pc) {
          if (!tc::mbar_wait(&full[gp % S], (gp / S) & 1, a.wait_ns)) {
            ok = false;
            break;
          }
          const int rot = (m.z0 - 1 + p + 3) % 3;
          const uint64_t ap = abase0 + (uint64_t)((gp % S) * (slot_bytes >> 4));
          const uint64_t wr = wbase + (uint64_t)(rot * 9 * 96);
          for (int t = me; t < T; t += NI) {
            // slot (z+1) mod 3 of this tile is drained and zeroed
            if (pc > 0 && !tc::mbar_wait(&acce[t], (pc - 1) & 1, a.wait_ns)) {
              ok = false;
              break;
            }
            tc::tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(t * 48);
            const uint64_t at = ap + (uint64_t)(128 * t);
#pragma unroll
            for (int t9 = 0; t9 < 9; ++t9)
              tc::mma_bf16(d, at + (uint64_t)toff[t9], wr + (uint64_t)(t9 * 96), IDESC,
                           p > 0 || t9 > 0);
            tc::mma_commit(&accf[t]);
            issued = true;
          }
          if (!ok) break;
          tc::mma_commit(&empty[gp % S]);  // the plane is read by this plane's MMAs only
        }
      }
      // every issuer arrives once; its MMAs must finish before TMEM is freed
      if (issued) tc::mma_commit(drain);
      else mbar_arrive(drain);
      if (!tc::mbar_wait(drain, 0, a.wait_ns)) ok = false;
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int q = warp & 3;
    const int grp = (warp - 1 - NI) >> 2;  // epilogue group (4 consecutive warps)
    const int row = q * 32 + lane;
    const uint32_t lanes = (uint32_t)(q * 32) << 16;
    uint32_t pc = 0;
    for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
      const Item m = decode(a, it);
      for (int p = 0; p < m.len && ok; ++p, ++pc) {
        const int zo = m.z0 - 2 + p;  // the output plane finished by input plane p
        const bool store = p >= 2;    // zo in z0 .. z0 + nout - 1
        const int k = (zo + 3) % 3;
        const int64_t zrow = ((int64_t)m.b * n + zo) * n;
        for (int t = grp; t < T; t += NE) {
          // (warp-uniform, for the .sync.aligned TMEM accesses below)
          const bool got = tc::mbar_wait(&accf[t], pc & 1, a.wait_ns);
          if (!__all_sync(0xffffffffu, got)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t col = (uint32_t)(t * 48 + k * 16);
          if (store) {
            float v[16];
            tc::tmem_ld16(tmem + lanes + col, v);
            const int pp = 128 * t + row;
            const int r = pp / xp, x = pp % xp - 1;
            if (r < a.ty && x >= 0 && m.y0 + r < n) {
              const int64_t e = ((zrow + m.y0 + r) * n + x) * 8;
#pragma unroll
              for (int i = 0; i < 16; ++i) v[i] *= a.out_scale;
              if (a.addend) {
                const uint4 u0 = *reinterpret_cast<const uint4*>(a.addend + e);
                const uint4 u1 = *reinterpret_cast<const uint4*>(a.addend + a.half + e);
                const __nv_bfloat16* b0 = reinterpret_cast<const __nv_bfloat16*>(&u0);
                const __nv_bfloat16* b1 = reinterpret_cast<const __nv_bfloat16*>(&u1);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                  v[i] += __bfloat162float(b0[i]);
                  v[8 + i] += __bfloat162float(b1[i]);
                }
              }
              uint4 o[2];
              __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(o);
#pragma unroll
              for (int i = 0; i < 16; ++i) ob[i] = __float2bfloat16_rn(v[i]);
              *reinterpret_cast<uint4*>(a.out + e) = o[0];
              *reinterpret_cast<uint4*>(a.out + a.half + e) = o[1];
            }
          }
          tc::tmem_zero16(tmem + lanes + col);
          tc::tc_fence_before();
          mbar_arrive(&acce[t]);
        }
      }
    }
  }
  if (!ok) atomicCAS(a.err, 0, 8);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 1) tc::tmem_free(tmem, (uint32_t)a.tmem_cols);
}

}  // namespace

// One single-source pass: out = conv(in, w[:, :, ci_off .. ci_off+15]) *
// scale (+ addend).  SSAM_ERR_UNSUPPORTED when the shape has no plan.
int conv3d_ring(const void* in, const void* addend, const void* w, int ci_total, int ci_off,
                void* out, int nb, int n, int dil, float out_scale, cudaStream_t s) {
  Plan p;
  // dilation 1: the z-stacked kernel (9 N = 48 MMAs per input plane and
  // tile); SSAM_CONV_RING27=1 in the environment keeps the 27-MMA kernel
  // (to check the two against each other)
  const char* e27 = getenv("SSAM_CONV_RING27");
  const bool ring27 = e27 && e27[0] == '1';
  // two CTAs a SM by default (two MMA-issuing CTAs share the tensor pipe:
  // 8 x 128^3 forward 4.62 -> 3.18 ms); SSAM_CONV_TWO_CTA=0 keeps one
  const char* e2 = getenv("SSAM_CONV_TWO_CTA");
  const bool two = !(e2 && e2[0] == '0');
  const bool zstack =
      dil == 1 && !ring27 && ((two && make_plan_zs2(n, &p)) || make_plan_zs(n, &p));
  // MMA-issuing warps of the z-stacked kernel: 3 by default (8 x 128^3
  // forward at two CTAs a SM, 1 / 2 / 3 / 4 issuers: 3.19 / 2.88 / 2.85 /
  // 2.84 ms with one epilogue group, - / 2.66 / 2.61 / 2.64 ms with two);
  // SSAM_CONV_ISSUERS=1..4 pins one; never more than tiles
  const char* ei = getenv("SSAM_CONV_ISSUERS");
  int issuers = (ei && ei[0] >= '1' && ei[0] <= '4') ? ei[0] - '0' : 3;
  issuers = std::min(issuers, p.tiles);
  if (!zstack && !make_plan(n, dil, &p)) return SSAM_ERR_UNSUPPORTED;
  ConvArgs a;
  a.in = (const __nv_bfloat16*)in;
  a.addend = (const __nv_bfloat16*)addend;
  a.w = (const __nv_bfloat16*)w;
  a.out = (__nv_bfloat16*)out;
  a.out_scale = out_scale;
  a.ci_total = ci_total;
  a.ci_off = ci_off;
  a.n = n;
  a.dil = dil;
  a.ty = p.ty;
  a.xp = p.xp;
  a.tiles = p.tiles;
  a.box_rows = p.box_rows;
  a.slab = p.slab;
  a.slots = p.slots;
  a.tmem_cols = p.ctas_per_sm == 2 ? 256 : 512;
  a.nyb = (n + p.ty - 1) / p.ty;
  a.half = (int64_t)nb * n * n * n * 8;
  a.wait_ns = 1000ull * 1000ull * 1000ull;
  int st = device_error_word(&a.err);
  if (st != SSAM_OK) return st;
  int dev = 0, sms = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  SSAM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // z chunk: fewest rounds x (planes per item incl. the d = 1 prologue)
  const int64_t cols = (int64_t)nb * a.nyb;
  int64_t best = -1;
  for (int nzc = 1; nzc <= n; nzc *= 2) {
    const int zc = (n + nzc - 1) / nzc;
    const int64_t items = cols * nzc;
    const int64_t slots_all = (int64_t)sms * p.ctas_per_sm;
    const int64_t rounds = (items + slots_all - 1) / slots_all;
    const int64_t cost = rounds * (dil == 1 ? zc + 2 : 3 * zc);
    if (best < 0 || cost < best) {
      best = cost;
      a.nzc = nzc;
      a.zc = zc;
      a.items = items;
    }
  }
  static bool attr_set = false;
  if (!attr_set) {
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_ring_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<3>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<4>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<2, 2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<3, 2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_zstack_kernel<4, 2>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    attr_set = true;
  }
  const int64_t grid = std::min<int64_t>(a.items, (int64_t)sms * p.ctas_per_sm);
  // epilogue groups: 2 by default where there are two tiles to share
  // (forward 2.89 -> 2.66 ms at two issuers); SSAM_CONV_EPI=1 keeps one
  // (one-issuer kernels have one)
  const char* ee = getenv("SSAM_CONV_EPI");
  const int epi = (ee && ee[0] == '1') || p.tiles < 2 ? 1 : 2;
  if (zstack && epi == 2 && issuers == 4)
    conv3d_zstack_kernel<4, 2><<<(unsigned)grid, 32 * 13, p.smem, s>>>(a);
  else if (zstack && epi == 2 && issuers == 3)
    conv3d_zstack_kernel<3, 2><<<(unsigned)grid, 32 * 12, p.smem, s>>>(a);
  else if (zstack && epi == 2 && issuers == 2)
    conv3d_zstack_kernel<2, 2><<<(unsigned)grid, 32 * 11, p.smem, s>>>(a);
  else if (zstack && issuers == 4)
    conv3d_zstack_kernel<4><<<(unsigned)grid, 32 * 9, p.smem, s>>>(a);
  else if (zstack && issuers == 3)
    conv3d_zstack_kernel<3><<<(unsigned)grid, 32 * 8, p.smem, s>>>(a);
  else if (zstack && issuers == 2)
    conv3d_zstack_kernel<2><<<(unsigned)grid, 32 * 7, p.smem, s>>>(a);
  else if (zstack)
    conv3d_zstack_kernel<1><<<(unsigned)grid, 32 * 6, p.smem, s>>>(a);
  else
    conv3d_ring_kernel<<<(unsigned)grid, kThreads, p.smem, s>>>(a);
  count_launch();
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

}  // namespace ssam
