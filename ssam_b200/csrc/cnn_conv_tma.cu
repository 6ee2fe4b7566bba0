// Persistent, TMA-fed implicit-GEMM 3D convolution for the warm-start CNN
// (forward, and the data gradient with mirrored / transposed weights).
//
// Shared-memory operand trick: the 27 taps of a 3x3x3 convolution read the
// same input shifted by (dz, dy, dx) * dilation.  A work item (grid b, output
// plane z, TY output rows from y0) stages, per source and per 8-channel half,
// the three input planes z - d, z, z + d as "slabs": TY + 2d rows of
// XP = n + d voxels, each row preceded by d zero voxels (the TMA box starts
// at x = -d, and the copy engine fills coordinates outside the grid with
// zeros).  In that padded, row-major layout a shift by (dy, dx) is a constant
// offset of (dy * XP + dx) * d voxels, and the zeros between rows are exactly
// the x-halo of both neighbouring rows.  So the A operand of every tap is the
// same slab seen from another start address: a K-major, no-swizzle UMMA
// descriptor whose 8-row core matrices are 8 consecutive voxels (SBO = 128 B)
// and whose two K halves (channels 0-7 / 8-15) are the two half-slabs (LBO).
// Nothing is gathered through registers.
//
// Output positions are enumerated in the same padded layout, 128 per MMA
// tile (TILES per item); positions in the gaps or past the last row are
// computed and discarded.
//
// Warp roles (one CTA per SM, persistent over items):
//   warp 0      TMA producer: 6 tiled 5D copies per (item, source) into one of
//               two stages (mbarrier full / empty ring)
//   warp 1      MMA issuer: TILES x 27 tcgen05.mma (128 x 16 x 16, BF16 in,
//               FP32 in TMEM) per (item, source); two accumulator buffers
//   warps 2-5   epilogue: tcgen05.ld of each tile's accumulators, scale,
//               round to BF16, store the valid voxels
// Every wait is bounded by %globaltimer; on expiry the kernel records error
// code 8 and winds down (drains its copies and MMAs, frees tensor memory).
#include <cudaTypedefs.h>
#include <string.h>

#include <algorithm>

#include "cnn_tc.cuh"

namespace ssam {

int device_error_word(int** out);
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

namespace {

constexpr int kFrontGuard = 8;  // voxels (16 B each) before every slab's box
constexpr int kMaxTiles = 8;    // 2 accumulator buffers x 8 tiles x 16 columns
constexpr int kThreads = 192;
constexpr int kSmemLimit = 227 * 1024;

struct TmaConvArgs {
  const __nv_bfloat16* w;  // [16][27][16 * NSRC]
  __nv_bfloat16* out;      // [nb][n][n][n][16]
  float out_scale;
  int n, dil, ty, xp, tiles, nyb, box_rows, slab_stride;
  int64_t items;
  int* err;
  unsigned long long wait_ns;
};

struct Plan {
  int ty, xp, tiles, box_rows, slab_stride, smem;
};

// Largest TY (rows per item) whose two stages and weights fit in shared memory
// with at most kMaxTiles MMA tiles per item.
bool make_plan(int n, int dil, int nsrc, Plan* p) {
  const int xp = n + dil;
  if (xp > 256) return false;
  for (int ty = std::min(n, 16); ty >= 1; ty /= 2) {
    const int box_rows = ty + 2 * dil;
    if (box_rows > 256) continue;
    const int tiles = (ty * xp + 127) / 128;
    if (tiles > kMaxTiles) continue;
    const int tail = tiles * 128 - ty * xp + dil;  // reach past the box of the last tile
    const int slab = ((kFrontGuard + box_rows * xp + tail) * 16 + 127) / 128 * 128;
    // (at least 120 KB, so that one CTA -- and its 256 TMEM columns -- is
    // alone on its SM)
    const int smem = std::max(1024 + 27 * nsrc * 512 + 2 * 6 * slab + 128, 120 * 1024);
    if (smem > kSmemLimit) continue;
    *p = Plan{ty, xp, tiles, box_rows, slab, smem};
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
// 5D tiled TMA load (no multicast); coordinates outside the tensor read zeros.
__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, int c4, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
      : "memory");
}

template <int NSRC>
__global__ void __launch_bounds__(kThreads, 1)
conv3d_tma_kernel(const __grid_constant__ CUtensorMap m00, const __grid_constant__ CUtensorMap m01,
                  const __grid_constant__ CUtensorMap m10, const __grid_constant__ CUtensorMap m11,
                  TmaConvArgs a) {
  constexpr uint32_t IDESC = tc::idesc_bf16(128, 16, 0, 0);
  constexpr int NK = 27 * NSRC;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* Ws = base;
  unsigned char* St = Ws + NK * 512;
  const int stage_bytes = 6 * a.slab_stride;
  uint64_t* full = (uint64_t*)(St + 2 * stage_bytes);
  uint64_t* empty = full + 2;
  uint64_t* accf = empty + 2;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_slot = (uint32_t*)(drain + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int box_bytes = a.box_rows * a.xp * 16;
  // weights -> canonical K-major B tiles (step ks = tap * NSRC + src)
  for (int idx = threadIdx.x; idx < NK * 32; idx += kThreads) {
    const int ks = idx >> 5, co = (idx >> 1) & 15, c = idx & 1;
    const uint4 v =
        *reinterpret_cast<const uint4*>(a.w + (size_t)co * NK * 16 + ks * 16 + c * 8);
    *reinterpret_cast<uint4*>(Ws + ks * 512 + (co >> 3) * 256 + c * 128 + (co & 7) * 16) = v;
  }
  // zero every slab's guards (the copies never write them)
  {
    const uint4 z = make_uint4(0, 0, 0, 0);
    const int front = kFrontGuard * 16, tail0 = front + box_bytes;
    const int per = (front + (a.slab_stride - tail0)) / 16;
    for (int idx = threadIdx.x; idx < 12 * per; idx += kThreads) {
      const int sl = idx / per, k = idx % per;
      const int off = k * 16 < front ? k * 16 : tail0 + (k * 16 - front);
      *reinterpret_cast<uint4*>(St + sl * a.slab_stride + off) = z;
    }
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&full[i], 1);
      tc::mbar_init(&empty[i], 1);
      tc::mbar_init(&accf[i], 1);
      tc::mbar_init(&acce[i], 128);
    }
    tc::mbar_init(drain, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tc::tmem_alloc(tmem_slot, 256);
  tc::fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int n = a.n, dil = a.dil, xp = a.xp;
  bool ok = true;
  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      uint32_t u = 0;
      for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x) {
        const int yb = (int)(it % a.nyb);
        const int z = (int)((it / a.nyb) % n);
        const int b = (int)(it / ((int64_t)a.nyb * n));
        const int y0 = yb * a.ty;
        for (int src = 0; src < NSRC; ++src, ++u) {
          const int s = u & 1;
          const uint32_t use = u >> 1;
          if (use > 0 && !tc::mbar_wait(&empty[s], (use - 1) & 1, a.wait_ns)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], (uint32_t)(6 * box_bytes));
          for (int h = 0; h < 2; ++h) {
            const CUtensorMap* map = src == 0 ? (h ? &m01 : &m00) : (h ? &m11 : &m10);
            for (int k = 0; k < 3; ++k) {
              const uint32_t dst = tc::smem_addr(St + s * stage_bytes +
                                                 (h * 3 + k) * a.slab_stride + kFrontGuard * 16);
              tma_load_5d(dst, map, 0, -dil, y0 - dil, z + (k - 1) * dil, b,
                          tc::smem_addr(&full[s]));
            }
          }
        }
      }
      // the last copies must land before the CTA exits
      for (uint32_t k = u > 2 ? u - 2 : 0; k < u; ++k)
        if (!tc::mbar_wait(&full[k & 1], (k >> 1) & 1, a.wait_ns)) ok = false;
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issuer
    if (lane == 0) {
      // descriptors are formed once: a tap's A operand is the stage's base
      // descriptor plus a constant offset (16-byte units in the address
      // field, which stays below 2^14 for every shared-memory address)
      int toff[27];
#pragma unroll
      for (int tap = 0; tap < 27; ++tap) {
        const int dz = tap / 9, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
        toff[tap] = dz * (a.slab_stride >> 4) + dil * xp + (dy * xp + dx) * dil;
      }
      const uint64_t abase0 = tc::smem_desc(St + kFrontGuard * 16,
                                            (uint32_t)(3 * a.slab_stride), 128);
      const uint64_t abase1 = abase0 + (uint64_t)(stage_bytes >> 4);
      const uint64_t wbase = tc::smem_desc(Ws, 128, 256);
      uint32_t u = 0, items_done = 0;
      bool issued = false;
      for (int64_t it = blockIdx.x; ok && it < a.items; it += gridDim.x, ++items_done) {
        const int ab = items_done & 1;
        const uint32_t ause = items_done >> 1;
        if (ause > 0 && !tc::mbar_wait(&acce[ab], (ause - 1) & 1, a.wait_ns)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        for (int src = 0; src < NSRC; ++src, ++u) {
          const int s = u & 1;
          if (!tc::mbar_wait(&full[s], (u >> 1) & 1, a.wait_ns)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          for (int t = 0; t < a.tiles; ++t) {
            const uint32_t d = tmem + (uint32_t)(ab * 128 + t * 16);
            const uint64_t at = (s ? abase1 : abase0) + (uint64_t)(128 * t);
#pragma unroll
            for (int tap = 0; tap < 27; ++tap)
              tc::mma_bf16(d, at + (uint64_t)toff[tap],
                           wbase + (uint64_t)((tap * NSRC + src) * 32), IDESC,
                           src > 0 || tap > 0);
          }
          tc::mma_commit(&empty[s]);
          issued = true;
        }
        if (!ok) break;
        tc::mma_commit(&accf[ab]);
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
    uint32_t items_done = 0;
    for (int64_t it = blockIdx.x; it < a.items; it += gridDim.x, ++items_done) {
      const int ab = items_done & 1;
      if (!tc::mbar_wait(&accf[ab], (items_done >> 1) & 1, a.wait_ns)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const int yb = (int)(it % a.nyb);
      const int z = (int)((it / a.nyb) % n);
      const int64_t b = it / ((int64_t)a.nyb * n);
      const int y0 = yb * a.ty;
      for (int t = 0; t < a.tiles; ++t) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(ab * 128 + t * 16), v);
        const int p = 128 * t + row;
        const int r = p / xp, x = p % xp - dil;
        if (r < a.ty && x >= 0 && y0 + r < n) {
          uint4 o[2];
          __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(o);
#pragma unroll
          for (int i = 0; i < 16; ++i) ob[i] = __float2bfloat16_rn(v[i] * a.out_scale);
          uint4* dst = reinterpret_cast<uint4*>(
              a.out + ((((b * n + z) * n) + y0 + r) * (int64_t)n + x) * 16);
          dst[0] = o[0];
          dst[1] = o[1];
        }
      }
      tc::tc_fence_before();
      mbar_arrive(&acce[ab]);
    }
  }
  if (!ok) atomicCAS(a.err, 0, 8);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 1) tc::tmem_free(tmem, 256);
}

int encode_half(CUtensorMap* map, const void* act, int half, int n, int64_t nb,
                const Plan& p) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(SSAM_ERR_UNSUPPORTED, "conv3d: no tensor-map encoder in the driver");
  const cuuint64_t un = (cuuint64_t)n;
  cuuint64_t dims[5] = {8, un, un, un, (cuuint64_t)nb};
  cuuint64_t strides[4] = {32, 32 * un, 32 * un * un, 32 * un * un * un};
  cuuint32_t box[5] = {8, (cuuint32_t)p.xp, (cuuint32_t)p.box_rows, 1, 1};
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  memset(map, 0, sizeof(*map));
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5,
                   (void*)((const char*)act + 16 * half), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SSAM_ERR_INVALID, "conv3d: cuTensorMapEncodeTiled failed");
  return SSAM_OK;
}

template <int NSRC>
int launch(const void* in0, const void* in1, const void* w, void* out, int nb, int n, int dil,
           float out_scale, const Plan& p, cudaStream_t s) {
  CUtensorMap m[4];
  int st = encode_half(&m[0], in0, 0, n, nb, p);
  if (st == SSAM_OK) st = encode_half(&m[1], in0, 1, n, nb, p);
  if (st == SSAM_OK && NSRC == 2) st = encode_half(&m[2], in1, 0, n, nb, p);
  if (st == SSAM_OK && NSRC == 2) st = encode_half(&m[3], in1, 1, n, nb, p);
  if (st != SSAM_OK) return st;
  if (NSRC == 1) m[2] = m[3] = m[0];
  TmaConvArgs a;
  a.w = (const __nv_bfloat16*)w;
  a.out = (__nv_bfloat16*)out;
  a.out_scale = out_scale;
  a.n = n;
  a.dil = dil;
  a.ty = p.ty;
  a.xp = p.xp;
  a.tiles = p.tiles;
  a.nyb = (n + p.ty - 1) / p.ty;
  a.box_rows = p.box_rows;
  a.slab_stride = p.slab_stride;
  a.items = (int64_t)nb * n * a.nyb;
  a.wait_ns = 1000ull * 1000ull * 1000ull;
  st = device_error_word(&a.err);
  if (st != SSAM_OK) return st;
  int dev = 0, sms = 0;
  SSAM_CUDA_TRY(cudaGetDevice(&dev));
  SSAM_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  static bool attr_set = false;
  if (!attr_set) {
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_tma_kernel<NSRC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemLimit));
    attr_set = true;
  }
  const int64_t grid = std::min<int64_t>(a.items, sms);
  conv3d_tma_kernel<NSRC><<<(unsigned)grid, kThreads, p.smem, s>>>(m[0], m[1], m[2], m[3], a);
  count_launch();
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

}  // namespace

// The TMA path of conv3d_fwd; SSAM_ERR_UNSUPPORTED when the shape does not
// fit it (the caller then uses the gather kernel).
int conv3d_fwd_tma(const void* in0, const void* in1, const void* w, void* out, int nb, int n,
                   int dil, float out_scale, cudaStream_t s) {
  Plan p;
  if (!make_plan(n, dil, in1 ? 2 : 1, &p) || tensor_map_encoder() == nullptr)
    return SSAM_ERR_UNSUPPORTED;
  return in1 ? launch<2>(in0, in1, w, out, nb, n, dil, out_scale, p, s)
             : launch<1>(in0, nullptr, w, out, nb, n, dil, out_scale, p, s);
}

}  // namespace ssam
