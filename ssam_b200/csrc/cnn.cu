// Warm-start CNN for the Poisson solver: hand-written implicit-GEMM 3D
// convolutions on the sm_100a tensor cores (tcgen05.mma, TMEM accumulators).
//
// Activations are BF16 in "planar halves": [2][b][z][y][x][8], channels 0-7
// of every voxel, then channels 8-15 (half = b * n^3 * 8 elements apart); a
// layer reads one or two 16-channel sources (the second is the skip
// connection of a U-Net decoder, so concatenation is never materialised).
// Weights are BF16 [co = 16][tap = 27][ci = 16 * nsrc]; tap = (kz*3 + ky)*3
// + kx reads the input at offset ((kz-1), (ky-1), (kx-1)) * dilation, zero
// outside the grid.
//
// The forward (and data-gradient, with mirrored / transposed weights)
// normally runs on the ring kernel of cnn_conv_ring.cu.  The gather kernel
// here is its cross-check (SSAM_CONV_GATHER=1) as a GEMM
//   D[voxel, co] = sum_k A[voxel, k] * B[co, k],  k = (tap, ci), both K-major:
// one CTA computes 128 voxels x 16 channels; every K step (one tap x 16
// channels) the 4 warps gather the 128 neighbour vectors into a shared-memory
// stage, one thread issues a 128x16x16 tcgen05.mma into TMEM, and a
// tcgen05.commit on the stage's mbarrier frees it for reuse four steps later.
// The epilogue reads the accumulators with tcgen05.ld and stores BF16.
#include <stdlib.h>

#include <algorithm>
#include <string>
#include <vector>

#include "cnn_tc.cuh"

namespace ssam {

int device_error_word(int** out);

namespace {

constexpr int kStages = 4;
constexpr int kTile = 128;            // voxels per CTA (MMA M)
constexpr int kAStageBytes = kTile * 16 * 2;  // 128 x 16 bf16
constexpr int kBStepBytes = 16 * 16 * 2;      // 16 x 16 bf16

template <int NSRC>
constexpr int conv_smem_bytes() {
  return 128 + 27 * NSRC * kBStepBytes + kStages * kAStageBytes + kStages * 8 + 16;
}

template <int NSRC>
__global__ void __launch_bounds__(128)
conv3d_fwd_kernel(const __nv_bfloat16* __restrict__ in0, const __nv_bfloat16* __restrict__ in1,
                  const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ out,
                  int log2n, int dil, float out_scale, int64_t half, int* err,
                  unsigned long long wait_ns) {
  constexpr int NK = 27 * NSRC;
  constexpr uint32_t IDESC = tc::idesc_bf16(kTile, 16, 0, 0);
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  unsigned char* Ws = base;
  unsigned char* As = Ws + NK * kBStepBytes;
  uint64_t* bars = (uint64_t*)(As + kStages * kAStageBytes);
  uint32_t* tmem_slot = (uint32_t*)(bars + kStages);

  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) tc::tmem_alloc(tmem_slot, 32);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) tc::mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights -> canonical K-major tiles: step ks, row co, 16-byte chunk c
  for (int idx = tid; idx < NK * 32; idx += 128) {
    const int ks = idx >> 5, co = (idx >> 1) & 15, c = idx & 1;
    const uint4 v = *reinterpret_cast<const uint4*>(w + (size_t)co * NK * 16 + ks * 16 + c * 8);
    *reinterpret_cast<uint4*>(Ws + ks * kBStepBytes + (co >> 3) * 256 + c * 128 +
                              (co & 7) * 16) = v;
  }
  tc::fence_async_smem();
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int n = 1 << log2n;
  const int64_t v = (int64_t)blockIdx.x * kTile + tid;  // my voxel (row of the tile)
  const int x = (int)(v & (n - 1)), y = (int)((v >> log2n) & (n - 1)),
            z = (int)((v >> (2 * log2n)) & (n - 1));
  const int64_t bofs = (v >> (3 * log2n)) << (3 * log2n);  // first voxel of my grid
  unsigned char* arow = As + (tid >> 3) * 256 + (tid & 7) * 16;
  bool ok = true;
  for (int ks = 0; ks < NK; ++ks) {
    const int stage = ks % kStages, use = ks / kStages;
    if (use > 0 && !tc::mbar_wait(&bars[stage], (use - 1) & 1, wait_ns)) ok = false;
    const int tap = ks / NSRC, src = ks % NSRC;
    const int zz = z + (tap / 9 - 1) * dil, yy = y + ((tap / 3) % 3 - 1) * dil,
              xx = x + (tap % 3 - 1) * dil;
    uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
    if ((unsigned)zz < (unsigned)n && (unsigned)yy < (unsigned)n && (unsigned)xx < (unsigned)n) {
      const __nv_bfloat16* p =
          (src == 0 ? in0 : in1) + (bofs + ((int64_t)zz << (2 * log2n)) + (yy << log2n) + xx) * 8;
      lo = __ldg(reinterpret_cast<const uint4*>(p));
      hi = __ldg(reinterpret_cast<const uint4*>(p + half));
    }
    unsigned char* a = arow + stage * kAStageBytes;
    *reinterpret_cast<uint4*>(a) = lo;
    *reinterpret_cast<uint4*>(a + 128) = hi;
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      const uint64_t da = tc::smem_desc(As + stage * kAStageBytes, 128, 256);
      const uint64_t db = tc::smem_desc(Ws + ks * kBStepBytes, 128, 256);
      tc::mma_bf16(tmem, da, db, IDESC, ks > 0);
      tc::mma_commit(&bars[stage]);
    }
  }
  const int last = NK - 1;
  if (!tc::mbar_wait(&bars[last % kStages], (last / kStages) & 1, wait_ns)) ok = false;
  tc::tc_fence_after();
  float acc[16];
  tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), acc);
  uint4 o[2];
  __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(o);
#pragma unroll
  for (int i = 0; i < 16; ++i) ob[i] = __float2bfloat16_rn(acc[i] * out_scale);
  *reinterpret_cast<uint4*>(out + v * 8) = o[0];
  *reinterpret_cast<uint4*>(out + half + v * 8) = o[1];
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 0) tc::tmem_free(tmem, 32);
  if (!ok && tid == 0) atomicCAS(err, 0, 6);
}

// Weight gradient: dW[co][tap][ci] = sum_v G[v][co] * X[v + off(tap)][ci].
// GEMM D[m = (tap, ci), n = co] = sum_k A[m, k] B[n, k] over voxels k, both
// operands MN-major (channels-last rows are contiguous in m / n).  A CTA owns
// one M tile (8 taps x 16 channels; the 4th tile is taps 24..26 padded with
// zeros) and one slab of voxels; it accumulates in TMEM and writes its
// partial 128 x 16 block, which a second kernel sums in a fixed order.
constexpr int kWgStepVox = 16;                   // voxels per MMA K step
constexpr int kWgStepsPerStage = 4;              // K steps per shared-memory stage
constexpr int kWgStageVox = kWgStepVox * kWgStepsPerStage;
constexpr int kWgAStep = 128 * kWgStepVox * 2;   // 4 KB
constexpr int kWgBStep = 16 * kWgStepVox * 2;    // 512 B
constexpr int kWgStages = 3;
// (+32 KB guard: the MN-major A tiles span up to 16 MN groups x 2 K groups;
// the guard keeps every address the descriptors can form inside the
// allocation)
constexpr int kWgSmem = 128 + kWgStages * kWgStepsPerStage * (kWgAStep + kWgBStep) + 64 +
                        32 * 1024;

template <int NSRC>
__global__ void __launch_bounds__(128)
conv3d_wgrad_kernel(const __nv_bfloat16* __restrict__ x0, const __nv_bfloat16* __restrict__ x1,
                    const __nv_bfloat16* __restrict__ g, float* __restrict__ partials,
                    int64_t nvox, int64_t slab, int log2n, int dil, int* err,
                    unsigned long long wait_ns) {
  // MN-major operand, no swizzle: core matrix = 8 K rows x 16 bytes (8 MN
  // elements); MN groups SBO = 128 B apart, K groups LBO apart.
  constexpr uint32_t IDESC = tc::idesc_bf16(128, 16, 1, 1);
  constexpr uint32_t A_SBO = 128, A_LBO = 16 * 128;  // 16 MN groups per K group
  constexpr uint32_t B_SBO = 128, B_LBO = 2 * 128;   // 2 MN groups per K group
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
  unsigned char* As = base;                                             // [stage][step] 4 KB
  unsigned char* Bs = As + kWgStages * kWgStepsPerStage * kWgAStep;     // [stage][step] 512 B
  uint64_t* bars = (uint64_t*)(Bs + kWgStages * kWgStepsPerStage * kWgBStep);
  uint32_t* tmem_slot = (uint32_t*)(bars + kWgStages);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int mtile = blockIdx.y;  // taps 8*mtile .. 8*mtile+7
  if (warp == 0) tc::tmem_alloc(tmem_slot, 32);
  if (tid == 0) {
    for (int s = 0; s < kWgStages; ++s) tc::mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int n = 1 << log2n;
  const int64_t v_begin = (int64_t)blockIdx.x * slab;
  const int64_t v_end = v_begin + slab < nvox ? v_begin + slab : nvox;
  const int64_t nstage_iters = (v_end - v_begin + kWgStageVox - 1) / kWgStageVox;
  bool ok = true;
  int issued = 0;
  for (int64_t it = 0; it < nstage_iters; ++it) {
    const int stage = (int)(it % kWgStages);
    const int use = (int)(it / kWgStages);
    if (use > 0 && !tc::mbar_wait(&bars[stage], (use - 1) & 1, wait_ns)) ok = false;
    const int64_t vs = v_begin + it * kWgStageVox;
    // A: 4 steps x 16 voxels x 8 taps x 2 chunks = 1024 pieces; B: 4 x 16 x 2 = 128
    for (int p = tid; p < kWgStepsPerStage * kWgStepVox * 8 * 2; p += 128) {
      const int c = p & 1, tl = (p >> 1) & 7, k = (p >> 4) & 15, st = p >> 8;
      const int64_t v = vs + st * kWgStepVox + k;
      const int tap = mtile * 8 + tl;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (v < v_end && tap < 27) {
        const int x = (int)(v & (n - 1)), y = (int)((v >> log2n) & (n - 1)),
                  z = (int)((v >> (2 * log2n)) & (n - 1));
        const int64_t bofs = (v >> (3 * log2n)) << (3 * log2n);
        const int zz = z + (tap / 9 - 1) * dil, yy = y + ((tap / 3) % 3 - 1) * dil,
                  xx = x + (tap % 3 - 1) * dil;
        if ((unsigned)zz < (unsigned)n && (unsigned)yy < (unsigned)n &&
            (unsigned)xx < (unsigned)n) {
          const int64_t nb = bofs + ((int64_t)zz << (2 * log2n)) + (yy << log2n) + xx;
          // NSRC sources: channel chunk c of source `src` -- handled by the caller
          // launching one M-tile set per source (x1 unused when NSRC == 1)
          const __nv_bfloat16* src = x0;
          val = __ldg(reinterpret_cast<const uint4*>(src + c * nvox * 8 + nb * 8));
        }
      }
      // m = tl*16 + c*8 .. +7 -> MN group tl*2 + c; K row k
      unsigned char* a = As + (stage * kWgStepsPerStage + st) * kWgAStep;
      *reinterpret_cast<uint4*>(a + (tl * 2 + c) * A_SBO + (k >> 3) * A_LBO + (k & 7) * 16) = val;
    }
    for (int p = tid; p < kWgStepsPerStage * kWgStepVox * 2; p += 128) {
      const int c = p & 1, k = (p >> 1) & 15, st = p >> 5;
      const int64_t v = vs + st * kWgStepVox + k;
      uint4 val = make_uint4(0, 0, 0, 0);
      if (v < v_end) val = __ldg(reinterpret_cast<const uint4*>(g + c * nvox * 8 + v * 8));
      unsigned char* b = Bs + (stage * kWgStepsPerStage + st) * kWgBStep;
      *reinterpret_cast<uint4*>(b + c * B_SBO + (k >> 3) * B_LBO + (k & 7) * 16) = val;
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::tc_fence_after();
      for (int st = 0; st < kWgStepsPerStage; ++st) {
        const uint64_t da = tc::smem_desc(As + (stage * kWgStepsPerStage + st) * kWgAStep, A_LBO, A_SBO);
        const uint64_t db = tc::smem_desc(Bs + (stage * kWgStepsPerStage + st) * kWgBStep, B_LBO, B_SBO);
        tc::mma_bf16(tmem, da, db, IDESC, issued > 0);
        ++issued;
      }
      tc::mma_commit(&bars[stage]);
    }
    __syncwarp();
    issued = __shfl_sync(0xffffffffu, issued, 0);
  }
  float acc[16];
  if (nstage_iters > 0) {
    const int64_t last = nstage_iters - 1;
    if (!tc::mbar_wait(&bars[last % kWgStages], (int)(last / kWgStages) & 1, wait_ns)) ok = false;
    tc::tc_fence_after();
    tc::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16), acc);
  } else {
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[i] = 0.f;
  }
  // partials[slab][mtile][m][co]
  float* dst = partials + (((int64_t)blockIdx.x * gridDim.y + mtile) * 128 + tid) * 16;
#pragma unroll
  for (int i = 0; i < 16; ++i) dst[i] = acc[i];
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  if (warp == 0) tc::tmem_free(tmem, 32);
  if (!ok && tid == 0) atomicCAS(err, 0, 7);
  (void)x1;
}

// dW[co][tap][src*16 + ci] (fp32) = sum over slabs, fixed order.
__global__ void wgrad_reduce_kernel(const float* __restrict__ partials, float* __restrict__ dw,
                                    int nslabs, int ci_total, int src) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (mtile, m, co)
  if (idx >= 4 * 128 * 16) return;
  const int co = idx & 15, m = (idx >> 4) & 127, mt = idx >> 11;
  const int tap = mt * 8 + (m >> 4), ci = m & 15;
  if (tap >= 27) return;
  float s = 0.f;
  for (int k = 0; k < nslabs; ++k) s += partials[((int64_t)k * 4 + mt) * 2048 + m * 16 + co];
  dw[((int64_t)co * 27 + tap) * ci_total + src * 16 + ci] = s;
}

int log2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return (1 << l) == n ? l : -1;
}

}  // namespace

int conv3d_ring(const void* in, const void* addend, const void* w, int ci_total, int ci_off,
                void* out, int nb, int n, int dil, float out_scale, cudaStream_t s);

// SSAM_CONV_GATHER=1 in the environment forces the gather kernel (to check
// it against the same oracle as the ring kernel).
static bool force_gather() {
  static const bool v = [] {
    const char* e = getenv("SSAM_CONV_GATHER");
    return e && e[0] == '1';
  }();
  return v;
}

// out = conv3d(in0 (+ in1 as channels 16..31), w) * out_scale over nb grids
// of n^3, planar-halves layout.  The ring kernel runs one source per pass; a
// second source is a second pass that adds the first one's (BF16) result.
int conv3d_fwd(const void* in0, const void* in1, const void* w, void* out, int nb, int n,
               int dil, float out_scale, cudaStream_t s) {
  if (in0 && w && out &&
      ((uintptr_t)in0 | (uintptr_t)w | (uintptr_t)out | (uintptr_t)in1) % 16 == 0 &&
      !force_gather()) {
    int st;
    if (in1) {
      st = conv3d_ring(in1, nullptr, w, 32, 16, out, nb, n, dil, out_scale, s);
      if (st == SSAM_OK) st = conv3d_ring(in0, out, w, 32, 0, out, nb, n, dil, out_scale, s);
    } else {
      st = conv3d_ring(in0, nullptr, w, 16, 0, out, nb, n, dil, out_scale, s);
    }
    if (st != SSAM_ERR_UNSUPPORTED) return st;
  }
  const int l2 = log2_exact(n);
  if (l2 < 0 || (int64_t)n * n * n % kTile != 0)
    return fail(SSAM_ERR_INVALID, "conv3d: n must be a power of two with n^3 % 128 == 0");
  if (!in0 || !w || !out) return fail(SSAM_ERR_INVALID, "conv3d: NULL tensor");
  if (((uintptr_t)in0 | (uintptr_t)w | (uintptr_t)out | (uintptr_t)in1) % 16)
    return fail(SSAM_ERR_INVALID, "conv3d: tensors must be 16-byte aligned");
  int* err = nullptr;
  int st = device_error_word(&err);
  if (st != SSAM_OK) return st;
  const int64_t tiles = (int64_t)nb * n * n * n / kTile;
  const int64_t half = (int64_t)nb * n * n * n * 8;
  const unsigned long long ns = 1000ull * 1000ull * 1000ull;
  if (in1) {
    constexpr int SM = conv_smem_bytes<2>();
    static bool attr = false;
    if (!attr) {
      SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_fwd_kernel<2>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, SM));
      attr = true;
    }
    conv3d_fwd_kernel<2><<<(unsigned)tiles, 128, SM, s>>>(
        (const __nv_bfloat16*)in0, (const __nv_bfloat16*)in1, (const __nv_bfloat16*)w,
        (__nv_bfloat16*)out, l2, dil, out_scale, half, err, ns);
  } else {
    constexpr int SM = conv_smem_bytes<1>();
    conv3d_fwd_kernel<1><<<(unsigned)tiles, 128, SM, s>>>(
        (const __nv_bfloat16*)in0, nullptr, (const __nv_bfloat16*)w, (__nv_bfloat16*)out, l2,
        dil, out_scale, half, err, ns);
  }
  count_launch();
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

// dW (fp32, [16][27][16 * nsrc]) for out = conv3d(x0 (+ x1), W): one pass per
// source.  `work` must hold nslabs * 4 * 128 * 16 floats (see
// conv3d_wgrad_work).
int64_t conv3d_wgrad_slabs(int64_t nvox) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int64_t slabs = std::max<int64_t>(1, std::min<int64_t>(sms * 2, nvox / 4096));
  return slabs;
}

int conv3d_wgrad(const void* x0, const void* x1, const void* g, float* dw, float* work, int nb,
                 int n, int dil, cudaStream_t s) {
  const int l2 = log2_exact(n);
  if (l2 < 0) return fail(SSAM_ERR_INVALID, "wgrad: n must be a power of two");
  int* err = nullptr;
  int st = device_error_word(&err);
  if (st != SSAM_OK) return st;
  const int64_t nvox = (int64_t)nb * n * n * n;
  const int64_t slabs = conv3d_wgrad_slabs(nvox);
  const int64_t slab = (nvox + slabs - 1) / slabs;
  static bool attr = false;
  if (!attr) {
    SSAM_CUDA_TRY(cudaFuncSetAttribute(conv3d_wgrad_kernel<1>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
    attr = true;
  }
  const int nsrc = x1 ? 2 : 1;
  for (int src = 0; src < nsrc; ++src) {
    conv3d_wgrad_kernel<1><<<dim3((unsigned)slabs, 4), 128, kWgSmem, s>>>(
        (const __nv_bfloat16*)(src ? x1 : x0), nullptr, (const __nv_bfloat16*)g, work, nvox,
        slab, l2, dil, err, 1000ull * 1000ull * 1000ull);
    count_launch();
    wgrad_reduce_kernel<<<(4 * 128 * 16 + 255) / 256, 256, 0, s>>>(work, dw, (int)slabs,
                                                                     16 * nsrc, src);
    count_launch();
    SSAM_CUDA_TRY(cudaGetLastError());
  }
  return SSAM_OK;
}

}  // namespace ssam

using namespace ssam;

extern "C" int ssam_cnn_conv3d_wgrad(const void* in0, const void* in1, const void* grad_out,
                                     float* dweight, int nbatch, int n, int dilation,
                                     void* stream) {
  if (!in0 || !grad_out || !dweight) return fail(SSAM_ERR_INVALID, "wgrad: NULL tensor");
  if (nbatch < 1 || dilation < 1) return fail(SSAM_ERR_INVALID, "wgrad: bad nbatch / dilation");
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nvox = (int64_t)nbatch * n * n * n;
  const int64_t slabs = conv3d_wgrad_slabs(nvox);
  void* work = nullptr;
  int st = scratch_alloc(&work, (size_t)slabs * 4 * 128 * 16 * sizeof(float), s);
  if (st != SSAM_OK) return st;
  st = conv3d_wgrad(in0, in1, grad_out, dweight, (float*)work, nbatch, n, dilation, s);
  scratch_free(work, s);
  return st;
}

extern "C" int ssam_cnn_conv3d(const void* in0, const void* in1, const void* weight, void* out,
                               int nbatch, int n, int dilation, float out_scale, void* stream) {
  if (nbatch < 1 || dilation < 1) return fail(SSAM_ERR_INVALID, "conv3d: bad nbatch / dilation");
  if (out && (out == in0 || out == in1))
    return fail(SSAM_ERR_INVALID, "conv3d: out must not alias an input");
  return conv3d_fwd(in0, in1, weight, out, nbatch, n, dilation, out_scale, (cudaStream_t)stream);
}
