// The Poisson warm-start network: a 3-level, 16-channel U-Net of 3x3x3
// convolutions (tcgen05 implicit GEMM, cnn.cu), trained and run on the GPU.
//
//   level 1 (n):    e1a, e1b ------------------------------ skip S1 ---+
//   level 2 (n/2):   pool -> e2a, e2b ------------ skip S2 ---+         |
//   level 3 (n/4):    pool -> b1 (dil 1), b2 (dil 2),         |         |
//                             b3 (dil 4), b4 (dil 8)          |         |
//   level 2:          up -> d2a(up, S2), d2b -----------------+         |
//   level 1:          up -> d1a(up, S1), d1b, head (1x1x1, 16 -> 1) ----+
//
// The map f -> u is linear, so the network is linear too (no activations,
// no biases, zero padding as the Dirichlet boundary): the warm start of -f
// is minus the warm start of f, and per-sample scaling commutes with it.
// The input is f / rms(f) in channel 0 of a 16-channel tensor; the output is
// head * rms(f) * kOutScale.  The bottom level's dilations give it a reach of
// +-60 cells at n = 128, close to the whole grid, which is what a Poisson
// solution needs (its Green's function is not local).
//
// Training: MSE against solver-produced solutions in the same normalised
// units, backward through every layer (data gradient = forward convolution
// with mirrored, transposed weights; weight gradient = cnn.cu's MN-major
// tcgen05 kernel), Adam on fp32 master weights, BF16 copies for the GEMMs.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <memory>
#include <random>
#include <string>
#include <vector>

#include "ssam_internal.cuh"

namespace ssam {

int conv3d_fwd(const void* in0, const void* in1, const void* w, void* out, int nb, int n,
               int dil, float out_scale, cudaStream_t s);
int conv3d_wgrad(const void* x0, const void* x1, const void* g, float* dw, float* work, int nb,
                 int n, int dil, cudaStream_t s);
int64_t conv3d_wgrad_slabs(int64_t nvox);

namespace {

constexpr float kOutScale = 0.03f;  // ~ 1 / (3 pi^2): size of u relative to f
constexpr int C = 16;

using bf16 = __nv_bfloat16;

// ----------------------------------------------------------------- kernels --

constexpr int kSumBlocks = 64;

// Per-block partial sums of f^2 (block x of right-hand side b); summed in a
// fixed order by sumsq_finish_kernel so the forward pass is deterministic.
__global__ void sumsq_kernel(const double* __restrict__ f, int64_t n3,
                             double* __restrict__ partial) {
  const int b = blockIdx.y;
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = f[b * n3 + i];
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double sh[32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    partial[b * kSumBlocks + blockIdx.x] = t;
  }
}

__global__ void sumsq_finish_kernel(const double* __restrict__ partial, double* __restrict__ out,
                                    int nb) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    double t = 0.0;
    for (int k = 0; k < kSumBlocks; ++k) t += partial[b * kSumBlocks + k];
    out[b] = t;
  }
}

// x[b][v][0] = f[b][v] / rms_b, channels 1..15 = 0 (planar halves)
__global__ void encode_kernel(const double* __restrict__ f, const double* __restrict__ sumsq,
                              bf16* __restrict__ x, int64_t n3, int nb) {
  const int64_t total = n3 * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int b = (int)(i / n3);
    const double rms = sqrt(sumsq[b] / (double)n3);
    const float v = rms > 0 ? (float)(f[i] / rms) : 0.f;
    uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
    reinterpret_cast<bf16*>(&lo)[0] = __float2bfloat16_rn(v);
    *reinterpret_cast<uint4*>(x + i * 8) = lo;
    *reinterpret_cast<uint4*>(x + total * 8 + i * 8) = hi;
  }
}

// The 16 channels of voxel i of a planar-halves tensor of `nvox` voxels.
__device__ __forceinline__ void load16(const bf16* t, int64_t i, int64_t nvox, float (&v)[16]) {
  const uint4 a = *reinterpret_cast<const uint4*>(t + i * 8);
  const uint4 b = *reinterpret_cast<const uint4*>(t + nvox * 8 + i * 8);
  const bf16* e = reinterpret_cast<const bf16*>(&a);
  const bf16* f = reinterpret_cast<const bf16*>(&b);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i] = __bfloat162float(e[i]);
    v[8 + i] = __bfloat162float(f[i]);
  }
}
__device__ __forceinline__ void store16(bf16* t, int64_t i, int64_t nvox, const float (&v)[16]) {
  uint4 a, b;
  bf16* e = reinterpret_cast<bf16*>(&a);
  bf16* f = reinterpret_cast<bf16*>(&b);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    e[i] = __float2bfloat16_rn(v[i]);
    f[i] = __float2bfloat16_rn(v[8 + i]);
  }
  *reinterpret_cast<uint4*>(t + i * 8) = a;
  *reinterpret_cast<uint4*>(t + nvox * 8 + i * 8) = b;
}

// 2x2x2 average pool (n -> n/2), 16 channels
__global__ void pool_kernel(const bf16* __restrict__ x, bf16* __restrict__ y, int nb, int n) {
  const int h = n / 2;
  const int64_t total = (int64_t)nb * h * h * h;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int xo = (int)(i % h), yo = (int)((i / h) % h), zo = (int)((i / h / h) % h);
    const int64_t b = i / ((int64_t)h * h * h);
    float acc[16] = {0};
    for (int d = 0; d < 8; ++d) {
      const int64_t src = ((b * n + 2 * zo + (d >> 2)) * n + 2 * yo + ((d >> 1) & 1)) * n +
                          2 * xo + (d & 1);
      float v[16];
      load16(x, src, total * 8, v);
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[c] += v[c];
    }
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c] *= 0.125f;
    store16(y, i, total, acc);
  }
}

// backward of the pool: every child gets gy / 8; accumulate into gx when add != 0
__global__ void pool_back_kernel(const bf16* __restrict__ gy, bf16* __restrict__ gx, int nb,
                                 int n, int add) {
  const int h = n / 2;
  const int64_t total = (int64_t)nb * n * n * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)((i / n / n) % n);
    const int64_t b = i / ((int64_t)n * n * n);
    const int64_t p = ((b * h + z / 2) * h + y / 2) * h + x / 2;
    float v[16], o[16];
    load16(gy, p, total / 8, v);
    if (add) load16(gx, i, total, o);
#pragma unroll
    for (int c = 0; c < 16; ++c) o[c] = (add ? o[c] : 0.f) + 0.125f * v[c];
    store16(gx, i, total, o);
  }
}

// nearest upsampling (n -> 2n)
__global__ void up_kernel(const bf16* __restrict__ x, bf16* __restrict__ y, int nb, int n) {
  const int m = 2 * n;
  const int64_t total = (int64_t)nb * m * m * m;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int xo = (int)(i % m), yo = (int)((i / m) % m), zo = (int)((i / m / m) % m);
    const int64_t b = i / ((int64_t)m * m * m);
    const int64_t src = ((b * n + zo / 2) * n + yo / 2) * n + xo / 2;
    const int64_t xv = total / 8;  // voxels of the coarse tensor
    *reinterpret_cast<uint4*>(y + i * 8) = *reinterpret_cast<const uint4*>(x + src * 8);
    *reinterpret_cast<uint4*>(y + total * 8 + i * 8) =
        *reinterpret_cast<const uint4*>(x + xv * 8 + src * 8);
  }
}

// backward of the upsampling: sum of the 8 children
__global__ void up_back_kernel(const bf16* __restrict__ gy, bf16* __restrict__ gx, int nb,
                               int n) {
  const int m = 2 * n;
  const int64_t total = (int64_t)nb * n * n * n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)((i / n) % n), z = (int)((i / n / n) % n);
    const int64_t b = i / ((int64_t)n * n * n);
    float acc[16] = {0};
    for (int d = 0; d < 8; ++d) {
      const int64_t src = ((b * m + 2 * z + (d >> 2)) * m + 2 * y + ((d >> 1) & 1)) * m +
                          2 * x + (d & 1);
      float v[16];
      load16(gy, src, total * 8, v);
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[c] += v[c];
    }
    store16(gx, i, total, acc);
  }
}

// a += b (16-channel BF16 tensors)
__global__ void add_kernel(bf16* __restrict__ a, const bf16* __restrict__ b, int64_t nvox) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox;
       i += (int64_t)gridDim.x * blockDim.x) {
    float u[16], v[16];
    load16(a, i, nvox, u);
    load16(b, i, nvox, v);
#pragma unroll
    for (int c = 0; c < 16; ++c) u[c] += v[c];
    store16(a, i, nvox, u);
  }
}

// head: u0[b][v] = rms_b * kOutScale * sum_c wh[c] x[v][c]   (fp64 out)
__global__ void head_kernel(const bf16* __restrict__ x, const float* __restrict__ wh,
                            const double* __restrict__ sumsq, double* __restrict__ u,
                            int64_t n3, int nb) {
  const int64_t total = n3 * nb;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v[16];
    load16(x, i, total, v);
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < 16; ++c) s = fmaf(wh[c], v[c], s);
    const int b = (int)(i / n3);
    u[i] = (double)s * sqrt(sumsq[b] / (double)n3) * (double)kOutScale;
  }
}

// Loss: the mean over right-hand sides of the relative squared error
//   L = (1/nb) sum_b sum_v (y - t)^2 / sum_v t^2,
// y = sum_c wh[c] x[v][c], t = target / (rms_b * kOutScale) (normalised
// units), so every right-hand side weighs the same whatever the size of its
// solution.  tsq[b] = sum_v target^2.  Writes dL/dx (BF16, into gx),
// accumulates dL/dwh (fp32) and L.
__global__ void head_loss_back_kernel(const bf16* __restrict__ x, const float* __restrict__ wh,
                                      const double* __restrict__ target,
                                      const double* __restrict__ sumsq,
                                      const double* __restrict__ tsq, bf16* __restrict__ gx,
                                      float* __restrict__ gwh, double* __restrict__ loss,
                                      int64_t n3, int nb) {
  const int64_t total = n3 * nb;
  float gw[16] = {0};
  double l = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v[16];
    load16(x, i, total, v);
    float y = 0.f;
#pragma unroll
    for (int c = 0; c < 16; ++c) y = fmaf(wh[c], v[c], y);
    const int b = (int)(i / n3);
    const double scale = sqrt(sumsq[b] / (double)n3) * (double)kOutScale;
    const double t = scale > 0 ? target[i] / scale : 0.0;
    // 1 / (nb * sum_v t^2) in normalised units
    const double wb = tsq[b] > 0 ? scale * scale / (tsq[b] * (double)nb) : 0.0;
    const double d = (double)y - t;
    l += wb * d * d;
    const float g = (float)(2.0 * d * wb);
    float o[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) {
      o[c] = g * wh[c];
      gw[c] = fmaf(g, v[c], gw[c]);
    }
    store16(gx, i, total, o);
  }
  for (int c = 0; c < 16; ++c) {
    float s = gw[c];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&gwh[c], s);
  }
  for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// fp32 master [16][27][ci] -> BF16 forward copy, and the data-gradient
// copies: for source s, Wt_s[ci][26 - tap][co] = W[co][tap][s*16 + ci]
__global__ void cast_weights_kernel(const float* __restrict__ w, bf16* __restrict__ wf,
                                    bf16* __restrict__ wt, int ci_total) {
  const int total = 16 * 27 * ci_total;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int co = i / (27 * ci_total), tap = (i / ci_total) % 27, ci = i % ci_total;
    const bf16 v = __float2bfloat16_rn(w[i]);
    wf[i] = v;
    const int s = ci / 16, c = ci % 16;
    wt[(((int64_t)s * 16 + c) * 27 + (26 - tap)) * 16 + co] = v;
  }
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, int count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

int grid_for(int64_t work) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((work + 255) / 256, 148 * 32));
}

// ---------------------------------------------------------------- network --

struct Layer {
  int level, nsrc, dil;
  size_t woff;  // offset of this layer's weights in the parameter vector
};

struct Net {
  int n = 0, nb_max = 0;
  std::vector<Layer> layers;
  size_t nparams = 0;  // conv weights + 16 head weights
  // device parameter state
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16 *wf = nullptr, *wt = nullptr;  // forward and data-gradient BF16 copies
  int64_t adam_t = 0;
  // activations (BF16, 16 channels) per level, allocated for nb_max
  std::vector<void*> bufs;
  void* wg_work = nullptr;
  double* scal = nullptr;  // sumsq[nb_max], loss, spare, kSumBlocks partials per rhs, tsq[nb_max]
  bool weights_dirty = true;
};

enum LayerId { E1A, E1B, E2A, E2B, B1, B2, B3, B4, D2A, D2B, D1A, D1B, NLAYERS };

void define_layers(Net& net) {
  const int spec[NLAYERS][3] = {
      {0, 1, 1}, {0, 1, 1}, {1, 1, 1}, {1, 1, 1}, {2, 1, 1}, {2, 1, 2},
      {2, 1, 4}, {2, 1, 8}, {1, 2, 1}, {1, 1, 1}, {0, 2, 1}, {0, 1, 1}};
  size_t off = 0;
  for (int i = 0; i < NLAYERS; ++i) {
    net.layers.push_back(Layer{spec[i][0], spec[i][1], spec[i][2], off});
    off += (size_t)16 * 27 * 16 * spec[i][1];
  }
  net.nparams = off + 16;  // + head
}

int level_n(const Net& net, int level) { return net.n >> level; }

// Activation buffer indices.
enum Buf {
  X0, A1, S1, P1, A2, S2, P2, T3a, T3b, U2, D2a, D2b, U1, D1a, D1b,
  // gradient buffers
  GA, GB, GS1, GS2, GL2a, GL2b, GL3a, GL3b, NBUF
};
int buf_level(int b) {
  switch (b) {
    case X0: case A1: case S1: case U1: case D1a: case D1b: case GA: case GB: case GS1:
      return 0;
    case P1: case A2: case S2: case U2: case D2a: case D2b: case GS2: case GL2a: case GL2b:
      return 1;
    default:
      return 2;
  }
}

const float* lw(const Net& net, int l) { return net.w + net.layers[l].woff; }
const bf16* lwf(const Net& net, int l) { return net.wf + net.layers[l].woff; }
const bf16* lwt(const Net& net, int l) { return net.wt + net.layers[l].woff; }

int refresh_weights(Net& net, cudaStream_t s) {
  if (!net.weights_dirty) return SSAM_OK;
  for (int l = 0; l < NLAYERS; ++l) {
    const int ci = 16 * net.layers[l].nsrc;
    cast_weights_kernel<<<grid_for(16 * 27 * ci), 256, 0, s>>>(
        net.w + net.layers[l].woff, net.wf + net.layers[l].woff, net.wt + net.layers[l].woff,
        ci);
    count_launch();
  }
  SSAM_CUDA_TRY(cudaGetLastError());
  net.weights_dirty = false;
  return SSAM_OK;
}

#define NET_TRY(x)                   \
  do {                               \
    int _st = (x);                   \
    if (_st != SSAM_OK) return _st;  \
  } while (0)

int conv(Net& net, int l, Buf in0, int in1, Buf out, int nb, cudaStream_t s) {
  const Layer& L = net.layers[l];
  return conv3d_fwd(net.bufs[in0], in1 >= 0 ? net.bufs[in1] : nullptr, lwf(net, l),
                    net.bufs[out], nb, level_n(net, L.level), L.dil, 1.f, s);
}

int forward(Net& net, const double* f, int nb, cudaStream_t s) {
  const int n = net.n;
  const int64_t n3 = (int64_t)n * n * n;
  NET_TRY(refresh_weights(net, s));
  SSAM_CUDA_TRY(cudaMemsetAsync(net.scal, 0, sizeof(double) * (net.nb_max + 1), s));
  sumsq_kernel<<<dim3(kSumBlocks, nb), 256, 0, s>>>(f, n3, net.scal + net.nb_max + 2);
  sumsq_finish_kernel<<<1, 32, 0, s>>>(net.scal + net.nb_max + 2, net.scal, nb);
  count_launch();
  encode_kernel<<<grid_for(n3 * nb), 256, 0, s>>>(f, net.scal, (bf16*)net.bufs[X0], n3, nb);
  count_launch();
  count_launch();
  NET_TRY(conv(net, E1A, X0, -1, A1, nb, s));
  NET_TRY(conv(net, E1B, A1, -1, S1, nb, s));
  pool_kernel<<<grid_for(n3 * nb / 8), 256, 0, s>>>((bf16*)net.bufs[S1], (bf16*)net.bufs[P1],
                                                    nb, n);
  count_launch();
  NET_TRY(conv(net, E2A, P1, -1, A2, nb, s));
  NET_TRY(conv(net, E2B, A2, -1, S2, nb, s));
  pool_kernel<<<grid_for(n3 * nb / 64), 256, 0, s>>>((bf16*)net.bufs[S2], (bf16*)net.bufs[P2],
                                                     nb, n / 2);
  count_launch();
  NET_TRY(conv(net, B1, P2, -1, T3a, nb, s));
  NET_TRY(conv(net, B2, T3a, -1, T3b, nb, s));
  NET_TRY(conv(net, B3, T3b, -1, T3a, nb, s));
  NET_TRY(conv(net, B4, T3a, -1, T3b, nb, s));
  up_kernel<<<grid_for(n3 * nb / 8), 256, 0, s>>>((bf16*)net.bufs[T3b], (bf16*)net.bufs[U2], nb,
                                                  n / 4);
  count_launch();
  NET_TRY(conv(net, D2A, U2, S2, D2a, nb, s));
  NET_TRY(conv(net, D2B, D2a, -1, D2b, nb, s));
  up_kernel<<<grid_for(n3 * nb), 256, 0, s>>>((bf16*)net.bufs[D2b], (bf16*)net.bufs[U1], nb,
                                              n / 2);
  count_launch();
  NET_TRY(conv(net, D1A, U1, S1, D1a, nb, s));
  NET_TRY(conv(net, D1B, D1a, -1, D1b, nb, s));
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

// Data gradient of layer l into gradient buffers (one per source); `out_g`
// is the gradient w.r.t. the layer's output.  Weight gradient into net.g.
int conv_back(Net& net, int l, Buf in0, int in1, Buf out_g, Buf gin0, int gin1, bool need_din,
              int nb, cudaStream_t s) {
  const Layer& L = net.layers[l];
  const int nl = level_n(net, L.level);
  NET_TRY(conv3d_wgrad(net.bufs[in0], in1 >= 0 ? net.bufs[in1] : nullptr, net.bufs[out_g],
                       net.g + L.woff, (float*)net.wg_work, nb, nl, L.dil, s));
  if (!need_din) return SSAM_OK;
  // data gradient: conv of out_g with the mirrored, transposed weights
  NET_TRY(conv3d_fwd(net.bufs[out_g], nullptr, lwt(net, l), net.bufs[gin0], nb, nl, L.dil, 1.f,
                     s));
  if (gin1 >= 0)
    NET_TRY(conv3d_fwd(net.bufs[out_g], nullptr, lwt(net, l) + 16 * 27 * 16, net.bufs[gin1], nb,
                       nl, L.dil, 1.f, s));
  return SSAM_OK;
}

int backward(Net& net, const double* target, int nb, cudaStream_t s) {
  const int n = net.n;
  const int64_t n3 = (int64_t)n * n * n;
  float* gh = net.g + (net.nparams - 16);
  SSAM_CUDA_TRY(cudaMemsetAsync(gh, 0, 16 * sizeof(float), s));
  double* part = net.scal + net.nb_max + 2;
  double* tsq = part + (size_t)kSumBlocks * net.nb_max;
  sumsq_kernel<<<dim3(kSumBlocks, nb), 256, 0, s>>>(target, n3, part);
  sumsq_finish_kernel<<<1, 32, 0, s>>>(part, tsq, nb);
  count_launch();
  count_launch();
  head_loss_back_kernel<<<grid_for(n3 * nb), 256, 0, s>>>(
      (const bf16*)net.bufs[D1b], net.w + (net.nparams - 16), target, net.scal, tsq,
      (bf16*)net.bufs[GA], gh, net.scal + net.nb_max, n3, nb);
  count_launch();
  // level 1 decoder
  NET_TRY(conv_back(net, D1B, D1a, -1, GA, GB, -1, true, nb, s));          // GB = dD1a
  NET_TRY(conv_back(net, D1A, U1, S1, GB, GA, GS1, true, nb, s));          // GA = dU1, GS1 = dS1
  up_back_kernel<<<grid_for(n3 * nb / 8), 256, 0, s>>>((bf16*)net.bufs[GA],
                                                       (bf16*)net.bufs[GL2a], nb, n / 2);
  count_launch();
  // level 2 decoder: GL2a = dD2b
  NET_TRY(conv_back(net, D2B, D2a, -1, GL2a, GL2b, -1, true, nb, s));      // GL2b = dD2a
  NET_TRY(conv_back(net, D2A, U2, S2, GL2b, GL2a, GS2, true, nb, s));      // GL2a = dU2
  up_back_kernel<<<grid_for(n3 * nb / 64), 256, 0, s>>>((bf16*)net.bufs[GL2a],
                                                        (bf16*)net.bufs[GL3a], nb, n / 4);
  count_launch();
  // bottom: GL3a = dB4out
  NET_TRY(conv_back(net, B4, T3a, -1, GL3a, GL3b, -1, true, nb, s));
  // recompute the bottom activations that were overwritten (T3a/T3b reuse)
  NET_TRY(conv(net, B1, P2, -1, T3a, nb, s));
  NET_TRY(conv(net, B2, T3a, -1, T3b, nb, s));
  NET_TRY(conv_back(net, B3, T3b, -1, GL3b, GL3a, -1, true, nb, s));
  NET_TRY(conv_back(net, B2, T3a, -1, GL3a, GL3b, -1, true, nb, s));
  NET_TRY(conv_back(net, B1, P2, -1, GL3b, GL3a, -1, true, nb, s));        // GL3a = dP2
  // pool back into dS2 (accumulate with the skip gradient)
  pool_back_kernel<<<grid_for(n3 * nb / 8), 256, 0, s>>>((bf16*)net.bufs[GL3a],
                                                         (bf16*)net.bufs[GS2], nb, n / 2, 1);
  count_launch();
  NET_TRY(conv_back(net, E2B, A2, -1, GS2, GL2a, -1, true, nb, s));        // GL2a = dA2
  NET_TRY(conv_back(net, E2A, P1, -1, GL2a, GL2b, -1, true, nb, s));       // GL2b = dP1
  pool_back_kernel<<<grid_for(n3 * nb), 256, 0, s>>>((bf16*)net.bufs[GL2b],
                                                     (bf16*)net.bufs[GS1], nb, n, 1);
  count_launch();
  NET_TRY(conv_back(net, E1B, A1, -1, GS1, GA, -1, true, nb, s));          // GA = dA1
  NET_TRY(conv_back(net, E1A, X0, -1, GA, GB, -1, false, nb, s));
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

void net_free(Net* net) {
  for (void* p : net->bufs) cudaFree(p);
  cudaFree(net->w);
  cudaFree(net->g);
  cudaFree(net->m);
  cudaFree(net->v);
  cudaFree(net->wf);
  cudaFree(net->wt);
  cudaFree(net->wg_work);
  cudaFree(net->scal);
  delete net;
}

}  // namespace
}  // namespace ssam

using namespace ssam;

extern "C" int ssam_cnn_create(int n, int nbatch_max, unsigned long long seed, void** handle) {
  if (!handle) return fail(SSAM_ERR_INVALID, "handle must not be NULL");
  *handle = nullptr;
  if (n < 32 || (n & (n - 1)) || nbatch_max < 1)
    return fail(SSAM_ERR_INVALID, "CNN grid n must be a power of two >= 32");
  Net* net = new Net();
  net->n = n;
  net->nb_max = nbatch_max;
  define_layers(*net);
  // He-style init scaled for a linear network: keep activations O(1)
  std::vector<float> w(net->nparams);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NLAYERS; ++l) {
    const int fan_in = 27 * 16 * net->layers[l].nsrc;
    std::normal_distribution<float> nd(0.f, sqrtf(1.f / fan_in));
    for (size_t i = 0; i < (size_t)16 * 27 * 16 * net->layers[l].nsrc; ++i)
      w[net->layers[l].woff + i] = nd(rng);
  }
  std::normal_distribution<float> nh(0.f, 0.25f);
  for (int c = 0; c < 16; ++c) w[net->nparams - 16 + c] = nh(rng);
  auto bail = [&](cudaError_t e, const char* what) {
    net_free(net);
    return fail_cuda(e, what);
  };
  const size_t pb = net->nparams * sizeof(float);
  cudaError_t e = cudaMalloc(&net->w, pb);
  if (e == cudaSuccess) e = cudaMalloc(&net->g, pb);
  if (e == cudaSuccess) e = cudaMalloc(&net->m, pb);
  if (e == cudaSuccess) e = cudaMalloc(&net->v, pb);
  if (e == cudaSuccess) e = cudaMalloc(&net->wf, net->nparams * sizeof(bf16));
  if (e == cudaSuccess) e = cudaMalloc(&net->wt, net->nparams * sizeof(bf16));
  if (e == cudaSuccess) e = cudaMalloc(&net->scal,
                                        sizeof(double) * (2 * (size_t)nbatch_max + 2 +
                                                          (size_t)kSumBlocks * nbatch_max));
  if (e != cudaSuccess) return bail(e, "cudaMalloc(cnn parameters)");
  e = cudaMemcpy(net->w, w.data(), pb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(net->g, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(net->m, 0, pb);
  if (e == cudaSuccess) e = cudaMemset(net->v, 0, pb);
  if (e != cudaSuccess) return bail(e, "cnn parameter init");
  net->bufs.assign(NBUF, nullptr);
  for (int b = 0; b < NBUF; ++b) {
    const int64_t nl = n >> buf_level(b);
    e = cudaMalloc(&net->bufs[b], (size_t)nbatch_max * nl * nl * nl * C * sizeof(bf16));
    if (e != cudaSuccess) return bail(e, "cudaMalloc(cnn activations)");
  }
  const int64_t slabs = conv3d_wgrad_slabs((int64_t)nbatch_max * n * n * n);
  e = cudaMalloc(&net->wg_work, (size_t)slabs * 4 * 128 * 16 * sizeof(float));
  if (e != cudaSuccess) return bail(e, "cudaMalloc(cnn wgrad work)");
  *handle = net;
  return SSAM_OK;
}

extern "C" int ssam_cnn_destroy(void* handle) {
  if (handle) net_free((Net*)handle);
  return SSAM_OK;
}

extern "C" int ssam_cnn_num_params(void* handle, int64_t* count) {
  if (!handle || !count) return fail(SSAM_ERR_INVALID, "NULL argument");
  *count = (int64_t)((Net*)handle)->nparams;
  return SSAM_OK;
}

extern "C" int ssam_cnn_get_params(void* handle, float* host_params, float* host_grads) {
  Net* net = (Net*)handle;
  if (!net) return fail(SSAM_ERR_INVALID, "NULL handle");
  const size_t pb = net->nparams * sizeof(float);
  if (host_params) SSAM_CUDA_TRY(cudaMemcpy(host_params, net->w, pb, cudaMemcpyDeviceToHost));
  if (host_grads) SSAM_CUDA_TRY(cudaMemcpy(host_grads, net->g, pb, cudaMemcpyDeviceToHost));
  return SSAM_OK;
}

extern "C" int ssam_cnn_set_params(void* handle, const float* host_params) {
  Net* net = (Net*)handle;
  if (!net || !host_params) return fail(SSAM_ERR_INVALID, "NULL argument");
  SSAM_CUDA_TRY(cudaMemcpy(net->w, host_params, net->nparams * sizeof(float),
                           cudaMemcpyHostToDevice));
  net->weights_dirty = true;
  return SSAM_OK;
}

extern "C" int ssam_cnn_forward(void* handle, const double* f, double* u0, int nbatch,
                                void* stream) {
  Net* net = (Net*)handle;
  if (!net || !f || !u0) return fail(SSAM_ERR_INVALID, "NULL argument");
  if (nbatch < 1 || nbatch > net->nb_max) return fail(SSAM_ERR_INVALID, "nbatch out of range");
  cudaStream_t s = (cudaStream_t)stream;
  NET_TRY(forward(*net, f, nbatch, s));
  const int64_t n3 = (int64_t)net->n * net->n * net->n;
  head_kernel<<<grid_for(n3 * nbatch), 256, 0, s>>>((const bf16*)net->bufs[D1b],
                                                    net->w + (net->nparams - 16), net->scal, u0,
                                                    n3, nbatch);
  count_launch();
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

namespace ssam {
// The network can serve a solve of nbatch right-hand sides on n^3.
int cnn_check(void* cnn, int n, int nbatch) {
  Net* net = (Net*)cnn;
  if (net->n != n) return fail(SSAM_ERR_INVALID, "network grid size differs from the solve's");
  if (nbatch > net->nb_max) return fail(SSAM_ERR_INVALID, "nbatch exceeds the network's nbatch_max");
  return SSAM_OK;
}

// c = network(r) for the defect-correction loop of the Poisson solver.
int cnn_apply(void* cnn, const double* r, double* c, int nbatch, cudaStream_t s) {
  return ssam_cnn_forward(cnn, r, c, nbatch, s);
}
}  // namespace ssam

// Forward + backward on (f, target); fills the gradient; returns the loss
// (normalised units) on the host.  Does not update the weights.
extern "C" int ssam_cnn_gradient(void* handle, const double* f, const double* target,
                                 int nbatch, double* loss, void* stream) {
  Net* net = (Net*)handle;
  if (!net || !f || !target) return fail(SSAM_ERR_INVALID, "NULL argument");
  if (nbatch < 1 || nbatch > net->nb_max) return fail(SSAM_ERR_INVALID, "nbatch out of range");
  cudaStream_t s = (cudaStream_t)stream;
  NET_TRY(forward(*net, f, nbatch, s));
  NET_TRY(backward(*net, target, nbatch, s));
  if (loss)
    SSAM_CUDA_TRY(cudaMemcpyAsync(loss, net->scal + net->nb_max, sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
  SSAM_CUDA_TRY(cudaStreamSynchronize(s));
  return SSAM_OK;
}

// One Adam step with the gradient of the last ssam_cnn_gradient call.
extern "C" int ssam_cnn_adam_step(void* handle, float lr, void* stream) {
  Net* net = (Net*)handle;
  if (!net) return fail(SSAM_ERR_INVALID, "NULL handle");
  const float b1 = 0.9f, b2 = 0.999f;
  net->adam_t += 1;
  const float c1 = 1.f - powf(b1, (float)net->adam_t), c2 = 1.f - powf(b2, (float)net->adam_t);
  adam_kernel<<<grid_for((int64_t)net->nparams), 256, 0, (cudaStream_t)stream>>>(
      net->w, net->g, net->m, net->v, (int)net->nparams, lr, b1, b2, 1e-8f, c1, c2);
  count_launch();
  net->weights_dirty = true;
  SSAM_CUDA_TRY(cudaGetLastError());
  return SSAM_OK;
}

// Weights as a little-endian float32 blob preceded by a one-line JSON header.
extern "C" int ssam_cnn_save(void* handle, const char* path) {
  Net* net = (Net*)handle;
  if (!net || !path) return fail(SSAM_ERR_INVALID, "NULL argument");
  std::vector<float> w(net->nparams);
  SSAM_CUDA_TRY(cudaMemcpy(w.data(), net->w, w.size() * sizeof(float), cudaMemcpyDeviceToHost));
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(SSAM_ERR_INVALID, std::string("cannot write ") + path);
  fprintf(fp, "{\"format\": \"ssam_cnn_v1\", \"n\": %d, \"params\": %zu, \"adam_steps\": %lld}\n",
          net->n, net->nparams, (long long)net->adam_t);
  const size_t wrote = fwrite(w.data(), sizeof(float), w.size(), fp);
  fclose(fp);
  if (wrote != w.size()) return fail(SSAM_ERR_INVALID, "short write");
  return SSAM_OK;
}

extern "C" int ssam_cnn_load(void* handle, const char* path) {
  Net* net = (Net*)handle;
  if (!net || !path) return fail(SSAM_ERR_INVALID, "NULL argument");
  FILE* fp = fopen(path, "rb");
  if (!fp) return fail(SSAM_ERR_INVALID, std::string("cannot read ") + path);
  char line[512];
  size_t params = 0;
  if (!fgets(line, sizeof line, fp) || !strstr(line, "ssam_cnn_v1") ||
      !strstr(line, "\"params\": ") ||
      sscanf(strstr(line, "\"params\": ") + 10, "%zu", &params) != 1 || params != net->nparams) {
    fclose(fp);
    return fail(SSAM_ERR_INVALID, "not an ssam_cnn_v1 file for this network");
  }
  std::vector<float> w(params);
  const size_t got = fread(w.data(), sizeof(float), params, fp);
  fclose(fp);
  if (got != params) return fail(SSAM_ERR_INVALID, "truncated weight file");
  SSAM_CUDA_TRY(cudaMemcpy(net->w, w.data(), params * sizeof(float), cudaMemcpyHostToDevice));
  net->weights_dirty = true;
  return SSAM_OK;
}
