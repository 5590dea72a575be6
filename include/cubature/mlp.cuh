// mlp.cuh -- the control-variate network g: 7 -> 128 -> 128 -> 128 -> 1,
// SiLU, BF16 weights and activations, FP32 accumulation; one independent
// network per integral (batched over integrals in grid.z).
//
// Every hidden-layer product runs on the tensor cores through one kernel,
// k_gemm (umma.cuh: D = A * B^T with A, B K-major), with three epilogues:
//
//   forward   Z = D + b;  H = silu(Z)         writes Z, H (row-major) and H^T
//   backward  dZ = D * silu'(Z)                writes dZ (row-major) and dZ^T
//   store     D as fp32                        (weight gradients)
//
// Keeping both layouts of every activation makes each product K-major on
// both sides:
//   forward      Z_l   = H_{l-1} W_l^T     A = H_{l-1} [s][in],  B = W_l  [out][in]
//   backward     dH_l  = dZ_{l+1} W_{l+1}  A = dZ_{l+1} [s][out], B = W^T [in][out]
//   gradients    dW_l  = dZ_l^T H_{l-1}    A = dZ_l^T [out][s],  B = H^T  [in][s]
// The 1-wide output layer, the loss and Adam run on the CUDA cores.
#pragma once

#include <cuda_bf16.h>

#include "umma.cuh"

namespace cubature {
namespace mlp {

constexpr int kIn = 7;      // network inputs
constexpr int kInPad = 16;  // padded to one MMA K-step
constexpr int kHidden = 128;

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float silu_grad(float z) {
  const float s = sigmoid(z);
  return s * (1.0f + z * (1.0f - s));
}

enum Epilogue : int { kEpiStore = 0, kEpiForward = 1, kEpiBackward = 2 };

struct EpiArgs {
  // kEpiStore: out[e * batch_out + row * ld_out + col] (fp32)
  float* out;
  long long ld_out, batch_out;
  // kEpiForward: bias[e * batch_bias + col]; z, h: [row][ld_act]; ht: [col][ld_t]
  const float* bias;
  long long batch_bias;
  __nv_bfloat16* z;
  __nv_bfloat16* h;
  __nv_bfloat16* ht;
  // kEpiBackward: zin [row][ld_act]; dz [row][ld_act]; dzt [col][ld_t]
  const __nv_bfloat16* zin;
  __nv_bfloat16* dz;
  __nv_bfloat16* dzt;
  long long ld_act, batch_act, ld_t, batch_t;
};

template <int N, int EPI>
__device__ __forceinline__ void epilogue(const EpiArgs& ep, int e, int row, int c0,
                                         const float* v, int cnt) {
  if (EPI == kEpiStore) {
    float* o = ep.out + (long long)e * ep.batch_out + (long long)row * ep.ld_out + c0;
    for (int i = 0; i < cnt; ++i) o[i] = v[i];
  } else if (EPI == kEpiForward) {
    const float* b = ep.bias + (long long)e * ep.batch_bias + c0;
    const long long ra = (long long)e * ep.batch_act + (long long)row * ep.ld_act + c0;
    const long long rt = (long long)e * ep.batch_t + row;
    for (int i = 0; i < cnt; ++i) {
      const float z = v[i] + b[i];
      const __nv_bfloat16 zb = __float2bfloat16(z);
      const __nv_bfloat16 hb = __float2bfloat16(silu(__bfloat162float(zb)));
      ep.z[ra + i] = zb;
      ep.h[ra + i] = hb;
      ep.ht[rt + (long long)(c0 + i) * ep.ld_t] = hb;
    }
  } else {
    const long long ra = (long long)e * ep.batch_act + (long long)row * ep.ld_act + c0;
    const long long rt = (long long)e * ep.batch_t + row;
    for (int i = 0; i < cnt; ++i) {
      const float dz = v[i] * silu_grad(__bfloat162float(ep.zin[ra + i]));
      const __nv_bfloat16 db = __float2bfloat16(dz);
      ep.dz[ra + i] = db;
      ep.dzt[rt + (long long)(c0 + i) * ep.ld_t] = db;
    }
  }
}

// Dynamic shared memory of k_gemm: the A chunk (16 KB), the B chunk (up to
// 16 KB), and slack up to 64 KB so that every operand read the descriptors
// can describe stays inside the CTA's allocation.
constexpr int kGemmSmem = 64 * 1024;

// One 128-row tile of D = A * B^T for batch entry blockIdx.z, row tile
// blockIdx.x, and its epilogue.  128 threads.

template <int N, int EPI>
__global__ void __launch_bounds__(128) k_gemm(umma::GemmArgs g, EpiArgs ep) {
  constexpr uint32_t kCols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
  extern __shared__ __align__(1024) uint8_t dsm[];
  uint8_t* sa = dsm;
  uint8_t* sb = dsm + umma::kTileM * umma::kChunkK * 2;
  __shared__ uint64_t bar;
  __shared__ uint32_t tmem_base;
  const int e = blockIdx.z, mt = blockIdx.x;
  if (threadIdx.x == 0) umma::mbar_init(&bar, 1);
  if (threadIdx.x < 32) umma::tmem_alloc(&tmem_base, kCols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tmem_base;
  uint32_t phase = 0;
  const bool ok = umma::gemm_tile<N>(g, e, mt, tmem, sa, sb, &bar, phase);
  if (ok) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row = mt * umma::kTileM + w * 32 + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(w * 32) << 16);
    if (N % 32 == 0) {
#pragma unroll 1
      for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        umma::tmem_load32(lane_addr + c0, v);
        epilogue<N, EPI>(ep, e, row, c0, v, 32);
      }
    } else {
#pragma unroll 1
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        umma::tmem_load16(lane_addr + c0, v);
        epilogue<N, EPI>(ep, e, row, c0, v, 16);
      }
    }
  } else {
    if (threadIdx.x == 0) atomicExch(g.error, 1);
    // the last commit may still be in flight: wait for it (bounded) before
    // the accumulator columns are released
    umma::mbar_wait(&bar, phase ^ 1);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) umma::tmem_dealloc(tmem, kCols);
}

// Layout of one network's fp32 parameter vector (also of its gradient and
// Adam moments).  W0 is [128][16] (out-major; inputs 7..15 are padding and
// stay zero), W1, W2 are [128][128] (out-major), w3 the output weights.
struct Layout {
  static constexpr int W0 = 0;
  static constexpr int B0 = W0 + kHidden * kInPad;
  static constexpr int W1 = B0 + kHidden;
  static constexpr int B1 = W1 + kHidden * kHidden;
  static constexpr int W2 = B1 + kHidden;
  static constexpr int B2 = W2 + kHidden * kHidden;
  static constexpr int W3 = B2 + kHidden;
  static constexpr int B3 = W3 + kHidden;
  static constexpr int kCount = B3 + 8;  // padded to 8 floats
};

// Inputs of network e: x in [0,1]^7 (fp64, [count][7]) -> bf16 (2x - 1),
// padded to 16, row-major X [count][16] and transposed XT [16][ld_t].
__global__ void k_prep_inputs(const double* x, long long count, long long batch_x,
                              __nv_bfloat16* X, __nv_bfloat16* XT, long long ld_t,
                              long long batch_X, long long batch_XT) {
  const int e = blockIdx.z;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < count;
       s += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int i = 0; i < kInPad; ++i) {
      const float v = i < kIn ? (float)(2.0 * x[e * batch_x + s * kIn + i] - 1.0) : 0.0f;
      const __nv_bfloat16 b = __float2bfloat16(v);
      X[e * batch_X + s * kInPad + i] = b;
      XT[e * batch_XT + (long long)i * ld_t + s] = b;
    }
  }
}

// Output layer on the CUDA cores, one thread per sample, 128 per block:
// g = H3 . w3 + b3.  Training (y != null): err = g - y; dZ3 = e w3 silu'(Z3)
// with e = 2 err / nbatch written row-major and transposed, and per-block
// partials part[blk] = (sum_s e H3[s][:], sum_s e, sum_s err^2).  Inference
// (g_out != null): g_out[s] = scale * g.
__global__ void __launch_bounds__(128) k_output(const float* P, const __nv_bfloat16* H3,
                                                const __nv_bfloat16* Z3, const float* y,
                                                long long batch_y, float inv_nbatch, __nv_bfloat16* dZ3,
                                                __nv_bfloat16* dZ3T, float* part,
                                                long long rows, long long valid,
                                                const float* scale, double* g_out,
                                                long long batch_g) {
  __shared__ float w3[kHidden];
  __shared__ float es[kHidden];
  const int e = blockIdx.z;
  const float* p = P + (long long)e * Layout::kCount;
  w3[threadIdx.x] = p[Layout::W3 + threadIdx.x];
  __syncthreads();
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long base = (long long)e * rows * kHidden;
  float g = p[Layout::B3];
  for (int j = 0; j < kHidden; ++j) g += __bfloat162float(H3[base + s * kHidden + j]) * w3[j];
  if (g_out) {
    if (s < valid) g_out[(long long)e * batch_g + s] = (double)scale[e] * (double)g;
    return;
  }
  const float err = g - y[(long long)e * batch_y + s];
  const float ec = 2.0f * err * inv_nbatch;
  es[threadIdx.x] = ec;
  for (int j = 0; j < kHidden; ++j) {
    const float dz = ec * w3[j] * silu_grad(__bfloat162float(Z3[base + s * kHidden + j]));
    const __nv_bfloat16 b = __float2bfloat16(dz);
    dZ3[base + s * kHidden + j] = b;
    dZ3T[base + (long long)j * rows + s] = b;
  }
  __syncthreads();
  // partial output-layer gradients of this block's 128 samples (fixed order)
  float* out = part + ((long long)e * gridDim.x + blockIdx.x) * (kHidden + 2);
  const long long s0 = (long long)blockIdx.x * blockDim.x;
  float acc = 0;
  for (int i = 0; i < 128; ++i)
    acc += es[i] * __bfloat162float(H3[base + (s0 + i) * kHidden + threadIdx.x]);
  out[threadIdx.x] = acc;
  // error sum and squared error, reduced by thread 0 in order
  __shared__ float sq[kHidden];
  sq[threadIdx.x] = err * err;
  __syncthreads();
  if (threadIdx.x == 0) {
    float se = 0, ss = 0;
    for (int i = 0; i < 128; ++i) {
      se += es[i];
      ss += sq[i];
    }
    out[kHidden] = se;
    out[kHidden + 1] = ss;
  }
}

// Sum the per-block partials in block order: gradients of w3 and b3, and
// the mean squared error of the batch.
__global__ void k_reduce_output(const float* part, int nblk, float* G, float* loss,
                                float inv_nbatch) {
  const int e = blockIdx.z;
  const float* pe = part + (long long)e * nblk * (kHidden + 2);
  for (int j = threadIdx.x; j < kHidden + 2; j += blockDim.x) {
    float a = 0;
    for (int b = 0; b < nblk; ++b) a += pe[(long long)b * (kHidden + 2) + j];
    if (j < kHidden)
      G[(long long)e * Layout::kCount + Layout::W3 + j] = a;
    else if (j == kHidden)
      G[(long long)e * Layout::kCount + Layout::B3] = a;
    else
      loss[e] = a * inv_nbatch;
  }
}

// Bias gradients: G[off + j] = sum_s dZT[j][s], a warp per j (fixed order).
__global__ void k_bias_grad(const __nv_bfloat16* dZT, long long rows, float* G, int off) {
  const int e = blockIdx.z;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= kHidden) return;
  const __nv_bfloat16* r = dZT + ((long long)e * kHidden + warp) * rows;
  float a = 0;
  for (long long s = lane; s < rows; s += 32) a += __bfloat162float(r[s]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) G[(long long)e * Layout::kCount + off + warp] = a;
}

// Adam on every parameter of every network (step t >= 1, bias-corrected).
__global__ void k_adam(float* P, const float* G, float* M, float* V, long long n, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float g = G[i];
    const float m = b1 * M[i] + (1 - b1) * g;
    const float v = b2 * V[i] + (1 - b2) * g * g;
    M[i] = m;
    V[i] = v;
    P[i] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  }
}

// bf16 copies of the weights for the tensor cores: W0, W1, W2 (out-major)
// and W1T, W2T (in-major).
__global__ void k_refresh_weights(const float* P, __nv_bfloat16* W0, __nv_bfloat16* W1,
                                  __nv_bfloat16* W1T, __nv_bfloat16* W2, __nv_bfloat16* W2T) {
  const int e = blockIdx.z;
  const float* p = P + (long long)e * Layout::kCount;
  const long long sq = (long long)kHidden * kHidden;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kHidden * kHidden;
       i += gridDim.x * blockDim.x) {
    const int r = i / kHidden, c = i % kHidden;
    const __nv_bfloat16 w1 = __float2bfloat16(p[Layout::W1 + i]);
    const __nv_bfloat16 w2 = __float2bfloat16(p[Layout::W2 + i]);
    W1[e * sq + i] = w1;
    W2[e * sq + i] = w2;
    W1T[e * sq + (long long)c * kHidden + r] = w1;
    W2T[e * sq + (long long)c * kHidden + r] = w2;
    if (i < kHidden * kInPad)
      W0[(long long)e * kHidden * kInPad + i] = __float2bfloat16(p[Layout::W0 + i]);
  }
}

// Targets of network e scaled by 1 / max |y| (scale[e] = max |y|, 1 if 0).
__global__ void k_scale_targets(const double* y, long long count, float* Y, float* scale) {
  const int e = blockIdx.z;
  __shared__ double red[256];
  double m = 0;
  for (long long s = threadIdx.x; s < count; s += blockDim.x) m = fmax(m, fabs(y[e * count + s]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  const double sc = red[0] > 0 ? red[0] : 1.0;
  if (threadIdx.x == 0) scale[e] = (float)sc;
  for (long long s = threadIdx.x; s < count; s += blockDim.x)
    Y[e * count + s] = (float)(y[e * count + s] / sc);
}

}  // namespace mlp
}  // namespace cubature
