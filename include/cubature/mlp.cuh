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

}  // namespace mlp
}  // namespace cubature
