// step_kernels.cuh -- stand-alone kernels behind the per-step C entry points
// (rule evaluation, split, reduction on caller-provided buffers).  The
// engine fuses the same work into its own iteration kernels.
#pragma once

#include "engine_kernels.cuh"

namespace cubature {

// Rule + classification over one integral's SoA list (INTEGRATE_GPU_PHASE1,
// GPUQuadPhases.cu:38-79).
template <int N, int K, class F>
__global__ void __launch_bounds__(256) k_step_rule(F f, RuleTables T, long long n,
                                                   const double* lo, const double* len,
                                                   long long ld, double epsrel, double epsabs,
                                                   double* avg, double* err, int* axis,
                                                   int* active) {
  __shared__ detail::ItemTable<N> tab;
  if (threadIdx.x == 0) tab.fill();
  __syncthreads();
  constexpr int kGroups = 256 / K;
  const int lane = threadIdx.x % K;
  const unsigned gmask =
      (K == 32) ? 0xffffffffu : (((1u << K) - 1u) << ((threadIdx.x & 31) & ~(K - 1)));
  for (long long i = (long long)blockIdx.x * kGroups + threadIdx.x / K; i < n;
       i += (long long)gridDim.x * kGroups) {
    double L[N], H[N];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      L[d] = lo[(long long)d * ld + i];
      H[d] = len[(long long)d * ld + i];
    }
    detail::RegionSums rs;
    detail::region_point_sums<N, K>(f, L, H, lane, tab, T.ratio, rs);
    if (K > 1) detail::reduce_lanes<K>(rs, gmask);
    if (lane == 0) {
      double jac = 1;
#pragma unroll
      for (int d = 0; d < N; ++d) jac = __dmul_rn(jac, H[d]);
      const detail::RegionResult r = detail::finish_region<N>(rs, T, jac, 0);
      avg[i] = r.avg;
      err[i] = r.err;
      axis[i] = r.axis;
      active[i] = (r.err / detail::max_err(r.avg, epsrel, epsabs)) > 1;
    }
  }
}

// Split, pass 1: active count per 32-region chunk.
static __global__ void k_step_count(long long n, const int* active, int* cnt) {
  const int lane = threadIdx.x & 31;
  const long long nchunk = (n + 31) / 32;
  for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; c < nchunk;
       c += (long long)gridDim.x * blockDim.x / 32) {
    const long long i = c * 32 + lane;
    const unsigned b = __ballot_sync(0xffffffffu, i < n && active[i] == 1);
    if (lane == 0) cnt[c] = __popc(b);
  }
}

// Split, pass 2: exclusive scan of the chunk counts (one block); writes the
// child count 2m.
static __global__ void __launch_bounds__(1024) k_step_scan(long long nchunk, const int* cnt, int* excl,
                                                    long long* count_out) {
  __shared__ long long wsum[32];
  __shared__ long long carry;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (long long base = 0; base < nchunk; base += 1024) {
    const long long c = base + tid;
    const long long v = c < nchunk ? cnt[c] : 0;
    long long incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      long long w = wsum[lane];
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, w, off);
        if (lane >= off) w += t;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const long long wb = wid > 0 ? wsum[wid - 1] : 0;
    if (c < nchunk) excl[c] = (int)(carry + wb + incl - v);
    __syncthreads();
    if (tid == 0) carry += wsum[31];
    __syncthreads();
  }
  if (tid == 0) *count_out = 2 * carry;
}

// Split, pass 3: write the children (alignRegions + divideIntervalsGPU,
// GPUKernelquad.cu:63-149).
template <int N>
__global__ void k_step_write(long long n, const double* lo, const double* len, long long ld,
                             const int* active, const int* axis, const int* excl,
                             const long long* count, double* olo, double* olen, long long old,
                             int layout) {
  const int lane = threadIdx.x & 31;
  const long long nchunk = (n + 31) / 32;
  const long long m = *count / 2;
  for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; c < nchunk;
       c += (long long)gridDim.x * blockDim.x / 32) {
    const long long i = c * 32 + lane;
    const bool act = i < n && active[i] == 1;
    const unsigned b = __ballot_sync(0xffffffffu, act);
    if (!act) continue;
    const long long j = excl[c] + __popc(b & ((1u << lane) - 1u));
    const long long d0 = layout == 0 ? j : 2 * j;
    const long long d1 = layout == 0 ? m + j : 2 * j + 1;
    const int ax = axis[i];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const double l = lo[(long long)d * ld + i], w = len[(long long)d * ld + i];
      const double h = w / 2;
      olo[(long long)d * old + d0] = l;
      olo[(long long)d * old + d1] = d == ax ? l + 1 * h : l;
      olen[(long long)d * old + d0] = d == ax ? h : w;
      olen[(long long)d * old + d1] = d == ax ? h : w;
    }
  }
}

// Reduction, pass 1: per-block partial sums (fixed grid, fixed order).
constexpr int kReduceBlocks = 1024;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

static __global__ void __launch_bounds__(256) k_step_reduce(long long n, const double* avg,
                                                     const double* err, const int* active,
                                                     double* part) {
  __shared__ double sm[8][4];
  double s[4] = {0, 0, 0, 0};
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = avg[i], e = err[i];
    s[0] += a;
    s[1] += e;
    if (active[i] != 1) {
      s[2] += a;
      s[3] += e;
    }
  }
  for (int q = 0; q < 4; ++q) s[q] = warp_sum(s[q]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0)
    for (int q = 0; q < 4; ++q) sm[wid][q] = s[q];
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0;
    for (int w = 0; w < 8; ++w) t += sm[w][threadIdx.x];
    part[blockIdx.x * 4 + threadIdx.x] = t;
  }
}

// Reduction, pass 2: one warp sums the block partials in a fixed order.
static __global__ void k_step_reduce_final(int nblocks, const double* part, double* out) {
  const int lane = threadIdx.x;
  double s[4] = {0, 0, 0, 0};
  for (int b = lane; b < nblocks; b += 32)
    for (int q = 0; q < 4; ++q) s[q] += part[b * 4 + q];
  for (int q = 0; q < 4; ++q) s[q] = warp_sum(s[q]);
  if (lane == 0)
    for (int q = 0; q < 4; ++q) out[q] = s[q];
}

}  // namespace cubature
