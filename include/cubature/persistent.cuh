// persistent.cuh -- the breadth-first loop as one persistent cooperative
// kernel, for region lists small enough that launch latency and host
// round trips would dominate (the reference pays ~10 cudaMalloc/cudaFree,
// four thrust reductions and two blocking copies per iteration,
// GPUKernelquad.cu:357-605).
//
// One launch runs iterations until no integral is running or the list
// grows past the kernel's range (the multi-launch driver takes over) or
// past the buffers (the host grows them and relaunches).  Per iteration:
//
//   eval   regions are evaluated by a block each (tiny lists) or a warp
//          each; the group that completes a 32-region chunk sums it, the
//          warp that completes an integral's last chunk takes its stop
//          decision, and the warp that decides the last integral assigns
//          the next segments -- "last arriver" atomics, no barrier;
//   grid barrier;
//   split  children written, segments handed over;
//   grid barrier.
//
// The grid barrier is a generation counter with a bounded spin: after
// ~4 s without progress it records a timeout and every block returns.
// All blocks are co-resident (cooperative launch).
#pragma once

#include "engine_kernels.cuh"

namespace cubature {

struct PersistArgs {
  EngineArgs base;       // lists of both buffers are rebound per iteration
  double* lo[2];
  double* len[2];
  int* rid[2];
  int max_n;             // leave when the list is longer than this
  int block_mode_max_n;  // block-per-region evaluation up to this length
};

namespace detail {

constexpr long long kBarrierSpins = 1ll << 25;  // x ~128 ns sleep: ~4 s

// Grid-wide barrier with a bounded wait.  Returns false once any block
// gave up waiting (all blocks then return).
__device__ __forceinline__ bool grid_barrier(Control* ctl, unsigned nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &ctl->bar_gen;
    const unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(&ctl->bar_count, 1u) == nblocks - 1) {
      atomicExch(&ctl->bar_count, 0u);
      __threadfence();
      atomicAdd(&ctl->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*vgen == g) {
        if (++spins > kBarrierSpins || *(volatile int*)&ctl->timeout) {
          atomicExch(&ctl->timeout, 1);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
    ok = *(volatile int*)&ctl->timeout == 0;
  }
  __syncthreads();
  return ok;
}

// Points of the rule, for evaluation with one thread per point: a 32-bit
// descriptor per point of sets 0..7 (set | d1<<4 | d2<<8 | d3<<12 |
// signs<<16), same order as the oracle's enumeration; the 2^N points of
// set 8 follow, their index is the sign pattern.
template <int N>
struct PointTable {
  static constexpr int kNonCube = 1 + 8 * N + 6 * N * (N - 1) + 4 * N * (N - 1) * (N - 2) / 3;
  static constexpr int kPoints = kNonCube + (1 << N);
  uint32_t desc[kNonCube];

  __device__ void fill() {
    int p = 0;
    desc[p++] = 0;
    for (int s = 1; s <= 4; ++s)
      for (int d = 0; d < N; ++d)
        for (int sg = 0; sg < 2; ++sg) desc[p++] = s | (d << 4) | (sg << 16);
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = d1 + 1; d2 < N; ++d2)
        for (int sg = 0; sg < 4; ++sg) desc[p++] = 5 | (d1 << 4) | (d2 << 8) | (sg << 16);
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = 0; d2 < N; ++d2)
        if (d2 != d1)
          for (int sg = 0; sg < 4; ++sg) desc[p++] = 6 | (d1 << 4) | (d2 << 8) | (sg << 16);
    for (int d1 = 0; d1 < N; ++d1)
      for (int d2 = d1 + 1; d2 < N; ++d2)
        for (int d3 = d2 + 1; d3 < N; ++d3)
          for (int sg = 0; sg < 8; ++sg)
            desc[p++] = 7 | (d1 << 4) | (d2 << 8) | (d3 << 12) | (sg << 16);
  }
};

template <int N>
__device__ __forceinline__ void point_coords(const PointTable<N>& pt, int p, const double (&L)[N],
                                             const double (&H)[N], const double (&C)[N],
                                             double (&x)[N], int& set) {
  if (p >= PointTable<N>::kNonCube) {
    const int s = p - PointTable<N>::kNonCube;
    set = 8;
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = fma(coef(kGenL, (s >> i) & 1), H[i], L[i]);
    return;
  }
  const uint32_t dsc = pt.desc[p];
  set = dsc & 15;
  const int d1 = (dsc >> 4) & 15, d2 = (dsc >> 8) & 15, d3 = (dsc >> 12) & 15;
  const int sg = dsc >> 16;
  const int nz = set == 0 ? 0 : (set <= 4 ? 1 : (set <= 6 ? 2 : 3));
  const double g1 = set == 2 ? kGenA2 : (set == 3 ? kGenA3 : (set == 4 ? kGenA4 : kGenA1));
  const double g2 = set == 6 ? kGenA2 : kGenA1;
  const double v1 = fma(coef(g1, sg & 1), pick(H, d1), pick(L, d1));
  const double v2 = fma(coef(g2, sg & 2), pick(H, d2), pick(L, d2));
  const double v3 = fma(coef(kGenA1, sg & 4), pick(H, d3), pick(L, d3));
#pragma unroll
  for (int i = 0; i < N; ++i)
    x[i] = (nz >= 1 && i == d1) ? v1
           : (nz >= 2 && i == d2) ? v2
           : (nz >= 3 && i == d3) ? v3
                                  : C[i];
}

template <int N>
struct BlockEvalSmem {
  PointTable<N> pt;
  double red[8][kNumSets];
  double fstage[4 * N + 1];
};

// One region evaluated by a whole 256-thread block, one point per thread
// per round.  Thread 0 returns the result.  All threads must call it.
template <int N, class F>
__device__ __forceinline__ RegionResult eval_region_block(const F& f, const double (&L)[N],
                                                          const double (&H)[N], const RuleTables& T,
                                                          BlockEvalSmem<N>& sm) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double C[N];
#pragma unroll
  for (int i = 0; i < N; ++i) C[i] = fma(0.5, H[i], L[i]);
  double S[kNumSets];
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) S[k] = 0;
  // points are sorted by set, so a thread's sets never decrease: keep one
  // running sum and flush it into S[set] when the set changes
  double acc = 0;
  int cur = 0;
  for (int p = tid; p < PointTable<N>::kPoints; p += 256) {
    double x[N];
    int set;
    point_coords<N>(sm.pt, p, L, H, C, x, set);
    const double fx = f(x);
    if (p <= 4 * N) sm.fstage[p] = fx;
    if (set != cur) {
#pragma unroll
      for (int k = 0; k < kNumSets; ++k)
        if (k == cur) S[k] += acc;
      acc = 0;
      cur = set;
    }
    acc += fx;
  }
#pragma unroll
  for (int k = 0; k < kNumSets; ++k)
    if (k == cur) S[k] += acc;
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) {
    double v = S[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if (lane == 0) sm.red[wid][k] = v;
  }
  __syncthreads();
  RegionResult r;
  r.avg = r.err = 0;
  r.axis = 0;
  if (wid == 0) {
    RegionSums rs;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) {
      double v = 0;
      for (int w = 0; w < 8; ++w) v += sm.red[w][k];
      rs.S[k] = v;
    }
    // fourth difference per axis from the staged centre and set-1/2 values
    rs.best = 0;
    rs.axis = -1;
    if (lane < N) {
      const double ratio = T.ratio;
      const double base = __dmul_rn(__dmul_rn(sm.fstage[0], 2.0), __dadd_rn(1.0, -ratio));
      const int d = lane;
      rs.best = fabs(__dadd_rn(
          __dadd_rn(base, __dmul_rn(ratio, __dadd_rn(sm.fstage[1 + 2 * d], sm.fstage[2 + 2 * d]))),
          -__dadd_rn(sm.fstage[1 + 2 * N + 2 * d], sm.fstage[2 + 2 * N + 2 * d])));
      rs.axis = rs.best > 0 ? d : -1;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, rs.best, off);
      const int oa = __shfl_xor_sync(0xffffffffu, rs.axis, off);
      const bool take = (ob > rs.best) || (ob == rs.best && oa >= 0 && (rs.axis < 0 || oa < rs.axis));
      if (take) {
        rs.best = ob;
        rs.axis = oa;
      }
    }
    if (lane == 0) {
      double jac = 1;
#pragma unroll
      for (int d = 0; d < N; ++d) jac = __dmul_rn(jac, H[d]);
      r = finish_region<N>(rs, T, jac, 0);
    }
  }
  __syncthreads();
  return r;
}

// Run by the warp that completed chunk c: sum the chunk; if it completed
// its integral, decide it; if that was the last integral, run the scan.
__device__ __forceinline__ void after_chunk_warp(const EngineArgs& a, long long c, int lane,
                                                 const IterState& st, IterState* next) {
  __threadfence();
  chunk_partial_warp(a, c, lane);
  const int k = a.rid[c * 32];
  unsigned last = 0;
  if (lane == 0) {
    a.chunk_cnt[c] = 0;
    __threadfence();
    const unsigned nc = (unsigned)((a.ist[k].seg_count + 31) / 32);
    last = atomicAdd(&a.int_cnt[k], 1u) == nc - 1;
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __threadfence();
  if (lane == 0) a.int_cnt[k] = 0;
  decide_warp(a, k, lane);
  __threadfence();
  unsigned all = 0;
  if (lane == 0) all = atomicAdd(&a.ctl->done_cnt, 1u) == (unsigned)st.n_running - 1;
  all = __shfl_sync(0xffffffffu, all, 0);
  if (!all) return;
  __threadfence();
  if (lane == 0) a.ctl->done_cnt = 0;
  scan_warp(a, st.n_left, next, lane);
  __threadfence();
}

}  // namespace detail

template <int N, class Src>
__global__ void __launch_bounds__(256) k_persistent(Src src, RuleTables T, PersistArgs p) {
  __shared__ detail::ItemTable<N> tab;
  __shared__ detail::BlockEvalSmem<N> bsm;
  __shared__ int flag;
  if (threadIdx.x == 0) {
    tab.fill();
    bsm.pt.fill();
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  Control* ctl = p.base.ctl;
  int cur = ctl->cur;
  int parity = 0;
  int reason = kExitDone;
  for (;;) {
    IterState st;
    {
      volatile IterState* v = &ctl->it[parity];
      st.n = v->n;
      st.n_running = v->n_running;
      st.n_left = v->n_left;
      st.overflow = v->overflow;
    }
    EngineArgs a = p.base;
    if (st.n_running == 0 || st.n == 0) {
      reason = kExitDone;
      break;
    }
    if (st.n > p.max_n) {
      reason = kExitLarge;
      break;
    }
    if (2ll * st.n + 32ll * a.nint > a.ncap ||
        (a.policy == kPolicyReference && (long long)st.n_left + 2ll * st.n > a.left_cap)) {
      reason = kExitCapacity;
      break;
    }
    a.lo = p.lo[cur];
    a.len = p.len[cur];
    a.rid = p.rid[cur];
    a.nlo = p.lo[cur ^ 1];
    a.nlen = p.len[cur ^ 1];
    a.nrid = p.rid[cur ^ 1];
    a.n = st.n;
    IterState* next = &ctl->it[parity ^ 1];

    if (st.n <= p.block_mode_max_n) {
      // one region per block
      for (long long slot = blockIdx.x; slot < st.n; slot += gridDim.x) {
        const int k = a.rid[slot];
        if (k >= 0) {
          double L[N], H[N];
#pragma unroll
          for (int d = 0; d < N; ++d) {
            L[d] = a.lo[(long long)d * a.cap + slot];
            H[d] = a.len[(long long)d * a.cap + slot];
          }
          const auto f = src.get(k);
          const detail::RegionResult r = detail::eval_region_block<N>(f, L, H, T, bsm);
          if (threadIdx.x == 0) detail::store_result(a, slot, r, a.ist[k]);
        } else if (threadIdx.x == 0) {
          detail::store_padding(a, slot);
        }
        if (threadIdx.x == 0) {
          __threadfence();
          flag = atomicAdd(&a.chunk_cnt[slot / 32], 1u) == 31;
        }
        __syncthreads();
        if (flag && threadIdx.x < 32) detail::after_chunk_warp(a, slot / 32, lane, st, next);
        __syncthreads();
      }
    } else {
      // one region per warp
      for (long long slot = gwarp; slot < st.n; slot += nwarp) {
        detail::eval_slot<N, 32>(src, T, a, slot, lane, 0xffffffffu, tab);
        unsigned last = 0;
        if (lane == 0) {
          __threadfence();
          last = atomicAdd(&a.chunk_cnt[slot / 32], 1u) == 31;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) detail::after_chunk_warp(a, slot / 32, lane, st, next);
      }
    }
    if (!detail::grid_barrier(ctl, gridDim.x)) {
      reason = kExitTimeout;
      break;
    }
    const long long nchunk = (st.n + 31) / 32;
    for (long long c = gwarp; c < nchunk; c += nwarp) detail::split_chunk_warp<N>(a, c, lane);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nint; k += gridDim.x * blockDim.x)
      detail::finish_integral(a, k);
    if (!detail::grid_barrier(ctl, gridDim.x)) {
      reason = kExitTimeout;
      break;
    }
    cur ^= 1;
    parity ^= 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->iters_done += 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctl->cur = cur;
    volatile IterState* v = &ctl->it[parity];
    ctl->host.n = v->n;
    ctl->host.n_running = v->n_running;
    ctl->host.n_left = v->n_left;
    ctl->host.overflow = 0;
    ctl->exit_reason = reason;
  }
}

}  // namespace cubature
