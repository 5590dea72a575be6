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
//   eval   each region is evaluated by a group of G = 256/R threads, one
//          rule point per thread per round (R = 1, 2, 4 or 8 regions per
//          block, the smallest R that covers the list in one pass);
//          consecutive regions go to different SMs.  The group that
//          completes a 32-region chunk sums it, the warp that completes an
//          integral's last chunk takes its stop decision, and the warp that
//          decides the last integral assigns the next segments -- "last
//          arriver" atomics, no barrier;
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
  EngineArgs base;  // lists of both buffers are rebound per iteration
  double* lo[2];
  double* len[2];
  int* rid[2];
  int max_n;        // leave when the list is longer than this
  int max_r;        // most regions a block evaluates at once (1, 2, 4 or 8)
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
        __nanosleep(64);
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
// signs<<16), in the oracle's enumeration order; the 2^N points of set 8
// follow, their index is the sign pattern.
template <int N>
struct PointTable {
  static constexpr int kNonCube = 1 + 8 * N + 6 * N * (N - 1) + 4 * N * (N - 1) * (N - 2) / 3;
  static constexpr int kPoints = kNonCube + (1 << N);
  uint32_t desc[kNonCube];

  // Descriptor of point p, decoded from its index.
  __host__ __device__ static uint32_t decode(int p) {
    if (p == 0) return 0;
    int q = p - 1;
    if (q < 8 * N) {  // sets 1..4: 2N points each, axis-major, + then -
      const int s = 1 + q / (2 * N), r = q % (2 * N);
      return s | ((r >> 1) << 4) | ((r & 1) << 16);
    }
    q -= 8 * N;
    const int npair = N * (N - 1) / 2;
    if (q < 4 * npair) {  // set 5: pairs d1 < d2, 4 sign patterns each
      int t = q >> 2;
      const int sg = q & 3;
      int d1 = 0;
      while (t >= N - 1 - d1) {
        t -= N - 1 - d1;
        ++d1;
      }
      return 5 | (d1 << 4) | ((d1 + 1 + t) << 8) | (sg << 16);
    }
    q -= 4 * npair;
    const int nord = N * (N - 1);
    if (q < 4 * nord) {  // set 6: ordered pairs d1 != d2
      const int t = q >> 2, sg = q & 3;
      const int d1 = t / (N - 1);
      int d2 = t % (N - 1);
      if (d2 >= d1) ++d2;
      return 6 | (d1 << 4) | (d2 << 8) | (sg << 16);
    }
    q -= 4 * nord;  // set 7: triples d1 < d2 < d3, 8 sign patterns each
    int t = q >> 3;
    const int sg = q & 7;
    int d1 = 0;
    for (;;) {
      const int m = N - 1 - d1, c = m * (m - 1) / 2;
      if (t < c) break;
      t -= c;
      ++d1;
    }
    int d2 = d1 + 1;
    for (;;) {
      const int c = N - 1 - d2;
      if (t < c) break;
      t -= c;
      ++d2;
    }
    return 7 | (d1 << 4) | (d2 << 8) | ((d2 + 1 + t) << 12) | (sg << 16);
  }

  __device__ void fill(int tid, int nthreads) {
    for (int p = tid; p < kNonCube; p += nthreads) desc[p] = decode(p);
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
struct GroupSmem {
  PointTable<N> pt;
  double red[8][kNumSets];      // one row per warp of the block
  double fstage[8][4 * N + 1];  // centre and set-1/2 values, per group
  int flag[8];
};

// Barrier for the groups of a block.  All groups of a block step through
// their slots in lockstep (eval_step), so a block-wide barrier serves every
// group size and no named barriers are needed.
template <int G>
__device__ __forceinline__ void group_sync(int) {
  __syncthreads();
}

// One region evaluated by the G threads of group g, one point per thread
// per round.  Thread 0 of the group returns the result.  Every thread of
// the block must call it (it contains block barriers); groups with
// active == false evaluate nothing.
template <int N, int G, class F>
__device__ __forceinline__ RegionResult eval_region_group(const F& f, const double (&L)[N],
                                                          const double (&H)[N], const RuleTables& T,
                                                          GroupSmem<N>& sm, int g, int t,
                                                          bool active) {
  constexpr int W = G / 32;
  const int lane = t & 31, wid = threadIdx.x >> 5;
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
  for (int p = active ? t : PointTable<N>::kPoints; p < PointTable<N>::kPoints; p += G) {
    double x[N];
    int set;
    point_coords<N>(sm.pt, p, L, H, C, x, set);
    const double fx = f(x);
    if (p <= 4 * N) sm.fstage[g][p] = fx;
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
    S[k] = v;
    if (W > 1 && lane == 0) sm.red[wid][k] = v;
  }
  group_sync<G>(g);
  RegionResult r;
  r.avg = r.err = 0;
  r.axis = 0;
  if (t < 32) {
    RegionSums rs;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) {
      if (W > 1) {
        double v = 0;
        for (int w = 0; w < W; ++w) v += sm.red[wid + w][k];
        rs.S[k] = v;
      } else {
        rs.S[k] = S[k];
      }
    }
    // fourth difference per axis from the staged centre and set-1/2 values
    rs.best = 0;
    rs.axis = -1;
    if (lane < N) {
      const double* fs = sm.fstage[g];
      const double ratio = T.ratio;
      const double base = __dmul_rn(__dmul_rn(fs[0], 2.0), __dadd_rn(1.0, -ratio));
      const int d = lane;
      rs.best = fabs(__dadd_rn(__dadd_rn(base, __dmul_rn(ratio, __dadd_rn(fs[1 + 2 * d], fs[2 + 2 * d]))),
                               -__dadd_rn(fs[1 + 2 * N + 2 * d], fs[2 + 2 * N + 2 * d])));
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
  group_sync<G>(g);
  return r;
}

// atomicAdd with acquire-release semantics at GPU scope: publishes the
// calling thread's earlier writes and, for the last arriver, makes every
// earlier arriver's writes visible -- cheaper than fence + add + fence.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Run by the warp that completed chunk c.  Small batches (few integrals):
// sum the chunk; the warp that completes the last chunk of the list
// decides every integral and runs the scan.  Large batches: the warp that
// completes an integral's last chunk decides it, the one that decides the
// last integral runs the scan.
__device__ __forceinline__ void after_chunk_warp(const EngineArgs& a, long long c, int lane,
                                                 const IterState& st, IterState* next, int it) {
  __syncwarp();
  chunk_partial_warp(a, c, lane);
  if (a.nint <= 32) {
    unsigned last = 0;
    if (lane == 0) {
      a.chunk_cnt[c] = 0;
      last = atom_add_acq_rel(&a.ctl->done_cnt, 1u) == (unsigned)(st.n / 32) - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __syncwarp();
    if (lane == 0) {
      a.ctl->done_cnt = 0;
      trace_mark(a.ctl, it, 5);
    }
    for (int k = 0; k < a.nint; ++k) {
      decide_warp(a, k, lane);
      __syncwarp();
    }
    if (lane == 0) trace_mark(a.ctl, it, 6);
    scan_warp(a, st.n_left, next, lane);
    __threadfence();
    if (lane == 0) trace_mark(a.ctl, it, 1);
    return;
  }
  __threadfence();
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
  if (lane == 0) trace_mark(a.ctl, it, 1);
}

// The eval step with groups of G threads (R = 256/G regions per block).
// The slots of round `base` are base + g * gridDim.x + blockIdx.x: group
// index interleaved over blocks, so consecutive regions land on different
// SMs.  Every group of a block runs the same number of rounds (groups past
// the end of the list idle through the block barriers).
template <int N, int G, class Src>
__device__ __forceinline__ void eval_step(const Src& src, const RuleTables& T, const EngineArgs& a,
                                          const IterState& st, IterState* next, GroupSmem<N>& sm,
                                          int it) {
  constexpr int R = 256 / G;
  const int g = threadIdx.x / G, t = threadIdx.x % G, lane = threadIdx.x & 31;
  const long long ngroups = (long long)R * gridDim.x;
  for (long long base = 0; base < st.n; base += ngroups) {
    const long long slot = base + (long long)g * gridDim.x + blockIdx.x;
    const bool live = slot < st.n;
    const int k = live ? a.rid[slot] : -1;
    {
      double L[N], H[N];
#pragma unroll
      for (int d = 0; d < N; ++d) {
        L[d] = k >= 0 ? a.lo[(long long)d * a.cap + slot] : 0.0;
        H[d] = k >= 0 ? a.len[(long long)d * a.cap + slot] : 1.0;
      }
      // groups without a region evaluate no point but join the barriers
      const auto f = src.get(k >= 0 ? k : 0);
      const RegionResult r = eval_region_group<N, G>(f, L, H, T, sm, g, t, k >= 0);
      if (t == 0 && k >= 0) store_result(a, slot, r, a.ist[k]);
    }
    if (t == 0 && live) {
      if (k < 0) store_padding(a, slot);
      sm.flag[g] = atom_add_acq_rel(&a.chunk_cnt[slot / 32], 1u) == 31;
    } else if (t == 0) {
      sm.flag[g] = 0;
    }
    __syncthreads();
    if (t < 32 && sm.flag[g]) after_chunk_warp(a, slot / 32, lane, st, next, it);
    __syncthreads();
  }
}

}  // namespace detail

template <int N, class Src>
__global__ void __launch_bounds__(256, 2) k_persistent(Src src, RuleTables T, PersistArgs p) {
  __shared__ detail::GroupSmem<N> sm;
  sm.pt.fill(threadIdx.x, blockDim.x);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  Control* ctl = p.base.ctl;
  int cur = ctl->cur;
  int parity = 0;
  int reason = kExitDone;
  const bool tracer = blockIdx.x == 0 && threadIdx.x == 0;
  for (int it = 0;; ++it) {
    if (tracer) trace_mark(ctl, it, 0);
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

    // smallest R (regions per block) that covers the list in one pass
    const long long per_block = (st.n + gridDim.x - 1) / gridDim.x;
    const int r = per_block <= 1 ? 1 : (per_block <= 2 ? 2 : (per_block <= 4 ? 4 : 8));
    switch (r < p.max_r ? r : p.max_r) {
      case 1: detail::eval_step<N, 256>(src, T, a, st, next, sm, it); break;
      case 2: detail::eval_step<N, 128>(src, T, a, st, next, sm, it); break;
      case 4: detail::eval_step<N, 64>(src, T, a, st, next, sm, it); break;
      default: detail::eval_step<N, 32>(src, T, a, st, next, sm, it); break;
    }
    if (tracer) trace_mark(ctl, it, 4);
    if (!detail::grid_barrier(ctl, gridDim.x)) {
      reason = kExitTimeout;
      break;
    }
    if (tracer) trace_mark(ctl, it, 2);
    const long long nchunk = (st.n + 31) / 32;
    for (long long c = gwarp; c < nchunk; c += nwarp) detail::split_chunk_warp<N>(a, c, lane);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nint; k += gridDim.x * blockDim.x)
      detail::finish_integral(a, k);
    if (!detail::grid_barrier(ctl, gridDim.x)) {
      reason = kExitTimeout;
      break;
    }
    if (tracer) trace_mark(ctl, it, 3);
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
