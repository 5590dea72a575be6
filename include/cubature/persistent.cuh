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
//          consecutive regions go to different SMs.  From the second
//          iteration of a launch on, no split step writes the list: the
//          group that evaluates slot s finds the parent region of s (the
//          region of rank s / 2 among the active regions of the previous
//          list, from per-chunk active masks and prefix counts), bisects
//          it and writes the child into the list itself;
//   chain  the group that completes a 32-region chunk sums it; small
//          batches: the warp that completes the last chunk decides every
//          integral and assigns the next segments; large batches: the warp
//          that completes an integral's last chunk decides it and the one
//          that decides the last integral assigns the segments -- "last
//          arriver" atomics, no barrier;
//   grid barrier (one per iteration).
//
// Leftover boxes of integrals handed to phase 2 are written at the start of
// the next iteration by all blocks.  Before the kernel returns it writes the
// pending list in full, so the host and the multi-launch driver always find
// a complete list.  The grid barrier is a monotonic counter with a bounded
// spin: after a few seconds without progress it records a timeout and every
// block returns.  All blocks are co-resident (cooperative launch).
#pragma once

#include "engine_kernels.cuh"

namespace cubature {

// Chunks of a list the persistent kernel stages in shared memory; the host
// hands lists longer than 32 * kStageChunks to the multi-launch driver.
constexpr int kStageChunks = 640;
// Batches up to this many integrals decide in one warp, one lane each.
constexpr int kSmallBatch = 32;

struct PersistArgs {
  EngineArgs base;     // lists and per-slot outputs are rebound per iteration
  double* lo[2];
  double* len[2];
  int* rid[2];
  int* axis[2];        // split axes, by iteration parity
  unsigned* cmask[2];  // active bit mask per chunk, by iteration parity
  int* excl[2];        // active regions before each chunk of its integral, by parity
  int* chunk_int;      // integral owning each chunk of the coming list (large batches)
  int max_n;           // leave when the list is longer than this
  int max_r;           // most regions a block evaluates at once (1, 2, 4 or 8)
  int iter_base;       // global index of the launch's first iteration
  // init != 0: the current list is the initial grid, not yet written; the
  // first iteration computes each slot's box (initial_box) and writes it
  int init;
  int divisions, per_integral, padded;
  const double* box;
  // When set (mapped pinned memory): at exit block 0 also stores the
  // control block and the integral states, host_words 8-byte words, there,
  // and the host needs no copy back.
  Control* host_out;
  int host_words;
  long long spin_limit;  // grid-barrier polls before giving up
  int hold_block;        // failure-detection tests: this block never arrives (-1: none)
};

// How the first step of an iteration obtains a slot's region.
enum SlotSource : int {
  kSlotStored = 0,  // read from the current list
  kSlotLazy = 1,    // bisect the parent in the previous list
  kSlotGrid = 2,    // compute the initial-grid box
};

namespace detail {

constexpr long long kBarrierSpins = 1ll << 23;  // x ~0.5 us per poll: a few seconds

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier on a monotonic arrival counter: the b-th barrier of a
// launch (b = 1, 2, ...) waits for b * gridDim.x arrivals.  Bounded wait
// (spin_limit polls); returns false when this block gave up waiting or saw
// that another block did (every block then returns: a block that passed
// this barrier meets the next one without the one that gave up).  A block
// with arrive == false waits without
// arriving: the failure-detection tests use it to make every wait run out.
// Ordering needs no separate fences: the block's writes precede thread 0's
// gpu-scope release through the CTA barrier, the release and acquire
// operations are cumulative, and the closing CTA barrier orders the
// block's later reads after thread 0's acquire.
// Only the arrival counter is read on the way through: the shared timeout
// flag is read every 64th poll, so a block that gave up is noticed within
// 64 polls (at the latest at the next barrier, which it does not reach),
// and a passing wait costs one acquire load after the last arrival.
__device__ __forceinline__ bool grid_barrier(Control* ctl, unsigned target, long long spin_limit,
                                             bool arrive) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (arrive) red_release_add(&ctl->bar_count, 1u);
    long long spins = 0;
    int good = 1;
    while (ld_acquire(&ctl->bar_count) < target) {
      if ((++spins & 63) == 0 && (spins > spin_limit || *(volatile int*)&ctl->timeout)) {
        atomicExch(&ctl->timeout, 1);
        good = 0;
        break;
      }
      __nanosleep(32);
    }
    ok = good;
  }
  __syncthreads();
  return ok;
}

// Points of the rule, for evaluation with one thread per point, in the
// oracle's enumeration order: sets 0..7 (decoded from the point index) then
// the 2^N points of set 8 (index = sign pattern).  Each point is stored as
// N 4-bit coefficient codes, so that its coordinates are
// x_i = fma(ctab[code_i], H_i, L_i) -- the same arithmetic as the
// structured evaluator: code 0 is the box centre (0.5), codes 1..10 are
// 0.5 -/+ g for the generators a1, a2, a3, a4 and the corner value.
template <int N>
struct PointTable {
  static constexpr int kNonCube = 1 + 8 * N + 6 * N * (N - 1) + 4 * N * (N - 1) * (N - 2) / 3;
  static constexpr int kPoints = kNonCube + (1 << N);
  static_assert(N <= 8, "4-bit codes of N axes must fit 32 bits");
  uint2 ent[kPoints];  // x: codes (axis i at bits 4i..4i+3), y: generator set
  double ctab[16];

  // Descriptor of non-corner point p decoded from its index:
  // set | d1<<4 | d2<<8 | d3<<12 | signs<<16.
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

  // Code of generator gi (0..3: a1..a4, 4: corner value) with sign `minus`.
  __host__ __device__ static uint32_t code(int gi, bool minus) {
    return 1u + 2u * (uint32_t)gi + (minus ? 1u : 0u);
  }

  // Codes and set of point p.
  __host__ __device__ static uint2 entry(int p) {
    uint32_t codes = 0;
    if (p >= kNonCube) {
      const int s = p - kNonCube;
      for (int i = 0; i < N; ++i) codes |= code(4, (s >> i) & 1) << (4 * i);
      return make_uint2(codes, 8u);
    }
    const uint32_t dsc = decode(p);
    const int set = dsc & 15;
    const int d1 = (dsc >> 4) & 15, d2 = (dsc >> 8) & 15, d3 = (dsc >> 12) & 15;
    const int sg = dsc >> 16;
    const int nz = set == 0 ? 0 : (set <= 4 ? 1 : (set <= 6 ? 2 : 3));
    const int g1 = set == 2 ? 1 : (set == 3 ? 2 : (set == 4 ? 3 : 0));
    const int g2 = set == 6 ? 1 : 0;
    if (nz >= 1) codes |= code(g1, sg & 1) << (4 * d1);
    if (nz >= 2) codes |= code(g2, sg & 2) << (4 * d2);
    if (nz >= 3) codes |= code(0, sg & 4) << (4 * d3);
    return make_uint2(codes, (uint32_t)set);
  }

  __device__ void fill(int tid, int nthreads) {
    if (tid < 16) {
      const double gen[5] = {kGenA1, kGenA2, kGenA3, kGenA4, kGenL};
      ctab[tid] = tid == 0 ? 0.5 : (tid <= 10 ? coef(gen[(tid - 1) >> 1], (tid - 1) & 1) : 0.0);
    }
    for (int p = tid; p < kPoints; p += nthreads) ent[p] = entry(p);
  }
};

// f(x, p) for functors that take the rule point's index (values computed
// ahead of the rule, e.g. the control-variate network), else f(x).
template <class F>
__device__ __forceinline__ auto call_point_(const F& f, const double* x, int p, int)
    -> decltype(f(x, p)) {
  return f(x, p);
}
template <class F>
__device__ __forceinline__ double call_point_(const F& f, const double* x, int, long) {
  return f(x);
}
template <class F>
__device__ __forceinline__ double call_point(const F& f, const double* x, int p) {
  return call_point_(f, x, p, 0);
}

// Two rule points in flight per thread, except for functors that carry
// several families' code (the unrolled loop would not fit the registers).
template <class F>
constexpr bool kTwoPointsInFlight = true;
template <int M>
constexpr bool kTwoPointsInFlight<MixedGenz<M>> = false;

template <int N>
struct GroupSmem {
  PointTable<N> pt;
  RuleTables tables;  // stage_tables copy of the kernel's tables
  double red[8][kNumSets];      // one row per warp of the block
  double fstage[8][4 * N + 1];  // centre and set-1/2 values, per group
  int flag[8];
  int owner[8];
};

// The set sums of the G threads of a group (S, per thread) combined into
// the region's result: warp shuffle trees, then the warps' partials in
// warp order; the fourth difference per axis from the staged centre and
// set-1/2 values (fst); value, error and split axis (finish_region's
// arithmetic, spread over five lanes).
// Thread 0 of the group returns the result.  Every thread of the block must
// call it (block barriers).
// The nine shuffle trees run level by level, so their latencies overlap;
// each set's tree adds in the same order as on its own.
template <int N, int G>
__device__ __forceinline__ RegionResult group_finish(double (&S)[kNumSets], const double (&H)[N],
                                                     const RuleTables& T,
                                                     double (&red)[8][kNumSets], const double* fst,
                                                     int t) {
  constexpr int W = G / 32;
  const int lane = t & 31, wid = threadIdx.x >> 5;
  // the Jacobian (box volume, axis order) before the barrier
  double jac = 1;
#pragma unroll
  for (int d = 0; d < N; ++d) jac = __dmul_rn(jac, H[d]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) S[k] += __shfl_xor_sync(0xffffffffu, S[k], off);
  }
  if (W > 1 && lane == 0) {
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) red[wid][k] = S[k];
  }
  __syncthreads();
  RegionResult r;
  r.avg = r.err = 0;
  r.axis = 0;
  if (t < 32) {
    RegionSums rs;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) {
      if (W > 1) {
        double v = 0;
        for (int w = 0; w < W; ++w) v += red[wid + w][k];
        rs.S[k] = v;
      } else {
        rs.S[k] = S[k];
      }
    }
    // fourth difference per axis from the staged centre and set-1/2 values
    rs.best = 0;
    rs.axis = -1;
    if (lane < N) {
      const double* fs = fst;
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
    // Value and error on five lanes: lane q forms rule q's sum, lanes 1-3
    // the null-rule errors, each with finish_region's arithmetic for its
    // rule (same operations, same order, so the same bits).  T is read by
    // lane index, so it must be a shared-memory copy (stage_tables).
    double sq = 0;
    if (lane < kNumRules) {
      double acc = 0;
#pragma unroll
      for (int k = 0; k < kNumSets; ++k) acc = __dadd_rn(acc, __dmul_rn(T.wt[k][lane], rs.S[k]));
      sq = __dmul_rn(acc, jac);
    }
    const double sq1 = __shfl_down_sync(0xffffffffu, sq, 1);
    double nq = 0;
    if (lane >= 1 && lane < kNumRules - 1) {
      double m = 0;
#pragma unroll
      for (int k = 0; k < kNumSets; ++k) {
        const double e =
            __dmul_rn(fabs(__dadd_rn(sq1, __dmul_rn(T.scale[k][lane], sq))), T.norm[k][lane]);
        m = (m > e) ? m : e;
      }
      nq = m;
    }
    const double n1 = __shfl_sync(0xffffffffu, nq, 1);
    const double n2 = __shfl_sync(0xffffffffu, nq, 2);
    const double n3 = __shfl_sync(0xffffffffu, nq, 3);
    if (lane == 0) {
      const double m12 = n1 > n2 ? n1 : n2;
      const double m123 = m12 > n3 ? m12 : n3;
      r.avg = sq;
      r.err = (__dmul_rn(5.0, n1) <= n2 && __dmul_rn(5.0, n2) <= n3) ? n1 : __dmul_rn(5.0, m123);
      r.axis = rs.axis >= 0 ? rs.axis : 0;
    }
  }
  __syncthreads();
  return r;
}

// Copy of the rule tables in shared memory, for group_finish (which reads
// them by lane index).  Every thread of the block calls it; a block
// barrier must follow before the copy is read.
__device__ __forceinline__ void stage_tables(const RuleTables& T, RuleTables& dst) {
  static_assert(sizeof(RuleTables) % 8 == 0, "tables are copied as 8-byte words");
  constexpr int kW = sizeof(RuleTables) / 8;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&T);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
  for (int i = threadIdx.x; i < kW; i += blockDim.x) d[i] = src[i];
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
  double S[kNumSets];
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) S[k] = 0;
  // Branch-free body, two points in flight per thread.  A thread's points
  // of one set are consecutive, so adding into S[set] directly gives the
  // same sums as a running sum flushed at set changes.
  const int p0 = active ? t : PointTable<N>::kPoints;
  auto point = [&](int p) {
    const uint2 e = sm.pt.ent[p];
    double x[N];
#pragma unroll
    for (int i = 0; i < N; ++i) x[i] = fma(sm.pt.ctab[(e.x >> (4 * i)) & 15u], H[i], L[i]);
    const double fx = call_point(f, x, p);
    if (p <= 4 * N) sm.fstage[g][p] = fx;
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) S[k] += (e.y == (unsigned)k) ? fx : 0.0;
  };
  if constexpr (kTwoPointsInFlight<F>) {
#pragma unroll 2
    for (int p = p0; p < PointTable<N>::kPoints; p += G) point(p);
  } else {
#pragma unroll 1
    for (int p = p0; p < PointTable<N>::kPoints; p += G) point(p);
  }
  return group_finish<N, G>(S, H, T, sm.red, sm.fstage[g], t);
}

// atomicAdd with acquire-release semantics at GPU scope: publishes the
// calling thread's earlier writes and, for the last arriver, makes every
// earlier arriver's writes visible -- cheaper than fence + add + fence.
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Position of the r-th (0-based) set bit of m; requires r < popcount(m).
__host__ __device__ __forceinline__ int nth_set_bit(unsigned m, int r) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const unsigned low = m & ((1u << w) - 1u);
#ifdef __CUDA_ARCH__
    const int c = __popc(low);
#else
    const int c = __builtin_popcount(low);
#endif
    if (r >= c) {
      r -= c;
      m >>= w;
      pos += w;
    }
  }
  return pos;
}

// Parent slot of the active region of rank i among the chunks
// [pc0, pc0 + pnc) of one integral in the parent list: the last chunk whose
// active-count prefix is <= i, then the matching set bit of its mask.
template <class Excl, class Mask>
__host__ __device__ __forceinline__ int parent_slot(int i, int pc0, int pnc, const Excl& excl,
                                                    const Mask& mask) {
  int lo = pc0, hi = pc0 + pnc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (excl(mid) <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo * 32 + nth_set_bit(mask(lo), i - excl(lo));
}

// The list the current one was split from, as the lazy split reads it.
struct Parent {
  const double* lo;
  const double* len;
  const int* axis;
  const unsigned* mask;
  const int* excl;
  long long cap;
};

// The list being written (current buffer).
struct Dest {
  double* lo;
  double* len;
  int* rid;
  long long cap;
};

// Child `side` (0 lower, 1 upper) of parent slot p: halved on the parent's
// split axis, the same arithmetic as split_chunk_warp.
template <int N>
__device__ __forceinline__ void child_box(const Parent& P, int p, int side, double (&L)[N],
                                          double (&H)[N]) {
  const int ax = P.axis[p];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const double l = P.lo[(long long)d * P.cap + p];
    const double w = P.len[(long long)d * P.cap + p];
    if (d == ax) {
      const double h = w / 2;
      L[d] = side ? l + 1 * h : l;
      H[d] = h;
    } else {
      L[d] = l;
      H[d] = w;
    }
  }
}

// Shared-memory copy of what the lazy split of one iteration looks up.
struct Stage {
  int excl[kStageChunks];       // parent list: active regions before each chunk
  unsigned mask[kStageChunks];  // parent list: active mask of each chunk
  int cint[kStageChunks];       // current list: owning integral (large batches)
  int seg_start[kSmallBatch], seg_count[kSmallBatch];
  int par_start[kSmallBatch], par_count[kSmallBatch];
  double epsrel[kSmallBatch], epsabs[kSmallBatch];
};

// Write the pending (lazily split) list in full, from global memory: run
// by every thread of the grid when the kernel leaves.
template <int N>
__device__ void materialize(const EngineArgs& a, const int* chunk_int, const Parent& P,
                            const Dest& D) {
  const bool small = a.nint <= kSmallBatch;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < a.n; s += stride) {
    int k = 0;
    if (small) {
      for (int q = 1; q < a.nint; ++q)
        if (a.ist[q].seg_start <= s) k = q;
    } else {
      k = chunk_int[s >> 5];
    }
    const IntegralState& is = a.ist[k];
    const int j = (int)(s - is.seg_start);
    if (j >= is.seg_count) {
      D.rid[s] = -1;
      continue;
    }
    const int par = parent_slot(
        j >> 1, is.par_start >> 5, (is.par_count + 31) >> 5, [&](int q) { return P.excl[q]; },
        [&](int q) { return P.mask[q]; });
    double L[N], H[N];
    child_box<N>(P, par, j & 1, L, H);
#pragma unroll
    for (int d = 0; d < N; ++d) {
      D.lo[(long long)d * D.cap + s] = L[d];
      D.len[(long long)d * D.cap + s] = H[d];
    }
    D.rid[s] = k;
  }
}

// Leftover boxes of the integrals handed to phase 2 by the previous
// iteration's decision (handoff_at == g_it): the children of their active
// regions in the parent list, written to the leftover list.  Warp per chunk.
template <int N>
__device__ void handoff(const EngineArgs& a, const Parent& P, const int* prid, long long pn,
                        int g_it) {
  const int lane = threadIdx.x & 31;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  for (long long c = gwarp; c < pn / 32; c += nwarp) {
    const long long i = c * 32 + lane;
    const int k = prid[i];
    const unsigned m = P.mask[c];
    bool act = k >= 0 && ((m >> lane) & 1u);
    if (act) act = a.ist[k].state == kStatePhase2 && a.ist[k].handoff_at == g_it;
    if (!act) continue;
    const int rank = P.excl[c] + __popc(m & ((1u << lane) - 1u));
    const long long dst = a.ist[k].left_start + 2ll * rank;
    const int ax = P.axis[i];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const double l = P.lo[(long long)d * P.cap + i];
      const double w = P.len[(long long)d * P.cap + i];
      double* dlo = a.left_lo + (long long)d * a.left_cap;
      double* dlen = a.left_len + (long long)d * a.left_cap;
      if (d == ax) {
        const double h = w / 2;
        dlo[dst] = l;
        dlo[dst + 1] = l + 1 * h;
        dlen[dst] = h;
        dlen[dst + 1] = h;
      } else {
        dlo[dst] = l;
        dlo[dst + 1] = l;
        dlen[dst] = w;
        dlen[dst + 1] = w;
      }
    }
    a.left_rid[dst] = k;
    a.left_rid[dst + 1] = k;
  }
}

// Small batches (nint <= kSmallBatch): the warp that completed the last
// chunk decides every integral (lane k: integral k), writes each chunk's
// active-count prefix, assigns the next segments (32-aligned, integral
// order) and leftover ranges, and moves every integral to its next segment
// (the current one becomes the parent segment).
static __device__ __noinline__ void decide_scan_small(const EngineArgs& a, const IterState& st,
                                               IterState* next, int lane, int g_next, int it) {
  const int nint = a.nint;
  const bool have = lane < nint;
  IntegralState& is = a.ist[have ? lane : 0];
  const bool run = have && is.state == kStateRunning;
  if (lane == 0) trace_mark(a.ctl, it, 3);
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int m = 0;
  if (nint == 1) {
    // one integral: lane-strided sums in the order of decide_warp
    const int nc = a.n / 32;
#pragma unroll 2
    for (int base = 0; base < nc; base += 32) {
      const int c = base + lane;
      double v0 = 0, v1 = 0, v2 = 0, v3 = 0;
      int na = 0;
      if (c < nc) {
        const ChunkPartial& pc = a.part[c];
        v0 = pc.sum_avg;
        v1 = pc.sum_err;
        v2 = pc.fin_avg;
        v3 = pc.fin_err;
        na = pc.nactive;
      }
      s0 += v0;
      s1 += v1;
      s2 += v2;
      s3 += v3;
      int incl = na;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
      }
      if (c < nc) a.chunk_excl[c] = m + incl - na;
      m += __shfl_sync(0xffffffffu, incl, 31);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, off);
      s1 += __shfl_xor_sync(0xffffffffu, s1, off);
      s2 += __shfl_xor_sync(0xffffffffu, s2, off);
      s3 += __shfl_xor_sync(0xffffffffu, s3, off);
    }
  } else if (run) {
    const int c0 = is.seg_start / 32, nc = (is.seg_count + 31) / 32;
    for (int q = 0; q < nc; ++q) {
      const ChunkPartial& pc = a.part[c0 + q];
      s0 += pc.sum_avg;
      s1 += pc.sum_err;
      s2 += pc.fin_avg;
      s3 += pc.fin_err;
      a.chunk_excl[c0 + q] = m;
      m += pc.nactive;
    }
  }
  if (lane == 0) trace_mark(a.ctl, it, 7);
  bool entered = false;
  if (run) {
    decide_integral(is, s0, s1, s2, s3, m, a);
    entered = is.state == kStatePhase2;
  }
  if (lane == 0) trace_mark(a.ctl, it, 6);
  const bool cont = run && is.state == kStateRunning;
  const int nextc = cont ? is.next_count : 0;
  const int vn = (nextc + 31) & ~31;
  const int vl = entered ? is.left_new : 0;
  int in = vn, il = vl;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int tn = __shfl_up_sync(0xffffffffu, in, off);
    const int tl = __shfl_up_sync(0xffffffffu, il, off);
    if (lane >= off) {
      in += tn;
      il += tl;
    }
  }
  const int tot_n = __shfl_sync(0xffffffffu, in, 31);
  const int tot_l = __shfl_sync(0xffffffffu, il, 31);
  const int nrun = __popc(__ballot_sync(0xffffffffu, nextc > 0));
  if (have) {
    const int ss = is.seg_start, sc = is.seg_count;
    is.par_start = ss;
    is.par_count = sc;
    is.next_start = in - vn;
    is.seg_start = in - vn;
    is.seg_count = nextc;
    if (vl > 0) {
      is.left_start = st.n_left + il - vl;
      is.left_count = vl;
      is.handoff_at = g_next;
    }
  }
  if (lane == 0) {
    IterState s;
    s.n = tot_n;
    s.n_running = nrun;
    s.n_left = st.n_left + tot_l;
    s.overflow = (tot_n > a.ncap) || (s.n_left > a.left_cap);
    s.handoff = tot_l > 0;
    *next = s;
  }
}

// Large batches: after every integral is decided, one warp assigns the
// next segments and leftover ranges (exclusive scan in integral order),
// moves each integral to its next segment and records the owner of every
// chunk of the next list.
static __device__ __noinline__ void scan_shift_warp(const EngineArgs& a, int n_left_in, IterState* out,
                                             int* chunk_int, int lane, int g_next) {
  int carry_n = 0, carry_l = n_left_in, nrun = 0;
  for (int base = 0; base < a.nint; base += 32) {
    const int k = base + lane;
    int vn = 0, vl = 0, r = 0;
    int state = kStateDone, next_count = 0, seg_start = 0, seg_count = 0;
    if (k < a.nint) {
      const IntegralState& is = a.ist[k];
      state = is.state;
      next_count = is.next_count;
      seg_start = is.seg_start;
      seg_count = is.seg_count;
      vn = state == kStateRunning ? (next_count + 31) & ~31 : 0;
      vl = is.left_count == 0 ? is.left_new : 0;  // each integral hands off once
      r = state == kStateRunning && next_count > 0;
    }
    int in = vn, il = vl;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int tn = __shfl_up_sync(0xffffffffu, in, off);
      const int tl = __shfl_up_sync(0xffffffffu, il, off);
      if (lane >= off) {
        in += tn;
        il += tl;
      }
    }
    if (k < a.nint) {
      IntegralState& is = a.ist[k];
      const int ns = carry_n + in - vn;
      is.par_start = seg_start;
      is.par_count = seg_count;
      is.next_start = ns;
      is.seg_start = ns;
      is.seg_count = state == kStateRunning ? next_count : 0;
      if (vl > 0) {
        is.left_start = carry_l + il - vl;
        is.left_count = vl;
        is.handoff_at = g_next;
      }
      for (int q = ns >> 5; q < (ns + vn) >> 5; ++q) chunk_int[q] = k;
    }
    carry_n += __shfl_sync(0xffffffffu, in, 31);
    carry_l += __shfl_sync(0xffffffffu, il, 31);
    nrun += __popc(__ballot_sync(0xffffffffu, r));
  }
  if (lane == 0) {
    IterState s;
    s.n = carry_n;
    s.n_running = nrun;
    s.n_left = carry_l;
    s.overflow = (carry_n > a.ncap) || (carry_l > a.left_cap);
    s.handoff = carry_l > n_left_in;
    *out = s;
  }
}

// Run by the warp that completed chunk c (owned by integral k).  Small
// batches: sum the chunk; the warp that completes the last chunk of the
// list decides every integral and assigns the next list.  Large batches:
// the warp that completes an integral's last chunk decides it, the one that
// decides the last integral assigns the next list.
static __device__ __noinline__ void after_chunk_warp(const EngineArgs& a, long long c, int k, int lane,
                                              const IterState& st, IterState* next,
                                              int* chunk_int, int it, int g_next) {
  __syncwarp();
  chunk_partial_warp(a, c, lane);
  if (a.nint <= kSmallBatch) {
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
    decide_scan_small(a, st, next, lane, g_next, it);
    // the next list becomes visible through the grid barrier's release
    if (lane == 0) trace_mark(a.ctl, it, 1);
    return;
  }
  unsigned last = 0;
  if (lane == 0) {
    a.chunk_cnt[c] = 0;
    const unsigned nc = (unsigned)((a.ist[k].seg_count + 31) / 32);
    last = atom_add_acq_rel(&a.int_cnt[k], 1u) == nc - 1;
  }
  last = __shfl_sync(0xffffffffu, last, 0);
  if (!last) return;
  __syncwarp();
  if (lane == 0) a.int_cnt[k] = 0;
  decide_warp(a, k, lane);
  __syncwarp();
  unsigned all = 0;
  if (lane == 0) all = atom_add_acq_rel(&a.ctl->done_cnt, 1u) == (unsigned)st.n_running - 1;
  all = __shfl_sync(0xffffffffu, all, 0);
  if (!all) return;
  __syncwarp();
  if (lane == 0) a.ctl->done_cnt = 0;
  scan_shift_warp(a, st.n_left, next, chunk_int, lane, g_next);
  // the next list becomes visible through the grid barrier's release
  if (lane == 0) trace_mark(a.ctl, it, 1);
}

// Where slot `slot` of a lazily split list comes from: its integral k (-1
// for padding), the integral's tolerances, and the parent slot and side.
struct Origin {
  int k, par, side;
  double epsrel, epsabs;
};

__device__ __forceinline__ Origin lazy_origin(const EngineArgs& a, const Stage& sg,
                                              long long slot) {
  Origin o;
  int ss, sc, ps, pc;
  if (a.nint <= kSmallBatch) {
    int k = 0;
    for (int q = 1; q < a.nint; ++q)
      if (sg.seg_start[q] <= slot) k = q;
    o.k = k;
    ss = sg.seg_start[k];
    sc = sg.seg_count[k];
    ps = sg.par_start[k];
    pc = sg.par_count[k];
    o.epsrel = sg.epsrel[k];
    o.epsabs = sg.epsabs[k];
  } else {
    o.k = sg.cint[slot >> 5];
    const IntegralState& is = a.ist[o.k];
    ss = is.seg_start;
    sc = is.seg_count;
    ps = is.par_start;
    pc = is.par_count;
    o.epsrel = is.epsrel;
    o.epsabs = is.epsabs;
  }
  const int j = (int)(slot - ss);
  o.side = j & 1;
  o.par = 0;
  if (j >= sc) {
    o.k = -1;
    return o;
  }
  o.par = parent_slot(
      j >> 1, ps >> 5, (pc + 31) >> 5, [&](int q) { return sg.excl[q]; },
      [&](int q) { return sg.mask[q]; });
  return o;
}

// Write the initial grid in full (the kernel leaves before evaluating it).
template <int N>
__device__ void grid_pass(const PersistArgs& p, const Dest& D, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
    double L[N], H[N];
    const int k = initial_box<N>(s, p.divisions, p.per_integral, p.padded, p.box, L, H);
    if (k >= 0) {
#pragma unroll
      for (int d = 0; d < N; ++d) {
        D.lo[(long long)d * D.cap + s] = L[d];
        D.len[(long long)d * D.cap + s] = H[d];
      }
    }
    D.rid[s] = k;
  }
}

// The eval step with groups of G threads (R = 256/G regions per block).
// The slots of round `base` are base + g * gridDim.x + blockIdx.x: group
// index interleaved over blocks, so consecutive regions land on different
// SMs.  Every group of a block runs the same number of rounds (groups past
// the end of the list idle through the block barriers).  Unless the slot's
// region is stored, the group first computes it (lazy split or initial
// grid) and writes it into the list.
template <int N, int G, class Src>
__device__ __forceinline__ void eval_step(const Src& src, const RuleTables& T, const EngineArgs& a,
                                          const PersistArgs& pa, const Parent& P, const Dest& D,
                                          const Stage& sg, int mode, const IterState& st,
                                          IterState* next, int* chunk_int, GroupSmem<N>& sm,
                                          int it, int g_next, const EngineArgs* sa) {
  constexpr int R = 256 / G;
  const int g = threadIdx.x / G, t = threadIdx.x % G, lane = threadIdx.x & 31;
  const long long ngroups = (long long)R * gridDim.x;
  for (long long base = 0; base < st.n; base += ngroups) {
    const long long slot = base + (long long)g * gridDim.x + blockIdx.x;
    const bool live = slot < st.n;
    int k = -1;
    double epsrel = 0, epsabs = 0;
    double L[N], H[N];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      L[d] = 0;
      H[d] = 1;
    }
    if (live && mode == kSlotGrid) {
      k = initial_box<N>(slot, pa.divisions, pa.per_integral, pa.padded, pa.box, L, H);
      if (k >= 0) {
        epsrel = a.ist[k].epsrel;
        epsabs = a.ist[k].epsabs;
      }
      if (t == 0) {
        if (k >= 0) {
#pragma unroll
          for (int d = 0; d < N; ++d) {
            D.lo[(long long)d * D.cap + slot] = L[d];
            D.len[(long long)d * D.cap + slot] = H[d];
          }
        }
        D.rid[slot] = k;
      }
    } else if (live && mode == kSlotStored) {
      k = a.rid[slot];
      if (k >= 0) {
#pragma unroll
        for (int d = 0; d < N; ++d) {
          L[d] = a.lo[(long long)d * a.cap + slot];
          H[d] = a.len[(long long)d * a.cap + slot];
        }
        epsrel = a.ist[k].epsrel;
        epsabs = a.ist[k].epsabs;
      }
    } else if (live) {
      const Origin o = lazy_origin(a, sg, slot);
      k = o.k;
      epsrel = o.epsrel;
      epsabs = o.epsabs;
      if (k >= 0) {
        child_box<N>(P, o.par, o.side, L, H);
        if (t == 0) {
#pragma unroll
          for (int d = 0; d < N; ++d) {
            D.lo[(long long)d * D.cap + slot] = L[d];
            D.len[(long long)d * D.cap + slot] = H[d];
          }
          D.rid[slot] = k;
        }
      } else if (t == 0) {
        D.rid[slot] = -1;
      }
    }
    {
      // groups without a region evaluate no point but join the barriers
      const auto f = src.get(k >= 0 ? k : 0);
      const RegionResult r = eval_region_group<N, G>(f, L, H, sm.tables, sm, g, t, k >= 0);
      if (t == 0 && k >= 0) store_result(a, slot, r, epsrel, epsabs);
    }
    if (t == 0 && live) {
      if (k < 0) store_padding(a, slot);
      sm.flag[g] = atom_add_acq_rel(&a.chunk_cnt[slot / 32], 1u) == 31;
      sm.owner[g] = k;
    } else if (t == 0) {
      sm.flag[g] = 0;
    }
    __syncthreads();
    if (t < 32 && sm.flag[g]) {
      // the chunk's owner: a padding slot only ends a segment, so the
      // chunk's first slot always holds a region
      const long long c = slot / 32;
      const int kc = sm.owner[g] >= 0 ? sm.owner[g] : a.rid[c * 32];
      after_chunk_warp(*sa, c, kc, lane, st, next, chunk_int, it, g_next);
    }
    __syncthreads();
  }
}

}  // namespace detail

template <int N, class Src>
__global__ void __launch_bounds__(256, 2) k_persistent(Src src, RuleTables T, PersistArgs p) {
  __shared__ detail::GroupSmem<N> sm;
  __shared__ detail::Stage sg;
  __shared__ EngineArgs sargs;
  sm.pt.fill(threadIdx.x, blockDim.x);
  detail::stage_tables(T, sm.tables);
  __syncthreads();
  Control* ctl = p.base.ctl;
  int cur = ctl->cur;
  int reason = kExitDone;
  long long prev_n = 0;
  unsigned barriers = 0;
  const bool tracer = blockIdx.x == 0 && threadIdx.x == 0;
  const bool small = p.base.nint <= kSmallBatch;
  IterState st;
  for (int it = 0;; ++it) {
    if (tracer) trace_mark(ctl, it, 0);
    const int parity = it & 1;
    const bool lazy = it > 0;
    if (lazy) {
      // Stage the lookups of the lazy split while the iteration state is
      // read: they depend only on the parent list and the integral states,
      // both complete at the grid barrier.  materialize and handoff do not
      // touch the staged copy.
      const int* pexcl = p.excl[parity ^ 1];
      const unsigned* pmask = p.cmask[parity ^ 1];
      const int pnc = (int)(prev_n / 32);
      for (int q = threadIdx.x; q < pnc; q += blockDim.x) {
        sg.excl[q] = pexcl[q];
        sg.mask[q] = pmask[q];
      }
      if (small) {
        for (int q = threadIdx.x; q < p.base.nint; q += blockDim.x) {
          const IntegralState& is = p.base.ist[q];
          sg.seg_start[q] = is.seg_start;
          sg.seg_count[q] = is.seg_count;
          sg.par_start[q] = is.par_start;
          sg.par_count[q] = is.par_count;
          sg.epsrel[q] = is.epsrel;
          sg.epsabs[q] = is.epsabs;
        }
      }
    }
    {
      volatile IterState* v = &ctl->it[parity];
      st.n = v->n;
      st.n_running = v->n_running;
      st.n_left = v->n_left;
      st.overflow = v->overflow;
      st.handoff = v->handoff;
    }
    const int mode = lazy ? kSlotLazy : (p.init ? kSlotGrid : kSlotStored);
    EngineArgs a = p.base;
    a.lo = p.lo[cur];
    a.len = p.len[cur];
    a.rid = p.rid[cur];
    a.axis = p.axis[parity];
    a.cmask = p.cmask[parity];
    a.chunk_excl = p.excl[parity];
    a.n = st.n;
    const detail::Parent P{p.lo[cur ^ 1],       p.len[cur ^ 1],     p.axis[parity ^ 1],
                           p.cmask[parity ^ 1], p.excl[parity ^ 1], a.cap};
    const detail::Dest D{p.lo[cur], p.len[cur], p.rid[cur], a.cap};
    const int* prid = p.rid[cur ^ 1];
    const int g_it = p.iter_base + it;

    if (st.n_running == 0 || st.n == 0)
      reason = kExitDone;
    else if (st.n > p.max_n)
      reason = kExitLarge;
    else if (2ll * st.n + 32ll * a.nint > a.ncap ||
             (a.policy == kPolicyReference && (long long)st.n_left + 2ll * st.n > a.left_cap))
      reason = kExitCapacity;
    else
      reason = 0;
    if (reason) {
      // leave a complete list behind
      if (lazy) {
        detail::materialize<N>(a, p.chunk_int, P, D);
        if (st.handoff) detail::handoff<N>(a, P, prid, prev_n, g_it);
      } else if (mode == kSlotGrid) {
        detail::grid_pass<N>(p, D, st.n);
      }
      break;
    }
    if (lazy && st.handoff) detail::handoff<N>(a, P, prid, prev_n, g_it);
    if (lazy && !small)
      for (int q = threadIdx.x; q < st.n / 32; q += blockDim.x) sg.cint[q] = p.chunk_int[q];
    IterState* next = &ctl->it[parity ^ 1];
    // The chain after a chunk runs out of line (one warp per chunk, cold
    // code shared by all group sizes); it reads the arguments from a
    // shared-memory copy so that the kernel's own copy stays in registers.
    if (threadIdx.x == 0) sargs = a;
    __syncthreads();  // also publishes the staged lookups

    // smallest R (regions per block) that covers the list in one pass
    const long long per_block = (st.n + gridDim.x - 1) / gridDim.x;
    const int r = per_block <= 1 ? 1 : (per_block <= 2 ? 2 : (per_block <= 4 ? 4 : 8));
    switch (r < p.max_r ? r : p.max_r) {
      case 1:
        detail::eval_step<N, 256>(src, T, a, p, P, D, sg, mode, st, next, p.chunk_int, sm, it, g_it + 1, &sargs);
        break;
      case 2:
        detail::eval_step<N, 128>(src, T, a, p, P, D, sg, mode, st, next, p.chunk_int, sm, it, g_it + 1, &sargs);
        break;
      case 4:
        detail::eval_step<N, 64>(src, T, a, p, P, D, sg, mode, st, next, p.chunk_int, sm, it, g_it + 1, &sargs);
        break;
      default:
        detail::eval_step<N, 32>(src, T, a, p, P, D, sg, mode, st, next, p.chunk_int, sm, it, g_it + 1, &sargs);
        break;
    }
    if (tracer) trace_mark(ctl, it, 4);
    ++barriers;
    if (!detail::grid_barrier(ctl, barriers * gridDim.x, p.spin_limit,
                              (int)blockIdx.x != p.hold_block)) {
      reason = kExitTimeout;
      break;
    }
    if (tracer) trace_mark(ctl, it, 2);
    cur ^= 1;
    prev_n = st.n;
    // a store, not a read-modify-write: the launch starts at iter_base
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->iters_done = p.iter_base + it + 1;
  }
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) {
      ctl->cur = cur;
      IterState h = st;
      h.overflow = 0;
      h.handoff = 0;
      ctl->host = h;
      ctl->exit_reason = reason;
    }
    if (p.host_out) {
      // the states were completed before the last grid barrier; the
      // control block's final fields just above
      __syncthreads();
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(ctl);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(p.host_out);
      for (int i = threadIdx.x; i < p.host_words; i += blockDim.x) dst[i] = src[i];
    }
  }
}

}  // namespace cubature
