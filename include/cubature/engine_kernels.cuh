// engine_kernels.cuh -- the device side of the breadth-first engine.
//
// One iteration of the reference's first phase (GPUKernelquad.cu:509-605)
// over a batch of independent integrals whose regions share one list:
//
//   eval      rule + fourth difference + error + classification per region
//             (INTEGRATE_GPU_PHASE1, GPUQuadPhases.cu:38-79)
//   partials  per 32-region chunk: value/error sums, finished sums, active
//             count (the reference's four thrust::reduce calls and the
//             exclusive scan, GPUKernelquad.cu:364-386,565-577)
//   decide    per integral: totals, the global stop test, the child count
//             (GPUKernelquad.cu:583-598)
//   scan      exclusive scan of child counts over integrals -> new segments
//   split     compaction + bisection of the active regions, written as
//             adjacent children (alignRegions + divideIntervalsGPU,
//             GPUKernelquad.cu:63-149)
//
// The steps are warp-level device functions shared by two drivers: one
// kernel launch per step (the throughput regime, engine.cuh) and the
// persistent cooperative kernel (the latency regime, persistent.cuh).
//
// Layout in HBM: region lists are SoA, lo[d * cap + i] and len[d * cap + i]
// (FP64), rid[i] = owning integral (-1 = padding).  Each integral owns a
// contiguous segment whose start is a multiple of 32, so a 32-region chunk
// never straddles two integrals and every reduction is a fixed-order tree
// (results are bit-reproducible run to run).
#pragma once

#include <cstdint>

#include "integrands.cuh"
#include "region_rule.cuh"

namespace cubature {

enum Policy : int { kPolicyReference = 0, kPolicyBreadth = 1 };

// Status of an integral whose sums stopped being finite (a NaN or infinite
// integrand value), CUB_STATUS_NONFINITE of the C ABI.
constexpr int kStatusNonFinite = 1 << 30;

enum IntegralStateCode : int {
  kStateRunning = 0,
  kStateDone = 1,      // converged or out of active regions
  kStatePhase2 = 2,    // handed to the depth-first second phase
  kStateCapacity = 3,  // stopped: region capacity or iteration limit
};

// Per-integral state, resident on the device for the whole run.
struct IntegralState {
  double epsrel, epsabs;
  double value, error;  // finished sums (final results when done)
  double last_value, last_error;
  unsigned long long nregions, neval;
  int state, status, iters;
  int left_new;                // leftover boxes produced this iteration
  int seg_start, seg_count;    // segment in the current list
  int next_start, next_count;  // segment in the next list
  int left_start, left_count;  // leftover boxes for phase 2
  // persistent kernel, where the next list is built lazily: the segment
  // of the list the current one was split from, and the global iteration
  // whose first step copies this integral's leftovers (hand-off to phase 2)
  int par_start, par_count;
  int handoff_at, pad;
};

struct ChunkPartial {
  double sum_avg, sum_err;  // all regions of the chunk
  double fin_avg, fin_err;  // finished regions only
  int nactive;
  unsigned mask;  // bit i: slot 32c + i stays active
};

// List sizes after one iteration's scan.
struct IterState {
  int n;          // slots in the list (padded)
  int n_running;  // integrals with regions in that list
  int n_left;     // leftover boxes queued for phase 2 so far
  int overflow;   // the list or the leftovers would exceed capacity
  int handoff;    // some integral was handed to phase 2 by this scan
};

// Control block shared by the host and both drivers.
struct Control {
  IterState host;      // result of the last scan (multi-launch driver)
  IterState it[2];     // double-buffered by iteration parity (persistent)
  int cur;             // index of the current list buffer
  int iters_done;      // breadth-first iterations completed
  int exit_reason;     // persistent kernel: why it returned
  int pad;
  unsigned done_cnt;   // integrals decided in this iteration
  unsigned bar_count;  // grid barrier arrivals since the launch (monotonic)
  unsigned exit_count;  // replicated kernel: blocks that have left this launch
  int timeout;         // a bounded wait gave up
  // globaltimer stamps (ns) of the persistent kernels' first kTraceIters
  // iterations, kTraceSlots per iteration (diagnostics, read back with the
  // control block).  Persistent kernel: 0 start, 1 next list assigned,
  // 2 grid barrier passed, 3 decider read its integral state, 4 block 0's
  // evaluations done, 5 last chunk summed, 6 integrals decided, 7 chunk sums
  // combined.  Replicated kernel (block 0): 0 start, 7 first region set up,
  // 4 evaluations done, 2 grid barrier passed, 3 chunk partials formed,
  // 1 per-integral sums formed (warp 0), 6 stop decision taken, 5 next
  // segments assigned.
  unsigned long long trace[64];
};
constexpr int kTraceIters = 8;
constexpr int kTraceSlots = 8;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void trace_mark(Control* ctl, int it, int slot) {
  if (it < kTraceIters) ctl->trace[kTraceSlots * it + slot] = global_ns();
}

enum ExitReason : int {
  kExitDone = 1,      // no integral left running
  kExitLarge = 2,     // the list grew past the persistent kernel's range
  kExitCapacity = 3,  // buffers must grow before the next iteration
  kExitTimeout = 4,   // a grid barrier wait ran out
};

struct EngineArgs {
  // current list
  const double* lo;
  const double* len;
  const int* rid;
  int n;  // padded slot count
  long long cap;
  // per-region outputs
  double* avg;
  double* err;
  int* axis;
  int* active;
  // chunk partials / prefix / arrival counters
  ChunkPartial* part;
  int* chunk_excl;
  unsigned* cmask;  // active bit mask per chunk (optional)
  unsigned* chunk_cnt;
  unsigned* int_cnt;
  // next list
  double* nlo;
  double* nlen;
  int* nrid;
  long long ncap;
  // leftovers for phase 2
  double* left_lo;
  double* left_len;
  int* left_rid;
  long long left_cap;
  // integrals
  IntegralState* ist;
  int nint;
  Control* ctl;
  int policy;
  int phase1_cap;  // child count that ends phase 1 (0 = never)
  int max_iters;   // phase-1 iteration limit
  int npoints;
};

namespace detail {

__host__ __device__ __forceinline__ double max_err(double avg, double epsrel, double epsabs) {
  const double a = epsrel * fabs(avg);
  return a > epsabs ? a : epsabs;
}

template <class F>
struct SingleSource {
  F f;
  __device__ __forceinline__ const F& get(int) const { return f; }
};

template <class F>
struct ParamSource {
  const GenzParams* params;
  __device__ __forceinline__ F get(int k) const { return F::load(params[k]); }
};

// Integrals of different families in one batch (family per integral).
template <int N>
struct MixedSource {
  const GenzParams* params;
  const int* families;
  __device__ __forceinline__ MixedGenz<N> get(int k) const {
    return MixedGenz<N>::make(params[k], families[k]);
  }
};

// Write one region's results (reference classification:
// fail when err / max(epsrel|avg|, epsabs) > 1, GPUQuadPhases.cu:63-74).
__device__ __forceinline__ void store_result(const EngineArgs& a, long long slot,
                                             const RegionResult& r, double epsrel, double epsabs) {
  const double ratio = r.err / max_err(r.avg, epsrel, epsabs);
  a.avg[slot] = r.avg;
  a.err[slot] = r.err;
  a.axis[slot] = r.axis;
  a.active[slot] = ratio > 1;
}

__device__ __forceinline__ void store_padding(const EngineArgs& a, long long slot) {
  a.avg[slot] = 0;
  a.err[slot] = 0;
  a.axis[slot] = 0;
  a.active[slot] = 0;
}

// Evaluate slot `slot` with the K lanes of a group (K <= 32, structured
// point enumeration); lane 0 of the group stores the result.
template <int N, int K, class Src>
__device__ __forceinline__ void eval_slot(const Src& src, const RuleTables& T,
                                          const EngineArgs& a, long long slot, int lane,
                                          unsigned gmask, const ItemTable<N>& tab) {
  const int k = a.rid[slot];
  if (k < 0) {
    if (lane == 0) store_padding(a, slot);
    return;
  }
  double L[N], H[N];
#pragma unroll
  for (int d = 0; d < N; ++d) {
    L[d] = a.lo[(long long)d * a.cap + slot];
    H[d] = a.len[(long long)d * a.cap + slot];
  }
  const auto f = src.get(k);
  RegionSums rs;
  region_point_sums<N, K>(f, L, H, lane, tab, T.ratio, rs);
  if (K > 1) reduce_lanes<K>(rs, gmask);
  if (lane == 0) {
    double jac = 1;
#pragma unroll
    for (int d = 0; d < N; ++d) jac = __dmul_rn(jac, H[d]);
    store_result(a, slot, finish_region<N>(rs, T, jac, 0), a.ist[k].epsrel, a.ist[k].epsabs);
  }
}

// A warp sums the 32 slots of chunk c into a.part[c].
__device__ __forceinline__ void chunk_partial_warp(const EngineArgs& a, long long c, int lane) {
  const long long i = c * 32 + lane;
  const bool valid = i < a.n && a.rid[i] >= 0;
  const double av = valid ? a.avg[i] : 0.0, er = valid ? a.err[i] : 0.0;
  const bool act = valid && a.active[i];
  double s0 = av, s1 = er, s2 = act ? 0.0 : av, s3 = act ? 0.0 : er;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    s3 += __shfl_xor_sync(0xffffffffu, s3, off);
  }
  const unsigned b = __ballot_sync(0xffffffffu, act);
  if (lane == 0) {
    ChunkPartial p;
    p.sum_avg = s0;
    p.sum_err = s1;
    p.fin_avg = s2;
    p.fin_err = s3;
    p.nactive = __popc(b);
    p.mask = b;
    a.part[c] = p;
    if (a.cmask) a.cmask[c] = b;
  }
}

// Stop decision for one running integral from the sums of its chunks and
// its active-region count m (GPUKernelquad.cu:565-605).  Sets the child
// count (next_count) or the leftover count (left_new) of phase 2.
__device__ __forceinline__ void decide_integral(IntegralState& is, double s0, double s1, double s2,
                                                double s3, int m, const EngineArgs& a) {
  const double rG = is.value + s0, errG = is.error + s1;
  is.value += s2;
  is.error += s3;
  is.last_value = rG;
  is.last_error = errG;
  is.nregions += (unsigned long long)is.seg_count;
  is.neval += (unsigned long long)is.seg_count * (unsigned long long)a.npoints;
  is.iters += 1;
  is.next_count = 0;
  is.left_new = 0;
  if (!isfinite(s0) || !isfinite(s1)) {
    // a NaN or infinite integrand value reached the sums: stop here
    is.value = rG;
    is.error = errG;
    is.state = kStateDone;
    is.status = kStatusNonFinite;
  } else if (errG <= max_err(rG, is.epsrel, is.epsabs)) {
    // global stop test (GPUKernelquad.cu:583-598)
    is.value = rG;
    is.error = errG;
    is.state = kStateDone;
    is.status = 0;
  } else if (m == 0) {
    // every region finished on its own tolerance
    is.state = kStateDone;
    is.status = 0;
  } else {
    const long long children = 2ll * m;
    const bool cap_hit = a.phase1_cap > 0 && children >= a.phase1_cap;
    const bool iter_hit = is.iters >= a.max_iters;
    if (cap_hit || iter_hit) {
      if (a.policy == kPolicyReference) {
        is.state = kStatePhase2;
        is.left_new = (int)children;
      } else {
        is.state = kStateCapacity;
        is.value = rG;
        is.error = errG;
        is.status = 1;
      }
    } else {
      is.next_count = (int)children;
    }
  }
}

// A warp combines integral k's chunk partials, writes the exclusive scan
// of active counts over its chunks, and takes the stop decision
// (GPUKernelquad.cu:565-605).
__device__ __forceinline__ void decide_warp(const EngineArgs& a, int k, int lane) {
  IntegralState& is = a.ist[k];
  if (is.state != kStateRunning) {
    if (lane == 0) {
      is.next_count = 0;
      is.left_new = 0;
    }
    return;
  }
  const int c0 = is.seg_start / 32;
  const int nc = (is.seg_count + 31) / 32;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  for (int c = lane; c < nc; c += 32) {
    const ChunkPartial p = a.part[c0 + c];
    s0 += p.sum_avg;
    s1 += p.sum_err;
    s2 += p.fin_avg;
    s3 += p.fin_err;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
    s3 += __shfl_xor_sync(0xffffffffu, s3, off);
  }
  int running = 0;
  for (int base = 0; base < nc; base += 32) {
    const int c = base + lane;
    const int v = c < nc ? a.part[c0 + c].nactive : 0;
    int incl = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += t;
    }
    if (c < nc) a.chunk_excl[c0 + c] = running + incl - v;
    running += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0) decide_integral(is, s0, s1, s2, s3, running, a);
}

// A single warp assigns the next segments (32-aligned) and the leftover
// ranges of all integrals: an exclusive scan in integral order.
__device__ __forceinline__ void scan_warp(const EngineArgs& a, int n_left_in, IterState* out,
                                          int lane) {
  int carry_n = 0, carry_l = n_left_in, nrun = 0;
  for (int base = 0; base < a.nint; base += 32) {
    const int k = base + lane;
    int vn = 0, vl = 0, r = 0;
    if (k < a.nint) {
      const IntegralState& is = a.ist[k];
      vn = is.state == kStateRunning ? (is.next_count + 31) & ~31 : 0;
      vl = is.left_count == 0 ? is.left_new : 0;  // each integral hands off once
      r = is.state == kStateRunning && is.next_count > 0;
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
      is.next_start = carry_n + in - vn;
      if (vl > 0) {
        is.left_start = carry_l + il - vl;
        is.left_count = vl;
      }
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
    s.handoff = 0;
    *out = s;
  }
}

// A warp writes the children of chunk c's active regions: two adjacent
// children per region, halved on its split axis, to the next list (running
// integrals) or the leftover list (integrals just handed to phase 2).
template <int N>
__device__ __forceinline__ void split_chunk_warp(const EngineArgs& a, long long c, int lane) {
  const long long i = c * 32 + lane;
  const int k = i < a.n ? a.rid[i] : -1;
  bool act = k >= 0 && a.active[i];
  int state = kStateDone;
  if (act) {
    state = a.ist[k].state;
    act = (state == kStateRunning && a.ist[k].next_count > 0) ||
          (state == kStatePhase2 && a.ist[k].left_new > 0);
  }
  const unsigned b = __ballot_sync(0xffffffffu, act);
  if (!act) return;
  const int rank = a.chunk_excl[c] + __popc(b & ((1u << lane) - 1u));
  const int ax = a.axis[i];
  double* dlo;
  double* dlen;
  int* drid;
  long long dcap, dst;
  if (state == kStatePhase2) {
    dlo = a.left_lo;
    dlen = a.left_len;
    drid = a.left_rid;
    dcap = a.left_cap;
    dst = a.ist[k].left_start + 2ll * rank;
  } else {
    dlo = a.nlo;
    dlen = a.nlen;
    drid = a.nrid;
    dcap = a.ncap;
    dst = a.ist[k].next_start + 2ll * rank;
  }
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const double l = a.lo[(long long)d * a.cap + i];
    const double w = a.len[(long long)d * a.cap + i];
    if (d == ax) {
      const double h = w / 2;
      dlo[(long long)d * dcap + dst] = l;
      dlo[(long long)d * dcap + dst + 1] = l + 1 * h;
      dlen[(long long)d * dcap + dst] = h;
      dlen[(long long)d * dcap + dst + 1] = h;
    } else {
      dlo[(long long)d * dcap + dst] = l;
      dlo[(long long)d * dcap + dst + 1] = l;
      dlen[(long long)d * dcap + dst] = w;
      dlen[(long long)d * dcap + dst + 1] = w;
    }
  }
  drid[dst] = k;
  drid[dst + 1] = k;
}

// Padding ids of integral k's next segment, and the segment hand-over
// (the next list becomes current).
__device__ __forceinline__ void finish_integral(const EngineArgs& a, int k) {
  IntegralState& is = a.ist[k];
  if (is.next_count > 0) {
    const int padded = (is.next_count + 31) & ~31;
    for (int j = is.next_count; j < padded; ++j) a.nrid[is.next_start + j] = -1;
  }
  if (is.state == kStateRunning) {
    is.seg_start = is.next_start;
    is.seg_count = is.next_count;
    if (is.next_count == 0) is.state = kStateDone;
  } else {
    is.seg_count = 0;
  }
}

}  // namespace detail

// ---------------------------------------------------------------------------
// Multi-launch driver kernels (one launch per step).
// ---------------------------------------------------------------------------
template <int N, int K, class Src>
// Two blocks per SM (at most 128 registers): the rule kernel is bound by
// FP64 latency, so warps in flight matter more than a few spilled values.
#ifndef CUB_EVAL_MIN_BLOCKS
#define CUB_EVAL_MIN_BLOCKS 2
#endif
__global__ void __launch_bounds__(256, CUB_EVAL_MIN_BLOCKS) k_eval(Src src, RuleTables T, EngineArgs a) {
  __shared__ detail::ItemTable<N> tab;
  if (threadIdx.x == 0) tab.fill();
  __syncthreads();
  constexpr int kGroups = 256 / K;
  const int lane = threadIdx.x % K;
  const unsigned gmask =
      (K == 32) ? 0xffffffffu : (((1u << K) - 1u) << ((threadIdx.x & 31) & ~(K - 1)));
  for (long long slot = (long long)blockIdx.x * kGroups + threadIdx.x / K; slot < a.n;
       slot += (long long)gridDim.x * kGroups)
    detail::eval_slot<N, K>(src, T, a, slot, lane, gmask, tab);
}

static __global__ void __launch_bounds__(256) k_partials(EngineArgs a) {
  const long long nchunk = (a.n + 31) / 32;
  for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; c < nchunk;
       c += (long long)gridDim.x * blockDim.x / 32)
    detail::chunk_partial_warp(a, c, threadIdx.x & 31);
}

static __global__ void __launch_bounds__(256) k_decide(EngineArgs a) {
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) / 32; k < a.nint;
       k += gridDim.x * blockDim.x / 32)
    detail::decide_warp(a, k, threadIdx.x & 31);
}

static __global__ void k_scan(EngineArgs a) {
  detail::scan_warp(a, a.ctl->host.n_left, &a.ctl->host, threadIdx.x & 31);
}

template <int N>
__global__ void __launch_bounds__(256) k_split(EngineArgs a) {
  if (a.ctl->host.overflow) return;
  const long long nchunk = (a.n + 31) / 32;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  for (long long c = gwarp; c < nchunk; c += nwarp) detail::split_chunk_warp<N>(a, c, threadIdx.x & 31);
}

static __global__ void k_advance(EngineArgs a) {
  if (a.ctl->host.overflow) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nint; k += gridDim.x * blockDim.x)
    detail::finish_integral(a, k);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->cur ^= 1;
    a.ctl->iters_done += 1;
  }
}

// Slot t of the initial grid: integral t / padded, cell t % padded of the
// d^N equal boxes of its integration box (box[k] = lo[N] then hi[N]; the
// unit cube when box is null), dimension 0 varying fastest
// (GPUKernelquad.cu:24-61,300-316).  Returns the integral, or -1 for a
// padding slot.
template <int N>
__device__ __forceinline__ int initial_box(long long t, int divisions, int per_integral,
                                           int padded, const double* box, double (&L)[N],
                                           double (&H)[N]) {
  const int k = (int)(t / padded);
  const int j = (int)(t % padded);
  if (j >= per_integral) return -1;
  int rem = j;
  const double* bx = box ? box + (long long)k * 2 * N : nullptr;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const int id = rem % divisions;
    rem /= divisions;
    const double blo = bx ? bx[d] : 0.0;
    const double w = (bx ? bx[N + d] - bx[d] : 1.0) / divisions;
    L[d] = blo + id * w;
    H[d] = w;
  }
  return k;
}

// Initial grid for every integral, written to the current list.
template <int N>
__global__ void k_init_grid(EngineArgs a, int divisions, int per_integral, int padded,
                            const double* box) {
  const long long total = (long long)a.nint * padded;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    double L[N], H[N];
    const int k = initial_box<N>(t, divisions, per_integral, padded, box, L, H);
    if (k >= 0) {
#pragma unroll
      for (int d = 0; d < N; ++d) {
        const_cast<double*>(a.lo)[(long long)d * a.cap + t] = L[d];
        const_cast<double*>(a.len)[(long long)d * a.cap + t] = H[d];
      }
    }
    const_cast<int*>(a.rid)[t] = k;
  }
}

}  // namespace cubature
