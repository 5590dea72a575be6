// replicated.cuh -- the breadth-first loop for small batches (at most
// kSmallBatch integrals) on short region lists, as one persistent
// cooperative kernel in which every block takes every decision itself.
//
// Per iteration:
//
//   eval    every region of the list is evaluated by a group of G = 256/R
//           threads (R = 1, 2, 4 or 8 regions per block, the smallest R that
//           covers the list in one pass); consecutive regions go to
//           different SMs.  From the second iteration of a launch on, the
//           group computes its region itself: the child of the parent of
//           rank s / 2 among the active regions of the previous list
//           (bisected on the parent's split axis), and writes it into the
//           list.  The group stores the region's value, error and axis.
//   barrier one grid barrier.
//   decide  every block reads every value and error of the list, forms
//           the chunk partials, the per-integral sums and the stop
//           decisions (GPUKernelquad.cu:565-605), the next segments and the
//           active prefix counts in its own shared memory -- the same
//           fixed-order arithmetic in every block, so every block holds
//           the same states.  No atomics, no chain of dependent global
//           round trips between the evaluation and the next iteration.
//
// The arithmetic is the persistent kernel's (persistent.cuh) step for step:
// the same rule points in the same per-thread order, the same reduction
// trees, the same chunk and integral sums.  Results are bit-identical to
// it; only the schedule differs.  The point loop is specialised per round
// at compile time: a round whose points all lie in one generator set adds
// into that set's sum directly, other rounds test only the sets their
// points can fall in, and coordinates come from byte offsets into the
// coefficient table.
//
// Leftover boxes of integrals handed to phase 2 are written by all blocks
// right after the decision.  When the kernel leaves (every integral
// stopped, the next list is longer than the kernel's range, or the buffers
// must grow), all blocks write the next list in full and block 0 stores the
// integral states, so the host and the other drivers find a complete list.
#pragma once

#include "persistent.cuh"

namespace cubature {

// Longest list the replicated kernel keeps (32 * kRepChunks slots).
constexpr int kRepChunks = 128;
// Batches up to this many integrals can start from states passed with the
// launch (RepArgs::param_state) instead of an upload.
constexpr int kParamStates = 4;

struct RepArgs {
  EngineArgs base;  // states, tolerances, policy, capacities, leftovers
  double* lo[2];    // list buffers
  double* len[2];
  int* rid[2];
  double* avg[2];  // per-slot results, by iteration parity
  double* err[2];
  int* axis[2];
  int max_n;      // leave when the next list is longer than this
  int max_r;      // most regions a block evaluates at once (1, 2, 4 or 8)
  int iter_base;  // global index of the launch's first iteration
  int init;       // the current list is the initial grid, not yet written
  int divisions, per_integral, padded;
  const double* box;
  Control* host_out;  // mapped pinned copy of the control block and states
  int host_words;
  long long spin_limit;  // grid-barrier polls before giving up
  int hold_block;        // failure-detection tests: this block never arrives (-1: none)
  // mapped pinned word that block 0 sets to `seq` once host_out is
  // complete, so the host can stop waiting before the grid has retired
  // (null: the host synchronises the stream)
  unsigned* done;
  unsigned seq;
  // param_state != 0: the launch starts from host0, cur0 and ist0[0..nint)
  // instead of the control block and states in device memory (no upload
  // before the launch; nint <= kParamStates).  The barrier counters must
  // then be zero on entry, which the last block of every launch of this
  // kernel leaves them.
  int param_state;
  int cur0;
  IterState host0;
  IntegralState ist0[kParamStates];
};

namespace detail {

// First point of generator set k (k = 0..9; set 9 = end) in the rule's
// enumeration order: centre, sets 1-4 (2N points each), set 5 (axis pairs,
// 4 signs), set 6 (ordered pairs, 4 signs), set 7 (triples, 8 signs), set 8
// (the 2^N corners).
template <int N>
__host__ __device__ constexpr int set_begin(int k) {
  const int b5 = 1 + 8 * N, b6 = b5 + 2 * N * (N - 1), b7 = b6 + 4 * N * (N - 1);
  const int b8 = b7 + 4 * N * (N - 1) * (N - 2) / 3;
  return k <= 0 ? 0 : k <= 5 ? (k == 5 ? b5 : 1 + 2 * N * (k - 1)) : k == 6 ? b6 : k == 7 ? b7
         : k == 8 ? b8 : b8 + (1 << N);
}

// Generator set of point p (empty sets are skipped).
template <int N>
__host__ __device__ constexpr int set_of(int p) {
  int k = 0;
  while (k < 8 && p >= set_begin<N>(k + 1)) ++k;
  return k;
}

// The rule's points for the replicated kernel: per point, byte i of `ent`
// (i < N) is 8 * code_i, the byte offset of coordinate i's coefficient in
// ctab (codes as in PointTable), so x_i = fma(ctab[code_i], H_i, L_i) costs
// a byte extract, a shared load and one FMA.
template <int N>
struct ByteTable {
  static constexpr int kPoints = PointTable<N>::kPoints;
  uint2 ent[kPoints];
  double ctab[16];

  __device__ void fill(int tid, int nthreads) {
    if (tid < 16) {
      const double gen[5] = {kGenA1, kGenA2, kGenA3, kGenA4, kGenL};
      ctab[tid] = tid == 0 ? 0.5 : (tid <= 10 ? coef(gen[(tid - 1) >> 1], (tid - 1) & 1) : 0.0);
    }
    for (int p = tid; p < kPoints; p += nthreads) {
      const uint32_t codes = PointTable<N>::entry(p).x;
      uint32_t w[2] = {0u, 0u};
#pragma unroll
      for (int i = 0; i < N; ++i) w[i >> 2] |= (((codes >> (4 * i)) & 15u) * 8u) << (8 * (i & 3));
      ent[p] = make_uint2(w[0], w[1]);
    }
  }
};

template <int N, class F>
__device__ __forceinline__ double byte_point(const F& f, const ByteTable<N>& tb,
                                             const double (&L)[N], const double (&H)[N], int p) {
  const uint2 e = tb.ent[p];
  const char* cbase = reinterpret_cast<const char*>(tb.ctab);
  double x[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const unsigned off = __byte_perm(i < 4 ? e.x : e.y, 0u, 0x4440u | (unsigned)(i & 3));
    x[i] = fma(*reinterpret_cast<const double*>(cbase + off), H[i], L[i]);
  }
  return call_point(f, x, p);
}

// Compile-time plan of the rounds of a group of G threads (round r holds
// points r * G .. r * G + G - 1).
template <int N, int G>
struct RoundPlan {
  static constexpr int P = ByteTable<N>::kPoints;
  static constexpr int kRounds = (P + G - 1) / G;
  static constexpr int lo(int r) { return r * G; }
  static constexpr int hi(int r) { return (r + 1) * G < P ? (r + 1) * G - 1 : P - 1; }
  static constexpr bool full(int r) { return (r + 1) * G <= P; }
  static constexpr int kmin(int r) { return set_of<N>(lo(r)); }
  static constexpr int kmax(int r) { return set_of<N>(hi(r)); }
  // a full round inside one set whose points are not staged
  static constexpr bool plain(int r) {
    return r < kRounds && full(r) && kmin(r) == kmax(r) && lo(r) > 4 * N;
  }
  // end of the run of plain rounds of set kmin(r) starting at r
  static constexpr int run_end(int r) {
    int e = r;
    while (plain(e) && kmin(e) == kmin(r)) ++e;
    return e;
  }
};

// Rounds R.. of a group's point loop, adding into the per-thread set sums S
// in round order (the order of eval_region_group).  fst receives the
// values of points 0..4N (centre and sets 1-2) for the fourth difference.
template <int N, int G, int R>
struct Rounds {
  template <class F>
  __device__ __forceinline__ static void run(const F& f, const ByteTable<N>& tb,
                                             const double (&L)[N], const double (&H)[N], int t,
                                             bool active, double (&S)[kNumSets], double* fst) {
    using Plan = RoundPlan<N, G>;
    if constexpr (R < Plan::kRounds) {
      constexpr int k0 = Plan::kmin(R), k1 = Plan::kmax(R);
      if constexpr (Plan::plain(R)) {
        constexpr int E = Plan::run_end(R);
        if (active) {
#pragma unroll 2
          for (int r = R; r < E; ++r) S[k0] += byte_point(f, tb, L, H, r * G + t);
        }
        Rounds<N, G, E>::run(f, tb, L, H, t, active, S, fst);
      } else {
        const int p = Plan::lo(R) + t;
        if (active && (Plan::full(R) || p < Plan::P)) {
          const double fx = byte_point(f, tb, L, H, p);
          if constexpr (Plan::lo(R) <= 4 * N) {
            if (p <= 4 * N) fst[p] = fx;
          }
#pragma unroll
          for (int k = k0; k <= k1; ++k)
            S[k] += (p >= set_begin<N>(k) && p < set_begin<N>(k + 1)) ? fx : 0.0;
        }
        Rounds<N, G, R + 1>::run(f, tb, L, H, t, active, S, fst);
      }
    }
  }
};

template <int N>
struct RepSmem {
  ByteTable<N> tb;
  double red[8][kNumSets];
  double fstage[8][4 * N + 1];
  IntegralState ist[kSmallBatch];   // this block's copy of every state
  ChunkPartial part[kRepChunks];    // chunk partials of the evaluated list
  int excl[kRepChunks];             // active regions before each chunk, per integral
  int owner[kRepChunks];            // integral owning each chunk of the evaluated list
  int entered[kSmallBatch];         // handed to phase 2 by the last decision
  IterState next;                   // sizes of the next list
  double box[8][2 * N];             // region of each group: lower corner, widths
  RuleTables tables;                // stage_tables copy of the kernel's tables
  int slot_k[8];                    // its integral (-1: padding or past the end)
};

// One region evaluated by the G threads of group g (replicated kernel).
template <int N, int G, class F>
__device__ __forceinline__ RegionResult rep_eval_region(const F& f, const double (&L)[N],
                                                        const double (&H)[N], const RuleTables& T,
                                                        RepSmem<N>& sm, int g, int t, bool active) {
  double S[kNumSets];
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) S[k] = 0;
  Rounds<N, G, 0>::run(f, sm.tb, L, H, t, active, S, sm.fstage[g]);
  return group_finish<N, G>(S, H, T, sm.red, sm.fstage[g], t);
}

// Integral owning slot s of a list whose segments are in the states
// (segments are in integral order; stopped integrals hold empty segments).
__device__ __forceinline__ int rep_slot_owner(const IntegralState* ist, int nint, long long s) {
  int k = 0;
  for (int q = 1; q < nint; ++q)
    if (ist[q].seg_start <= s) k = q;
  return k;
}

// Dimension d of slot t of the initial grid (initial_box, one axis).
// Returns the slot's integral, or -1 for a padding slot.
template <int N>
__device__ __forceinline__ int initial_box_axis(long long t, int divisions, int per_integral,
                                                int padded, const double* box, int d, double& L,
                                                double& H) {
  const int k = (int)(t / padded);
  const int j = (int)(t % padded);
  if (j >= per_integral) return -1;
  int rem = j;
  for (int q = 0; q < d; ++q) rem /= divisions;
  const int id = rem % divisions;
  const double* bx = box ? box + (long long)k * 2 * N : nullptr;
  const double blo = bx ? bx[d] : 0.0;
  const double w = (bx ? bx[N + d] - bx[d] : 1.0) / divisions;
  L = blo + id * w;
  H = w;
  return k;
}

// The eval step: every slot of the list (n slots) by groups of G threads.
// mode: kSlotGrid (initial grid, computed and written), kSlotStored (read
// from the list), kSlotLazy (child of a parent in the previous list,
// computed and written).  The first warp of a group sets up the group's
// region (lane d: axis d) and hands it to the group through shared memory.
template <int N, int G, class Src>
__device__ __forceinline__ void rep_eval_step(const Src& src, const RuleTables& T,
                                              const RepArgs& p, RepSmem<N>& sm, int mode, int n,
                                              int cur, int par, int it) {
  constexpr int R = 256 / G;
  const int g = threadIdx.x / G, t = threadIdx.x % G;
  const int nint = p.base.nint;
  const long long cap = p.base.cap;
  double* dlo = p.lo[cur];
  double* dlen = p.len[cur];
  int* drid = p.rid[cur];
  const double* plo = p.lo[cur ^ 1];
  const double* plen = p.len[cur ^ 1];
  const int* pax = p.axis[par ^ 1];
  const long long ngroups = (long long)R * gridDim.x;
  for (long long base = 0; base < n; base += ngroups) {
    const long long slot = base + (long long)g * gridDim.x + blockIdx.x;
    const bool live = slot < n;
    if (t < 32) {
      const int d = t;
      int k = -1;
      double Ld = 0, Hd = 1;
      bool write = false;
      if (live && mode == kSlotGrid) {
        k = initial_box_axis<N>(slot, p.divisions, p.per_integral, p.padded, p.box,
                                d < N ? d : 0, Ld, Hd);
        write = true;
      } else if (live && mode == kSlotStored) {
        k = drid[slot];
        if (k >= 0 && d < N) {
          Ld = dlo[(long long)d * cap + slot];
          Hd = dlen[(long long)d * cap + slot];
        }
      } else if (live) {
        const int kk = rep_slot_owner(sm.ist, nint, slot);
        const IntegralState& is = sm.ist[kk];
        const int j = (int)(slot - is.seg_start);
        if (j < is.seg_count) {
          k = kk;
          const int pp = parent_slot(
              j >> 1, is.par_start >> 5, (is.par_count + 31) >> 5,
              [&](int q) { return sm.excl[q]; }, [&](int q) { return sm.part[q].mask; });
          const int ax = __ldcg(pax + pp);
          if (d < N) {
            const double l = __ldcg(plo + (long long)d * cap + pp);
            const double w = __ldcg(plen + (long long)d * cap + pp);
            if (d == ax) {
              const double h = w / 2;
              Ld = (j & 1) ? l + 1 * h : l;
              Hd = h;
            } else {
              Ld = l;
              Hd = w;
            }
          }
        }
        write = true;
      }
      if (d < N) {
        sm.box[g][d] = Ld;
        sm.box[g][N + d] = Hd;
        if (write && k >= 0) {
          dlo[(long long)d * cap + slot] = Ld;
          dlen[(long long)d * cap + slot] = Hd;
        }
      }
      if (d == 0) {
        sm.slot_k[g] = live ? k : -1;
        if (write) drid[slot] = k;
      }
    }
    __syncthreads();
    if (base == 0 && blockIdx.x == 0 && threadIdx.x == 0) trace_mark(p.base.ctl, it, 7);
    const int k = sm.slot_k[g];
    double L[N], H[N];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      L[d] = sm.box[g][d];
      H[d] = sm.box[g][N + d];
    }
    const auto f = src.get(k >= 0 ? k : 0);
    const RegionResult r = rep_eval_region<N, G>(f, L, H, T, sm, g, t, k >= 0);
    if (t == 0 && live) {
      p.avg[par][slot] = k >= 0 ? r.avg : 0.0;
      p.err[par][slot] = k >= 0 ? r.err : 0.0;
      p.axis[par][slot] = k >= 0 ? r.axis : 0;
    }
  }
}

// The decision after an evaluated list of n slots (parity par), taken by
// every block from the stored values and errors: chunk partials (the
// arithmetic of chunk_partial_warp), per-integral sums, stop decisions and
// the next segments (decide_scan_small), active prefix counts per chunk.
// Leaves the next list's sizes in sm.next and the states updated.
template <int N>
__device__ __forceinline__ void rep_decide(const RepArgs& p, RepSmem<N>& sm, int n, int par,
                                           int n_left_in, int it) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool tracer = blockIdx.x == 0 && threadIdx.x == 0;
  const int nint = p.base.nint;
  const int nc = n / 32;
  const double* avg = p.avg[par];
  const double* err = p.err[par];
  for (int c = threadIdx.x; c < nc; c += blockDim.x)
    sm.owner[c] = rep_slot_owner(sm.ist, nint, (long long)c * 32);
  __syncthreads();
  // a warp's chunks in batches of four: the loads of a batch are in flight
  // together
  constexpr int kBatch = 4;
  const int nw = blockDim.x / 32;
  for (int c0 = warp; c0 < nc; c0 += kBatch * nw) {
    double avb[kBatch], erb[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const long long i = (long long)(c0 + u * nw) * 32 + lane;
      const bool in = c0 + u * nw < nc;
      avb[u] = in ? __ldcg(avg + i) : 0.0;
      erb[u] = in ? __ldcg(err + i) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      const int c = c0 + u * nw;
      if (c >= nc) break;
      const int k = sm.owner[c];
      const double av = avb[u], er = erb[u];
      const bool act = er / max_err(av, sm.ist[k].epsrel, sm.ist[k].epsabs) > 1;
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
        ChunkPartial q;
        q.sum_avg = s0;
        q.sum_err = s1;
        q.fin_avg = s2;
        q.fin_err = s3;
        q.nactive = __popc(b);
        q.mask = b;
        sm.part[c] = q;
      }
    }
  }
  __syncthreads();
  if (tracer) trace_mark(p.base.ctl, it, 3);
  if (warp == 0) {
    const bool have = lane < nint;
    IntegralState& is = sm.ist[have ? lane : 0];
    const bool run = have && is.state == kStateRunning;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int m = 0;
    if (nint == 1) {
      // one integral: lane-strided sums in the order of decide_warp
      for (int base = 0; base < nc; base += 32) {
        const int c = base + lane;
        double v0 = 0, v1 = 0, v2 = 0, v3 = 0;
        int na = 0;
        if (c < nc) {
          const ChunkPartial& pc = sm.part[c];
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
        if (c < nc) sm.excl[c] = m + incl - na;
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
      const int c0 = is.seg_start / 32, ncq = (is.seg_count + 31) / 32;
      for (int q = 0; q < ncq; ++q) {
        const ChunkPartial& pc = sm.part[c0 + q];
        s0 += pc.sum_avg;
        s1 += pc.sum_err;
        s2 += pc.fin_avg;
        s3 += pc.fin_err;
        sm.excl[c0 + q] = m;
        m += pc.nactive;
      }
    }
    // The two timestamps around the decision are volatile asm, which the
    // compiler does not move code across.  Without them it interleaved the
    // decision with the sums above, and this warp's section took ~6 us per
    // iteration instead of ~1 us (8-D corner peak, measured on a B200).
    if (tracer) trace_mark(p.base.ctl, it, 1);
    bool entered = false;
    if (run) {
      decide_integral(is, s0, s1, s2, s3, m, p.base);
      entered = is.state == kStatePhase2;
    }
    if (tracer) trace_mark(p.base.ctl, it, 6);
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
      sm.entered[lane] = entered;
      is.par_start = is.seg_start;
      is.par_count = is.seg_count;
      is.next_start = in - vn;
      is.seg_start = in - vn;
      is.seg_count = nextc;
      if (vl > 0) {
        is.left_start = n_left_in + il - vl;
        is.left_count = vl;
      }
    }
    if (lane == 0) {
      IterState s;
      s.n = tot_n;
      s.n_running = nrun;
      s.n_left = n_left_in + tot_l;
      s.overflow = (tot_n > p.base.ncap) || (s.n_left > p.base.left_cap);
      s.handoff = tot_l > 0;
      sm.next = s;
    }
    if (tracer) trace_mark(p.base.ctl, it, 5);
  }
  __syncthreads();
}

// Children of the active regions of the evaluated list (n slots, buffer
// cur, parity par) for the integrals in `sel`: to the next list (buffer
// cur ^ 1, next segments) or, for integrals just handed to phase 2, to the
// leftover list.  Warp per chunk over the whole grid; reads the block's own
// masks and prefix counts.
template <int N>
__device__ __forceinline__ void rep_write_children(const RepArgs& p, const RepSmem<N>& sm, int n,
                                                   int cur, int par, bool to_next) {
  const int lane = threadIdx.x & 31;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  const long long cap = p.base.cap;
  const double* lo = p.lo[cur];
  const double* len = p.len[cur];
  const int* ax = p.axis[par];
  for (long long c = gwarp; c < n / 32; c += nwarp) {
    const int k = sm.owner[c];
    const IntegralState& is = sm.ist[k];
    const bool handed = sm.entered[k] != 0;
    const bool want = to_next ? (is.state == kStateRunning && is.seg_count > 0) : handed;
    const unsigned m = sm.part[c].mask;
    if (!want || !((m >> lane) & 1u)) continue;
    const int rank = sm.excl[c] + __popc(m & ((1u << lane) - 1u));
    const long long i = c * 32 + lane;
    double* dlo;
    double* dlen;
    int* drid;
    long long dcap, dst;
    if (to_next) {
      dlo = p.lo[cur ^ 1];
      dlen = p.len[cur ^ 1];
      drid = p.rid[cur ^ 1];
      dcap = cap;
      dst = is.seg_start + 2ll * rank;
    } else {
      dlo = p.base.left_lo;
      dlen = p.base.left_len;
      drid = p.base.left_rid;
      dcap = p.base.left_cap;
      dst = is.left_start + 2ll * rank;
    }
    const int a = __ldcg(ax + i);
#pragma unroll
    for (int d = 0; d < N; ++d) {
      const double l = __ldcg(lo + (long long)d * cap + i);
      const double w = __ldcg(len + (long long)d * cap + i);
      if (d == a) {
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
  if (to_next) {
    // padding ids at the end of every next segment
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long gt = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    for (int k = 0; k < p.base.nint; ++k) {
      const IntegralState& is = sm.ist[k];
      if (is.state != kStateRunning || is.seg_count == 0) continue;
      const int padded = (is.seg_count + 31) & ~31;
      for (long long j = is.seg_count + gt; j < padded; j += stride)
        p.rid[cur ^ 1][is.seg_start + j] = -1;
    }
  }
}

}  // namespace detail

template <int N, class Src>
__global__ void __launch_bounds__(256, 2) k_replicated(Src src, RuleTables T, RepArgs p) {
  __shared__ detail::RepSmem<N> sm;
  const int nint = p.base.nint;
  Control* ctl = p.base.ctl;
  sm.tb.fill(threadIdx.x, blockDim.x);
  detail::stage_tables(T, sm.tables);
  IterState st;
  int cur;
  if (p.param_state) {
    for (int q = threadIdx.x; q < nint; q += blockDim.x) sm.ist[q] = p.ist0[q];
    st = p.host0;
    cur = p.cur0;
    // the trace rows describe this launch only
    if (blockIdx.x == 0)
      for (int i = threadIdx.x; i < kTraceIters * kTraceSlots; i += blockDim.x) ctl->trace[i] = 0;
  } else {
    for (int q = threadIdx.x; q < nint; q += blockDim.x) sm.ist[q] = p.base.ist[q];
    volatile IterState* v = &ctl->host;
    st.n = v->n;
    st.n_running = v->n_running;
    st.n_left = v->n_left;
    cur = ctl->cur;
  }
  st.overflow = 0;
  st.handoff = 0;
  __syncthreads();
  const bool tracer = blockIdx.x == 0 && threadIdx.x == 0;
  const long long ncap = p.base.ncap;
  const bool ref = p.base.policy == kPolicyReference;
  int reason = 0;
  unsigned barriers = 0;
  int it = 0;

  // the starting list: leave before evaluating it when it is out of range
  if (st.n_running == 0 || st.n == 0)
    reason = kExitDone;
  else if (st.n > p.max_n)
    reason = kExitLarge;
  else if (2ll * st.n + 32ll * nint > ncap || (ref && (long long)st.n_left + 2ll * st.n > p.base.left_cap))
    reason = kExitCapacity;
  if (reason) {
    if (p.init && reason != kExitDone) {
      // write the initial grid the kernel would have evaluated
      const long long stride = (long long)gridDim.x * blockDim.x;
      for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < st.n; s += stride) {
        double L[N], H[N];
        const int k = initial_box<N>(s, p.divisions, p.per_integral, p.padded, p.box, L, H);
        if (k >= 0) {
#pragma unroll
          for (int d = 0; d < N; ++d) {
            p.lo[cur][(long long)d * p.base.cap + s] = L[d];
            p.len[cur][(long long)d * p.base.cap + s] = H[d];
          }
        }
        p.rid[cur][s] = k;
      }
    }
  } else {
    int mode = p.init ? kSlotGrid : kSlotStored;
    for (;; ++it) {
      const int par = it & 1;
      if (tracer) trace_mark(ctl, it, 0);
      const long long per_block = (st.n + gridDim.x - 1) / gridDim.x;
      const int r = per_block <= 1 ? 1 : (per_block <= 2 ? 2 : (per_block <= 4 ? 4 : 8));
      switch (r < p.max_r ? r : p.max_r) {
        case 1: detail::rep_eval_step<N, 256>(src, sm.tables, p, sm, mode, st.n, cur, par, it); break;
        case 2: detail::rep_eval_step<N, 128>(src, sm.tables, p, sm, mode, st.n, cur, par, it); break;
        case 4: detail::rep_eval_step<N, 64>(src, sm.tables, p, sm, mode, st.n, cur, par, it); break;
        default: detail::rep_eval_step<N, 32>(src, sm.tables, p, sm, mode, st.n, cur, par, it); break;
      }
      if (tracer) trace_mark(ctl, it, 4);
      ++barriers;
      if (!detail::grid_barrier(ctl, barriers * gridDim.x, p.spin_limit,
                                (int)blockIdx.x != p.hold_block)) {
        reason = kExitTimeout;
        break;
      }
      if (tracer) trace_mark(ctl, it, 2);
      detail::rep_decide<N>(p, sm, st.n, par, st.n_left, it);
      const IterState nx = sm.next;
      if (nx.handoff) detail::rep_write_children<N>(p, sm, st.n, cur, par, false);
      if (nx.n_running == 0 || nx.n == 0)
        reason = kExitDone;
      else if (nx.n > p.max_n)
        reason = kExitLarge;
      else if (2ll * nx.n + 32ll * nint > ncap ||
               (ref && (long long)nx.n_left + 2ll * nx.n > p.base.left_cap))
        reason = kExitCapacity;
      if (reason) {
        if (reason != kExitDone) detail::rep_write_children<N>(p, sm, st.n, cur, par, true);
        cur ^= 1;
        st = nx;
        ++it;
        break;
      }
      cur ^= 1;
      st = nx;
      mode = kSlotLazy;
    }
  }
  if (blockIdx.x == 0) {
    for (int q = threadIdx.x; q < nint; q += blockDim.x) p.base.ist[q] = sm.ist[q];
    if (threadIdx.x == 0) {
      ctl->cur = cur;
      IterState h = st;
      h.overflow = 0;
      h.handoff = 0;
      ctl->host = h;
      ctl->exit_reason = reason;
      ctl->iters_done = p.iter_base + it;
    }
    if (p.host_out) {
      __syncthreads();
      const unsigned long long* s = reinterpret_cast<const unsigned long long*>(ctl);
      unsigned long long* dst = reinterpret_cast<unsigned long long*>(p.host_out);
      for (int i = threadIdx.x; i < p.host_words; i += blockDim.x) dst[i] = s[i];
      if (p.done) {
        // the block's stores to host_out, then the sequence number, at
        // system scope
        __syncthreads();
        if (threadIdx.x == 0) {
          __threadfence_system();
          asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p.done), "r"(p.seq) : "memory");
        }
      }
    }
  }
  // The last block to leave zeroes the barrier counters for the next launch
  // (every other block has passed its last barrier by then; block 0 has
  // stored the control block first).
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&ctl->exit_count, 1u) == gridDim.x - 1) {
      ctl->bar_count = 0;
      ctl->timeout = 0;
      ctl->exit_count = 0;
    }
  }
}

}  // namespace cubature
