// phase2_kernels.cuh -- depth-first refinement of leftover boxes.
//
// The reference's second phase (BLOCK_INTEGRATE_GPU_PHASE2,
// quad/GPUquad/GPUQuadPhases.cu:424-536) refines every box left over by the
// first phase on its own: serial Cuhre with the box's own tolerance
// (ERR <= max(epsrel |RESULT|, epsabs)) and at most 2048 bisections.
//
// Re-design for sm_100a: one warp per leftover box, persistent warps pulling
// boxes from an atomic counter.  Each step bisects the box's exact maximum
// error subregion (a binary heap kept by lane 0, each entry holding the
// subregion's error beside its index), and the two children are
// evaluated in parallel by the two 16-lane halves of the warp: rule point
// p on lane p % 16, in rounds whose generator sets are fixed at compile
// time (the replicated kernel's coefficient-code table and round plan), so
// the 16 lanes carry the same number of points.  Subregions
// live in a per-warp slab of global memory preallocated by the host, so
// there is no device malloc and the footprint is fixed by the grid size.
// Every loop is bounded (at most max_regions steps per box).
#pragma once

#include "engine_kernels.cuh"
#include "replicated.cuh"

namespace cubature {

struct LeftoverResult {
  double value, error;
  int nregions, failed;
};

// One subregion of a leftover box, in the box's local [0,1]^N coordinates.
template <int N>
struct P2Region {
  double avg, err;
  int axis, div;
  double lo[N], hi[N];
};

// Heap entry: a subregion's error (the key) beside its pool index, so that
// a heap level costs one read, not a read of the index and a dependent read
// of the subregion.
struct P2HeapEnt {
  double err;
  int idx;
  int pad;
};

struct Phase2Args {
  const double* left_lo;  // [N][left_cap]
  const double* left_len;
  const int* left_rid;
  long long left_cap;
  int n_left;
  int max_regions;  // bisections per box (MAX_GLOBALPOOL_SIZE, quad.h:9)
  void* slab;       // per-warp pools: nwarps * (max_regions + 2) regions
  P2HeapEnt* heap;  // per-warp heaps: nwarps * (max_regions + 2) entries
  int* next_box;    // work counter
  LeftoverResult* out;
  const IntegralState* ist;
  // 0: the counter walks the leftover list in its own order.  h > 0: the
  // list holds the two children of h regions adjacently (2j, 2j + 1), and
  // the counter walks it in the reference's order, first children then
  // second children (position q < h is box 2q, q >= h is box 2(q - h) + 1),
  // so that a contiguous range of positions is the reference's
  // multi-device share (GPUKernelquad.cu:759-768)
  int pair_half;
};

namespace detail {

// Max-heap on the error, sifting with a hole: the same comparisons, and so
// the same order, as swapping the entries level by level.
__device__ __forceinline__ void heap_push(P2HeapEnt* heap, int& hn, int idx, double err) {
  int i = hn++;
  const P2HeapEnt e{err, idx, 0};
  while (i > 0) {
    const int p = (i - 1) / 2;
    const P2HeapEnt pe = heap[p];
    if (pe.err >= e.err) break;
    heap[i] = pe;
    i = p;
  }
  heap[i] = e;
}

__device__ __forceinline__ int heap_pop(P2HeapEnt* heap, int& hn) {
  const int top = heap[0].idx;
  const P2HeapEnt e = heap[--hn];
  int i = 0;
  for (;;) {
    const int l = 2 * i + 1, r = l + 1;
    int m = i;
    double km = e.err;
    if (l < hn) {
      const double kl = heap[l].err;
      if (kl > km) {
        m = l;
        km = kl;
      }
    }
    if (r < hn && heap[r].err > km) m = r;
    if (m == i) break;
    heap[i] = heap[m];
    i = m;
  }
  heap[i] = e;
  return top;
}

// The same heap with keys and indices in separate arrays (shared memory:
// 12 bytes an entry).  Same comparisons in the same order as heap_push /
// heap_pop, so the same bisection order.
__device__ __forceinline__ void heap_push_soa(double* key, int* id, int& hn, int idx, double err) {
  int i = hn++;
  while (i > 0) {
    const int p = (i - 1) / 2;
    const double pk = key[p];
    if (pk >= err) break;
    key[i] = pk;
    id[i] = id[p];
    i = p;
  }
  key[i] = err;
  id[i] = idx;
}

__device__ __forceinline__ int heap_pop_soa(double* key, int* id, int& hn) {
  const int top = id[0];
  --hn;
  const double ek = key[hn];
  const int ei = id[hn];
  int i = 0;
  for (;;) {
    const int l = 2 * i + 1, r = l + 1;
    int m = i;
    double km = ek;
    if (l < hn) {
      const double kl = key[l];
      if (kl > km) {
        m = l;
        km = kl;
      }
    }
    if (r < hn && key[r] > km) m = r;
    if (m == i) break;
    key[i] = key[m];
    id[i] = id[m];
    i = m;
  }
  key[i] = ek;
  id[i] = ei;
  return top;
}

// A warp's heap: in the global slab (kShared = false) or in the block's
// dynamic shared memory (keys of the block's four warps, then their
// indices).
template <bool kShared>
struct P2Heap;

template <>
struct P2Heap<false> {
  P2HeapEnt* h;
  __device__ __forceinline__ void push(int& hn, int idx, double err) { heap_push(h, hn, idx, err); }
  __device__ __forceinline__ int pop(int& hn) { return heap_pop(h, hn); }
};

template <>
struct P2Heap<true> {
  double* key;
  int* id;
  __device__ __forceinline__ void push(int& hn, int idx, double err) {
    heap_push_soa(key, id, hn, idx, err);
  }
  __device__ __forceinline__ int pop(int& hn) { return heap_pop_soa(key, id, hn); }
};

// Dynamic shared memory of one block of the shared-heap phase-2 kernel.
inline size_t phase2_heap_smem(int max_regions) {
  return (size_t)4 * (size_t)(max_regions + 2) * (sizeof(double) + sizeof(int));
}

// Evaluate subregion `reg` of box (BL, BW) with the 16 lanes of a half
// warp, table-driven: round r holds points 16 r .. 16 r + 15 (Rounds<N,
// 16>), the lanes' set sums are combined by shuffles within the half, and
// the fourth difference comes from the staged centre and set-1/2 values
// (fst, one staging row per half warp).  Every lane of the half returns
// the result.
template <int N, class F>
__device__ __forceinline__ RegionResult eval_sub_tab(const F& f, const double (&BL)[N],
                                                     const double (&BW)[N], const P2Region<N>& reg,
                                                     int hlane, unsigned hmask,
                                                     const ByteTable<N>& tb, double* fst,
                                                     const RuleTables& T) {
  double L[N], H[N];
  int widest = 0;
  double wmax = 0;
#pragma unroll
  for (int d = 0; d < N; ++d) {
    L[d] = fma(reg.lo[d], BW[d], BL[d]);
    H[d] = (reg.hi[d] - reg.lo[d]) * BW[d];
    const double w = reg.hi[d] - reg.lo[d];
    if (w > wmax) {  // widest local side (GPUQuadSample.cu:118-125)
      wmax = w;
      widest = d;
    }
  }
  RegionSums rs;
#pragma unroll
  for (int k = 0; k < kNumSets; ++k) rs.S[k] = 0;
  Rounds<N, 16, 0>::run(f, tb, L, H, hlane, true, rs.S, fst);
#pragma unroll
  for (int off = 8; off > 0; off >>= 1) {
#pragma unroll
    for (int k = 0; k < kNumSets; ++k) rs.S[k] += __shfl_xor_sync(hmask, rs.S[k], off);
  }
  __syncwarp(hmask);
  // fourth difference per axis (lanes 0..N-1 of the half), then the
  // largest, the smallest axis on ties
  rs.best = 0;
  rs.axis = -1;
  if (hlane < N) {
    const double ratio = T.ratio;
    const double base = __dmul_rn(__dmul_rn(fst[0], 2.0), __dadd_rn(1.0, -ratio));
    const int d = hlane;
    rs.best = fabs(__dadd_rn(__dadd_rn(base, __dmul_rn(ratio, __dadd_rn(fst[1 + 2 * d], fst[2 + 2 * d]))),
                             -__dadd_rn(fst[1 + 2 * N + 2 * d], fst[2 + 2 * N + 2 * d])));
    rs.axis = rs.best > 0 ? d : -1;
  }
#pragma unroll
  for (int off = 8; off > 0; off >>= 1) {
    const double ob = __shfl_xor_sync(hmask, rs.best, off);
    const int oa = __shfl_xor_sync(hmask, rs.axis, off);
    const bool take = (ob > rs.best) || (ob == rs.best && oa >= 0 && (rs.axis < 0 || oa < rs.axis));
    if (take) {
      rs.best = ob;
      rs.axis = oa;
    }
  }
  __syncwarp(hmask);  // fst is rewritten by the next evaluation
  double jac = 1;
#pragma unroll
  for (int d = 0; d < N; ++d) jac = __dmul_rn(jac, H[d]);
  return finish_region<N>(rs, T, jac, widest);
}

}  // namespace detail

// kShared = false: three blocks (12 warps) per SM, each warp's heap in the
// global slab -- each warp refines its box serially, so warps in flight
// hide the latency of the heap and the rule; the register cap this sets
// costs a few spilled words.  kShared = true: the heaps in shared memory
// (phase2_heap_smem bytes a block, two blocks per SM at the default 2048
// bisections), so a heap level costs a shared-memory access instead of an
// L2 round trip.
template <int N, class Src, bool kShared = false>
__global__ void __launch_bounds__(128, kShared ? 2 : 3) k_phase2(Src src, RuleTables T,
                                                                 Phase2Args a) {
  __shared__ detail::ByteTable<N> tb;
  __shared__ double fstage[8][4 * N + 1];  // per half warp
  extern __shared__ double p2_dyn[];
  tb.fill(threadIdx.x, blockDim.x);
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int half = lane >> 4, hlane = lane & 15;
  const unsigned hmask = half ? 0xffff0000u : 0x0000ffffu;
  double* fst = fstage[threadIdx.x >> 4];
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const int stride = a.max_regions + 2;
  P2Region<N>* pool = reinterpret_cast<P2Region<N>*>(a.slab) + gwarp * stride;
  detail::P2Heap<kShared> heap;
  if constexpr (kShared) {
    const int w = threadIdx.x >> 5;
    heap.key = p2_dyn + (size_t)w * stride;
    heap.id = reinterpret_cast<int*>(p2_dyn + (size_t)4 * stride) + (size_t)w * stride;
  } else {
    heap.h = a.heap + gwarp * stride;
  }

  for (;;) {
    int box = 0;
    if (lane == 0) box = atomicAdd(a.next_box, 1);
    box = __shfl_sync(0xffffffffu, box, 0);
    if (box >= a.n_left) break;
    if (a.pair_half) box = box < a.pair_half ? 2 * box : 2 * (box - a.pair_half) + 1;
    const int k = a.left_rid[box];
    const IntegralState& is = a.ist[k];
    const double epsrel = is.epsrel, epsabs = is.epsabs;
    double BL[N], BW[N];
#pragma unroll
    for (int d = 0; d < N; ++d) {
      BL[d] = a.left_lo[(long long)d * a.left_cap + box];
      BW[d] = a.left_len[(long long)d * a.left_cap + box];
    }
    const auto f = src.get(k);

    // the whole box as the first subregion (INIT_REGION_POOL, :110-182)
    P2Region<N> r0;
#pragma unroll
    for (int d = 0; d < N; ++d) { r0.lo[d] = 0; r0.hi[d] = 1; }
    r0.div = 0;
    {
      // both halves evaluate it; half 0's result is used
      const detail::RegionResult rr = detail::eval_sub_tab<N>(f, BL, BW, r0, hlane, hmask, tb, fst, T);
      r0.avg = rr.avg;
      r0.err = rr.err;
      r0.axis = rr.axis;
    }
    int hn = 0, used = 1;
    double ERR = r0.err, RESULT = r0.avg;
    if (lane == 0) {
      pool[0] = r0;
      heap.push(hn, 0, r0.err);
    }
    __syncwarp();
    int nreg = 1;
    for (; nreg <= a.max_regions &&
           (nreg == 1 || ERR > detail::max_err(RESULT, epsrel, epsabs));
         ++nreg) {
      int pi = 0;
      if (lane == 0) pi = heap.pop(hn);
      pi = __shfl_sync(0xffffffffu, pi, 0);
      __syncwarp();
      const P2Region<N> parent = pool[pi];
      P2Region<N> child = parent;
      const int ax = parent.axis;
      const double mid = 0.5 * (parent.lo[ax] + parent.hi[ax]);
      child.div = parent.div + 1;
#pragma unroll
      for (int d = 0; d < N; ++d) {
        if (d == ax) {
          if (half == 0) child.hi[d] = mid;
          else child.lo[d] = mid;
        }
      }
      const detail::RegionResult rr = detail::eval_sub_tab<N>(f, BL, BW, child, hlane, hmask, tb, fst, T);
      const double avgR = __shfl_sync(0xffffffffu, rr.avg, 16);
      const double errR0 = __shfl_sync(0xffffffffu, rr.err, 16);
      const int axR = __shfl_sync(0xffffffffu, rr.axis, 16);
      if (lane == 0) {
        // Cuhre error refinement (GPUQuadPhases.cu:498-515)
        double errL = rr.err, errR = errR0;
        const double diff = fabs(.25 * (rr.avg + avgR - parent.avg));
        const double e = errL + errR;
        if (e > 0) {
          const double c = 1 + 2 * diff / e;
          errL *= c;
          errR *= c;
        }
        errL += diff;
        errR += diff;
        ERR += errL + errR - parent.err;
        RESULT += rr.avg + avgR - parent.avg;
        P2Region<N> left = parent, right = parent;
        left.div = right.div = parent.div + 1;
#pragma unroll
        for (int d = 0; d < N; ++d) {
          if (d == ax) {
            left.hi[d] = mid;
            right.lo[d] = mid;
          }
        }
        left.avg = rr.avg;
        left.err = errL;
        left.axis = rr.axis;
        right.avg = avgR;
        right.err = errR;
        right.axis = axR;
        pool[pi] = left;
        pool[used] = right;
        heap.push(hn, pi, errL);
        heap.push(hn, used, errR);
      }
      ++used;
      ERR = __shfl_sync(0xffffffffu, ERR, 0);
      RESULT = __shfl_sync(0xffffffffu, RESULT, 0);
      __syncwarp();
    }
    if (lane == 0) {
      int failed = ERR > detail::max_err(RESULT, epsrel, epsabs);
      if (ERR > 1e10) {  // GPUQuadPhases.cu:519-527
        RESULT = 0.0;
        ERR = 0.0;
        failed = 1;
      }
      LeftoverResult o;
      o.value = RESULT;
      o.error = ERR;
      o.nregions = nreg;
      o.failed = failed;
      a.out[box] = o;
    }
    __syncwarp();
  }
}

// Per-integral sums of the phase-2 results, one warp per integral, and the
// final status (GPUKernelquad.cu:870-892, GPUquad.h:713-714).
// final_test: apply the reference's status test (GPUquad.h:713) to the
// integral's total; 0 for a share of the boxes (the combined total is
// tested by the caller), whose status is then its failed-box count.
static __global__ void k_phase2_collect(IntegralState* ist, int nint, const LeftoverResult* res,
                                        int npoints, int final_test) {
  const int lane = threadIdx.x & 31;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) / 32; k < nint;
       k += gridDim.x * blockDim.x / 32) {
    IntegralState& is = ist[k];
    if (is.state != kStatePhase2) continue;
    double v = 0, e = 0;
    unsigned long long nr = 0, nb = 0;
    int nf = 0;
    for (int j = lane; j < is.left_count; j += 32) {
      const LeftoverResult r = res[is.left_start + j];
      v += r.value;
      e += r.error;
      nr += (unsigned long long)r.nregions;
      nb += r.nregions > 0 ? 1ull : 0ull;  // boxes refined here (all, unless sharded)
      nf += r.failed;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      v += __shfl_xor_sync(0xffffffffu, v, off);
      e += __shfl_xor_sync(0xffffffffu, e, off);
      nr += __shfl_xor_sync(0xffffffffu, nr, off);
      nb += __shfl_xor_sync(0xffffffffu, nb, off);
      nf += __shfl_xor_sync(0xffffffffu, nf, off);
    }
    if (lane == 0) {
      const unsigned long long n = nb;
      is.value += v;
      is.error += e;
      is.nregions += nr;
      is.neval += (nr - n) * (unsigned long long)npoints * 2ull + n * (unsigned long long)npoints;
      is.status = nf;
      if (final_test && is.error <= detail::max_err(is.value, is.epsrel, is.epsabs)) is.status = 0;
      if (!isfinite(v) || !isfinite(e)) is.status = kStatusNonFinite;
      is.state = kStateDone;
    }
  }
}

}  // namespace cubature
