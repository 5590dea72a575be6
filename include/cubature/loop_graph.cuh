// loop_graph.cuh -- the multi-launch iteration as a device-driven loop.
//
// While the region list is long (beyond the persistent kernels' range), an
// iteration is a chain of launches: the rule over the list (k_eval), the
// chunk partials, the per-integral decisions, the scan, the split and the
// hand-over (engine_kernels.cuh).  The host used to launch that chain once
// per iteration and read the control block back in between, as the
// reference's loop does with its blocking copies (GPUKernelquad.cu:609-668).
// Here the chain is the body of a CUDA graph's conditional WHILE node:
//
//   bind     reads the list length and buffer parity from the control block,
//            binds the iteration's arguments and picks the rule kernel's
//            lanes per region (a SWITCH node over three k_eval variants);
//   eval, partials, decide, scan, split, advance
//            the multi-launch kernels, reading their arguments from device
//            memory instead of launch parameters;
//   test     continues while integrals are running, the next list fits the
//            buffers and is still longer than the persistent kernels take.
//
// One graph launch runs iterations until the host has to act (grow the
// buffers, hand over to a persistent kernel, stop).  The kernels and their
// order are those of the host-driven loop, so the results are identical.
#pragma once

#include "engine_kernels.cuh"

namespace cubature {

// Arguments of the loop in device memory, written by the host before each
// launch of the loop graph.
template <class Src>
struct LoopArgs {
  EngineArgs base[2];  // lists bound for buffer parity 0 and 1 (n unset)
  EngineArgs it;       // this iteration's binding (k_loop_bind)
  Src src;
  long long cap;       // list capacity (and the caller's limit): 2n + 32 nint must fit
  long long left_cap;  // reference policy: n_left + 4n + 1 leftovers must fit
  int ref_policy;
  int hand_back;    // leave when the next list is at most this long
  int k1_min;       // lists at least this long: one lane per region
  int k8_min;       // at least this long: 8 lanes per region (else 32)
  int forced_lanes;  // 1, 8 or 32: always that many (0: by length)
  int pad;
  // results of the launch
  unsigned long long regions;  // regions evaluated
  long long peak_need;         // largest 2n + 32 nint met
  int iterations;
  int pad2;
};

// Lanes per region of the multi-launch rule kernel for a list of n slots
// (0, 1, 2: 1, 8, 32 lanes).
template <class Src>
__device__ __forceinline__ int loop_lane_case(const LoopArgs<Src>& la, long long n) {
  const int k = la.forced_lanes ? la.forced_lanes : (n >= la.k1_min ? 1 : (n >= la.k8_min ? 8 : 32));
  return k == 1 ? 0 : (k == 8 ? 1 : 2);
}

template <class Src>
__global__ void k_loop_bind(LoopArgs<Src>* la, cudaGraphConditionalHandle lanes) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Control* ctl = la->base[0].ctl;
  const int cur = ctl->cur;
  const long long n = ctl->host.n;
  EngineArgs a = la->base[cur];
  a.n = (int)n;
  la->it = a;
  la->regions += (unsigned long long)n;
  la->iterations += 1;
  const long long need = 2 * n + 32ll * a.nint;
  if (need > la->peak_need) la->peak_need = need;
  cudaGraphSetConditional(lanes, (unsigned)loop_lane_case(*la, n));
}

// The iteration's arguments and integrand source in shared memory (one
// copy per block).
template <class Src>
struct LoopShared {
  EngineArgs a;
  Src src;
};

template <class Src>
__device__ __forceinline__ void loop_load(const LoopArgs<Src>* la, LoopShared<Src>& sh) {
  static_assert(sizeof(EngineArgs) % 4 == 0, "copied as 4-byte words");
  const unsigned* s0 = reinterpret_cast<const unsigned*>(&la->it);
  unsigned* d0 = reinterpret_cast<unsigned*>(&sh.a);
  for (int i = threadIdx.x; i < (int)(sizeof(EngineArgs) / 4); i += blockDim.x) d0[i] = s0[i];
  const unsigned char* s2 = reinterpret_cast<const unsigned char*>(&la->src);
  unsigned char* d2 = reinterpret_cast<unsigned char*>(&sh.src);
  for (int i = threadIdx.x; i < (int)sizeof(Src); i += blockDim.x) d2[i] = s2[i];
}

// The other loop kernels copy the iteration's arguments into registers
// (every thread reads the same words, served by L1): from shared memory the
// compiler would have to reread them after every global store, which might
// alias them.
//
// The rule tables come as a launch parameter (fixed per dimension when the
// graph is built): the rule's finish then reads them as constant operands,
// as k_eval does; from shared memory the one-lane-per-region variant
// spilled.  Blocks beyond the list's end leave before loading anything.
template <int N, int K, class Src>
__global__ void __launch_bounds__(256, CUB_EVAL_MIN_BLOCKS) k_loop_eval(const LoopArgs<Src>* la,
                                                                        RuleTables T) {
  constexpr int kGroups = 256 / K;
  if ((long long)blockIdx.x * kGroups >= la->it.n) return;
  __shared__ detail::ItemTable<N> tab;
  __shared__ LoopShared<Src> sh;
  if (threadIdx.x == 0) tab.fill();
  loop_load(la, sh);
  __syncthreads();
  const int lane = threadIdx.x % K;
  const unsigned gmask =
      (K == 32) ? 0xffffffffu : (((1u << K) - 1u) << ((threadIdx.x & 31) & ~(K - 1)));
  const EngineArgs& a = sh.a;
  for (long long slot = (long long)blockIdx.x * kGroups + threadIdx.x / K; slot < a.n;
       slot += (long long)gridDim.x * kGroups)
    detail::eval_slot<N, K>(sh.src, T, a, slot, lane, gmask, tab);
}

template <class Src>
__global__ void __launch_bounds__(256) k_loop_partials(const LoopArgs<Src>* la) {
  const EngineArgs a = la->it;
  const long long nchunk = (a.n + 31) / 32;
  for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32; c < nchunk;
       c += (long long)gridDim.x * blockDim.x / 32)
    detail::chunk_partial_warp(a, c, threadIdx.x & 31);
}

template <class Src>
__global__ void __launch_bounds__(256) k_loop_decide(const LoopArgs<Src>* la) {
  const EngineArgs a = la->it;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) / 32; k < a.nint;
       k += gridDim.x * blockDim.x / 32)
    detail::decide_warp(a, k, threadIdx.x & 31);
}

template <class Src>
__global__ void k_loop_scan(const LoopArgs<Src>* la) {
  const EngineArgs a = la->it;
  detail::scan_warp(a, a.ctl->host.n_left, &a.ctl->host, threadIdx.x & 31);
}

template <int N, class Src>
__global__ void __launch_bounds__(256) k_loop_split(const LoopArgs<Src>* la) {
  const EngineArgs a = la->it;
  if (a.ctl->host.overflow) return;
  const long long nchunk = (a.n + 31) / 32;
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) / 32;
  const long long nwarp = (long long)gridDim.x * blockDim.x / 32;
  for (long long c = gwarp; c < nchunk; c += nwarp)
    detail::split_chunk_warp<N>(a, c, threadIdx.x & 31);
}

template <class Src>
__global__ void k_loop_advance(const LoopArgs<Src>* la) {
  const EngineArgs a = la->it;
  if (a.ctl->host.overflow) return;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < a.nint; k += gridDim.x * blockDim.x)
    detail::finish_integral(a, k);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.ctl->cur ^= 1;
    a.ctl->iters_done += 1;
  }
}

// The WHILE node's test after an iteration: another iteration when
// integrals are running, the scan did not overflow, the next list fits the
// buffers (and, under the reference policy, the leftover buffer) and it is
// longer than the persistent kernels take.
template <class Src>
__global__ void k_loop_test(const LoopArgs<Src>* la, cudaGraphConditionalHandle again) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const IterState nx = la->it.ctl->host;
  const long long n = nx.n;
  bool more = nx.n_running > 0 && n > 0 && !nx.overflow && n > la->hand_back &&
              2 * n + 32ll * la->it.nint <= la->cap;
  if (la->ref_policy) more = more && (long long)nx.n_left + 4 * n + 1 <= la->left_cap;
  cudaGraphSetConditional(again, more ? 1u : 0u);
}

}  // namespace cubature
