// engine.cuh -- host driver of the breadth-first + depth-first engine.
//
// Header-only so user code can integrate its own device functors (the
// reference's integrate(..., F* f, ...) takes any functor type,
// quad/GPUquad/GPUquad.h:611-620); the prebuilt library instantiates it for
// the built-in families.
//
// Two drivers share the device state (region lists, per-integral states,
// control block):
//   * the persistent cooperative kernel (persistent.cuh) runs whole
//     stretches of iterations while the region list is short, with no host
//     round trip;
//   * the multi-launch driver runs one iteration per round of launches
//     (thread-per-region rule kernel) once the list is long, where launch
//     latency is negligible against the rule kernel.
// The host switches between them at iteration boundaries.  All device
// memory lives in a Workspace that grows geometrically and is reused across
// calls (the reference mallocs and frees ~10 buffers per iteration,
// GPUKernelquad.cu:357-605).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "engine_kernels.cuh"
#include "persistent.cuh"
#include "loop_graph.cuh"
#include "phase2_kernels.cuh"
#include "replicated.cuh"
#include "rule9.hpp"

namespace cubature {

struct Options {
  int policy = kPolicyReference;  // two-phase reference semantics
  int phase1_cap = 1 << 14;       // FIRST_PHASE_MAXREGIONS (quad.h:21)
  int max_iters = 100;            // phase-1 iterations (GPUKernelquad.cu:631)
  int phase2_max_regions = 2048;  // MAX_GLOBALPOOL_SIZE (quad.h:9)
  long long max_slots = 0;        // region-list capacity; 0 = from free device memory
  int lanes = 0;                  // lanes per region in the multi-launch rule kernel; 0 auto
  int persistent = 1;             // use the persistent kernel for short lists
  int persistent_max_n = 0;       // list length where it hands over; 0 auto
  int persistent_max_r = 0;       // most regions per block in the persistent kernel (1,2,4,8); 0 = 8
  int replicated = 1;             // small batches: the replicated-decision kernel for short lists
  int device_loop = 1;            // long lists: iterations driven by a conditional graph loop
  long long barrier_spins = 0;    // grid-barrier polls before a timeout; 0 = kBarrierSpins
  int hold_block = -1;            // tests: this block never arrives at a grid barrier
  // Second phase on share shard_rank of shard_world of the leftover boxes
  // (the reference's multi-device cut, GPUKernelquad.cu:759-768).  The
  // results then hold only the share's depth-first sums, regions and
  // failed boxes; Workspace::phase1_out receives the first phase's.
  int shard_rank = 0;
  int shard_world = 1;
};

struct Result {
  double value, error;
  unsigned long long nregions, neval;
  int status;      // reference errorFlag: 0 = converged
  int iterations;  // phase-1 iterations
  int state;       // IntegralStateCode at exit
  int pad;
};

// Error codes of the host layer (negative; positive values are numerical
// statuses of individual integrals).
enum ErrorCode : int {
  kOk = 0,
  kErrInvalid = -1,
  kErrCuda = -2,
  kErrCapacity = -3,
  kErrUnsupported = -4,
  kErrTimeout = -5,
};

// Counters of the work a context has launched (reset by the caller).
struct Stats {
  double ms_eval = 0;            // device time of the multi-launch rule kernel (timing on)
  long long eval_launches = 0;   // multi-launch rule-kernel launches
  long long launches = 0;        // all kernel launches
  long long regions_evaluated = 0;
  long long iterations = 0;      // breadth-first iterations
  long long phase2_boxes = 0;    // leftover boxes refined depth-first
  double ms_phase2 = 0;          // device time of the phase-2 kernel (timing on)
  long long h2d_bytes = 0;       // host-to-device copies issued
  long long d2h_bytes = 0;       // device-to-host copies issued
  double ms_persistent = 0;      // device time of the persistent kernel (timing on)
  long long persistent_launches = 0;
  long long persistent_iterations = 0;
  long long replicated_launches = 0;  // persistent launches of the replicated kernel
  long long device_loops = 0;         // launches of the device-driven loop graph
  long long persistent_regions = 0;   // regions evaluated by both persistent kernels
};

inline const char* state_name(int s) {
  switch (s) {
    case kStateRunning: return "running";
    case kStateDone: return "done";
    case kStatePhase2: return "phase2";
    case kStateCapacity: return "capacity";
  }
  return "?";
}

inline long long auto_max_slots(int ndim, int policy);

class Workspace {
 public:
  explicit Workspace(int device = 0) : device_(device) {}
  ~Workspace() { release(); }
  Workspace(const Workspace&) = delete;
  Workspace& operator=(const Workspace&) = delete;

  // Free every device and pinned buffer; the next run reserves afresh.
  void release() {
    drop_launch_graphs();
    drop_loops();
    if (done_host_) cudaFreeHost(done_host_);
    done_host_ = nullptr;
    done_dev_ = nullptr;
    for (auto& p : bufs_)
      if (p.first) cudaFree(p.first);
    bufs_.clear();
    bytes_ = 0;
    if (host_block_) cudaFreeHost(host_block_);
    host_block_ = nullptr;
    host_block_dev_ = nullptr;
    ctl_host_ = nullptr;
    ist_host_ = nullptr;
    ctl_block_ = nullptr;
    for (auto& e : ev) {
      if (e) cudaEventDestroy(e);
      e = nullptr;
    }
    for (int b = 0; b < 2; ++b) lo[b] = len[b] = nullptr, rid[b] = nullptr;
    avg = err = nullptr;
    axis = active = chunk_excl = nullptr;
    part = nullptr;
    chunk_cnt = int_cnt = nullptr;
    axis_alt = excl_alt = chunk_int = nullptr;
    avg_alt = err_alt = nullptr;
    cmask = nullptr;
    box = nullptr;
    box_cap_ = 0;
    left_lo = left_len = nullptr;
    left_rid = nullptr;
    left_res = nullptr;
    ist = nullptr;
    ctl = nullptr;
    slab = nullptr;
    heap = counter = nullptr;
    cap_ = left_cap_ = 0;
    left_ndim_ = 0;
    heap_ints_ = 0;
    for (auto& v : auto_slots_) v = 0;
    nint_cap_ = 0;
    slab_bytes_ = 0;
    ndim_ = 0;
  }

  int device() const { return device_; }
  bool timing = false;  // record CUDA events around the rule, persistent and phase-2 kernels
  // list capacity (2n + 32 per integral) that the widest iteration of the
  // last run_batch needed
  long long peak_need = 0;
  const std::string& error() const { return err_; }
  void set_error(const std::string& m) { err_ = m; }
  Stats& stats() { return stats_; }

  // Buffers (valid after the reserve_* calls).
  double* lo[2] = {nullptr, nullptr};
  double* len[2] = {nullptr, nullptr};
  int* rid[2] = {nullptr, nullptr};
  double* avg = nullptr;
  double* err = nullptr;
  int* axis = nullptr;
  int* active = nullptr;
  ChunkPartial* part = nullptr;
  int* chunk_excl = nullptr;
  unsigned* chunk_cnt = nullptr;
  // second parity of the persistent kernel's lazy split
  int* axis_alt = nullptr;
  int* excl_alt = nullptr;
  // second parity of the replicated kernel's per-slot values and errors
  double* avg_alt = nullptr;
  double* err_alt = nullptr;
  unsigned* cmask = nullptr;  // two arrays of nchunk masks
  int* chunk_int = nullptr;
  double* box = nullptr;  // integration boxes of the current batch
  unsigned* int_cnt = nullptr;
  double* left_lo = nullptr;
  double* left_len = nullptr;
  int* left_rid = nullptr;
  LeftoverResult* left_res = nullptr;
  IntegralState* ist = nullptr;
  Control* ctl = nullptr;
  // The control block and the integral states share one device allocation
  // (ctl, then ist at kStateOffset) and one pinned host copy (ctl_host_,
  // ist_host_), so one copy moves both each way.
  Control* ctl_host_ = nullptr;
  IntegralState* ist_host_ = nullptr;
  static constexpr size_t kStateOffset = (sizeof(Control) + 255) & ~size_t(255);
  size_t state_bytes(int nint) const { return kStateOffset + sizeof(IntegralState) * nint; }
  // Device address of the pinned state copy, when a persistent launch of
  // nint integrals should write its final states there itself (small
  // batches: one block stores them in less time than a copy takes to
  // start); null otherwise.
  static constexpr int kDirectStatesMax = 64;
  static_assert(sizeof(IntegralState) % 8 == 0 && kStateOffset % 8 == 0,
                "the kernel stores the states as 8-byte words");
  Control* direct_states(int nint) const {
    return nint <= kDirectStatesMax ? static_cast<Control*>(host_block_dev_) : nullptr;
  }
  void* slab = nullptr;
  int* heap = nullptr;
  int* counter = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // When set, run_batch stores each integral's first-phase result here
  // before its second phase (integrals without leftover boxes: the final
  // result).
  Result* phase1_out = nullptr;
  int counter_host = 0;  // host source of the phase-2 box counter's start

  long long cap() const { return cap_; }
  long long left_cap() const { return left_cap_; }

  // Region lists for `slots` regions of dimension ndim; list `cur` keeps
  // its first `keep` slots when the buffers grow.  Growth doubles, capped at
  // `limit` slots; everything but the preserved list is freed before the
  // new buffers are allocated, so the peak is one old list plus the new set.
  bool reserve_lists(int ndim, long long slots, int cur, long long keep, cudaStream_t s,
                     long long limit = 1ll << 30) {
    if (slots <= cap_ && ndim == ndim_) return true;
    long long ncap;
    if (ndim != ndim_ || keep == 0) {
      // nothing to preserve: free first, size for this request only
      release_lists();
      ncap = std::max<long long>(slots, 1 << 16);
    } else {
      ncap = std::max<long long>(slots, cap_ * 2);
      free_buf(lo[cur ^ 1]);
      free_buf(len[cur ^ 1]);
      free_buf(rid[cur ^ 1]);
      free_buf(avg);
      free_buf(err);
      free_buf(axis);
      free_buf(active);
      free_scratch();
    }
    ncap = std::max<long long>(slots, std::min<long long>(ncap, limit));
    ncap = (ncap + 31) & ~31ll;
    double *nlo[2] = {nullptr, nullptr}, *nlen[2] = {nullptr, nullptr};
    int* nrid[2] = {nullptr, nullptr};
    for (int b = 0; b < 2; ++b) {
      if (!alloc(&nlo[b], sizeof(double) * ndim * ncap) ||
          !alloc(&nlen[b], sizeof(double) * ndim * ncap) || !alloc(&nrid[b], sizeof(int) * ncap))
        return false;
    }
    if (keep > 0 && ndim == ndim_) {
      for (int d = 0; d < ndim; ++d) {
        if (!ck(cudaMemcpyAsync(nlo[cur] + d * ncap, lo[cur] + d * cap_, sizeof(double) * keep,
                                cudaMemcpyDeviceToDevice, s)) ||
            !ck(cudaMemcpyAsync(nlen[cur] + d * ncap, len[cur] + d * cap_, sizeof(double) * keep,
                                cudaMemcpyDeviceToDevice, s)))
          return false;
      }
      if (!ck(cudaMemcpyAsync(nrid[cur], rid[cur], sizeof(int) * keep, cudaMemcpyDeviceToDevice,
                              s)))
        return false;
      if (!ck(cudaStreamSynchronize(s))) return false;
    }
    for (int b = 0; b < 2; ++b) {
      free_buf(lo[b]);
      free_buf(len[b]);
      free_buf(rid[b]);
      lo[b] = nlo[b];
      len[b] = nlen[b];
      rid[b] = nrid[b];
    }
    free_scratch();
    const long long nchunk = ncap / 32 + 1;
    if (!alloc(&avg, sizeof(double) * ncap) || !alloc(&err, sizeof(double) * ncap) ||
        !alloc(&axis, sizeof(int) * ncap) || !alloc(&active, sizeof(int) * ncap) ||
        !alloc(&part, sizeof(ChunkPartial) * nchunk) || !alloc(&chunk_excl, sizeof(int) * nchunk) ||
        !alloc(&chunk_cnt, sizeof(unsigned) * nchunk) || !alloc(&axis_alt, sizeof(int) * ncap) ||
        !alloc(&excl_alt, sizeof(int) * nchunk) || !alloc(&cmask, sizeof(unsigned) * 2 * nchunk) ||
        !alloc(&chunk_int, sizeof(int) * nchunk) || !alloc(&avg_alt, sizeof(double) * ncap) ||
        !alloc(&err_alt, sizeof(double) * ncap))
      return false;
    if (!ck(cudaMemsetAsync(chunk_cnt, 0, sizeof(unsigned) * nchunk, s))) return false;
    cap_ = ncap;
    ndim_ = ndim;
    return true;
  }

  bool reserve_leftovers(int ndim, long long slots, long long keep, cudaStream_t s) {
    if (slots <= left_cap_ && ndim == left_ndim_) return true;
    long long ncap;
    if (ndim != left_ndim_ || keep == 0) {
      free_buf(left_lo);
      free_buf(left_len);
      free_buf(left_rid);
      free_buf(left_res);
      left_cap_ = 0;
      ncap = std::max<long long>(slots, 1 << 14);
    } else {
      ncap = std::max<long long>(slots, left_cap_ * 2);
    }
    double *nlo = nullptr, *nlen = nullptr;
    int* nrid = nullptr;
    LeftoverResult* nres = nullptr;
    if (!alloc(&nlo, sizeof(double) * ndim * ncap) || !alloc(&nlen, sizeof(double) * ndim * ncap) ||
        !alloc(&nrid, sizeof(int) * ncap) || !alloc(&nres, sizeof(LeftoverResult) * ncap))
      return false;
    if (keep > 0 && ndim == left_ndim_) {
      for (int d = 0; d < ndim; ++d) {
        if (!ck(cudaMemcpyAsync(nlo + d * ncap, left_lo + d * left_cap_, sizeof(double) * keep,
                                cudaMemcpyDeviceToDevice, s)) ||
            !ck(cudaMemcpyAsync(nlen + d * ncap, left_len + d * left_cap_, sizeof(double) * keep,
                                cudaMemcpyDeviceToDevice, s)))
          return false;
      }
      if (!ck(cudaMemcpyAsync(nrid, left_rid, sizeof(int) * keep, cudaMemcpyDeviceToDevice, s)))
        return false;
      if (!ck(cudaStreamSynchronize(s))) return false;
    }
    free_buf(left_lo);
    free_buf(left_len);
    free_buf(left_rid);
    free_buf(left_res);
    left_lo = nlo;
    left_len = nlen;
    left_rid = nrid;
    left_res = nres;
    left_cap_ = ncap;
    left_ndim_ = ndim;
    return true;
  }

  // Automatic region capacity for (ndim, policy), measured once (free
  // device memory) and kept until release().
  long long auto_slots(int ndim, int policy) {
    const int i = 2 * ndim + (policy == kPolicyReference ? 1 : 0);
    if (ndim < 0 || ndim > kMaxDim) return auto_max_slots(ndim, policy);
    if (!auto_slots_[i]) auto_slots_[i] = auto_max_slots(ndim, policy);
    return auto_slots_[i];
  }

  // Free the region lists and their per-slot scratch.
  void release_lists() {
    for (int b = 0; b < 2; ++b) {
      free_buf(lo[b]);
      free_buf(len[b]);
      free_buf(rid[b]);
    }
    free_scratch();
    cap_ = 0;
    ndim_ = 0;
  }

  // Per-slot and per-chunk scratch of the lists.
  void free_scratch() {
    free_buf(avg);
    free_buf(err);
    free_buf(axis);
    free_buf(active);
    free_buf(part);
    free_buf(chunk_excl);
    free_buf(chunk_cnt);
    free_buf(axis_alt);
    free_buf(excl_alt);
    free_buf(cmask);
    free_buf(chunk_int);
    free_buf(avg_alt);
    free_buf(err_alt);
  }

  bool reserve_integrals(int nint, cudaStream_t s) {
    if (!ev[0]) {
      for (auto& e : ev)
        if (!ck(cudaEventCreate(&e))) return false;
    }
    if (!counter && !alloc(&counter, sizeof(int) * 4)) return false;
    if (nint <= nint_cap_) return true;
    free_buf(ctl_block_);
    ctl = nullptr;
    ist = nullptr;
    free_buf(int_cnt);
    if (host_block_) cudaFreeHost(host_block_);
    host_block_ = nullptr;
    host_block_dev_ = nullptr;
    ctl_host_ = nullptr;
    ist_host_ = nullptr;
    nint_cap_ = 0;
    const int n = std::max(nint, 64);
    if (!alloc(&ctl_block_, state_bytes(n)) || !alloc(&int_cnt, sizeof(unsigned) * n)) return false;
    // mapped, so that a persistent launch can write its final states here
    // itself; without a device address the copy engine does it
    if (!ck(cudaHostAlloc(&host_block_, state_bytes(n), cudaHostAllocMapped))) return false;
    if (cudaHostGetDevicePointer(&host_block_dev_, host_block_, 0) != cudaSuccess) {
      host_block_dev_ = nullptr;
      cudaGetLastError();
    }
    ctl = static_cast<Control*>(ctl_block_);
    ist = reinterpret_cast<IntegralState*>(static_cast<char*>(ctl_block_) + kStateOffset);
    ctl_host_ = static_cast<Control*>(host_block_);
    ist_host_ = reinterpret_cast<IntegralState*>(static_cast<char*>(host_block_) + kStateOffset);
    if (!ck(cudaMemsetAsync(ctl, 0, sizeof(Control), s))) return false;
    if (!ck(cudaMemsetAsync(int_cnt, 0, sizeof(unsigned) * n, s))) return false;
    barrier_clean = true;
    nint_cap_ = n;
    return true;
  }

  bool reserve_boxes(size_t doubles) {
    if (doubles <= box_cap_) return true;
    free_buf(box);
    box_cap_ = 0;
    if (!alloc(&box, sizeof(double) * doubles)) return false;
    box_cap_ = doubles;
    return true;
  }

  bool reserve_slab(size_t bytes, size_t heap_ints) {
    if (bytes <= slab_bytes_ && heap_ints <= heap_ints_) return true;
    free_buf(slab);
    free_buf(heap);
    if (!alloc(&slab, bytes) || !alloc(&heap, sizeof(int) * heap_ints)) return false;
    slab_bytes_ = bytes;
    heap_ints_ = heap_ints;
    return true;
  }

  bool ck(cudaError_t e) {
    if (e != cudaSuccess) {
      err_ = std::string("CUDA: ") + cudaGetErrorString(e);
      return false;
    }
    return true;
  }

  // Device-driven loops of the multi-launch iteration (loop_graph.cuh):
  // one graph per dimension and integrand source, built on first use, with
  // its argument block in device memory and a pinned staging copy.
  struct LoopEntry {
    const void* key = nullptr;  // identifies the instantiation (its bind kernel)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void* dargs = nullptr;  // LoopArgs<Src> on the device
    void* hargs = nullptr;  // pinned staging copy
  };
  LoopEntry* find_loop(const void* key) {
    for (auto& e : loops_)
      if (e.key == key) return &e;
    return nullptr;
  }
  LoopEntry* add_loop(const LoopEntry& e) {
    loops_.push_back(e);
    return &loops_.back();
  }
  bool loops_failed = false;  // a loop graph could not be built here: the host drives

  // The device control block's barrier counters are zero: set when the
  // block is cleared or uploaded and after a replicated launch (its last
  // block zeroes them), cleared after a launch of the persistent kernel.
  bool barrier_clean = true;

  // Completion word of replicated launches: a mapped pinned word that the
  // kernel sets to the launch's sequence number after storing its final
  // states in the pinned block, so the host stops waiting then, not when
  // the whole grid has retired.  Null when mapped memory is unavailable.
  unsigned* done_word() {
    if (!done_host_ && !done_failed_) {
      if (cudaHostAlloc(reinterpret_cast<void**>(&done_host_), 64, cudaHostAllocMapped) !=
              cudaSuccess ||
          cudaHostGetDevicePointer(reinterpret_cast<void**>(&done_dev_), done_host_, 0) !=
              cudaSuccess) {
        if (done_host_) cudaFreeHost(done_host_);
        done_host_ = nullptr;
        done_dev_ = nullptr;
        done_failed_ = true;
        cudaGetLastError();
      } else {
        *done_host_ = 0;
      }
    }
    return done_dev_;
  }
  unsigned next_seq() {
    if (++done_seq_ == 0) ++done_seq_;
    return done_seq_;
  }

  // Wait until the completion word holds seq.  The stream is queried now
  // and then, so a launch that failed (or finished without storing) ends
  // the wait with its error instead of spinning.
  bool wait_done(unsigned seq, cudaStream_t s) {
    for (unsigned i = 1;; ++i) {
      if (__atomic_load_n(done_host_, __ATOMIC_ACQUIRE) == seq) return true;
      if ((i & 4095) == 0) {
        const cudaError_t e = cudaStreamQuery(s);
        if (e == cudaErrorNotReady) continue;
        if (e != cudaSuccess) return ck(e);
        if (__atomic_load_n(done_host_, __ATOMIC_ACQUIRE) == seq) return true;
        err_ = "replicated launch finished without storing its states";
        return false;
      }
    }
  }

  // One replicated launch as a replay: the upload of `bytes` bytes of the
  // pinned control block and states (none when bytes is 0: the launch
  // carries its starting states), then the cooperative launch of `func`
  // on `blocks` blocks of 256 threads with `args`.  The two are captured
  // into a CUDA graph on first use, and again when the kernel, the grid or
  // the copy changes; later calls set the kernel node's arguments and
  // launch the graph, which costs the host less than a copy plus a
  // cooperative launch.  Returns false on a CUDA error; a capture that is
  // not possible here (the stream is being captured by the caller, say)
  // falls back to the copy and launch.
  bool launch_replicated(const void* func, unsigned blocks, void** args, size_t bytes,
                         cudaStream_t s) {
    // one graph per kernel and copy, so that calls alternating between
    // integrands reuse theirs (the oldest of kLaunchGraphs is dropped)
    LaunchGraph* gp = nullptr;
    for (auto& e : lg_)
      if (e.exec && e.func == func && e.blocks == blocks && e.bytes == bytes && e.dst == ctl &&
          e.src == ctl_host_)
        gp = &e;
    if (!gp) {
      gp = &lg_[0];
      for (auto& e : lg_)
        if (!e.exec || e.used < gp->used) gp = &e;
      drop_launch_graph(*gp);
    }
    LaunchGraph& g = *gp;
    g.used = ++lg_clock_;
    if (!g.exec && !graph_failed_) {
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t e1 = bytes ? cudaMemcpyAsync(ctl, ctl_host_, bytes, cudaMemcpyHostToDevice, s)
                               : cudaSuccess;
        if (e1 == cudaSuccess)
          e1 = cudaLaunchCooperativeKernel(func, dim3(blocks), dim3(256), args, 0, s);
        e = cudaStreamEndCapture(s, &graph);
        if (e == cudaSuccess) e = e1;
      }
      cudaGraphNode_t knode = nullptr;
      if (e == cudaSuccess) {
        size_t nn = 0;
        e = cudaGraphGetNodes(graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess) e = cudaGraphGetNodes(graph, nodes.data(), &nn);
        for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            knode = nodes[i];
        }
      }
      if (e == cudaSuccess && knode) e = cudaGraphInstantiate(&g.exec, graph, 0);
      if (e != cudaSuccess || !knode || !g.exec) {
        if (graph) cudaGraphDestroy(graph);
        g.exec = nullptr;
        graph_failed_ = true;
        cudaGetLastError();
      } else {
        g.graph = graph;
        g.kernel = knode;
        g.func = func;
        g.blocks = blocks;
        g.bytes = bytes;
        g.dst = ctl;
        g.src = ctl_host_;
        // the recorded launch holds this call's arguments already
        return ck(cudaGraphLaunch(g.exec, s));
      }
    }
    if (!g.exec) {
      return (!bytes || ck(cudaMemcpyAsync(ctl, ctl_host_, bytes, cudaMemcpyHostToDevice, s))) &&
             ck(cudaLaunchCooperativeKernel(func, dim3(blocks), dim3(256), args, 0, s));
    }
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void*>(func);
    kp.gridDim = dim3(blocks);
    kp.blockDim = dim3(256);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return ck(cudaGraphExecKernelNodeSetParams(g.exec, g.kernel, &kp)) &&
           ck(cudaGraphLaunch(g.exec, s));
  }

  size_t bytes_reserved() const { return bytes_; }

 private:
  template <class T>
  bool alloc(T** p, size_t bytes) {
    void* q = nullptr;
    if (!ck(cudaMalloc(&q, bytes))) return false;
    *p = static_cast<T*>(q);
    bufs_.push_back({q, bytes});
    bytes_ += bytes;
    return true;
  }
  template <class T>
  void free_buf(T*& p) {
    if (!p) return;
    for (auto& q : bufs_)
      if (q.first == p) {
        cudaFree(q.first);
        bytes_ -= q.second;
        q.first = nullptr;
        q.second = 0;
      }
    p = nullptr;
  }

  int device_;
  long long auto_slots_[2 * (kMaxDim + 1)] = {};
  std::vector<std::pair<void*, size_t>> bufs_;
  long long cap_ = 0, left_cap_ = 0;
  int ndim_ = 0, left_ndim_ = 0;
  int nint_cap_ = 0;
  size_t slab_bytes_ = 0, heap_ints_ = 0;
  size_t box_cap_ = 0;
  void* ctl_block_ = nullptr;
  void* host_block_ = nullptr;
  void* host_block_dev_ = nullptr;  // device address of host_block_ (mapped)
  // the graphs of launch_replicated and what each was recorded for
  struct LaunchGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t kernel = nullptr;
    const void* func = nullptr;
    unsigned blocks = 0;
    size_t bytes = 0;
    const void* dst = nullptr;
    const void* src = nullptr;
    unsigned long long used = 0;  // lg_clock_ at the last use
  };
  static constexpr int kLaunchGraphs = 8;
  LaunchGraph lg_[kLaunchGraphs];
  unsigned long long lg_clock_ = 0;
  bool graph_failed_ = false;
  std::vector<LoopEntry> loops_;
  void drop_loops() {
    for (auto& e : loops_) {
      if (e.exec) cudaGraphExecDestroy(e.exec);
      if (e.graph) cudaGraphDestroy(e.graph);
      if (e.dargs) cudaFree(e.dargs);
      if (e.hargs) cudaFreeHost(e.hargs);
    }
    loops_.clear();
  }
  static void drop_launch_graph(LaunchGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    g = LaunchGraph();
  }
  void drop_launch_graphs() {
    for (auto& g : lg_) drop_launch_graph(g);
  }
  unsigned* done_host_ = nullptr;  // completion word (pinned, mapped)
  unsigned* done_dev_ = nullptr;
  unsigned done_seq_ = 0;
  bool done_failed_ = false;
  size_t bytes_ = 0;
  std::string err_;
  Stats stats_;
};

inline int sm_count(int device) {
  // queried once per device (every call needs it)
  static std::atomic<int> cache[64];
  const int d = device >= 0 && device < 64 ? device : 0;
  int n = cache[d].load(std::memory_order_relaxed);
  if (n > 0 && device == d) return n;
  n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  n = n > 0 ? n : 148;
  if (device == d) cache[d].store(n, std::memory_order_relaxed);
  return n;
}

// Region-list capacity when the caller leaves it to the library: the slots
// that fit in 40% of the device's free memory (two lists of FP64 bounds plus
// per-slot results and chunk scratch, and leftover boxes under the reference
// policy), between 2^20 and 2^30.
inline long long auto_max_slots(int ndim, int policy) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || free_b == 0) return 1ll << 26;
  double per_slot = 2.0 * (16.0 * ndim + 4) + 28 + 64.0 / 32;
  if (policy == kPolicyReference) per_slot += 2.0 * (16.0 * ndim + 4 + 24);
  const double slots = 0.4 * (double)free_b / per_slot;
  return std::max<long long>(1ll << 20, std::min<long long>(1ll << 30, (long long)slots));
}

// Divisions per axis of the initial grid (GPUKernelquad.cu:300-311).
inline int grid_divisions(int ndim) { return ndim > 10 ? 1 : (ndim >= 5 ? 2 : 4); }

template <int N, int K, class Src>
inline void launch_eval(const Src& src, const RuleTables& T, const EngineArgs& a, int sms,
                        cudaStream_t s) {
  const long long threads = (long long)a.n * K;
  long long blocks = (threads + 255) / 256;
  blocks = std::max<long long>(1, std::min<long long>(blocks, (long long)sms * 32));
  k_eval<N, K, Src><<<(unsigned)blocks, 256, 0, s>>>(src, T, a);
}

namespace detail {

// Host copy of a batch's starting point: integral k owns the k-th padded
// segment of the initial grid.  Fills the pinned states behind
// ws.ctl_host_ and returns the control block the first launch starts from.
inline Control initial_states(Workspace& ws, int nint, const double* epsrel,
                              const double* epsabs, int per, int padded, long long n0) {
  IntegralState* h = ws.ist_host_;
  for (int k = 0; k < nint; ++k) {
    IntegralState& is = h[k];
    std::memset(&is, 0, sizeof(is));
    is.epsrel = epsrel[k];
    is.epsabs = epsabs[k];
    is.state = kStateRunning;
    is.seg_start = k * padded;
    is.seg_count = per;
  }
  Control c0;
  std::memset(&c0, 0, sizeof(c0));
  c0.host.n = (int)n0;
  c0.host.n_running = nint;
  return c0;
}

// Results from the final integral states.
inline void state_results(const IntegralState* h, int nint, Result* out) {
  for (int k = 0; k < nint; ++k) {
    const IntegralState& is = h[k];
    Result& r = out[k];
    r.nregions = is.nregions;
    r.neval = is.neval;
    r.iterations = is.iters;
    r.state = is.state;
    r.pad = 0;
    if (is.state == kStateRunning || is.state == kStateCapacity) {
      // stopped early: report the last full estimate, not converged
      r.value = is.last_value;
      r.error = is.last_error;
      r.status = is.last_error <= detail::max_err(is.last_value, is.epsrel, is.epsabs) ? 0 : 1;
    } else {
      r.value = is.value;
      r.error = is.error;
      r.status = is.status;
    }
  }
}

// Blocks per SM of a cooperative launch of `kernel` (256 threads), cached
// per device and kernel instantiation in `cache` (0: not yet queried,
// else 1 + blocks per SM, or 1 when the device has no cooperative launch).
// The query is idempotent, so concurrent first calls from several host
// threads store the same value.
inline int coop_blocks(std::atomic<int>* cache, int device, const void* kernel, int sms) {
  const int dev = device & 63;
  int v = cache[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    int per_sm = 0, coop = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    v = 1 + (coop ? per_sm : 0);
    cache[dev].store(v, std::memory_order_relaxed);
  }
  return (v - 1) * sms;
}

// Blocks of a cooperative k_persistent<N, Src> launch on the workspace's
// device; 0 when the device has no cooperative launch.
template <int N, class Src>
int persistent_blocks(const Workspace& ws, int sms) {
  static std::atomic<int> cache[64];
  return coop_blocks(cache, ws.device(), (const void*)k_persistent<N, Src>, sms);
}

// The same for k_replicated<N, Src>.
template <int N, class Src>
int replicated_blocks(const Workspace& ws, int sms) {
  static std::atomic<int> cache[64];
  return coop_blocks(cache, ws.device(), (const void*)k_replicated<N, Src>, sms);
}

// Longest list a persistent launch keeps iterating on.
inline int persistent_limit(const Options& opt, int pblocks) {
  return std::min(opt.persistent_max_n > 0 ? opt.persistent_max_n : pblocks * 8 * 8,
                  32 * kStageChunks);
}

// Engine arguments of a batch; bind_lists points them at list `cur`.
inline EngineArgs engine_args(const Workspace& ws, int nint, const Options& opt, int npoints) {
  EngineArgs a;
  std::memset(&a, 0, sizeof(a));
  a.ist = ws.ist;
  a.nint = nint;
  a.ctl = ws.ctl;
  a.policy = opt.policy;
  a.phase1_cap = opt.policy == kPolicyReference ? opt.phase1_cap : 0;
  a.max_iters = opt.max_iters;
  a.npoints = npoints;
  return a;
}

inline void bind_lists(const Workspace& ws, EngineArgs& a, int cur, long long n) {
  a.lo = ws.lo[cur];
  a.len = ws.len[cur];
  a.rid = ws.rid[cur];
  a.n = (int)n;
  a.cap = ws.cap();
  a.avg = ws.avg;
  a.err = ws.err;
  a.axis = ws.axis;
  a.active = ws.active;
  a.part = ws.part;
  a.chunk_excl = ws.chunk_excl;
  a.chunk_cnt = ws.chunk_cnt;
  a.int_cnt = ws.int_cnt;
  a.nlo = ws.lo[cur ^ 1];
  a.nlen = ws.len[cur ^ 1];
  a.nrid = ws.rid[cur ^ 1];
  a.ncap = ws.cap();
  a.left_lo = ws.left_lo;
  a.left_len = ws.left_len;
  a.left_rid = ws.left_rid;
  a.left_cap = ws.left_cap();
}

// Arguments of a persistent launch over the lists bound in `a`.
inline PersistArgs persist_args(const Workspace& ws, const EngineArgs& a, const Options& opt,
                                int iter_base, int pmax, bool init, int dv, int per, int padded,
                                const double* d_box) {
  PersistArgs p;
  p.base = a;
  const long long nchunk = ws.cap() / 32 + 1;
  for (int b = 0; b < 2; ++b) {
    p.lo[b] = ws.lo[b];
    p.len[b] = ws.len[b];
    p.rid[b] = ws.rid[b];
    p.cmask[b] = ws.cmask + b * nchunk;
  }
  p.axis[0] = ws.axis;
  p.axis[1] = ws.axis_alt;
  p.excl[0] = ws.chunk_excl;
  p.excl[1] = ws.excl_alt;
  p.chunk_int = ws.chunk_int;
  p.iter_base = iter_base;
  p.max_n = pmax;
  p.max_r = opt.persistent_max_r > 0 ? opt.persistent_max_r : 8;
  p.init = init ? 1 : 0;
  p.divisions = dv;
  p.per_integral = per;
  p.padded = padded;
  p.box = d_box;
  p.host_out = nullptr;
  p.host_words = 0;
  p.spin_limit = opt.barrier_spins > 0 ? opt.barrier_spins : detail::kBarrierSpins;
  p.hold_block = opt.hold_block;
  return p;
}

// Arguments of a replicated-kernel launch over the lists bound in `a`.
inline RepArgs rep_args(const Workspace& ws, const EngineArgs& a, const Options& opt,
                        int iter_base, int rmax, bool init, int dv, int per, int padded,
                        const double* d_box) {
  RepArgs p;
  p.base = a;
  for (int b = 0; b < 2; ++b) {
    p.lo[b] = ws.lo[b];
    p.len[b] = ws.len[b];
    p.rid[b] = ws.rid[b];
  }
  p.avg[0] = ws.avg;
  p.avg[1] = ws.avg_alt;
  p.err[0] = ws.err;
  p.err[1] = ws.err_alt;
  p.axis[0] = ws.axis;
  p.axis[1] = ws.axis_alt;
  p.max_n = rmax;
  p.max_r = opt.persistent_max_r > 0 ? opt.persistent_max_r : 8;
  p.iter_base = iter_base;
  p.init = init ? 1 : 0;
  p.divisions = dv;
  p.per_integral = per;
  p.padded = padded;
  p.box = d_box;
  p.host_out = nullptr;
  p.host_words = 0;
  p.spin_limit = opt.barrier_spins > 0 ? opt.barrier_spins : detail::kBarrierSpins;
  p.hold_block = opt.hold_block;
  p.done = nullptr;
  p.seq = 0;
  p.param_state = 0;
  p.cur0 = 0;
  std::memset(&p.host0, 0, sizeof(p.host0));
  return p;
}

// Longest list a replicated launch evaluates.
inline int replicated_limit(const Options& opt, int rblocks) {
  return std::min(opt.persistent_max_n > 0 ? opt.persistent_max_n : rblocks * 8,
                  32 * kRepChunks);
}

// Pinned control block for a persistent launch starting from `hs`.
inline void persistent_control(Workspace& ws, const IterState& hs, int cur) {
  ws.ctl_host_->host = hs;
  ws.ctl_host_->it[0] = hs;
  ws.ctl_host_->cur = cur;
  ws.ctl_host_->done_cnt = 0;
  ws.ctl_host_->bar_count = 0;
  ws.ctl_host_->exit_count = 0;
  ws.ctl_host_->timeout = 0;
  ws.ctl_host_->exit_reason = 0;
  std::memset(ws.ctl_host_->trace, 0, sizeof(ws.ctl_host_->trace));
}

}  // namespace detail

namespace detail {

// The device-driven loop of dimension N and integrand source Src, built on
// first use: WHILE { bind; SWITCH { rule with 1 | 8 | 32 lanes per region };
// partials; decide; scan; split; advance; test }.  Grids are the largest
// the host-driven loop uses for the lane count or step (the kernels stride
// over the list).  Null when a graph with conditional nodes cannot be built
// here; the host then drives the iterations.
template <int N, class Src>
Workspace::LoopEntry* loop_graph(Workspace& ws, int sms) {
  const void* key = (const void*)k_loop_split<N, Src>;
  if (Workspace::LoopEntry* found = ws.find_loop(key)) return found;
  if (ws.loops_failed) return nullptr;
  Workspace::LoopEntry e;
  e.key = key;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle again = 0, lanes = 0;
  bool ok = cudaMalloc(&e.dargs, sizeof(LoopArgs<Src>)) == cudaSuccess &&
            cudaHostAlloc(&e.hargs, sizeof(LoopArgs<Src>), cudaHostAllocDefault) == cudaSuccess &&
            cudaGraphCreate(&g, 0) == cudaSuccess &&
            cudaGraphConditionalHandleCreate(&again, g, 1, cudaGraphCondAssignDefault) ==
                cudaSuccess &&
            cudaGraphConditionalHandleCreate(&lanes, g, 0, 0) == cudaSuccess;
  cudaGraph_t body = nullptr;
  if (ok) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = again;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn;
    ok = cudaGraphAddNode(&wn, g, nullptr, 0, &cp) == cudaSuccess;
    if (ok) body = cp.conditional.phGraph_out[0];
  }
  auto kernel = [&](cudaGraph_t gr, cudaGraphNode_t* dep, const void* fn, int grid, int block,
                    void** args, cudaGraphNode_t* out) {
    cudaKernelNodeParams kp = {};
    kp.func = const_cast<void*>(fn);
    kp.gridDim = dim3((unsigned)grid);
    kp.blockDim = dim3((unsigned)block);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return cudaGraphAddKernelNode(out, gr, dep, dep ? 1 : 0, &kp) == cudaSuccess;
  };
  LoopArgs<Src>* la = static_cast<LoopArgs<Src>*>(e.dargs);
  const LoopArgs<Src>* lac = la;
  void* a_bind[] = {(void*)&la, (void*)&lanes};
  void* a_la[] = {(void*)&lac};
  const RuleTables T = make_rule9_tables(N);
  void* a_eval[] = {(void*)&lac, (void*)&T};
  void* a_test[] = {(void*)&lac, (void*)&again};
  cudaGraphNode_t n_bind = nullptr, n_sw = nullptr, n_part = nullptr, n_dec = nullptr,
                  n_scan = nullptr, n_split = nullptr, n_adv = nullptr, n_test = nullptr, n_ev;
  ok = ok && kernel(body, nullptr, (const void*)k_loop_bind<Src>, 1, 32, a_bind, &n_bind);
  cudaGraph_t arms[3] = {nullptr, nullptr, nullptr};
  if (ok) {
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = lanes;
    cp.conditional.type = cudaGraphCondTypeSwitch;
    cp.conditional.size = 3;
    ok = cudaGraphAddNode(&n_sw, body, &n_bind, 1, &cp) == cudaSuccess;
    if (ok)
      for (int i = 0; i < 3; ++i) arms[i] = cp.conditional.phGraph_out[i];
  }
  ok = ok && kernel(arms[0], nullptr, (const void*)k_loop_eval<N, 1, Src>, sms * 32, 256, a_eval, &n_ev);
  ok = ok && kernel(arms[1], nullptr, (const void*)k_loop_eval<N, 8, Src>, sms * 16, 256, a_eval, &n_ev);
  ok = ok && kernel(arms[2], nullptr, (const void*)k_loop_eval<N, 32, Src>, sms * 8, 256, a_eval, &n_ev);
  ok = ok && kernel(body, &n_sw, (const void*)k_loop_partials<Src>, sms * 16, 256, a_la, &n_part);
  ok = ok && kernel(body, &n_part, (const void*)k_loop_decide<Src>, sms * 16, 256, a_la, &n_dec);
  ok = ok && kernel(body, &n_dec, (const void*)k_loop_scan<Src>, 1, 32, a_la, &n_scan);
  ok = ok && kernel(body, &n_scan, (const void*)k_loop_split<N, Src>, sms * 16, 256, a_la, &n_split);
  ok = ok && kernel(body, &n_split, (const void*)k_loop_advance<Src>, sms, 256, a_la, &n_adv);
  ok = ok && kernel(body, &n_adv, (const void*)k_loop_test<Src>, 1, 32, a_test, &n_test);
  ok = ok && cudaGraphInstantiate(&e.exec, g, 0) == cudaSuccess;
  if (!ok) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (g) cudaGraphDestroy(g);
    if (e.dargs) cudaFree(e.dargs);
    if (e.hargs) cudaFreeHost(e.hargs);
    ws.loops_failed = true;
    cudaGetLastError();
    return nullptr;
  }
  e.graph = g;
  return ws.add_loop(e);
}

}  // namespace detail

// Rule evaluation step of the multi-launch driver when the caller supplies
// its own (NoHook: the engine's k_eval).  A hook's eval(args, n, stream)
// evaluates the n slots of the current list into args.avg/err/axis/active
// and returns 0 or an error code; with a hook the persistent kernel is not
// used.
struct NoHook {
  static constexpr bool kActive = false;
  int eval(const EngineArgs&, long long, cudaStream_t) const { return 0; }
};

// Run one batch: `nint` integrals of one family and dimension N, each over
// its box (h_box[k] = lo[N] then hi[N], host memory; the unit cube when
// h_box is null).  Results go to out[0..nint).
template <int N, class Src, class Hook = NoHook>
int run_batch(Workspace& ws, const Src& src, int nint, const double* epsrel,
              const double* epsabs, const Options& opt, Result* out, cudaStream_t s,
              const double* h_box = nullptr, const Hook& hook = Hook()) {
  static_assert(N >= 2 && N <= kMaxDim, "dimension out of range");
  const long long max_slots = opt.max_slots > 0 ? opt.max_slots : ws.auto_slots(N, opt.policy);
  if (nint <= 0) return kErrInvalid;
  static const RuleTables T = make_rule9_tables(N);
  const int sms = sm_count(ws.device());
  const int dv = grid_divisions(N);
  int per = 1;
  for (int d = 0; d < N; ++d) per *= dv;
  const int padded = (per + 31) & ~31;
  long long n_cur = (long long)nint * padded;
  Stats& st = ws.stats();

  ws.peak_need = 0;
  if (!ws.reserve_integrals(nint, s)) return kErrCuda;
  if (!ws.reserve_lists(N, std::min<long long>(std::max<long long>(1 << 20, 4 * n_cur), max_slots),
                        0, 0, s, max_slots))
    return kErrCuda;
  if (!ws.reserve_leftovers(N, 1, 0, s)) return kErrCuda;

  // integral states
  IntegralState* h = ws.ist_host_;
  Control c0 = detail::initial_states(ws, nint, epsrel, epsabs, per, padded, n_cur);
  *ws.ctl_host_ = c0;
  // The control block and the states go to the device with the first
  // launch (one copy); the initial grid is written by k_init_grid or, when
  // the persistent kernel runs first, by its first iteration.
  bool uploaded = false;
  bool grid_pending = true;
  const double* d_box = nullptr;
  if (h_box) {
    const size_t nb = (size_t)nint * 2 * N;
    if (!ws.reserve_boxes(nb)) return kErrCuda;
    if (!ws.ck(cudaMemcpyAsync(ws.box, h_box, sizeof(double) * nb, cudaMemcpyHostToDevice, s)))
      return kErrCuda;
    st.h2d_bytes += (long long)(sizeof(double) * nb);
    d_box = ws.box;
  }

  int cur = 0;
  EngineArgs a = detail::engine_args(ws, nint, opt, T.npoints);
  auto bind = [&](long long n) { detail::bind_lists(ws, a, cur, n); };
  bind(n_cur);

  // persistent kernel geometry (queried once per device and instantiation)
  const int pblocks =
      opt.persistent && !Hook::kActive ? detail::persistent_blocks<N, Src>(ws, sms) : 0;
  const int pmax = detail::persistent_limit(opt, pblocks);
  const int rblocks = opt.persistent && opt.replicated && !Hook::kActive && nint <= kSmallBatch
                          ? detail::replicated_blocks<N, Src>(ws, sms)
                          : 0;
  const int rmax = detail::replicated_limit(opt, rblocks);

  IterState hs = c0.host;
  long long n_left = 0;
  bool states_fresh = true;  // h holds the device states after the last kernel
  // regions of each integral before a persistent launch (statistics)
  unsigned long long nreg_small[kSmallBatch];
  std::vector<unsigned long long> nreg_big(nint > kSmallBatch ? nint : 0);
  unsigned long long* nreg_before = nint > kSmallBatch ? nreg_big.data() : nreg_small;
  int status = kOk;
  while (hs.n_running > 0 && hs.n > 0) {
    n_cur = hs.n;
    // capacity for the worst case of the coming iteration(s)
    const long long need = 2 * n_cur + 32ll * nint;
    ws.peak_need = std::max(ws.peak_need, need);
    if (need > max_slots) {
      status = kErrCapacity;
      break;
    }
    if (!ws.reserve_lists(N, std::min<long long>(std::max<long long>(need, 4 * n_cur), max_slots),
                          cur, n_cur, s, max_slots))
      return kErrCuda;
    if (opt.policy == kPolicyReference &&
        !ws.reserve_leftovers(N, n_left + 4 * n_cur + 1, n_left, s))
      return kErrCuda;
    bind(n_cur);

    const bool use_rep = rblocks > 0 && n_cur <= rmax;
    if (use_rep || (pblocks > 0 && n_cur <= pmax)) {
      // a stretch of iterations in one persistent launch: the
      // replicated-decision kernel for small batches on short lists, else
      // the persistent kernel
      detail::persistent_control(ws, hs, cur);
      // the replicated kernel reads the states every launch (its blocks
      // keep their own copies); the persistent kernel keeps them on the
      // device between its launches
      const size_t up = uploaded && !use_rep ? sizeof(Control) : ws.state_bytes(nint);
      if (use_rep && uploaded && !states_fresh) {
        // the device holds the newer states (multi-launch steps ran since
        // the last copy back): fetch them before re-uploading
        if (!ws.ck(cudaMemcpyAsync(ws.ist_host_, ws.ist, sizeof(IntegralState) * nint,
                                   cudaMemcpyDeviceToHost, s)) ||
            !ws.ck(cudaStreamSynchronize(s)))
          return kErrCuda;
        st.d2h_bytes += (long long)(sizeof(IntegralState) * nint);
        detail::persistent_control(ws, hs, cur);
      }
      // small batches on the replicated kernel: the upload and the launch
      // replayed from a graph, and the wait ends when the kernel has stored
      // its states (launch_replicated, wait_done)
      const bool fast = use_rep && !ws.timing && ws.direct_states(nint) && ws.done_word();
      // a batch of up to kParamStates integrals passes its starting states
      // with the launch when the barrier counters are known to be zero
      const bool pstate = fast && nint <= kParamStates && ws.barrier_clean;
      if (!fast && !ws.ck(cudaMemcpyAsync(ws.ctl, ws.ctl_host_, up, cudaMemcpyHostToDevice, s)))
        return kErrCuda;
      uploaded = true;
      st.h2d_bytes += (long long)up;
      // the host copy of the states is current unless multi-launch steps ran
      // since it was read (the replicated path fetched it above)
      const bool count_regions = use_rep || states_fresh;
      if (count_regions)
        for (int k = 0; k < nint; ++k) nreg_before[k] = h[k].nregions;
      if (ws.timing) ws.ck(cudaEventRecord(ws.ev[0], s));
      unsigned seq = 0;  // completion word value of a fast launch
      if (use_rep) {
        RepArgs p = detail::rep_args(ws, a, opt, c0.iters_done, rmax, grid_pending, dv, per,
                                     padded, d_box);
        p.host_out = ws.direct_states(nint);
        p.host_words = (int)(ws.state_bytes(nint) / 8);
        if (fast) {
          p.done = ws.done_word();
          p.seq = seq = ws.next_seq();
        }
        if (pstate) {
          p.param_state = 1;
          p.cur0 = cur;
          p.host0 = hs;
          for (int k = 0; k < nint; ++k) p.ist0[k] = h[k];
        }
        void* args[] = {(void*)&src, (void*)&T, (void*)&p};
        if (fast) {
          if (!ws.launch_replicated((const void*)k_replicated<N, Src>, (unsigned)rblocks, args,
                                    pstate ? 0 : up, s))
            return kErrCuda;
        } else if (!ws.ck(cudaLaunchCooperativeKernel((const void*)k_replicated<N, Src>,
                                                      dim3(rblocks), dim3(256), args, 0, s))) {
          return kErrCuda;
        }
      } else {
        PersistArgs p = detail::persist_args(ws, a, opt, c0.iters_done, pmax, grid_pending, dv,
                                             per, padded, d_box);
        p.host_out = ws.direct_states(nint);
        p.host_words = (int)(ws.state_bytes(nint) / 8);
        void* args[] = {(void*)&src, (void*)&T, (void*)&p};
        if (!ws.ck(cudaLaunchCooperativeKernel((const void*)k_persistent<N, Src>,
                                               dim3(pblocks), dim3(256), args, 0, s)))
          return kErrCuda;
      }
      grid_pending = false;
      ws.barrier_clean = use_rep;
      if (ws.timing) ws.ck(cudaEventRecord(ws.ev[1], s));
      st.launches += 1;
      st.persistent_launches += 1;
      // the states come back with the control block (stored by the kernel
      // itself for small batches): when the launch finished every
      // integral, no further round trip is needed
      if (!ws.direct_states(nint) &&
          !ws.ck(cudaMemcpyAsync(ws.ctl_host_, ws.ctl, ws.state_bytes(nint),
                                 cudaMemcpyDeviceToHost, s)))
        return kErrCuda;
      if (seq) {
        if (!ws.wait_done(seq, s)) return kErrCuda;
      } else if (!ws.ck(cudaStreamSynchronize(s))) {
        return kErrCuda;
      }
      st.d2h_bytes += (long long)ws.state_bytes(nint);
      states_fresh = true;
      if (ws.timing) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ws.ev[0], ws.ev[1]);
        st.ms_persistent += ms;
      }
      const Control& c = *ws.ctl_host_;
      const int before = c0.iters_done;
      st.iterations += c.iters_done - before;
      st.persistent_iterations += c.iters_done - before;
      if (use_rep) st.replicated_launches += 1;
      if (count_regions)
        for (int k = 0; k < nint; ++k)
          st.persistent_regions += (long long)(h[k].nregions - nreg_before[k]);
      c0.iters_done = c.iters_done;
      if (c.exit_reason == kExitTimeout || c.timeout) {
        ws.ck(cudaErrorLaunchTimeout);
        return kErrTimeout;
      }
      cur = c.cur;
      hs = c.host;
      n_left = hs.n_left;
      continue;  // done, too large or capacity: the loop re-checks
    }

    // one iteration, one launch per step
    states_fresh = false;
    if (!uploaded) {
      if (!ws.ck(cudaMemcpyAsync(ws.ctl, ws.ctl_host_, ws.state_bytes(nint),
                                 cudaMemcpyHostToDevice, s)))
        return kErrCuda;
      st.h2d_bytes += (long long)ws.state_bytes(nint);
      uploaded = true;
    }
    if (grid_pending) {
      const long long blocks = std::min<long long>((n_cur + 255) / 256, (long long)sms * 8);
      k_init_grid<N><<<(unsigned)std::max<long long>(blocks, 1), 256, 0, s>>>(a, dv, per, padded,
                                                                            d_box);
      st.launches += 1;
      grid_pending = false;
    }
    // Device-driven iterations (loop_graph.cuh): one graph launch runs them
    // until the list needs larger buffers, goes back to a persistent
    // kernel's range or no integral is running.  Timing keeps the
    // host-driven loop, which records events around each rule launch.
    Workspace::LoopEntry* loop = nullptr;
    if constexpr (!Hook::kActive) {
      if (opt.device_loop && !ws.timing) loop = detail::loop_graph<N, Src>(ws, sms);
    }
    if (loop) {
      LoopArgs<Src>& la = *static_cast<LoopArgs<Src>*>(loop->hargs);
      std::memset(&la, 0, sizeof(la));
      for (int b = 0; b < 2; ++b) {
        EngineArgs ab = a;
        detail::bind_lists(ws, ab, b, 0);
        la.base[b] = ab;
      }
      la.src = src;
      // the host's own limit too: the buffers may be larger than max_slots
      // (grown by an earlier call), and a list beyond it stops the run
      la.cap = std::min<long long>(ws.cap(), max_slots);
      la.left_cap = ws.left_cap();
      la.ref_policy = opt.policy == kPolicyReference ? 1 : 0;
      const int hb_p = pblocks > 0 ? pmax : 0;
      const int hb_r = rblocks > 0 ? rmax : 0;
      la.hand_back = std::max(hb_p, hb_r);
      la.k1_min = sms * 512;
      la.k8_min = sms * 64;
      la.forced_lanes = opt.lanes > 0 ? opt.lanes : 0;
      if (!ws.ck(cudaMemcpyAsync(loop->dargs, loop->hargs, sizeof(la), cudaMemcpyHostToDevice, s)) ||
          !ws.ck(cudaGraphLaunch(loop->exec, s)) ||
          !ws.ck(cudaMemcpyAsync(loop->hargs, loop->dargs, sizeof(la), cudaMemcpyDeviceToHost, s)) ||
          !ws.ck(cudaMemcpyAsync(ws.ctl_host_, ws.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s)) ||
          !ws.ck(cudaStreamSynchronize(s)))
        return kErrCuda;
      st.h2d_bytes += (long long)sizeof(la);
      st.d2h_bytes += (long long)(sizeof(la) + sizeof(Control));
      st.iterations += la.iterations;
      st.eval_launches += la.iterations;
      st.regions_evaluated += (long long)la.regions;
      st.launches += 8ll * la.iterations;  // bind, rule, partials, decide, scan, split, advance, test
      st.device_loops += 1;
      ws.peak_need = std::max(ws.peak_need, la.peak_need);
      c0.iters_done = ws.ctl_host_->iters_done;
      const IterState nx = ws.ctl_host_->host;
      if (nx.overflow) {
        status = kErrCapacity;
        break;
      }
      cur = ws.ctl_host_->cur;
      hs = nx;
      n_left = nx.n_left;
      continue;
    }
    int K = opt.lanes;
    if (K <= 0) K = n_cur >= (long long)sms * 512 ? 1 : (n_cur >= (long long)sms * 64 ? 8 : 32);
    if (ws.timing) ws.ck(cudaEventRecord(ws.ev[0], s));
    if constexpr (Hook::kActive) {
      const int hr = hook.eval(a, n_cur, s);
      if (hr) return hr;
    } else {
      switch (K) {
        case 1: launch_eval<N, 1>(src, T, a, sms, s); break;
        case 8: launch_eval<N, 8>(src, T, a, sms, s); break;
        default: launch_eval<N, 32>(src, T, a, sms, s); break;
      }
    }
    if (ws.timing) ws.ck(cudaEventRecord(ws.ev[1], s));
    st.eval_launches += 1;
    st.regions_evaluated += n_cur;
    const long long nchunk = (n_cur + 31) / 32;
    const unsigned pb =
        (unsigned)std::max<long long>(1, std::min<long long>((nchunk + 7) / 8, sms * 16ll));
    k_partials<<<pb, 256, 0, s>>>(a);
    const unsigned db = (unsigned)std::max(1, std::min((nint + 7) / 8, sms * 16));
    k_decide<<<db, 256, 0, s>>>(a);
    k_scan<<<1, 32, 0, s>>>(a);
    k_split<N><<<pb, 256, 0, s>>>(a);
    k_advance<<<(unsigned)std::max(1, std::min((nint + 255) / 256, sms)), 256, 0, s>>>(a);
    st.launches += 6;
    if (!ws.ck(cudaMemcpyAsync(ws.ctl_host_, ws.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s)))
      return kErrCuda;
    if (!ws.ck(cudaStreamSynchronize(s))) return kErrCuda;
    st.iterations += 1;
    st.d2h_bytes += (long long)sizeof(Control);
    c0.iters_done = ws.ctl_host_->iters_done;
    if (ws.timing) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ws.ev[0], ws.ev[1]);
      st.ms_eval += ms;
    }
    const IterState nx = ws.ctl_host_->host;
    if (nx.overflow) {
      status = kErrCapacity;
      break;
    }
    cur ^= 1;
    hs = nx;
    n_left = nx.n_left;
  }

  // a share of the second phase (cub_integrate_shard sets phase1_out; one
  // share of one is the whole second phase, reported the same way)
  const bool shard = ws.phase1_out != nullptr;
  if (status == kOk && n_left > 0 && (ws.phase1_out || shard)) {
    // the first phase's results, before the second phase adds to them
    if (!states_fresh) {
      if (!ws.ck(cudaMemcpyAsync(h, ws.ist, sizeof(IntegralState) * nint,
                                 cudaMemcpyDeviceToHost, s)) ||
          !ws.ck(cudaStreamSynchronize(s)))
        return kErrCuda;
      st.d2h_bytes += (long long)(sizeof(IntegralState) * nint);
      states_fresh = true;
    }
    if (ws.phase1_out) detail::state_results(h, nint, ws.phase1_out);
    if (shard) {
      // the share's sums start from zero
      for (int k = 0; k < nint; ++k)
        if (h[k].state == kStatePhase2) {
          h[k].value = h[k].error = 0;
          h[k].nregions = h[k].neval = 0;
        }
      if (!ws.ck(cudaMemcpyAsync(ws.ist, h, sizeof(IntegralState) * nint,
                                 cudaMemcpyHostToDevice, s)))
        return kErrCuda;
      st.h2d_bytes += (long long)(sizeof(IntegralState) * nint);
    }
  } else if (ws.phase1_out && status == kOk) {
    ws.phase1_out = nullptr;  // filled from the final results below
  }
  long long box0 = 0, box1 = n_left;
  if (shard && n_left > 0 && opt.shard_world > 1) {
    const long long each = n_left / opt.shard_world;
    box0 = (long long)opt.shard_rank * each;
    box1 = opt.shard_rank == opt.shard_world - 1 ? n_left : box0 + each;
  }
  if (status == kOk && n_left > 0) {
    // phase 2 on the leftover boxes [box0, box1)
    states_fresh = false;
    // the heaps in shared memory when two blocks of them fit on an SM (the
    // default 2048 bisections: 98 KB a block), else in the global slab
    const size_t heap_smem = detail::phase2_heap_smem(opt.phase2_max_regions);
    const bool smem_heap =
        heap_smem <= 100 * 1024 &&
        cudaFuncSetAttribute(k_phase2<N, Src, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)heap_smem) == cudaSuccess;
    if (!smem_heap) cudaGetLastError();
    int dev_blocks = 0;
    if (smem_heap)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dev_blocks, k_phase2<N, Src, true>, 128,
                                                    heap_smem);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&dev_blocks, k_phase2<N, Src, false>, 128, 0);
    dev_blocks = std::max(1, dev_blocks);
    long long blocks = std::min<long long>((long long)sms * dev_blocks, (box1 - box0 + 3) / 4);
    blocks = std::max<long long>(blocks, 1);
    const long long nwarps = blocks * 4;
    const int stride = opt.phase2_max_regions + 2;
    if (!ws.reserve_slab(sizeof(P2Region<N>) * nwarps * stride,
                         smem_heap ? 1 : (size_t)nwarps * stride * (sizeof(P2HeapEnt) / sizeof(int))))
      return kErrCuda;
    if (shard) {
      // boxes of other shares contribute nothing to the collection
      if (!ws.ck(cudaMemsetAsync(ws.left_res, 0, sizeof(LeftoverResult) * n_left, s)))
        return kErrCuda;
      ws.counter_host = (int)box0;
      if (!ws.ck(cudaMemcpyAsync(ws.counter, &ws.counter_host, sizeof(int),
                                 cudaMemcpyHostToDevice, s)))
        return kErrCuda;
    } else if (!ws.ck(cudaMemsetAsync(ws.counter, 0, sizeof(int), s))) {
      return kErrCuda;
    }
    Phase2Args p;
    p.left_lo = ws.left_lo;
    p.left_len = ws.left_len;
    p.left_rid = ws.left_rid;
    p.left_cap = ws.left_cap();
    p.n_left = (int)box1;
    p.max_regions = opt.phase2_max_regions;
    p.slab = ws.slab;
    p.heap = reinterpret_cast<P2HeapEnt*>(ws.heap);
    p.next_box = ws.counter;
    p.out = ws.left_res;
    p.ist = ws.ist;
    // one integral's shares follow the reference's leftover order
    p.pair_half = shard && opt.shard_world > 1 && nint == 1 ? (int)(n_left / 2) : 0;
    if (ws.timing) ws.ck(cudaEventRecord(ws.ev[2], s));
    if (smem_heap)
      k_phase2<N, Src, true><<<(unsigned)blocks, 128, heap_smem, s>>>(src, T, p);
    else
      k_phase2<N, Src, false><<<(unsigned)blocks, 128, 0, s>>>(src, T, p);
    if (ws.timing) ws.ck(cudaEventRecord(ws.ev[3], s));
    st.phase2_boxes += box1 - box0;
    const unsigned cb = (unsigned)std::max(1, std::min((nint + 7) / 8, sms * 16));
    k_phase2_collect<<<cb, 256, 0, s>>>(ws.ist, nint, ws.left_res, T.npoints, shard ? 0 : 1);
    st.launches += 2;
  }

  if (!states_fresh) {
    if (!ws.ck(cudaMemcpyAsync(h, ws.ist, sizeof(IntegralState) * nint, cudaMemcpyDeviceToHost, s)))
      return kErrCuda;
    st.d2h_bytes += (long long)(sizeof(IntegralState) * nint);
    if (!ws.ck(cudaStreamSynchronize(s))) return kErrCuda;
  }
  if (!ws.ck(cudaGetLastError())) return kErrCuda;
  if (ws.timing && status == kOk && n_left > 0) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ws.ev[2], ws.ev[3]);
    st.ms_phase2 += ms;
  }
  detail::state_results(h, nint, out);
  return status;
}

// A batch prepared for replay, for instance from a CUDA graph: the stream
// work of run_batch's first persistent launch (upload of the starting
// states, one cooperative launch that lays out the initial grid and runs
// every breadth-first iteration while the list stays within the persistent
// limit, download of the states).  Every buffer is reserved by
// replay_prepare, so the pointers in the recorded work stay valid for the
// workspace's lifetime as long as nothing else reserves in it.
//
// One replay completes the batch when every integral stops inside the
// launch (converged, or out of iterations) without phase-2 boxes;
// replay_finish says whether it did.  The launch is the one run_batch makes
// first, so a completed replay equals run_batch's result; otherwise the
// caller integrates the batch with run_batch.
struct Replay {
  int nint = 0;
  int pblocks = 0;
  int per = 0, padded = 0;
  long long n0 = 0;
  PersistArgs p;
  // batches of up to kSmallBatch integrals whose initial grid is within the
  // replicated kernel's range launch it instead, as run_batch does
  bool rep = false;
  int rblocks = 0;
  RepArgs rp;
};

template <int N, class Src>
int replay_prepare(Workspace& ws, int nint, const Options& opt, cudaStream_t s, Replay* r) {
  static_assert(N >= 2 && N <= kMaxDim, "dimension out of range");
  if (nint <= 0 || !r) return kErrInvalid;
  const long long max_slots = opt.max_slots > 0 ? opt.max_slots : ws.auto_slots(N, opt.policy);
  const int sms = sm_count(ws.device());
  const int dv = grid_divisions(N);
  int per = 1;
  for (int d = 0; d < N; ++d) per *= dv;
  const int padded = (per + 31) & ~31;
  const long long n0 = (long long)nint * padded;
  const int pblocks = opt.persistent ? detail::persistent_blocks<N, Src>(ws, sms) : 0;
  const int pmax = detail::persistent_limit(opt, pblocks);
  if (pblocks <= 0 || n0 > pmax) {
    ws.set_error("replay needs the persistent kernel and an initial grid of at most " +
                 std::to_string(pmax) + " regions");
    return kErrUnsupported;
  }
  // Lists for the longest list the launch iterates on: it leaves on length
  // (n > pmax) before the capacity test (2n + 32 nint > cap) can stop it,
  // as in run_batch, whose first reservation is larger.  Leftover room as
  // run_batch reserves before its first launch.
  const long long need = 2 * n0 + 32ll * nint;
  if (need > max_slots) return kErrCapacity;
  if (!ws.reserve_integrals(nint, s)) return kErrCuda;
  if (!ws.reserve_lists(N, std::min<long long>(2ll * pmax + 32ll * nint + 64, max_slots), 0, 0,
                        s, max_slots))
    return kErrCuda;
  if (!ws.reserve_leftovers(N, opt.policy == kPolicyReference ? 4 * n0 + 1 : 1, 0, s))
    return kErrCuda;
  const RuleTables T = make_rule9_tables(N);
  EngineArgs a = detail::engine_args(ws, nint, opt, T.npoints);
  detail::bind_lists(ws, a, 0, n0);
  r->nint = nint;
  r->pblocks = pblocks;
  r->per = per;
  r->padded = padded;
  r->n0 = n0;
  r->p = detail::persist_args(ws, a, opt, 0, pmax, true, dv, per, padded, nullptr);
  r->p.host_out = ws.direct_states(nint);
  r->p.host_words = (int)(ws.state_bytes(nint) / 8);
  const int rblocks = opt.persistent && opt.replicated && nint <= kSmallBatch
                          ? detail::replicated_blocks<N, Src>(ws, sms)
                          : 0;
  const int rmax = detail::replicated_limit(opt, rblocks);
  r->rep = rblocks > 0 && n0 <= rmax;
  if (r->rep) {
    r->rblocks = rblocks;
    r->rp = detail::rep_args(ws, a, opt, 0, rmax, true, dv, per, padded, nullptr);
    r->rp.host_out = ws.direct_states(nint);
    r->rp.host_words = (int)(ws.state_bytes(nint) / 8);
  }
  return kOk;
}

// Starting states of one replay (pinned host memory; read by the upload
// that replay_enqueue records).
inline void replay_states(Workspace& ws, const Replay& r, const double* epsrel,
                          const double* epsabs) {
  const Control c0 = detail::initial_states(ws, r.nint, epsrel, epsabs, r.per, r.padded, r.n0);
  *ws.ctl_host_ = c0;
  detail::persistent_control(ws, c0.host, 0);
}

// Record (or issue) the replay's stream work on s; nothing here waits for
// the device, so the calls may be captured.
template <int N, class Src>
int replay_enqueue(Workspace& ws, const Src& src, const Replay& r, cudaStream_t s) {
  static const RuleTables T = make_rule9_tables(N);
  const size_t bytes = ws.state_bytes(r.nint);
  if (!ws.ck(cudaMemcpyAsync(ws.ctl, ws.ctl_host_, bytes, cudaMemcpyHostToDevice, s)))
    return kErrCuda;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(r.rep ? r.rblocks : r.pblocks));
  cfg.blockDim = dim3(256);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (r.rep) {
    if (!ws.ck(cudaLaunchKernelEx(&cfg, k_replicated<N, Src>, src, T, r.rp))) return kErrCuda;
  } else if (!ws.ck(cudaLaunchKernelEx(&cfg, k_persistent<N, Src>, src, T, r.p))) {
    return kErrCuda;
  }
  if (!r.p.host_out &&
      !ws.ck(cudaMemcpyAsync(ws.ctl_host_, ws.ctl, bytes, cudaMemcpyDeviceToHost, s)))
    return kErrCuda;
  return kOk;
}

// After the replay's work has completed: 1 and the results in out[0..nint)
// when the launch finished the batch, 0 when it did not (the list outgrew
// the persistent limit, or boxes went to phase 2), or a negative ErrorCode.
inline int replay_finish(Workspace& ws, const Replay& r, Result* out) {
  const Control& c = *ws.ctl_host_;
  Stats& st = ws.stats();
  st.launches += 1;
  st.persistent_launches += 1;
  st.iterations += c.iters_done;
  st.persistent_iterations += c.iters_done;
  st.h2d_bytes += (long long)ws.state_bytes(r.nint);
  st.d2h_bytes += (long long)ws.state_bytes(r.nint);
  if (c.exit_reason == kExitTimeout || c.timeout) {
    ws.ck(cudaErrorLaunchTimeout);
    return kErrTimeout;
  }
  const IterState& hs = c.host;
  if ((hs.n_running > 0 && hs.n > 0) || hs.n_left > 0) return 0;
  detail::state_results(ws.ist_host_, r.nint, out);
  return 1;
}

}  // namespace cubature
