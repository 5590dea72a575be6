// graph.cu -- replayable batches: the persistent launch of one or more
// batches captured once in a CUDA graph and replayed by every call.
//
// Each entry of a graph is a batch of `count` integrals of one family and
// dimension over the unit cube, with its own workspace (region lists, the
// control block and its pinned host copy) and a pinned parameter buffer.
// The graph holds, per entry in order: the parameter upload, the state
// upload, the cooperative persistent launch and the state download.  A call
// writes parameters and starting states into the pinned buffers, launches
// the graph once and waits once.  An entry whose launch did not finish its
// batch (the list outgrew the persistent kernel's limit, or boxes went to
// phase 2) is integrated again by cub_integrate_batch on the context's own
// workspace, so every result equals cub_integrate_batch's.
#include <cstring>

#include "capi_internal.h"

using namespace cubature;
using namespace cubature::capi;

struct cub_graph {
  struct Entry {
    int family = 0, ndim = 0, count = 0, offset = 0;
    Workspace* ws = nullptr;
    GenzParams* d_params = nullptr;
    GenzParams* h_params = nullptr;  // pinned
    Replay r;
  };
  cub_ctx* ctx = nullptr;
  std::vector<Entry> entries;
  int total = 0;
  cub_options opt;
  bool has_opt = false;
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long replays = 0, reruns = 0;
};

namespace {

using PrepareFn = int (*)(int, Workspace&, int, const Options&, cudaStream_t, Replay*);
using EnqueueFn = int (*)(int, Workspace&, const GenzParams*, const Replay&, cudaStream_t);

PrepareFn prepare_fn(int ndim) {
  switch (ndim) {
    case 2: return replay_prepare_dim_2;
    case 3: return replay_prepare_dim_3;
    case 4: return replay_prepare_dim_4;
    case 5: return replay_prepare_dim_5;
    case 6: return replay_prepare_dim_6;
    case 7: return replay_prepare_dim_7;
    case 8: return replay_prepare_dim_8;
  }
  return nullptr;
}

EnqueueFn enqueue_fn(int ndim) {
  switch (ndim) {
    case 2: return replay_enqueue_dim_2;
    case 3: return replay_enqueue_dim_3;
    case 4: return replay_enqueue_dim_4;
    case 5: return replay_enqueue_dim_5;
    case 6: return replay_enqueue_dim_6;
    case 7: return replay_enqueue_dim_7;
    case 8: return replay_enqueue_dim_8;
  }
  return nullptr;
}

// Map an engine code from an entry's workspace to the C ABI.
int entry_status(const Workspace& ws, int rc, const char* what) {
  switch (rc) {
    case kOk:
      return 0;
    case kErrCuda:
      set_error(std::string(what) + ": " + ws.error());
      return CUB_ERR_CUDA;
    case kErrTimeout:
      set_error("a device-side grid barrier wait ran out (persistent kernel)");
      return CUB_ERR_TIMEOUT;
    case kErrCapacity:
      set_error(std::string(what) + ": the initial grid does not fit the region capacity");
      return CUB_ERR_CAPACITY;
    case kErrUnsupported:
      set_error(std::string(what) + ": " + ws.error());
      return CUB_ERR_UNSUPPORTED;
    default:
      set_error(std::string(what) + ": invalid argument");
      return rc < 0 ? rc : CUB_ERR_INVALID;
  }
}

void free_graph(cub_graph* g) {
  if (!g) return;
  cudaSetDevice(g->ctx->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto& e : g->entries) {
    delete e.ws;
    if (e.d_params) cudaFree(e.d_params);
    if (e.h_params) cudaFreeHost(e.h_params);
  }
  if (g->capture) cudaStreamDestroy(g->capture);
  delete g;
}

}  // namespace

extern "C" {

int cub_graph_create(cub_ctx* ctx, int nentries, const int* families, const int* ndims,
                     const int* counts, const cub_options* opt, cub_graph** out) {
  if (!ctx || nentries <= 0 || !families || !ndims || !counts || !out) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  *out = nullptr;
  for (int i = 0; i < nentries; ++i) {
    if (ndims[i] < CUB_MIN_NDIM || ndims[i] > CUB_MAX_NDIM || families[i] < CUB_GAUSSIAN ||
        families[i] > CUB_COSSUM || counts[i] <= 0) {
      set_error("graph entry " + std::to_string(i) + ": family, ndim or count out of range");
      return CUB_ERR_INVALID;
    }
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  cub_graph* g = new cub_graph();
  g->ctx = ctx;
  if (opt) {
    g->opt = *opt;
    g->has_opt = true;
  }
  const Options o = to_options(opt);
  if ((e = cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking)) != cudaSuccess) {
    free_graph(g);
    return cuda_error(e, "cudaStreamCreateWithFlags");
  }
  for (int i = 0; i < nentries; ++i) {
    cub_graph::Entry en;
    en.family = families[i];
    en.ndim = ndims[i];
    en.count = counts[i];
    en.offset = g->total;
    g->total += counts[i];
    g->entries.push_back(en);
    cub_graph::Entry& x = g->entries.back();
    x.ws = new Workspace(ctx->device);
    if ((e = cudaMalloc(&x.d_params, sizeof(GenzParams) * x.count)) != cudaSuccess ||
        (e = cudaMallocHost(&x.h_params, sizeof(GenzParams) * x.count)) != cudaSuccess) {
      free_graph(g);
      return cuda_error(e, "graph parameter buffers");
    }
    std::memset(x.h_params, 0, sizeof(GenzParams) * x.count);
    const int rc = prepare_fn(x.ndim)(x.family, *x.ws, x.count, o, g->capture, &x.r);
    if (rc != kOk) {
      const int c = entry_status(*x.ws, rc, ("graph entry " + std::to_string(i)).c_str());
      free_graph(g);
      return c;
    }
  }
  if ((e = cudaStreamSynchronize(g->capture)) != cudaSuccess) {
    free_graph(g);
    return cuda_error(e, "cudaStreamSynchronize");
  }
  // record every entry's work once
  if ((e = cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
    free_graph(g);
    return cuda_error(e, "cudaStreamBeginCapture");
  }
  int rc = kOk;
  size_t bad = 0;
  for (size_t i = 0; i < g->entries.size() && rc == kOk; ++i) {
    cub_graph::Entry& x = g->entries[i];
    bad = i;
    if (cudaMemcpyAsync(x.d_params, x.h_params, sizeof(GenzParams) * x.count,
                        cudaMemcpyHostToDevice, g->capture) != cudaSuccess) {
      rc = kErrCuda;
      x.ws->set_error("parameter upload could not be recorded");
    } else {
      rc = enqueue_fn(x.ndim)(x.family, *x.ws, x.d_params, x.r, g->capture);
    }
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(g->capture, &graph);
  g->graph = graph;
  if (rc != kOk) {
    const int c = entry_status(*g->entries[bad].ws, rc, "graph capture");
    free_graph(g);
    return c;
  }
  if (ec != cudaSuccess) {
    free_graph(g);
    return cuda_error(ec, "cudaStreamEndCapture");
  }
  if ((e = cudaGraphInstantiate(&g->exec, g->graph, 0)) != cudaSuccess) {
    free_graph(g);
    return cuda_error(e, "cudaGraphInstantiate");
  }
  *out = g;
  return 0;
}

int cub_graph_launch(cub_graph* g, const cub_genz_params* params, const double* epsrel,
                     const double* epsabs, cub_result* out) {
  if (!g || !params || !epsrel || !epsabs || !out) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  for (int k = 0; k < g->total; ++k)
    if (!(epsrel[k] >= 0) || !(epsabs[k] >= 0)) {
      set_error("epsrel/epsabs must be >= 0");
      return CUB_ERR_INVALID;
    }
  cub_ctx* ctx = g->ctx;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  static_assert(sizeof(cub_genz_params) == sizeof(GenzParams), "params layout");
  for (auto& x : g->entries) {
    std::memcpy(x.h_params, params + x.offset, sizeof(GenzParams) * x.count);
    replay_states(*x.ws, x.r, epsrel + x.offset, epsabs + x.offset);
  }
  if ((e = cudaGraphLaunch(g->exec, ctx->stream)) != cudaSuccess)
    return cuda_error(e, "cudaGraphLaunch");
  if ((e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess)
    return cuda_error(e, "cudaStreamSynchronize");
  g->replays += 1;
  std::vector<Result> res;
  int status = 0;
  for (auto& x : g->entries) {
    res.assign(x.count, Result());
    const int rc = replay_finish(*x.ws, x.r, res.data());
    if (rc < 0) return entry_status(*x.ws, rc, "graph launch");
    if (rc == 1) {
      for (int k = 0; k < x.count; ++k) result_to_c(res[k], out + x.offset + k);
      continue;
    }
    // the launch stopped short of the end: the ordinary path finishes it
    g->reruns += 1;
    const int r = cub_integrate_batch(ctx, x.family, x.ndim, x.count, params + x.offset,
                                      epsrel + x.offset, epsabs + x.offset, 0.0, 0.0,
                                      g->has_opt ? &g->opt : nullptr, out + x.offset);
    if (r < 0 && r != CUB_ERR_CAPACITY) return r;
    if (r == CUB_ERR_CAPACITY) status = r;
  }
  return status;
}

int cub_graph_info(const cub_graph* g, long long* replays, long long* reruns) {
  if (!g) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  if (replays) *replays = g->replays;
  if (reruns) *reruns = g->reruns;
  return 0;
}

void cub_graph_destroy(cub_graph* g) { free_graph(g); }

}  // extern "C"
