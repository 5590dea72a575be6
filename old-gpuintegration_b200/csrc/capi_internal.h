// capi_internal.h -- shared declarations of the C ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "cubature.h"
#include "cubature/engine.cuh"

struct cub_ctx {
  int device = 0;
  // share of the second phase the next integrate call refines
  // (cub_integrate_shard); 0 of 1 otherwise
  int shard_rank = 0;
  int shard_world = 1;
  cudaStream_t stream = nullptr;
  cubature::Workspace* ws = nullptr;
  cubature::GenzParams* d_params = nullptr;
  int params_cap = 0;
  double* d_aux = nullptr;  // per-integral scalars of the table integrands
  int aux_cap = 0;
  int* d_fams = nullptr;  // per-integral families of mixed batches
  int fams_cap = 0;
};

namespace cubature {
namespace capi {

void set_error(const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
// Map an engine return code to the C ABI (sets the message).
int engine_status(cub_ctx* ctx, int rc);
void result_to_c(const Result& r, cub_result* c);
cudaStream_t as_stream(void* s);
Options to_options(const cub_options* opt);

// Per-dimension entry points, one translation unit per dimension
// (capi_dim.cu compiled with -DCUB_DIM=N).
#define CUB_DECLARE_DIM(N)                                                                     \
  int run_dim_##N(cub_ctx* ctx, int family, int count, const GenzParams* h_params,             \
                  const GenzParams* d_params, const double* epsrel, const double* epsabs,      \
                  const Options& opt, Result* out, const double* h_box);                       \
  int run_mixed_dim_##N(cub_ctx* ctx, int count, const GenzParams* d_params, const int* d_fams,  \
                        const double* epsrel, const double* epsabs, const Options& opt,         \
                        Result* out);                                                           \
  int rule_eval_dim_##N(int family, const GenzParams& p, long long n, const double* lo,        \
                        const double* len, long long ld, double epsrel, double epsabs,         \
                        double* avg, double* err, int* axis, int* active, cudaStream_t s);     \
  int split_dim_##N(long long n, const double* lo, const double* len, long long ld,            \
                    const int* active, const int* axis, double* olo, double* olen,             \
                    long long old, int layout, long long* count, int* cnt, int* excl,          \
                    cudaStream_t s);                                                           \
  int replay_prepare_dim_##N(int family, Workspace& ws, int count, const Options& opt,          \
                             cudaStream_t s, Replay* r);                                        \
  int replay_enqueue_dim_##N(int family, Workspace& ws, const GenzParams* d_params,             \
                             const Replay& r, cudaStream_t s);
CUB_DECLARE_DIM(2)
CUB_DECLARE_DIM(3)
CUB_DECLARE_DIM(4)
CUB_DECLARE_DIM(5)
CUB_DECLARE_DIM(6)
CUB_DECLARE_DIM(7)
CUB_DECLARE_DIM(8)
#undef CUB_DECLARE_DIM

// Integrate `count` independent integrals in groups that share one region
// list.  run(idx, out) integrates the integrals idx (indices into the batch)
// and returns an engine code.  Under the reference policy an integral's list
// stays below 2 * phase1_cap + 96 slots, so groups of max_slots / that size
// always fit.  Under the breadth policy lists are unbounded: with `ws` given
// (the workspace run uses) and at least 4 * kProbeGroup integrals, the first
// kProbeGroup integrals run as a group of their own, and later groups are
// sized so that their widest iteration needs about 3/4 of max_slots at the
// capacity per integral that the probe group needed; otherwise the whole
// batch is tried at once.  Integrals still running when the capacity ran out
// are integrated again in groups a quarter the size.  Integrals are
// independent, so a rerun gives the same result up to the order in which
// points are summed: the list length of a group decides whether the
// persistent or the multi-launch rule kernel evaluates an iteration.  Returns kOk,
// kErrCapacity (some integral never fit; its result is the last estimate)
// or the first error.
constexpr int kProbeGroup = 256;

template <class Run>
int grouped_batch(int count, const Options& o, Run&& run, std::vector<Result>& res,
                  const Workspace* ws = nullptr) {
  res.assign(count, Result());
  int group = count;
  const bool bounded = o.policy == kPolicyReference && o.phase1_cap > 0;
  if (bounded) {
    const long long per = 2ll * o.phase1_cap + 96;
    group = (int)std::max<long long>(1, std::min<long long>(count, o.max_slots / per));
  }
  int probe = (!bounded && ws && o.max_slots > 0 && count >= 4 * kProbeGroup) ? kProbeGroup : 0;
  std::vector<int> todo(count), idx;
  for (int k = 0; k < count; ++k) todo[k] = k;
  std::vector<Result> gres;
  int rc = kOk;
  while (!todo.empty()) {
    std::vector<int> again;
    for (size_t g0 = 0; g0 < todo.size();) {
      const int gn = (int)std::min<size_t>(probe ? probe : group, todo.size() - g0);
      idx.assign(todo.begin() + g0, todo.begin() + g0 + gn);
      gres.assign(gn, Result());
      const int r = run(idx, gres.data());
      if (r != kOk && r != kErrCapacity) return r;
      for (int j = 0; j < gn; ++j) {
        res[idx[j]] = gres[j];
        if (r == kErrCapacity && group > 1 && gres[j].state == kStateRunning)
          again.push_back(idx[j]);
      }
      if (r == kErrCapacity && (group == 1 || again.empty())) rc = kErrCapacity;
      if (probe) {
        probe = 0;
        if (r == kOk && ws->peak_need > 0) {
          const long long per = std::max<long long>(1, ws->peak_need / gn);
          group = (int)std::max<long long>(1, std::min<long long>(count, o.max_slots * 3 / 4 / per));
        }
      }
      g0 += gn;
    }
    todo.swap(again);
    group = std::max(1, group / 4);
  }
  return rc;
}

}  // namespace capi
}  // namespace cubature
