// capi.cu -- the C ABI (include/cubature.h): contexts, dispatch by
// dimension and family, per-step entry points.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "capi_internal.h"
#include "cubature/step_kernels.cuh"

namespace cubature {
namespace capi {

namespace {
thread_local std::string g_error;
}

void set_error(const std::string& msg) { g_error = msg; }

int cuda_error(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return CUB_ERR_CUDA;
}

int engine_status(cub_ctx* ctx, int rc) {
  switch (rc) {
    case kOk:
      return 0;
    case kErrCuda:
      if (!ctx->ws->error().empty()) set_error(ctx->ws->error());
      return CUB_ERR_CUDA;
    case kErrTimeout:
      set_error("a device-side grid barrier wait ran out (persistent kernel)");
      return CUB_ERR_TIMEOUT;
    case kErrCapacity:
      set_error("region capacity exceeded; results are the last estimates");
      return CUB_ERR_CAPACITY;
    default:
      set_error("invalid argument");
      return rc < 0 ? rc : CUB_ERR_INVALID;
  }
}

void result_to_c(const Result& r, cub_result* c) {
  c->value = r.value;
  c->error = r.error;
  c->nregions = r.nregions;
  c->neval = r.neval;
  c->status = r.status;
  c->iterations = r.iterations;
  c->state = r.state;
  c->reserved = 0;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

Options to_options(const cub_options* opt) {
  Options o;
  if (!opt) return o;
  o.policy = opt->policy;
  if (opt->phase1_cap > 0) o.phase1_cap = opt->phase1_cap;
  if (opt->max_iters > 0) o.max_iters = opt->max_iters;
  if (opt->phase2_max_regions > 0) o.phase2_max_regions = opt->phase2_max_regions;
  if (opt->max_slots > 0) o.max_slots = opt->max_slots;
  o.lanes = opt->lanes;
  o.persistent = opt->no_persistent ? 0 : 1;
  if (opt->persistent_max_n > 0) o.persistent_max_n = opt->persistent_max_n;
  if (opt->persistent_max_r > 0) o.persistent_max_r = opt->persistent_max_r;
  o.replicated = opt->no_replicated ? 0 : 1;
  if (opt->barrier_spins > 0) o.barrier_spins = opt->barrier_spins;
  o.hold_block = opt->test_hold_block > 0 ? opt->test_hold_block - 1 : -1;
  o.device_loop = opt->no_device_loop ? 0 : 1;
  return o;
}

namespace {

bool check_ndim(int ndim) {
  if (ndim < CUB_MIN_NDIM || ndim > CUB_MAX_NDIM) {
    set_error("ndim " + std::to_string(ndim) + " outside the built range [" +
              std::to_string(CUB_MIN_NDIM) + ", " + std::to_string(CUB_MAX_NDIM) + "]");
    return false;
  }
  return true;
}

bool check_family(int family) {
  if (family < CUB_GAUSSIAN || family > CUB_COSSUM) {
    set_error("unknown integrand family " + std::to_string(family));
    return false;
  }
  return true;
}

int cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  return CUB_ERR_CUDA;
}

int dispatch_run(cub_ctx* ctx, int family, int ndim, int count, const GenzParams* h,
                 const GenzParams* d, const double* er, const double* ea, const Options& o,
                 Result* out, const double* box) {
  switch (ndim) {
    case 2: return run_dim_2(ctx, family, count, h, d, er, ea, o, out, box);
    case 3: return run_dim_3(ctx, family, count, h, d, er, ea, o, out, box);
    case 4: return run_dim_4(ctx, family, count, h, d, er, ea, o, out, box);
    case 5: return run_dim_5(ctx, family, count, h, d, er, ea, o, out, box);
    case 6: return run_dim_6(ctx, family, count, h, d, er, ea, o, out, box);
    case 7: return run_dim_7(ctx, family, count, h, d, er, ea, o, out, box);
    case 8: return run_dim_8(ctx, family, count, h, d, er, ea, o, out, box);
  }
  return CUB_ERR_INVALID;
}

void to_c(const Result& r, cub_result* c) {
  c->value = r.value;
  c->error = r.error;
  c->nregions = r.nregions;
  c->neval = r.neval;
  c->status = r.status;
  c->iterations = r.iterations;
  c->state = r.state;
  c->reserved = 0;
}

}  // namespace
}  // namespace capi
}  // namespace cubature

using namespace cubature;
using namespace cubature::capi;

extern "C" {

int cub_version(void) { return (0 << 16) | 1; }

const char* cub_last_error(void) { return g_error.c_str(); }

void cub_default_options(cub_options* opt) {
  if (!opt) return;
  const Options o;
  std::memset(opt, 0, sizeof(*opt));
  opt->policy = o.policy;
  opt->phase1_cap = o.phase1_cap;
  opt->max_iters = o.max_iters;
  opt->phase2_max_regions = o.phase2_max_regions;
  opt->max_slots = o.max_slots;
  opt->lanes = o.lanes;
  opt->no_persistent = o.persistent ? 0 : 1;
  opt->persistent_max_n = o.persistent_max_n;
  opt->persistent_max_r = o.persistent_max_r;
  opt->no_replicated = o.replicated ? 0 : 1;
  opt->barrier_spins = 0;
  opt->test_hold_block = 0;
  opt->no_device_loop = o.device_loop ? 0 : 1;
}

cub_ctx* cub_create(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
    return nullptr;
  }
  if (device < 0 || device >= n) {
    set_error("device index out of range");
    return nullptr;
  }
  if ((e = cudaSetDevice(device)) != cudaSuccess) {
    set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return nullptr;
  }
  cub_ctx* ctx = new cub_ctx();
  ctx->device = device;
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) {
    set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    delete ctx;
    return nullptr;
  }
  ctx->ws = new Workspace(device);
  return ctx;
}

void cub_destroy(cub_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  delete ctx->ws;
  if (ctx->d_params) cudaFree(ctx->d_params);
  if (ctx->d_aux) cudaFree(ctx->d_aux);
  if (ctx->d_fams) cudaFree(ctx->d_fams);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

size_t cub_ctx_bytes(const cub_ctx* ctx) { return ctx && ctx->ws ? ctx->ws->bytes_reserved() : 0; }

void* cub_ctx_stream(cub_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int cub_ctx_stats(const cub_ctx* ctx, cub_stats* out) {
  if (!ctx || !out) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const Stats& s = ctx->ws->stats();
  out->ms_eval = s.ms_eval;
  out->ms_phase2 = s.ms_phase2;
  out->eval_launches = s.eval_launches;
  out->launches = s.launches;
  out->regions_evaluated = s.regions_evaluated;
  out->iterations = s.iterations;
  out->phase2_boxes = s.phase2_boxes;
  out->h2d_bytes = s.h2d_bytes;
  out->d2h_bytes = s.d2h_bytes;
  out->ms_persistent = s.ms_persistent;
  out->persistent_launches = s.persistent_launches;
  out->persistent_iterations = s.persistent_iterations;
  out->replicated_launches = s.replicated_launches;
  out->persistent_regions = s.persistent_regions;
  out->device_loops = s.device_loops;
  return 0;
}

int cub_ctx_trace(const cub_ctx* ctx, unsigned long long* out) {
  if (!ctx || !out) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const Control* c = ctx->ws->ctl_host_;
  for (int i = 0; i < 64; ++i) out[i] = c ? c->trace[i] : 0;
  return 0;
}

void cub_ctx_release(cub_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  ctx->ws->release();
  if (ctx->d_params) cudaFree(ctx->d_params);
  ctx->d_params = nullptr;
  ctx->params_cap = 0;
  if (ctx->d_aux) cudaFree(ctx->d_aux);
  ctx->d_aux = nullptr;
  ctx->aux_cap = 0;
  if (ctx->d_fams) cudaFree(ctx->d_fams);
  ctx->d_fams = nullptr;
  ctx->fams_cap = 0;
}

void cub_ctx_reset_stats(cub_ctx* ctx) {
  if (ctx) ctx->ws->stats() = Stats();
}

void cub_ctx_set_timing(cub_ctx* ctx, int on) {
  if (ctx) ctx->ws->timing = on != 0;
}

namespace {

// Shared body of the integrate entry points; lo/hi are [count][ndim] host
// arrays (both null: the unit cube).
int integrate_impl(cub_ctx* ctx, int family, int ndim, int count, const cub_genz_params* params,
                   const double* lo, const double* hi, const double* epsrel,
                   const double* epsabs, double epsrel0, double epsabs0, const cub_options* opt,
                   cub_result* out) {
  if (!ctx || !params || !out || count <= 0 || (!lo) != (!hi)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  if (!check_ndim(ndim) || !check_family(family)) return CUB_ERR_INVALID;
  if (lo) {
    for (long long i = 0; i < (long long)count * ndim; ++i)
      if (!(std::isfinite(lo[i]) && std::isfinite(hi[i]) && hi[i] > lo[i])) {
        set_error("integration box needs finite bounds with hi > lo");
        return CUB_ERR_INVALID;
      }
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  static_assert(sizeof(cub_genz_params) == sizeof(GenzParams), "params layout");
  const GenzParams* h = reinterpret_cast<const GenzParams*>(params);
  if (count == 1) {
    // one integral (the drop-in call): no grouping and no staging vectors;
    // the same run as a group of one
    const double er1 = epsrel ? epsrel[0] : epsrel0, ea1 = epsabs ? epsabs[0] : epsabs0;
    if (!(er1 >= 0) || !(ea1 >= 0)) {
      set_error("epsrel/epsabs must be >= 0");
      return CUB_ERR_INVALID;
    }
    Options o = to_options(opt);
    if (o.max_slots <= 0) o.max_slots = ctx->ws->auto_slots(ndim, o.policy);
    o.shard_rank = ctx->shard_rank;
    o.shard_world = ctx->shard_world;
    double box[2 * kMaxDim];
    if (lo)
      for (int d = 0; d < ndim; ++d) {
        box[d] = lo[d];
        box[ndim + d] = hi[d];
      }
    Result r{};
    const int rc = dispatch_run(ctx, family, ndim, 1, h, nullptr, &er1, &ea1, o, &r,
                                lo ? box : nullptr);
    if (rc == kErrCuda) {
      set_error(ctx->ws->error());
      return CUB_ERR_CUDA;
    }
    if (rc == kErrTimeout) {
      set_error("a device-side grid barrier wait ran out (persistent kernel)");
      return CUB_ERR_TIMEOUT;
    }
    if (rc == kErrCapacity) set_error("region capacity exceeded; results are the last estimates");
    if (rc < 0 && rc != kErrCapacity) return rc;
    to_c(r, out);
    return rc == kErrCapacity ? CUB_ERR_CAPACITY : 0;
  }
  std::vector<double> er(count), ea(count);
  for (int k = 0; k < count; ++k) {
    er[k] = epsrel ? epsrel[k] : epsrel0;
    ea[k] = epsabs ? epsabs[k] : epsabs0;
    if (!(er[k] >= 0) || !(ea[k] >= 0)) {
      set_error("epsrel/epsabs must be >= 0");
      return CUB_ERR_INVALID;
    }
  }
  if (count > 1 && count > ctx->params_cap) {
    if (ctx->d_params) cudaFree(ctx->d_params);
    ctx->d_params = nullptr;
    ctx->params_cap = 0;
    if ((e = cudaMalloc(&ctx->d_params, sizeof(GenzParams) * count)) != cudaSuccess)
      return cuda_fail(e, "cudaMalloc(params)");
    ctx->params_cap = count;
  }
  Options o = to_options(opt);
  if (o.max_slots <= 0) o.max_slots = ctx->ws->auto_slots(ndim, o.policy);
  o.shard_rank = ctx->shard_rank;
  o.shard_world = ctx->shard_world;
  std::vector<Result> res;
  std::vector<GenzParams> hp;
  std::vector<double> ger, gea, gbox;
  const int rc = grouped_batch(count, o, [&](const std::vector<int>& idx, Result* gout) {
    const int gn = (int)idx.size();
    hp.resize(gn);
    ger.resize(gn);
    gea.resize(gn);
    for (int j = 0; j < gn; ++j) {
      hp[j] = h[idx[j]];
      ger[j] = er[idx[j]];
      gea[j] = ea[idx[j]];
    }
    if (lo) {
      // per integral: lo[ndim] then hi[ndim]
      gbox.resize((size_t)gn * 2 * ndim);
      for (int j = 0; j < gn; ++j)
        for (int d = 0; d < ndim; ++d) {
          gbox[(size_t)j * 2 * ndim + d] = lo[(size_t)idx[j] * ndim + d];
          gbox[(size_t)j * 2 * ndim + ndim + d] = hi[(size_t)idx[j] * ndim + d];
        }
    }
    const GenzParams* d = nullptr;
    if (gn > 1) {
      if (cudaMemcpyAsync(ctx->d_params, hp.data(), sizeof(GenzParams) * gn,
                          cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        return (int)kErrCuda;
      ctx->ws->stats().h2d_bytes += (long long)(sizeof(GenzParams) * gn);
      d = ctx->d_params;
    }
    return dispatch_run(ctx, family, ndim, gn, hp.data(), d, ger.data(), gea.data(), o, gout,
                        lo ? gbox.data() : nullptr);
  }, res, ctx->ws);
  if (rc == kErrCuda) {
    set_error(ctx->ws->error());
    return CUB_ERR_CUDA;
  }
  if (rc == kErrTimeout) {
    set_error("a device-side grid barrier wait ran out (persistent kernel)");
    return CUB_ERR_TIMEOUT;
  }
  if (rc == kErrCapacity) set_error("region capacity exceeded; results are the last estimates");
  if (rc < 0 && rc != kErrCapacity) return rc;
  for (int k = 0; k < count; ++k) to_c(res[k], &out[k]);
  return rc == kErrCapacity ? CUB_ERR_CAPACITY : 0;
}

}  // namespace

int cub_integrate_batch(cub_ctx* ctx, int family, int ndim, int count,
                        const cub_genz_params* params, const double* epsrel,
                        const double* epsabs, double epsrel0, double epsabs0,
                        const cub_options* opt, cub_result* out) {
  return integrate_impl(ctx, family, ndim, count, params, nullptr, nullptr, epsrel, epsabs,
                        epsrel0, epsabs0, opt, out);
}

int cub_integrate_batch_box(cub_ctx* ctx, int family, int ndim, int count,
                            const cub_genz_params* params, const double* lo, const double* hi,
                            const double* epsrel, const double* epsabs, double epsrel0,
                            double epsabs0, const cub_options* opt, cub_result* out) {
  return integrate_impl(ctx, family, ndim, count, params, lo, hi, epsrel, epsabs, epsrel0,
                        epsabs0, opt, out);
}

int cub_integrate(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                  double epsrel, double epsabs, const cub_options* opt, cub_result* out) {
  return integrate_impl(ctx, family, ndim, 1, params, nullptr, nullptr, nullptr, nullptr, epsrel,
                        epsabs, opt, out);
}

int cub_integrate_shard(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                        double epsrel, double epsabs, const cub_options* opt, int rank,
                        int world, cub_result* phase1, cub_result* part) {
  if (!ctx || !phase1 || !part || world < 1 || rank < 0 || rank >= world) {
    set_error("invalid argument: need 0 <= rank < world and both outputs");
    return CUB_ERR_INVALID;
  }
  cub_options o;
  if (opt)
    o = *opt;
  else
    cub_default_options(&o);
  Result p1{};
  ctx->ws->phase1_out = &p1;
  ctx->shard_rank = rank;
  ctx->shard_world = world;
  const int rc = integrate_impl(ctx, family, ndim, 1, params, nullptr, nullptr, nullptr, nullptr,
                                epsrel, epsabs, &o, part);
  const bool split = ctx->ws->phase1_out != nullptr;
  ctx->ws->phase1_out = nullptr;
  ctx->shard_rank = 0;
  ctx->shard_world = 1;
  if (rc < 0) return rc;
  if (split) {
    result_to_c(p1, phase1);
  } else {
    // finished in the first phase: every rank holds the whole result
    *phase1 = *part;
    std::memset(part, 0, sizeof(*part));
  }
  return 0;
}

int cub_integrate_box(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                      const double* lo, const double* hi, double epsrel, double epsabs,
                      const cub_options* opt, cub_result* out) {
  if (!lo || !hi) {
    set_error("invalid argument: lo and hi are required");
    return CUB_ERR_INVALID;
  }
  return integrate_impl(ctx, family, ndim, 1, params, lo, hi, nullptr, nullptr, epsrel, epsabs,
                        opt, out);
}

int cub_rule_tables(int ndim, double* wt, double* scale, double* norm, int* count) {
  if (ndim < 2 || ndim > CUB_MAXDIM) {
    set_error("ndim out of range");
    return CUB_ERR_INVALID;
  }
  const RuleTables T = make_rule9_tables(ndim);
  if (wt) std::memcpy(wt, T.wt, sizeof(T.wt));
  if (scale) std::memcpy(scale, T.scale, sizeof(T.scale));
  if (norm) std::memcpy(norm, T.norm, sizeof(T.norm));
  if (count) std::memcpy(count, T.count, sizeof(T.count));
  return 0;
}

int cub_rule_eval(int family, int ndim, const cub_genz_params* params, long long n,
                  const double* d_lo, const double* d_len, long long ld, double epsrel,
                  double epsabs, double* d_avg, double* d_err, int* d_axis, int* d_active,
                  void* stream) {
  if (!check_ndim(ndim) || !check_family(family)) return CUB_ERR_INVALID;
  if (!params || n < 0 || ld < n || (n > 0 && (!d_lo || !d_len || !d_avg || !d_err || !d_axis ||
                                                 !d_active))) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  if (n == 0) return 0;
  const GenzParams& p = *reinterpret_cast<const GenzParams*>(params);
  const cudaStream_t s = as_stream(stream);
  int rc = CUB_ERR_INVALID;
  switch (ndim) {
#define CUB_RULE_CASE(N)                                                                        \
  case N:                                                                                      \
    rc = rule_eval_dim_##N(family, p, n, d_lo, d_len, ld, epsrel, epsabs, d_avg, d_err, d_axis, \
                           d_active, s);                                                       \
    break;
    CUB_RULE_CASE(2) CUB_RULE_CASE(3) CUB_RULE_CASE(4) CUB_RULE_CASE(5) CUB_RULE_CASE(6)
    CUB_RULE_CASE(7) CUB_RULE_CASE(8)
#undef CUB_RULE_CASE
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "rule kernel launch");
  return rc;
}

size_t cub_split_scratch_bytes(long long n) {
  const long long nchunk = (n + 31) / 32;
  return sizeof(int) * 2 * (size_t)(nchunk + 1);
}

size_t cub_reduce_scratch_bytes(long long) { return sizeof(double) * 4 * kReduceBlocks; }

int cub_split(int ndim, long long n, const double* d_lo, const double* d_len, long long ld,
              const int* d_active, const int* d_axis, double* d_out_lo, double* d_out_len,
              long long out_ld, int layout, long long* d_count, void* d_scratch,
              size_t scratch_bytes, void* stream) {
  if (!check_ndim(ndim)) return CUB_ERR_INVALID;
  if (n < 0 || ld < n || !d_count || (layout != 0 && layout != 1) ||
      scratch_bytes < cub_split_scratch_bytes(n) || (n > 0 && !d_scratch)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const cudaStream_t s = as_stream(stream);
  if (n == 0) {
    const cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(long long), s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "cudaMemsetAsync");
  }
  int* cnt = static_cast<int*>(d_scratch);
  int* excl = cnt + (n + 31) / 32 + 1;
  int rc = CUB_ERR_INVALID;
  switch (ndim) {
#define CUB_SPLIT_CASE(N)                                                                      \
  case N:                                                                                     \
    rc = split_dim_##N(n, d_lo, d_len, ld, d_active, d_axis, d_out_lo, d_out_len, out_ld,     \
                       layout, d_count, cnt, excl, s);                                        \
    break;
    CUB_SPLIT_CASE(2) CUB_SPLIT_CASE(3) CUB_SPLIT_CASE(4) CUB_SPLIT_CASE(5) CUB_SPLIT_CASE(6)
    CUB_SPLIT_CASE(7) CUB_SPLIT_CASE(8)
#undef CUB_SPLIT_CASE
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "split kernel launch");
  return rc;
}

int cub_reduce(long long n, const double* d_avg, const double* d_err, const int* d_active,
               double* d_out, void* d_scratch, size_t scratch_bytes, void* stream) {
  if (n < 0 || !d_out || scratch_bytes < cub_reduce_scratch_bytes(n) || !d_scratch ||
      (n > 0 && (!d_avg || !d_err || !d_active))) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const cudaStream_t s = as_stream(stream);
  double* part = static_cast<double*>(d_scratch);
  const long long want = (n + 255) / 256;
  const int blocks = (int)std::max<long long>(1, std::min<long long>(want, kReduceBlocks));
  k_step_reduce<<<blocks, 256, 0, s>>>(n, d_avg, d_err, d_active, part);
  k_step_reduce_final<<<1, 32, 0, s>>>(blocks, part, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "reduce kernel launch");
  return 0;
}

}  // extern "C"

int cub_autotune_batch(cub_ctx* ctx, int family, int ndim, int count,
                       const cub_genz_params* params, double epsrel, double epsabs, int sample,
                       const cub_options* opt, cub_options* best, double* best_ms) {
  if (!ctx || !params || !best || count <= 0) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const int n = sample > 0 ? std::min(sample, count) : count;
  cub_options base;
  if (opt)
    base = *opt;
  else
    cub_default_options(&base);
  std::vector<cub_options> cands;
  for (int r : {1, 2, 4, 8})
    for (int pm : {0, 4096}) {
      cub_options c = base;
      c.no_persistent = 0;
      c.persistent_max_r = r;
      c.persistent_max_n = pm;
      cands.push_back(c);
    }
  for (int lanes : {1, 8, 32}) {
    cub_options c = base;
    c.no_persistent = 1;
    c.lanes = lanes;
    cands.push_back(c);
  }
  std::vector<cub_result> out(n);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    return cuda_fail(cudaGetLastError(), "cudaEventCreate");
  double bt = 1e300;
  int bi = -1;
  int rc = 0;
  for (size_t i = 0; i < cands.size() && rc == 0; ++i) {
    double t = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
      cudaEventRecord(e0, ctx->stream);
      const int r = cub_integrate_batch(ctx, family, ndim, n, params, nullptr, nullptr, epsrel,
                                        epsabs, &cands[i], out.data());
      cudaEventRecord(e1, ctx->stream);
      if (r < 0 && r != CUB_ERR_CAPACITY) {
        rc = r;
        break;
      }
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r == 0) t = std::min(t, (double)ms);
    }
    if (t < bt) {
      bt = t;
      bi = (int)i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (bi < 0) {
    set_error("autotune: no candidate completed the batch");
    return CUB_ERR_CAPACITY;
  }
  *best = cands[bi];
  if (best_ms) *best_ms = bt;
  return 0;
}

int cub_integrate_mixed_batch(cub_ctx* ctx, int ndim, int count, const int* families,
                              const cub_genz_params* params, const double* epsrel,
                              const double* epsabs, double epsrel0, double epsabs0,
                              const cub_options* opt, cub_result* out) {
  if (!ctx || !families || !params || !out || count <= 0) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  if (!check_ndim(ndim)) return CUB_ERR_INVALID;
  for (int k = 0; k < count; ++k)
    if (!check_family(families[k])) return CUB_ERR_INVALID;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  std::vector<double> er(count), ea(count);
  for (int k = 0; k < count; ++k) {
    er[k] = epsrel ? epsrel[k] : epsrel0;
    ea[k] = epsabs ? epsabs[k] : epsabs0;
    if (!(er[k] >= 0) || !(ea[k] >= 0)) {
      set_error("epsrel/epsabs must be >= 0");
      return CUB_ERR_INVALID;
    }
  }
  if (count > ctx->params_cap) {
    if (ctx->d_params) cudaFree(ctx->d_params);
    ctx->d_params = nullptr;
    ctx->params_cap = 0;
    if ((e = cudaMalloc(&ctx->d_params, sizeof(GenzParams) * count)) != cudaSuccess)
      return cuda_fail(e, "cudaMalloc(params)");
    ctx->params_cap = count;
  }
  if (count > ctx->fams_cap) {
    if (ctx->d_fams) cudaFree(ctx->d_fams);
    ctx->d_fams = nullptr;
    ctx->fams_cap = 0;
    if ((e = cudaMalloc(&ctx->d_fams, sizeof(int) * count)) != cudaSuccess)
      return cuda_fail(e, "cudaMalloc(families)");
    ctx->fams_cap = count;
  }
  Options o = to_options(opt);
  if (o.max_slots <= 0) o.max_slots = ctx->ws->auto_slots(ndim, o.policy);
  const GenzParams* h = reinterpret_cast<const GenzParams*>(params);
  std::vector<GenzParams> hp;
  std::vector<int> hf;
  std::vector<double> ger, gea;
  std::vector<Result> res;
  const int rc = grouped_batch(count, o, [&](const std::vector<int>& idx, Result* gout) {
    const int gn = (int)idx.size();
    hp.resize(gn);
    hf.resize(gn);
    ger.resize(gn);
    gea.resize(gn);
    for (int j = 0; j < gn; ++j) {
      hp[j] = h[idx[j]];
      hf[j] = families[idx[j]];
      ger[j] = er[idx[j]];
      gea[j] = ea[idx[j]];
    }
    if (cudaMemcpyAsync(ctx->d_params, hp.data(), sizeof(GenzParams) * gn,
                        cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaMemcpyAsync(ctx->d_fams, hf.data(), sizeof(int) * gn, cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess)
      return (int)kErrCuda;
    ctx->ws->stats().h2d_bytes += (long long)((sizeof(GenzParams) + sizeof(int)) * gn);
    switch (ndim) {
      case 2: return run_mixed_dim_2(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 3: return run_mixed_dim_3(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 4: return run_mixed_dim_4(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 5: return run_mixed_dim_5(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 6: return run_mixed_dim_6(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 7: return run_mixed_dim_7(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
      case 8: return run_mixed_dim_8(ctx, gn, ctx->d_params, ctx->d_fams, ger.data(), gea.data(), o, gout);
    }
    return (int)kErrInvalid;
  }, res, ctx->ws);
  if (rc != kOk && rc != kErrCapacity) return engine_status(ctx, rc);
  for (int k = 0; k < count; ++k) result_to_c(res[k], &out[k]);
  return engine_status(ctx, rc);
}
