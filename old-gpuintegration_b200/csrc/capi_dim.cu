// capi_dim.cu -- instantiations of the engine for one dimension (compiled
// once per dimension with -DCUB_DIM=N) and the built-in integrand families.
#include "capi_internal.h"
#include "cubature/step_kernels.cuh"

#ifndef CUB_DIM
#error "compile with -DCUB_DIM=<ndim>"
#endif

#define CUB_CAT2(a, b) a##b
#define CUB_CAT(a, b) CUB_CAT2(a, b)

namespace cubature {
namespace capi {
namespace {

constexpr int N = CUB_DIM;

template <template <int> class Fam>
int run_family(cub_ctx* ctx, int count, const GenzParams* h_params, const GenzParams* d_params,
               const double* epsrel, const double* epsabs, const Options& opt, Result* out,
               const double* h_box) {
  if (count == 1) {
    detail::SingleSource<Fam<N>> src{Fam<N>::load(h_params[0])};
    return run_batch<N>(*ctx->ws, src, 1, epsrel, epsabs, opt, out, ctx->stream, h_box);
  }
  detail::ParamSource<Fam<N>> src{d_params};
  return run_batch<N>(*ctx->ws, src, count, epsrel, epsabs, opt, out, ctx->stream, h_box);
}

template <template <int> class Fam>
int rule_family(const GenzParams& p, long long n, const double* lo, const double* len,
                long long ld, double epsrel, double epsabs, double* avg, double* err, int* axis,
                int* active, cudaStream_t s) {
  const RuleTables T = make_rule9_tables(N);
  const Fam<N> f = Fam<N>::load(p);
  int dev = 0;
  cudaGetDevice(&dev);
  const int sms = sm_count(dev);
  if (n >= (long long)sms * 512) {
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)sms * 32);
    k_step_rule<N, 1><<<(unsigned)blocks, 256, 0, s>>>(f, T, n, lo, len, ld, epsrel, epsabs, avg,
                                                       err, axis, active);
  } else {
    const long long blocks = std::max<long long>(1, (n * 32 + 255) / 256);
    k_step_rule<N, 32><<<(unsigned)std::min<long long>(blocks, (long long)sms * 32), 256, 0, s>>>(
        f, T, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active);
  }
  return 0;
}

// A batch of one family for replay: its integrands read their parameters
// from device memory, so one recording serves every call.
template <template <int> class Fam>
int replay_prepare_family(Workspace& ws, int count, const Options& opt, cudaStream_t s,
                          Replay* r) {
  return replay_prepare<N, detail::ParamSource<Fam<N>>>(ws, count, opt, s, r);
}

template <template <int> class Fam>
int replay_enqueue_family(Workspace& ws, const GenzParams* d_params, const Replay& r,
                          cudaStream_t s) {
  return replay_enqueue<N>(ws, detail::ParamSource<Fam<N>>{d_params}, r, s);
}

}  // namespace

int CUB_CAT(replay_prepare_dim_, CUB_DIM)(int family, Workspace& ws, int count,
                                          const Options& opt, cudaStream_t s, Replay* r) {
  switch (family) {
    case kGaussian: return replay_prepare_family<Gaussian>(ws, count, opt, s, r);
    case kOscillatory: return replay_prepare_family<Oscillatory>(ws, count, opt, s, r);
    case kCornerPeak: return replay_prepare_family<CornerPeak>(ws, count, opt, s, r);
    case kProductPeak: return replay_prepare_family<ProductPeak>(ws, count, opt, s, r);
    case kContinuous: return replay_prepare_family<Continuous>(ws, count, opt, s, r);
    case kDiscontinuous: return replay_prepare_family<Discontinuous>(ws, count, opt, s, r);
    case kCosSum: return replay_prepare_family<CosSum>(ws, count, opt, s, r);
  }
  return CUB_ERR_INVALID;
}

int CUB_CAT(replay_enqueue_dim_, CUB_DIM)(int family, Workspace& ws, const GenzParams* d_params,
                                          const Replay& r, cudaStream_t s) {
  switch (family) {
    case kGaussian: return replay_enqueue_family<Gaussian>(ws, d_params, r, s);
    case kOscillatory: return replay_enqueue_family<Oscillatory>(ws, d_params, r, s);
    case kCornerPeak: return replay_enqueue_family<CornerPeak>(ws, d_params, r, s);
    case kProductPeak: return replay_enqueue_family<ProductPeak>(ws, d_params, r, s);
    case kContinuous: return replay_enqueue_family<Continuous>(ws, d_params, r, s);
    case kDiscontinuous: return replay_enqueue_family<Discontinuous>(ws, d_params, r, s);
    case kCosSum: return replay_enqueue_family<CosSum>(ws, d_params, r, s);
  }
  return CUB_ERR_INVALID;
}

int CUB_CAT(run_mixed_dim_, CUB_DIM)(cub_ctx* ctx, int count, const GenzParams* d_params,
                                     const int* d_fams, const double* epsrel,
                                     const double* epsabs, const Options& opt, Result* out) {
  detail::MixedSource<N> src{d_params, d_fams};
  return run_batch<N>(*ctx->ws, src, count, epsrel, epsabs, opt, out, ctx->stream);
}

int CUB_CAT(run_dim_, CUB_DIM)(cub_ctx* ctx, int family, int count, const GenzParams* h_params,
                               const GenzParams* d_params, const double* epsrel,
                               const double* epsabs, const Options& opt, Result* out,
                               const double* h_box) {
  switch (family) {
    case kGaussian: return run_family<Gaussian>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kOscillatory: return run_family<Oscillatory>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kCornerPeak: return run_family<CornerPeak>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kProductPeak: return run_family<ProductPeak>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kContinuous: return run_family<Continuous>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kDiscontinuous: return run_family<Discontinuous>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
    case kCosSum: return run_family<CosSum>(ctx, count, h_params, d_params, epsrel, epsabs, opt, out, h_box);
  }
  return CUB_ERR_INVALID;
}

int CUB_CAT(rule_eval_dim_, CUB_DIM)(int family, const GenzParams& p, long long n,
                                     const double* lo, const double* len, long long ld,
                                     double epsrel, double epsabs, double* avg, double* err,
                                     int* axis, int* active, cudaStream_t s) {
  switch (family) {
    case kGaussian: return rule_family<Gaussian>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kOscillatory: return rule_family<Oscillatory>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kCornerPeak: return rule_family<CornerPeak>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kProductPeak: return rule_family<ProductPeak>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kContinuous: return rule_family<Continuous>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kDiscontinuous: return rule_family<Discontinuous>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
    case kCosSum: return rule_family<CosSum>(p, n, lo, len, ld, epsrel, epsabs, avg, err, axis, active, s);
  }
  return CUB_ERR_INVALID;
}

int CUB_CAT(split_dim_, CUB_DIM)(long long n, const double* lo, const double* len, long long ld,
                                 const int* active, const int* axis, double* olo, double* olen,
                                 long long old, int layout, long long* count, int* cnt,
                                 int* excl, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int sms = sm_count(dev);
  const long long nchunk = (n + 31) / 32;
  const unsigned blocks =
      (unsigned)std::max<long long>(1, std::min<long long>((nchunk + 7) / 8, (long long)sms * 16));
  k_step_count<<<blocks, 256, 0, s>>>(n, active, cnt);
  k_step_scan<<<1, 1024, 0, s>>>(nchunk, cnt, excl, count);
  k_step_write<N><<<blocks, 256, 0, s>>>(n, lo, len, ld, active, axis, excl, count, olo, olen,
                                         old, layout);
  return 0;
}

}  // namespace capi
}  // namespace cubature
