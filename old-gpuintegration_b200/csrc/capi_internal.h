// capi_internal.h -- shared declarations of the C ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "cubature.h"
#include "cubature/engine.cuh"

struct cub_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cubature::Workspace* ws = nullptr;
  cubature::GenzParams* d_params = nullptr;
  int params_cap = 0;
  double* d_aux = nullptr;  // per-integral scalars of the table integrands
  int aux_cap = 0;
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
  int rule_eval_dim_##N(int family, const GenzParams& p, long long n, const double* lo,        \
                        const double* len, long long ld, double epsrel, double epsabs,         \
                        double* avg, double* err, int* axis, int* active, cudaStream_t s);     \
  int split_dim_##N(long long n, const double* lo, const double* len, long long ld,            \
                    const int* active, const int* axis, double* olo, double* olen,             \
                    long long old, int layout, long long* count, int* cnt, int* excl,          \
                    cudaStream_t s);
CUB_DECLARE_DIM(2)
CUB_DECLARE_DIM(3)
CUB_DECLARE_DIM(4)
CUB_DECLARE_DIM(5)
CUB_DECLARE_DIM(6)
CUB_DECLARE_DIM(7)
CUB_DECLARE_DIM(8)
#undef CUB_DECLARE_DIM

}  // namespace capi
}  // namespace cubature
