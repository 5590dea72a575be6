// mlp.cu -- C ABI of the control-variate network's tensor-core kernels
// (include/cubature/mlp.cuh, umma.cuh).
#include <cuda_bf16.h>

#include "capi_internal.h"
#include "cubature/mlp.cuh"

using namespace cubature;
using namespace cubature::capi;

namespace {

int* error_flag() {
  // one device flag per process and device, set by a kernel whose bounded
  // wait gave up
  static int* flags[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!flags[dev]) {
    if (cudaMalloc(&flags[dev], sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(flags[dev], 0, sizeof(int));
  }
  return flags[dev];
}

template <int N, int EPI>
cudaError_t launch_gemm(dim3 grid, cudaStream_t s, const umma::GemmArgs& g,
                        const mlp::EpiArgs& ep) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!configured[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(mlp::k_gemm<N, EPI>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         mlp::kGemmSmem);
    if (e != cudaSuccess) return e;
    configured[dev & 63] = true;
  }
  mlp::k_gemm<N, EPI><<<grid, 128, mlp::kGemmSmem, s>>>(g, ep);
  return cudaGetLastError();
}

}  // namespace

int cub_mlp_gemm_bf16(int batch, int m, int n, int k, const void* d_a, long long lda,
                      const void* d_b, long long ldb, float* d_d, long long ldd, void* stream) {
  if (batch <= 0 || m <= 0 || m % umma::kTileM || k <= 0 || k % 16 || (n != 16 && n != 128) ||
      !d_a || !d_b || !d_d || lda < k || ldb < k || ldd < n || lda % 8 || ldb % 8) {
    set_error("cub_mlp_gemm_bf16: m % 128, k % 16, n in {16, 128}, lda/ldb % 8 required");
    return CUB_ERR_INVALID;
  }
  int* err = error_flag();
  if (!err) return cuda_error(cudaErrorMemoryAllocation, "error flag");
  cudaStream_t s = as_stream(stream);
  umma::GemmArgs g;
  g.a = static_cast<const __nv_bfloat16*>(d_a);
  g.b = static_cast<const __nv_bfloat16*>(d_b);
  g.lda = lda;
  g.ldb = ldb;
  g.batch_a = lda * m;
  g.batch_b = ldb * n;
  g.m = m;
  g.k = k;
  g.error = err;
  mlp::EpiArgs ep{};
  ep.out = d_d;
  ep.ld_out = ldd;
  ep.batch_out = ldd * m;
  const dim3 grid(m / umma::kTileM, 1, batch);
  cudaError_t e;
  if (n == 16) {
    e = launch_gemm<16, mlp::kEpiStore>(grid, s, g, ep);
  } else {
    e = launch_gemm<128, mlp::kEpiStore>(grid, s, g, ep);
  }
  if (e != cudaSuccess) return cuda_error(e, "k_gemm launch");
  int h_err = 0;
  if ((e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_error(e, "k_gemm");
  if (h_err) {
    cudaMemsetAsync(err, 0, sizeof(int), s);
    set_error("tensor-core GEMM: a bounded wait gave up");
    return CUB_ERR_TIMEOUT;
  }
  return 0;
}
