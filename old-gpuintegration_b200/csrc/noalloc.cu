// noalloc.cu -- cub_split_noalloc: the scan + compact + bisect step with its
// scratch in a fixed device array, for callers that cannot allocate.
//
// cub_split needs a small scratch buffer (two ints per 32 regions) that the
// caller provides.  Some callers cannot obtain one at call time: code whose
// device memory is owned entirely by another allocator or framework, and
// hot loops where a cudaMalloc/cudaFree (which may synchronise the device)
// is not acceptable.  This variant uses a file-scope __device__ array
// instead, so the call itself allocates nothing.
//
// Costs and rules of that choice:
//   * the array is a fixed 1 MiB (two ints per 32 regions for up to
//     kNoAllocMaxRegions = 2^22 regions); every GPU that loads this library
//     holds it until the process exits;
//   * larger lists are rejected with CUB_ERR_INVALID and a message;
//   * all calls share the one array per device, so two calls whose work
//     overlaps on the GPU (different streams, or different host threads)
//     race on it; serialise them;
//   * the array keeps whatever the last call left in it; every entry a call
//     reads is written earlier in the same call, so nothing needs clearing;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture.
#include <mutex>
#include <string>

#include "capi_internal.h"

namespace {

constexpr long long kNoAllocMaxRegions = 1ll << 22;
constexpr long long kNoAllocChunks = kNoAllocMaxRegions / 32 + 1;
constexpr int kMaxDevices = 64;

// chunk counts followed by their exclusive prefix
static __device__ __align__(256) int g_split_scratch[2 * kNoAllocChunks];

std::mutex g_mu;
int* g_scratch_addr[kMaxDevices] = {};

// Device address of g_split_scratch on the current device (set up once).
int* scratch_on_current_device(int* dev_out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cubature::capi::set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return nullptr;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    cubature::capi::set_error("device index beyond the no-alloc table");
    return nullptr;
  }
  *dev_out = dev;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_split_scratch);
    if (e != cudaSuccess || !p) {
      cubature::capi::set_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return nullptr;
    }
    g_scratch_addr[dev] = static_cast<int*>(p);
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int cub_split_noalloc(int ndim, long long n, const double* d_lo, const double* d_len,
                                 long long ld, const int* d_active, const int* d_axis,
                                 double* d_out_lo, double* d_out_len, long long out_ld,
                                 int layout, long long* d_count, void* stream) {
  using namespace cubature::capi;
  if (ndim < CUB_MIN_NDIM || ndim > CUB_MAX_NDIM) {
    set_error("ndim " + std::to_string(ndim) + " outside the built range");
    return CUB_ERR_INVALID;
  }
  if (n > kNoAllocMaxRegions) {
    set_error("cub_split_noalloc: " + std::to_string(n) + " regions exceed its fixed limit of " +
              std::to_string(kNoAllocMaxRegions) + "; use cub_split with caller scratch");
    return CUB_ERR_INVALID;
  }
  if (n < 0 || ld < n || !d_count || (layout != 0 && layout != 1)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  const cudaStream_t s = as_stream(stream);
  if (n == 0) {
    const cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(long long), s);
    if (e != cudaSuccess) {
      set_error(std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
      return CUB_ERR_CUDA;
    }
    return 0;
  }
  int dev = 0;
  int* base = scratch_on_current_device(&dev);
  if (!base) return CUB_ERR_CUDA;
  int* cnt = base;
  int* excl = base + kNoAllocChunks;
  int rc = CUB_ERR_INVALID;
  switch (ndim) {
#define CUB_NOALLOC_CASE(N)                                                                    \
  case N:                                                                                     \
    rc = cubature::capi::split_dim_##N(n, d_lo, d_len, ld, d_active, d_axis, d_out_lo,        \
                                       d_out_len, out_ld, layout, d_count, cnt, excl, s);     \
    break;
    CUB_NOALLOC_CASE(2) CUB_NOALLOC_CASE(3) CUB_NOALLOC_CASE(4) CUB_NOALLOC_CASE(5)
    CUB_NOALLOC_CASE(6) CUB_NOALLOC_CASE(7) CUB_NOALLOC_CASE(8)
#undef CUB_NOALLOC_CASE
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("split kernel launch: ") + cudaGetErrorString(e));
    return CUB_ERR_CUDA;
  }
  return rc;
}
