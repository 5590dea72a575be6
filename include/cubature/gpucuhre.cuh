// gpucuhre.cuh -- C++ front end with the reference's API, for integrands
// written as device functors: the drop-in for quad::GPUcuhre<T>
// (quad/GPUquad/GPUquad.h:46-63,611-727) and its Volume
// (quad/GPUquad/GPUQuadVolume.cu:4-25).
//
// Compile the including file with nvcc for sm_100a.  Each dimension in
// [CUB_FRONT_MIN_DIM, CUB_FRONT_MAX_DIM] (default 2..8) instantiates the
// engine once per functor type; narrow the range to shorten compilation.
//
// Differences from the reference, all deliberate: the constructor neither
// parses argv nor resets devices; the domain box is FP64; errors come back
// as negative return values instead of exit(); the engine runs on its own
// stream with pooled device memory reused across calls.
#pragma once

#include <cuda_runtime.h>

#include "engine.cuh"

#ifndef CUB_FRONT_MIN_DIM
#define CUB_FRONT_MIN_DIM 2
#endif
#ifndef CUB_FRONT_MAX_DIM
#define CUB_FRONT_MAX_DIM 8
#endif

namespace cubature {

// Integration box [lows, highs] (the reference's Volume<T>, in FP64 here).
template <typename T = double>
struct Volume {
  T lows[kMaxDim];
  T highs[kMaxDim];
  Volume() {
    for (int i = 0; i < kMaxDim; ++i) {
      lows[i] = 0;
      highs[i] = 1;
    }
  }
  Volume(const T* lo, const T* hi, int dim) : Volume() {
    for (int i = 0; i < dim && i < kMaxDim; ++i) {
      lows[i] = lo[i];
      highs[i] = hi[i];
    }
  }
};

namespace detail {

// The reference's functors take (double x[], int dim) and may have a
// non-const call operator; the engine calls f(const double* x) const.
template <class F, int N>
struct RefCall {
  mutable F f;
  __device__ __forceinline__ double operator()(const double* x) const {
    double y[N];
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = x[i];
    return f(y, N);
  }
};

}  // namespace detail

template <typename T = double>
class GPUcuhre {
 public:
  // The reference's constructor signature.  argv is not parsed, no device is
  // reset; only key 0 or 9 (the degree-9 rule) exists.  The device is the
  // current one.
  GPUcuhre(int /*argc*/, char** /*argv*/, int dim, int key = 0, int verbose = 0,
           int /*numDevices*/ = 1)
      : GPUcuhre(dim, current_device()) {
    key_ = key;
    verbose_ = verbose;
  }

  explicit GPUcuhre(int dim, int device = 0, const Options& opt = Options())
      : dim_(dim), device_(device), ws_(device), opt_(opt) {
    cudaSetDevice(device_);
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
  }

  ~GPUcuhre() {
    cudaSetDevice(device_);
    ws_.release();
    if (stream_) cudaStreamDestroy(stream_);
  }

  GPUcuhre(const GPUcuhre&) = delete;
  GPUcuhre& operator=(const GPUcuhre&) = delete;

  Options& options() { return opt_; }
  Stats& stats() { return ws_.stats(); }
  cudaStream_t stream() const { return stream_; }
  const std::string& last_error() const { return err_; }

  // The reference's integrate (GPUquad.h:611-727): integral, error,
  // nregions and neval are ADDED to the caller's variables, as there.
  // Returns the reference's errorFlag (0 = converged, > 0 = failed phase-2
  // boxes) or a negative error code (ErrorCode).
  template <class F>
  int integrate(T epsrel, T epsabs, T& integral, T& error, size_t& nregions, size_t& neval, F* f,
                const Volume<T>* vol = nullptr) {
    if (!f) return kErrInvalid;
    Result r;
    const int rc = run(*f, (double)epsrel, (double)epsabs, vol, &r);
    if (rc < 0 && rc != kErrCapacity) return rc;
    integral += (T)r.value;
    error += (T)r.error;
    nregions += (size_t)r.nregions;
    neval += (size_t)r.neval;
    return rc == kErrCapacity ? rc : r.status;
  }

  // Value form: one integral, results returned; rc (if given) receives the
  // engine's return code (0, or a negative ErrorCode).
  template <class F>
  Result integrate(const F& f, double epsrel, double epsabs, const Volume<T>* vol = nullptr,
                   int* rc = nullptr) {
    Result r;
    std::memset(&r, 0, sizeof(r));
    const int c = run(f, epsrel, epsabs, vol, &r);
    if (rc) *rc = c;
    return r;
  }

 private:
  static int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
  }

  template <class F>
  int run(const F& f, double epsrel, double epsabs, const Volume<T>* vol, Result* r) {
    if (!(epsrel >= 0) || !(epsabs >= 0)) return kErrInvalid;
    if (cudaSetDevice(device_) != cudaSuccess) return kErrCuda;
    switch (dim_) {
#define CUB_FRONT_CASE(n)                                                          \
  case n:                                                                          \
    if constexpr (n >= CUB_FRONT_MIN_DIM && n <= CUB_FRONT_MAX_DIM && n <= kMaxDim) \
      return run_dim<n>(f, epsrel, epsabs, vol, r);                               \
    break;
      CUB_FRONT_CASE(2)
      CUB_FRONT_CASE(3)
      CUB_FRONT_CASE(4)
      CUB_FRONT_CASE(5)
      CUB_FRONT_CASE(6)
      CUB_FRONT_CASE(7)
      CUB_FRONT_CASE(8)
#undef CUB_FRONT_CASE
      default:
        break;
    }
    err_ = "dimension not instantiated in this build";
    return kErrUnsupported;
  }

  template <int N, class F>
  int run_dim(const F& f, double epsrel, double epsabs, const Volume<T>* vol, Result* r) {
    double box[2 * N];
    if (vol) {
      for (int i = 0; i < N; ++i) {
        box[i] = (double)vol->lows[i];
        box[N + i] = (double)vol->highs[i];
        if (!(box[N + i] > box[i])) return kErrInvalid;
      }
    }
    detail::SingleSource<detail::RefCall<F, N>> src{detail::RefCall<F, N>{f}};
    const int rc = run_batch<N>(ws_, src, 1, &epsrel, &epsabs, opt_, r, stream_,
                                vol ? box : nullptr);
    if (rc < 0) err_ = ws_.error();
    return rc;
  }

  int dim_;
  int device_;
  int key_ = 0;
  int verbose_ = 0;
  cudaStream_t stream_ = nullptr;
  Workspace ws_;
  Options opt_;
  std::string err_;
};

}  // namespace cubature

// The reference's spelling, for callers that switch by changing the include.
namespace quad {
template <typename T>
using GPUcuhre = cubature::GPUcuhre<T>;
template <typename T>
using Volume = cubature::Volume<T>;
}  // namespace quad
