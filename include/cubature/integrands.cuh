// integrands.cuh -- built-in integrand families as device functors.
//
// Each functor is templated on the dimension N and evaluates f(x) for a
// point x held in registers (double x[N]).  The families are Genz's test
// families (the ones the reference's drivers draw from, function.cu:70-214,
// and the north-star configurations) plus the reference driver's own
// cosine-sum integrand (cudaCuhre.cu:9-23).
//
// Parameters travel as GenzParams (one per integral); load() turns them
// into the functor's register form, folding constant work (a^2, a^-2).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

#include "rule9.hpp"

namespace cubature {

// Family identifiers (shared with the C ABI, include/cubature.h).
enum Family : int {
  kGaussian = 1,
  kOscillatory = 2,
  kCornerPeak = 3,
  kProductPeak = 4,
  kContinuous = 5,
  kDiscontinuous = 6,
  kCosSum = 7,
};

struct GenzParams {
  double a[kMaxDim];
  double u[kMaxDim];
};

// exp(-sum a_i^2 (x_i - u_i)^2)
template <int N>
struct Gaussian {
  double a[N], u[N];
  __host__ __device__ static Gaussian load(const GenzParams& p) {
    Gaussian g;
#pragma unroll
    for (int i = 0; i < N; ++i) { g.a[i] = p.a[i]; g.u[i] = p.u[i]; }
    return g;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double t = a[i] * (x[i] - u[i]);
      s += t * t;
    }
    return exp(-s);
  }
};

// cos(2 pi u_0 + sum a_i x_i)
template <int N>
struct Oscillatory {
  double a[N], phase;
  __host__ __device__ static Oscillatory load(const GenzParams& p) {
    Oscillatory o;
#pragma unroll
    for (int i = 0; i < N; ++i) o.a[i] = p.a[i];
    o.phase = 2 * CUDART_PI * p.u[0];
    return o;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = phase;
#pragma unroll
    for (int i = 0; i < N; ++i) s += a[i] * x[i];
    return cos(s);
  }
};

// (1 + sum a_i x_i)^-(N+1)
template <int N>
struct CornerPeak {
  double a[N];
  __host__ __device__ static CornerPeak load(const GenzParams& p) {
    CornerPeak c;
#pragma unroll
    for (int i = 0; i < N; ++i) c.a[i] = p.a[i];
    return c;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = 1;
#pragma unroll
    for (int i = 0; i < N; ++i) s += a[i] * x[i];
    double p = 1;
#pragma unroll
    for (int k = 0; k <= N; ++k) p *= s;
    return 1 / p;
  }
};

// prod 1/(a_i^-2 + (x_i - u_i)^2)
template <int N>
struct ProductPeak {
  double ia2[N], u[N];
  __host__ __device__ static ProductPeak load(const GenzParams& p) {
    ProductPeak q;
#pragma unroll
    for (int i = 0; i < N; ++i) { q.ia2[i] = 1 / (p.a[i] * p.a[i]); q.u[i] = p.u[i]; }
    return q;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double den = 1;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double t = x[i] - u[i];
      den *= ia2[i] + t * t;
    }
    return 1 / den;
  }
};

// exp(-sum a_i |x_i - u_i|)
template <int N>
struct Continuous {
  double a[N], u[N];
  __host__ __device__ static Continuous load(const GenzParams& p) {
    Continuous c;
#pragma unroll
    for (int i = 0; i < N; ++i) { c.a[i] = p.a[i]; c.u[i] = p.u[i]; }
    return c;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) s += a[i] * fabs(x[i] - u[i]);
    return exp(-s);
  }
};

// 0 if x_0 > u_0 or x_1 > u_1, else exp(sum a_i x_i)
template <int N>
struct Discontinuous {
  double a[N], u0, u1;
  __host__ __device__ static Discontinuous load(const GenzParams& p) {
    Discontinuous c;
#pragma unroll
    for (int i = 0; i < N; ++i) c.a[i] = p.a[i];
    c.u0 = p.u[0];
    c.u1 = N > 1 ? p.u[1] : 2.0;
    return c;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) s += a[i] * x[i];
    const bool out = x[0] > u0 || (N > 1 && x[N > 1 ? 1 : 0] > u1);
    return out ? 0.0 : exp(s);
  }
};

// -sum cos(10 x_i) / 0.054402111088937 / 2   (cudaCuhre.cu:11-22)
template <int N>
struct CosSum {
  __host__ __device__ static CosSum load(const GenzParams&) { return CosSum(); }
  __device__ __forceinline__ double operator()(const double* x) const {
    double s = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) s = s - cos(10.0 * x[i]) / 0.054402111088937;
    return s / 2.0;
  }
};

// One integrand of any built-in family, chosen per integral: the family's
// functor is built once (per region, by the source) and called unchanged,
// so a mixed batch computes exactly what single-family batches compute.
template <int N>
struct MixedGenz {
  int family;
  union {
    Gaussian<N> g;
    Oscillatory<N> o;
    CornerPeak<N> c;
    ProductPeak<N> p;
    Continuous<N> ct;
    Discontinuous<N> d;
  } f;
  __host__ __device__ static MixedGenz make(const GenzParams& q, int family) {
    MixedGenz m;
    m.family = family;
    switch (family) {
      case kGaussian: m.f.g = Gaussian<N>::load(q); break;
      case kOscillatory: m.f.o = Oscillatory<N>::load(q); break;
      case kCornerPeak: m.f.c = CornerPeak<N>::load(q); break;
      case kProductPeak: m.f.p = ProductPeak<N>::load(q); break;
      case kContinuous: m.f.ct = Continuous<N>::load(q); break;
      case kDiscontinuous: m.f.d = Discontinuous<N>::load(q); break;
      default: break;
    }
    return m;
  }
  __device__ __forceinline__ double operator()(const double* x) const {
    switch (family) {
      case kGaussian: return f.g(x);
      case kOscillatory: return f.o(x);
      case kCornerPeak: return f.c(x);
      case kProductPeak: return f.p(x);
      case kContinuous: return f.ct(x);
      case kDiscontinuous: return f.d(x);
      default: return CosSum<N>()(x);
    }
  }
};

}  // namespace cubature
