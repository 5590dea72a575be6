// tables.cuh -- FP64 device tables and the integrands built on them.
//
//   * Interp2D: bilinear interpolation on a rectilinear grid, the reference's
//     quad::Interp2D (GPUQuadInterp2D.cu:50-106) in FP64 with a binary
//     search for the cell (the reference reads FP32 textures and searches
//     linearly).  Cell convention as there: the cell left of the first knot
//     >= t, clamped to the table (points outside extrapolate linearly from
//     the end cells; the reference reads past the table there).
//   * Spline1D: natural cubic spline (Numerical Recipes form) with the same
//     cell search.
//   * LcLt: the reference's 3-D physics integrand over (lt, zt, lc), five
//     tables on one grid (lc_lt_t.h:18-52), in FP64.
//   * Table7: the 7-D integrand spline(x0) * bilinear(x1, x2) *
//     exp(-(4 x3 - mu(x))^2 / 2 sigma^2), mu = offset + 2 x4 + 0.1 (x5 + x6).
//
// Tables live in device memory owned by the caller; the functors hold raw
// pointers and are copied by value to the device, as the reference's are.
#pragma once

#include <cuda_runtime.h>

namespace cubature {

// Cell [xs[i], xs[i+1]] for t: i = (index of the first knot >= t among
// xs[1..n-1]) - 1, clamped to [0, n-2].
__host__ __device__ __forceinline__ int table_cell(const double* xs, int n, double t) {
  int lo = 1, hi = n - 1;  // first index in [1, n-1] with xs[i] >= t, or n-1
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (xs[mid] >= t)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo - 1;
}

// Lookup hint of a knot array: x0 and 1 / spacing for knots that are
// uniform to rounding (inv_dx = 0: no hint).  Set on the host.
struct KnotHint {
  double x0 = 0;
  double inv_dx = 0;
};

// table_cell from a guess: cell floor((t - x0) / dx), corrected by walking
// down while xs[g - 1] >= t and up while xs[g] < t.  The predicate
// xs[i] >= t is monotone in i for ascending knots, so the walk ends on the
// binary search's answer whatever the guess; a hint only saves reads (two
// independent ones on a uniform table instead of log2(n) dependent ones).
// NaN takes the binary search.
__host__ __device__ __forceinline__ int table_cell(const double* xs, int n, double t,
                                                   const KnotHint& h) {
  const double u = (t - h.x0) * h.inv_dx;
  if (h.inv_dx > 0 && u == u) {
    int g = u < 0 ? 1 : (u >= (double)(n - 2) ? n - 1 : (int)u + 1);
    while (g > 1 && xs[g - 1] >= t) --g;
    while (g < n - 1 && xs[g] < t) ++g;
    return g - 1;
  }
  return table_cell(xs, n, t);
}

struct Interp2D {
  const double* xs;  // row coordinates, nx, ascending
  const double* ys;  // column coordinates, ny, ascending
  const double* zs;  // values, row-major: zs[i * ny + j] at (xs[i], ys[j])
  int nx, ny;
  KnotHint hx, hy;

  // Value at (x, y) in a known cell (i, j).
  __host__ __device__ __forceinline__ double at_cell(int i, int j, double x, double y) const {
    const double x1 = xs[i], x2 = xs[i + 1], y1 = ys[j], y2 = ys[j + 1];
    const double q11 = zs[i * ny + j], q21 = zs[(i + 1) * ny + j];
    const double q12 = zs[i * ny + j + 1], q22 = zs[(i + 1) * ny + j + 1];
    const double d = (x2 - x1) * (y2 - y1);
    const double t1 = (y2 - y) / d, t2 = (y - y1) / d;
    return (q11 * (x2 - x) + q21 * (x - x1)) * t1 + (q12 * (x2 - x) + q22 * (x - x1)) * t2;
  }

  __host__ __device__ __forceinline__ double operator()(double x, double y) const {
    return at_cell(table_cell(xs, nx, x, hx), table_cell(ys, ny, y, hy), x, y);
  }
};

struct Spline1D {
  const double* xs;  // knots, ascending
  const double* ys;  // values
  const double* y2;  // second derivatives (natural spline: y2[0] = y2[n-1] = 0)
  int n;
  KnotHint h;

  __host__ __device__ __forceinline__ double operator()(double t) const {
    const int i = table_cell(xs, n, t, h);
    const double h = xs[i + 1] - xs[i];
    const double a = (xs[i + 1] - t) / h, b = (t - xs[i]) / h;
    return a * ys[i] + b * ys[i + 1] +
           ((a * a * a - a) * y2[i] + (b * b * b - b) * y2[i + 1]) * (h * h) / 6.0;
  }
};

// The reference's LC_LT integrand (lc_lt_t.h:18-52) in FP64: x = (lt, zt,
// lc); tau, mu, sigma, fmsk, fprj from five tables over (lt, zt) that share
// one grid (one cell search serves all five).
template <int N>
struct LcLt {
  static_assert(N == 3, "LC_LT is a 3-D integrand");
  const double* xs;  // lt knots
  const double* ys;  // zt knots
  const double* z[5];  // tau, mu, sigma, fmsk, fprj, each row-major nx x ny
  int nx, ny;
  KnotHint hx, hy;

  __device__ __forceinline__ double operator()(const double* x) const {
    const double lt = x[0], zt = x[1], lc = x[2];
    const int i = table_cell(xs, nx, lt, hx), j = table_cell(ys, ny, zt, hy);
    double v[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) v[q] = Interp2D{xs, ys, z[q], nx, ny, hx, hy}.at_cell(i, j, lt, zt);
    const double tau = v[0], mu = v[1], sigma = v[2], fmsk = v[3], fprj = v[4];
    const double exptau = exp(tau * (2.0 * mu + tau * sigma * sigma - 2.0 * lc) / 2.0);
    const double r2s = sqrt(2.0) * sigma;
    const double mts = mu + tau * sigma * sigma;
    const double zg = (lc - mu) / sigma;
    const double gauss = exp(-zg * zg / 2.0) * 0.3989422804014327 / sigma;  // 1/sqrt(2 pi)
    return (1.0 - fmsk) * (1.0 - fprj) * gauss +
           0.5 * ((1.0 - fmsk) * fprj * tau + fmsk * fprj / lt) * exptau * erfc((mts - lc) / r2s) +
           0.5 * fmsk / lt * (erfc((lc - mu) / r2s) - erfc((lc + lt - mu) / r2s)) -
           0.5 * fmsk * fprj / lt * (exp(-tau * lt) * exptau * erfc((mts - lc - lt) / r2s));
  }
};

// spline(x0) * bilinear(x1, x2) * exp(-(4 x3 - mu)^2 / (2 sigma^2)),
// mu = offset + 2 x4 + 0.1 (x5 + x6).
template <int N>
struct Table7 {
  static_assert(N == 7, "the table integrand is 7-D");
  Spline1D spline;
  Interp2D grid;
  double inv2s2;  // 1 / (2 sigma^2)
  double offset;

  __device__ __forceinline__ double operator()(const double* x) const {
    const double mu = offset + 2.0 * x[4] + 0.1 * (x[5] + x[6]);
    const double r = 4.0 * x[3] - mu;
    return spline(x[0]) * grid(x[1], x[2]) * exp(-r * r * inv2s2);
  }
};

namespace detail {

// Source of Table7 integrands with one offset per integral (device array).
struct Table7Source {
  Table7<7> base;
  const double* offsets;
  __device__ __forceinline__ Table7<7> get(int k) const {
    Table7<7> t = base;
    t.offset = offsets[k];
    return t;
  }
};

}  // namespace detail
}  // namespace cubature
