// capi_tables.cu -- C ABI of the integrands on device tables
// (include/cubature/tables.cuh): the reference's LC_LT over five Interp2D
// tables (lc_lt_t.h:18-52, GPUQuadInterp2D.cu:50-106) and the 7-D spline x
// bilinear x Gaussian-kernel integrand.  The engine is instantiated here
// for n = 3 and n = 7 only.
#include <cmath>
#include <vector>

#include "capi_internal.h"
#include "cubature/tables.cuh"

using namespace cubature;
using namespace cubature::capi;

namespace {

bool valid_grid(const cub_interp2d& g) {
  return g.xs && g.ys && g.zs && g.nx >= 2 && g.ny >= 2;
}

bool valid_spline(const cub_spline1d& s) { return s.xs && s.ys && s.y2 && s.n >= 2; }

// Lookup hint of caller knots in device memory: uniform to within 1e-9 of
// the spacing gives x0 and 1 / spacing, anything else (or a failed copy)
// no hint.  The hint changes no result, only the number of knot reads.
KnotHint knot_hint(const double* d_xs, int n) {
  KnotHint h;
  if (n < 3) return h;
  std::vector<double> x(n);
  if (cudaMemcpy(x.data(), d_xs, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return h;
  }
  const double dx = (x[n - 1] - x[0]) / (n - 1);
  if (!(dx > 0) || !std::isfinite(dx)) return h;
  for (int i = 0; i < n; ++i)
    if (!(std::fabs(x[i] - (x[0] + i * dx)) <= 1e-9 * dx)) return h;
  h.x0 = x[0];
  h.inv_dx = 1.0 / dx;
  return h;
}

bool valid_box(const double* lo, const double* hi, int n) {
  for (int i = 0; i < n; ++i)
    if (!(std::isfinite(lo[i]) && std::isfinite(hi[i]) && hi[i] > lo[i])) return false;
  return true;
}

}  // namespace

int cub_spline_second_derivatives(int n, const double* xs, const double* ys, double* y2) {
  if (n < 2 || !xs || !ys || !y2) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  for (int i = 1; i < n; ++i)
    if (!(xs[i] > xs[i - 1])) {
      set_error("spline knots must be strictly increasing");
      return CUB_ERR_INVALID;
    }
  // natural end conditions; forward elimination and back substitution of
  // h_{i-1} y2_{i-1} + 2 (h_{i-1} + h_i) y2_i + h_i y2_{i+1} = 6 (d_i - d_{i-1})
  std::vector<double> c(n, 0.0), r(n, 0.0);
  y2[0] = 0;
  y2[n - 1] = 0;
  for (int i = 1; i < n - 1; ++i) {
    const double hl = xs[i] - xs[i - 1], hr = xs[i + 1] - xs[i];
    const double rhs = 6.0 * ((ys[i + 1] - ys[i]) / hr - (ys[i] - ys[i - 1]) / hl);
    const double den = 2.0 * (hl + hr) - hl * c[i - 1];
    c[i] = hr / den;
    r[i] = (rhs - hl * r[i - 1]) / den;
  }
  for (int i = n - 2; i >= 1; --i) y2[i] = r[i] - c[i] * y2[i + 1];
  return 0;
}

int cub_integrate_lclt(cub_ctx* ctx, const cub_lclt_tables* tables, const double* lo,
                       const double* hi, double epsrel, double epsabs, const cub_options* opt,
                       cub_result* out) {
  if (!ctx || !tables || !lo || !hi || !out || !(epsrel >= 0) || !(epsabs >= 0)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  for (int q = 0; q < 5; ++q)
    if (!tables->t[q].zs || !valid_grid(tables->t[0])) {
      set_error("LC_LT needs five tables on one grid of at least 2 x 2 knots");
      return CUB_ERR_INVALID;
    }
  if (!valid_box(lo, hi, 3)) {
    set_error("integration box needs finite bounds with hi > lo");
    return CUB_ERR_INVALID;
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  LcLt<3> f;
  f.xs = tables->t[0].xs;
  f.ys = tables->t[0].ys;
  f.nx = tables->t[0].nx;
  f.ny = tables->t[0].ny;
  for (int q = 0; q < 5; ++q) f.z[q] = tables->t[q].zs;
  f.hx = knot_hint(f.xs, f.nx);
  f.hy = knot_hint(f.ys, f.ny);
  double box[6] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
  Options o = to_options(opt);
  if (o.max_slots <= 0) o.max_slots = ctx->ws->auto_slots(3, o.policy);
  Result r;
  detail::SingleSource<LcLt<3>> src{f};
  const int rc = run_batch<3>(*ctx->ws, src, 1, &epsrel, &epsabs, o, &r, ctx->stream, box);
  if (rc != kOk && rc != kErrCapacity) return engine_status(ctx, rc);
  result_to_c(r, out);
  return engine_status(ctx, rc);
}

int cub_integrate_table7_batch(cub_ctx* ctx, const cub_table7* tables, int count,
                               const double* offsets, const double* epsrel, const double* epsabs,
                               double epsrel0, double epsabs0, const cub_options* opt,
                               cub_result* out) {
  if (!ctx || !tables || !offsets || !out || count <= 0 || !valid_spline(tables->spline) ||
      !valid_grid(tables->grid) || !(tables->sigma > 0)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  std::vector<double> er(count), ea(count);
  for (int k = 0; k < count; ++k) {
    er[k] = epsrel ? epsrel[k] : epsrel0;
    ea[k] = epsabs ? epsabs[k] : epsabs0;
    if (!(er[k] >= 0) || !(ea[k] >= 0) || !std::isfinite(offsets[k])) {
      set_error("epsrel/epsabs must be >= 0 and offsets finite");
      return CUB_ERR_INVALID;
    }
  }
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  Options o = to_options(opt);
  if (o.max_slots <= 0) o.max_slots = ctx->ws->auto_slots(7, o.policy);
  if (count > ctx->aux_cap) {
    if (ctx->d_aux) cudaFree(ctx->d_aux);
    ctx->d_aux = nullptr;
    ctx->aux_cap = 0;
    if ((e = cudaMalloc(&ctx->d_aux, sizeof(double) * count)) != cudaSuccess)
      return cuda_error(e, "cudaMalloc(offsets)");
    ctx->aux_cap = count;
  }
  detail::Table7Source src;
  src.base.spline = Spline1D{tables->spline.xs, tables->spline.ys, tables->spline.y2,
                             tables->spline.n, knot_hint(tables->spline.xs, tables->spline.n)};
  src.base.grid = Interp2D{tables->grid.xs, tables->grid.ys, tables->grid.zs, tables->grid.nx,
                           tables->grid.ny, knot_hint(tables->grid.xs, tables->grid.nx),
                           knot_hint(tables->grid.ys, tables->grid.ny)};
  src.base.inv2s2 = 1.0 / (2.0 * tables->sigma * tables->sigma);
  src.base.offset = 0;
  src.offsets = ctx->d_aux;
  std::vector<double> goff, ger, gea;
  std::vector<Result> res;
  const int rc = grouped_batch(count, o, [&](const std::vector<int>& idx, Result* gout) {
    const int gn = (int)idx.size();
    goff.resize(gn);
    ger.resize(gn);
    gea.resize(gn);
    for (int j = 0; j < gn; ++j) {
      goff[j] = offsets[idx[j]];
      ger[j] = er[idx[j]];
      gea[j] = ea[idx[j]];
    }
    if (cudaMemcpyAsync(ctx->d_aux, goff.data(), sizeof(double) * gn, cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess)
      return (int)kErrCuda;
    return run_batch<7>(*ctx->ws, src, gn, ger.data(), gea.data(), o, gout, ctx->stream);
  }, res, ctx->ws);
  if (rc != kOk && rc != kErrCapacity) return engine_status(ctx, rc);
  for (int k = 0; k < count; ++k) result_to_c(res[k], &out[k]);
  return engine_status(ctx, rc);
}
