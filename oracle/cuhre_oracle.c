/*
 * cuhre_oracle.c -- CPU oracle for the adaptive cubature hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  Nothing in the product library links or calls this file.
 *
 * Restates, in plain C, the algorithm of marcpaterno/old-gpuintegration:
 *   rule construction      quad/GPUquad/GPUQuadRule.cu:31-390
 *   region rule            quad/GPUquad/GPUQuadSample.cu:35-220
 *   phase-1 classify       quad/GPUquad/GPUQuadPhases.cu:38-79
 *   phase-1 loop/reduce    quad/GPUquad/GPUKernelquad.cu:509-668
 *   scan/compact/bisect    quad/GPUquad/GPUKernelquad.cu:63-149,357-505
 *   initial grid           quad/GPUquad/GPUKernelquad.cu:24-61,272-354
 *   phase 2 (per region)   quad/GPUquad/GPUQuadPhases.cu:424-536
 *   final status           quad/GPUquad/GPUquad.h:611-727
 *
 * Deliberate, documented differences from the reference's arithmetic (all
 * are re-associations of the same sums; none changes the algorithm):
 *   - points are enumerated in this file's own order (the orbit of each
 *     generator), keeping the reference's convention that points 1..4n are
 *     (+a e_d, -a e_d) for sets 1 and 2, which the fourth difference reads;
 *   - the five rule sums are formed from per-set sums of f
 *     (sum_k w[k][r] S_k) instead of per-point weighted sums, and the
 *     Jacobian is applied once per region;
 *   - phase 2 bisects the exact maximum-error region (the reference's
 *     128-slot shared pool falls back to an approximate top-64 once full,
 *     GPUQuadPhases.cu:253-277,384-394).
 */
#include "cuhre_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_rule {
  int ndim;
  int npts;
  int count[ORC_NSETS];
  double gen[ORC_NSETS][ORC_MAXDIM];
  double wt[ORC_NSETS][ORC_NRULES];
  double scale[ORC_NSETS][ORC_NRULES];
  double norm[ORC_NSETS][ORC_NRULES];
  double* g;  /* [npts][ndim] */
  int* set;   /* [npts]       */
};

int orc_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Number of points of the degree-9 rule, quad/quad.h:83-85. */
int orc_npoints_formula(int n)
{
  return 1 + 8 * n + 6 * n * (n - 1) + 4 * n * (n - 1) * (n - 2) / 3 + (1 << n);
}

/* ------------------------------------------------------------------------
 * Rule tables.  Weights are polynomials in n; generators and the null-rule
 * normalisation follow GPUQuadRule.cu:31-228.  The numeric table defines
 * the rule, so its values (and the evaluation order of each polynomial,
 * which fixes the rounding) are the reference's.
 * ---------------------------------------------------------------------- */
static void rule_weights(int ndim, double wt[ORC_NSETS][ORC_NRULES])
{
  const double n = (double)ndim;
  const double p0 = n * (n * (n * (-.0023611709677855117884) + .11415390023857325268) +
                         (-.63833920076702389094)) + .74849988504685208004;
  const double p1 = n * (n * (n * (-.0014324017033399125142) + .057471507864489725949) +
                         (-.14225104571434243234)) - (-.062875028738286979989);
  const double q0 = n * (n * .0035417564516782676826 + (-.072609367395893679605)) +
                    .10557491625218991012;
  const double q1 = n * (n * .0021486025550098687713 + (-.032268563892953949998)) +
                    .010636783990231217481;
  const double r0 = n * (-.04508628929435784076) + .21415883524352793401;
  const double r1 = n * (-.027351546526545644722) + .054941067048711234101;
  const double s0 = .015532417276607053264 - n * .0035417564516782676826;
  const double s1 = .0035328099607090870236 - n * .0021486025550098687713;
  const double t0 = .25150011495314791996 / (double)(1 << ndim);
  const double t1 = -.062875028738286979989 / (double)(1 << ndim);

  const double table[ORC_NSETS][ORC_NRULES] = {
    {p0, p1, n * (.254591133248959089) - p1,
     n * (n * (-1.207328566678236261) + .89567365764160676508) - 1 + p0,
     n * (-.36479356986049146661) + 1 - p0},
    {q0, q1, .014689102496143490175 - q1,
     n * .51134708346467591431 + .45976448120806344646 + q0,
     .18239678493024573331 - q0},
    {r0, r1, .11937596202570775297 - r1, n * .65089519391920250593 + .14744939829434460168,
     -r0},
    {.057693384490973483573, .034999626602143583822, -.057693384490973483573,
     -1.3868627719278281436, -.057693384490973483573},
    {0, 0, -.2386668732575008879, 0, 0},
    {s0, s1, -s1, .09231719987444221619 + .015532417276607053264 - n * .0035417564516782676826,
     -s0},
    {.02254314464717892038, .013675773263272822361, -.013675773263272822361,
     -.32544759695960125297, -.02254314464717892038},
    {.0017708782258391338413, .0010743012775049343856, -.0010743012775049343856,
     .0017708782258391338413, -.0017708782258391338413},
    {t0, t1, -t1, t0, -t0}};
  memcpy(wt, table, sizeof(table));
}

/* Generator magnitudes, GPUQuadRule.cu:159-163. */
static const double kGen[5] = {.47795365790226950619, .20302858736911986780,
                               .44762735462617812882, .125, .34303789878087814570};

static void put_point(orc_rule* r, int p, int set, const int* axes,
                      const double* vals, int k)
{
  double* g = r->g + (size_t)p * r->ndim;
  for (int d = 0; d < r->ndim; ++d) g[d] = 0.0;
  for (int j = 0; j < k; ++j) g[axes[j]] = vals[j];
  r->set[p] = set;
}

/* Emit the 2^k sign patterns of k nonzero coordinates: bit j of the pattern
 * makes coordinate j negative. */
static int put_signed(orc_rule* r, int p, int set, const int* axes,
                      const double* mag, int k)
{
  double v[ORC_MAXDIM];
  for (int s = 0; s < (1 << k); ++s) {
    for (int j = 0; j < k; ++j) v[j] = ((s >> j) & 1) ? -mag[j] : mag[j];
    put_point(r, p++, set, axes, v, k);
  }
  return p;
}

orc_rule* orc_rule_new(int ndim)
{
  if (ndim < 2 || ndim > ORC_MAXDIM) return NULL;
  orc_rule* r = (orc_rule*)calloc(1, sizeof(orc_rule));
  const int n = ndim;
  r->ndim = n;
  r->npts = orc_npoints_formula(n);
  const int cnt[ORC_NSETS] = {1, 2 * n, 2 * n, 2 * n, 2 * n, 2 * n * (n - 1), 4 * n * (n - 1),
                              4 * n * (n - 1) * (n - 2) / 3, 1 << n};
  memcpy(r->count, cnt, sizeof(cnt));
  rule_weights(n, r->wt);

  /* generator vectors, GPUQuadRule.cu:179-207 */
  r->gen[1][0] = kGen[0];
  r->gen[2][0] = kGen[1];
  r->gen[3][0] = kGen[2];
  r->gen[4][0] = kGen[3];
  r->gen[5][0] = r->gen[5][1] = kGen[0];
  r->gen[6][0] = kGen[0];
  r->gen[6][1] = kGen[1];
  r->gen[7][0] = r->gen[7][1] = r->gen[7][2] = kGen[0];
  for (int d = 0; d < n; ++d) r->gen[8][d] = kGen[4];

  /* null-rule scale and norm, GPUQuadRule.cu:209-227 */
  for (int k = 0; k < ORC_NSETS; ++k) {
    for (int q = 1; q < ORC_NRULES - 1; ++q) {
      double scale = (r->wt[k][q] == 0) ? 100 : -r->wt[k][q + 1] / r->wt[k][q];
      double sum = 0;
      for (int x = 0; x < ORC_NSETS; ++x)
        sum += r->count[x] * fabs(r->wt[x][q + 1] + scale * r->wt[x][q]);
      r->scale[k][q] = scale;
      r->norm[k][q] = 1 / sum;
    }
  }

  /* the points: each generator's orbit under sign changes and permutations */
  r->g = (double*)calloc((size_t)r->npts * n, sizeof(double));
  r->set = (int*)calloc((size_t)r->npts, sizeof(int));
  int p = 0, ax[ORC_MAXDIM];
  double mag[ORC_MAXDIM];
  put_point(r, p++, 0, ax, mag, 0);
  for (int k = 1; k <= 4; ++k)
    for (int d = 0; d < n; ++d) {
      ax[0] = d;
      mag[0] = r->gen[k][0];
      p = put_signed(r, p, k, ax, mag, 1);
    }
  for (int d1 = 0; d1 < n; ++d1)
    for (int d2 = d1 + 1; d2 < n; ++d2) {
      ax[0] = d1; ax[1] = d2;
      mag[0] = mag[1] = kGen[0];
      p = put_signed(r, p, 5, ax, mag, 2);
    }
  for (int d1 = 0; d1 < n; ++d1)
    for (int d2 = 0; d2 < n; ++d2) {
      if (d2 == d1) continue;
      ax[0] = d1; ax[1] = d2;
      mag[0] = kGen[0]; mag[1] = kGen[1];
      p = put_signed(r, p, 6, ax, mag, 2);
    }
  for (int d1 = 0; d1 < n; ++d1)
    for (int d2 = d1 + 1; d2 < n; ++d2)
      for (int d3 = d2 + 1; d3 < n; ++d3) {
        ax[0] = d1; ax[1] = d2; ax[2] = d3;
        mag[0] = mag[1] = mag[2] = kGen[0];
        p = put_signed(r, p, 7, ax, mag, 3);
      }
  for (int d = 0; d < n; ++d) { ax[d] = d; mag[d] = kGen[4]; }
  p = put_signed(r, p, 8, ax, mag, n);
  if (p != r->npts) { orc_rule_free(r); return NULL; }
  return r;
}

void orc_rule_free(orc_rule* r)
{
  if (!r) return;
  free(r->g);
  free(r->set);
  free(r);
}

int orc_rule_ndim(const orc_rule* r) { return r->ndim; }
int orc_rule_npoints(const orc_rule* r) { return r->npts; }

void orc_rule_tables(const orc_rule* r, double* gen, double* wt, double* scale,
                     double* norm, int* count)
{
  for (int k = 0; k < ORC_NSETS; ++k) {
    if (gen) for (int d = 0; d < r->ndim; ++d) gen[k * r->ndim + d] = r->gen[k][d];
    for (int q = 0; q < ORC_NRULES; ++q) {
      if (wt) wt[k * ORC_NRULES + q] = r->wt[k][q];
      if (scale) scale[k * ORC_NRULES + q] = r->scale[k][q];
      if (norm) norm[k * ORC_NRULES + q] = r->norm[k][q];
    }
    if (count) count[k] = r->count[k];
  }
}

void orc_rule_points(const orc_rule* r, double* g, int* set)
{
  if (g) memcpy(g, r->g, sizeof(double) * (size_t)r->npts * r->ndim);
  if (set) memcpy(set, r->set, sizeof(int) * (size_t)r->npts);
}

/* ------------------------------------------------------------------------
 * Integrand families (Genz 1984 test families; COSSUM is the reference's
 * own driver integrand, cudaCuhre.cu:11-22).
 * ---------------------------------------------------------------------- */
/* ------------------------------------------------------------------------
 * Tables: cell search (the cell left of the first knot >= t among
 * xs[1..n-1], as the reference's SmallNearestN, GPUQuadInterp2D.cu:50-67,
 * clamped to the table), bilinear interpolation, natural cubic spline.
 * ---------------------------------------------------------------------- */
int orc_table_cell(const double* xs, int n, double t)
{
  int i = 1;
  while (i < n - 1 && xs[i] < t) ++i;
  return i - 1;
}

double orc_interp2d_eval(const orc_interp2d* t, double x, double y)
{
  const int i = orc_table_cell(t->xs, t->nx, x), j = orc_table_cell(t->ys, t->ny, y);
  const double x1 = t->xs[i], x2 = t->xs[i + 1], y1 = t->ys[j], y2 = t->ys[j + 1];
  const double q11 = t->zs[i * t->ny + j], q21 = t->zs[(i + 1) * t->ny + j];
  const double q12 = t->zs[i * t->ny + j + 1], q22 = t->zs[(i + 1) * t->ny + j + 1];
  const double d = (x2 - x1) * (y2 - y1);
  return (q11 * (x2 - x) + q21 * (x - x1)) * ((y2 - y) / d) +
         (q12 * (x2 - x) + q22 * (x - x1)) * ((y - y1) / d);
}

double orc_spline_eval(const orc_spline1d* s, double t)
{
  const int i = orc_table_cell(s->xs, s->n, t);
  const double h = s->xs[i + 1] - s->xs[i];
  const double a = (s->xs[i + 1] - t) / h, b = (t - s->xs[i]) / h;
  return a * s->ys[i] + b * s->ys[i + 1] +
         ((a * a * a - a) * s->y2[i] + (b * b * b - b) * s->y2[i + 1]) * (h * h) / 6.0;
}

void orc_spline_second_derivs(int n, const double* xs, const double* ys, double* y2)
{
  /* natural end conditions; Thomas algorithm on the interior equations
   * h_{i-1} y2_{i-1} + 2 (h_{i-1} + h_i) y2_i + h_i y2_{i+1} = 6 (d_i - d_{i-1}) */
  double* c = (double*)malloc(sizeof(double) * (size_t)n);
  double* r = (double*)malloc(sizeof(double) * (size_t)n);
  y2[0] = 0;
  y2[n - 1] = 0;
  c[0] = 0;
  r[0] = 0;
  for (int i = 1; i < n - 1; ++i) {
    const double hl = xs[i] - xs[i - 1], hr = xs[i + 1] - xs[i];
    const double rhs = 6.0 * ((ys[i + 1] - ys[i]) / hr - (ys[i] - ys[i - 1]) / hl);
    const double den = 2.0 * (hl + hr) - hl * c[i - 1];
    c[i] = hr / den;
    r[i] = (rhs - hl * r[i - 1]) / den;
  }
  for (int i = n - 2; i >= 1; --i) y2[i] = r[i] - c[i] * y2[i + 1];
  free(c);
  free(r);
}

static double lclt_eval(const orc_tables* T, const double* x)
{
  const double lt = x[0], zt = x[1], lc = x[2];
  double v[5];
  for (int q = 0; q < 5; ++q) v[q] = orc_interp2d_eval(&T->lclt[q], lt, zt);
  const double tau = v[0], mu = v[1], sigma = v[2], fmsk = v[3], fprj = v[4];
  /* lc_lt_t.h:36-50 */
  const double exptau = exp(tau * (2.0 * mu + tau * sigma * sigma - 2.0 * lc) / 2.0);
  const double r2s = sqrt(2.0) * sigma;
  const double mts = mu + tau * sigma * sigma;
  const double zg = (lc - mu) / sigma;
  const double gauss = exp(-zg * zg / 2.0) * 0.3989422804014327 / sigma;
  return (1.0 - fmsk) * (1.0 - fprj) * gauss +
         0.5 * ((1.0 - fmsk) * fprj * tau + fmsk * fprj / lt) * exptau * erfc((mts - lc) / r2s) +
         0.5 * fmsk / lt * (erfc((lc - mu) / r2s) - erfc((lc + lt - mu) / r2s)) -
         0.5 * fmsk * fprj / lt * (exp(-tau * lt) * exptau * erfc((mts - lc - lt) / r2s));
}

static double table7_eval(const orc_tables* T, const double* x)
{
  const double mu = T->offset + 2.0 * x[4] + 0.1 * (x[5] + x[6]);
  const double r = 4.0 * x[3] - mu;
  return orc_spline_eval(&T->spline, x[0]) * orc_interp2d_eval(&T->grid, x[1], x[2]) *
         exp(-r * r / (2.0 * T->sigma * T->sigma));
}

double orc_eval_integrand(const orc_integrand* f, const double* x)
{
  const int n = f->ndim;
  switch (f->family) {
    case ORC_LCLT:
      return lclt_eval(f->tables, x);
    case ORC_TABLE7:
      return table7_eval(f->tables, x);
    case ORC_GAUSSIAN: {
      double s = 0;
      for (int d = 0; d < n; ++d) {
        double t = f->a[d] * (x[d] - f->u[d]);
        s += t * t;
      }
      return exp(-s);
    }
    case ORC_OSCILLATORY: {
      double s = 2 * M_PI * f->u[0];
      for (int d = 0; d < n; ++d) s += f->a[d] * x[d];
      return cos(s);
    }
    case ORC_CORNER_PEAK: {
      double s = 1;
      for (int d = 0; d < n; ++d) s += f->a[d] * x[d];
      double p = 1;
      for (int k = 0; k <= n; ++k) p *= s;
      return 1 / p;
    }
    case ORC_PRODUCT_PEAK: {
      double p = 1;
      for (int d = 0; d < n; ++d) {
        double t = x[d] - f->u[d];
        p *= 1 / (1 / (f->a[d] * f->a[d]) + t * t);
      }
      return p;
    }
    case ORC_CONTINUOUS: {
      double s = 0;
      for (int d = 0; d < n; ++d) s += f->a[d] * fabs(x[d] - f->u[d]);
      return exp(-s);
    }
    case ORC_DISCONTINUOUS: {
      if (x[0] > f->u[0] || (n > 1 && x[1] > f->u[1])) return 0;
      double s = 0;
      for (int d = 0; d < n; ++d) s += f->a[d] * x[d];
      return exp(s);
    }
    case ORC_COSSUM: {
      double s = 0;
      for (int d = 0; d < n; ++d) s = s - cos(10.0 * x[d]) / 0.054402111088937;
      return s / 2.0;
    }
    default:
      return NAN;
  }
}

/* Analytic integrals over [0,1]^n. */
double orc_exact(const orc_integrand* f)
{
  const int n = f->ndim;
  if (f->has_box) {
    /* closed forms over a box for the separable families */
    double p = 1;
    for (int d = 0; d < n; ++d) {
      const double a = f->a[d], u = f->u[d], l = f->box_lo[d], h = f->box_hi[d];
      if (f->family == ORC_GAUSSIAN)
        p *= sqrt(M_PI) / (2 * a) * (erf(a * (h - u)) - erf(a * (l - u)));
      else if (f->family == ORC_PRODUCT_PEAK)
        p *= a * (atan(a * (h - u)) - atan(a * (l - u)));
      else
        return NAN;
    }
    return p;
  }
  switch (f->family) {
    case ORC_GAUSSIAN: {
      double p = 1;
      for (int d = 0; d < n; ++d) {
        double a = f->a[d], u = f->u[d];
        p *= sqrt(M_PI) / (2 * a) * (erf(a * (1 - u)) + erf(a * u));
      }
      return p;
    }
    case ORC_OSCILLATORY: {
      /* Re[e^{i 2 pi u0} prod (e^{i a} - 1)/(i a)] */
      double re = cos(2 * M_PI * f->u[0]), im = sin(2 * M_PI * f->u[0]);
      for (int d = 0; d < n; ++d) {
        double a = f->a[d];
        double zr = sin(a) / a, zi = (1 - cos(a)) / a; /* (e^{ia}-1)/(ia) */
        double nr = re * zr - im * zi, ni = re * zi + im * zr;
        re = nr;
        im = ni;
      }
      return re;
    }
    case ORC_CORNER_PEAK: {
      double fact = 1, prod = 1, acc = 0;
      for (int d = 1; d <= n; ++d) fact *= d;
      for (int d = 0; d < n; ++d) prod *= f->a[d];
      for (unsigned s = 0; s < (1u << n); ++s) {
        double t = 1;
        int bits = 0;
        for (int d = 0; d < n; ++d)
          if (s >> d & 1) { t += f->a[d]; ++bits; }
        acc += ((bits & 1) ? -1.0 : 1.0) / t;
      }
      return acc / (fact * prod);
    }
    case ORC_PRODUCT_PEAK: {
      double p = 1;
      for (int d = 0; d < n; ++d) {
        double a = f->a[d], u = f->u[d];
        p *= a * (atan(a * (1 - u)) + atan(a * u));
      }
      return p;
    }
    case ORC_CONTINUOUS: {
      double p = 1;
      for (int d = 0; d < n; ++d) {
        double a = f->a[d], u = f->u[d];
        p *= (2 - exp(-a * u) - exp(-a * (1 - u))) / a;
      }
      return p;
    }
    case ORC_DISCONTINUOUS: {
      double p = 1;
      for (int d = 0; d < n; ++d) {
        double a = f->a[d];
        double hi = (d < 2) ? (f->u[d] < 1 ? f->u[d] : 1) : 1;
        p *= (exp(a * hi) - 1) / a;
      }
      return p;
    }
    case ORC_COSSUM:
      return -n * sin(10.0) / 10.0 / 0.054402111088937 / 2.0;
    default:
      return NAN;
  }
}

/* ------------------------------------------------------------------------
 * One region: rule sums, fourth-difference split axis, null-rule error
 * (GPUQuadSample.cu:102-220, computePermutation :35-97).
 * ---------------------------------------------------------------------- */
void orc_eval_region(const orc_rule* r, const orc_integrand* f, const double* L,
                     const double* W, const double* llo, const double* lhi, int div,
                     orc_result* out)
{
  const int n = r->ndim;
  double range[ORC_MAXDIM], lo[ORC_MAXDIM], hi[ORC_MAXDIM], x[ORC_MAXDIM];
  double jac = 1;
  for (int d = 0; d < n; ++d) {
    double U = L[d] + W[d];
    range[d] = U - L[d];
    jac = jac * range[d];
    lo[d] = llo ? llo[d] : 0.0;
    hi[d] = lhi ? lhi[d] : 1.0;
  }
  /* fallback split axis: the widest local side (GPUQuadSample.cu:118-125) */
  int maxdim = 0;
  double maxrange = 0;
  for (int d = 0; d < n; ++d) {
    double w = hi[d] - lo[d];
    if (w > maxrange) { maxrange = w; maxdim = d; }
  }

  double S[ORC_NSETS] = {0}, Sabs[ORC_NSETS] = {0};
  double fv[4 * ORC_MAXDIM + 1];
  for (int p = 0; p < r->npts; ++p) {
    const double* g = r->g + (size_t)p * n;
    for (int d = 0; d < n; ++d) {
      double xl = (.5 + g[d]) * lo[d] + (.5 - g[d]) * hi[d];
      x[d] = L[d] + xl * range[d];
    }
    double fx = orc_eval_integrand(f, x);
    S[r->set[p]] += fx;
    Sabs[r->set[p]] += fabs(fx);
    if (p <= 4 * n) fv[p] = fx;
  }
  {
    double m = 0;
    for (int k = 0; k < ORC_NSETS; ++k) m += fabs(r->wt[k][0]) * Sabs[k];
    out->mag = m * jac * ldexp(1., -div);
  }

  /* fourth divided difference per axis (GPUQuadSample.cu:152-172) */
  const double ratio = (r->gen[2][0] / r->gen[1][0]) * (r->gen[2][0] / r->gen[1][0]);
  const double base = fv[0] * 2 * (1 - ratio);
  double best = 0, second = 0;
  int axis = maxdim;
  for (int d = 0; d < n; ++d) {
    double fd = fabs(base + ratio * (fv[1 + 2 * d] + fv[2 + 2 * d]) -
                     (fv[1 + 2 * n + 2 * d] + fv[2 + 2 * n + 2 * d]));
    if (fd > best) {
      second = best;
      best = fd;
      axis = d;
    } else if (fd > second) {
      second = fd;
    }
  }
  out->axis = axis;
  out->axis_margin = best > 0 ? (best - second) / best : 1.0;

  /* rule sums and the null-rule error (GPUQuadSample.cu:195-216) */
  double sum[ORC_NRULES];
  for (int q = 0; q < ORC_NRULES; ++q) {
    double acc = 0;
    for (int k = 0; k < ORC_NSETS; ++k) acc += r->wt[k][q] * S[k];
    sum[q] = acc * jac;
  }
  double nul[ORC_NRULES];
  for (int q = 1; q < ORC_NRULES - 1; ++q) {
    double m = 0;
    for (int k = 0; k < ORC_NSETS; ++k) {
      double e = fabs(sum[q + 1] + r->scale[k][q] * sum[q]) * r->norm[k][q];
      m = (m > e) ? m : e;
    }
    nul[q] = m;
  }
  const double vol = ldexp(1., -div);
  out->avg = vol * sum[0];
  double m12 = nul[1] > nul[2] ? nul[1] : nul[2];
  double m123 = m12 > nul[3] ? m12 : nul[3];
  out->err = vol * ((5 * nul[1] <= nul[2] && 5 * nul[2] <= nul[3]) ? 1 * nul[1] : 5 * m123);
}

static double max_err(double avg, double epsrel, double epsabs)
{
  double a = epsrel * fabs(avg);
  return a > epsabs ? a : epsabs;
}

void orc_phase1_eval(const orc_rule* r, const orc_integrand* f, size_t n, const double* lo,
                     const double* len, double epsrel, double epsabs, double* avg,
                     double* err, int* axis, int* active, double* margin, double* ratio,
                     double* mag, int nthreads)
{
  const int nd = r->ndim;
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
  for (long long i = 0; i < (long long)n; ++i) {
    double L[ORC_MAXDIM], W[ORC_MAXDIM];
    for (int d = 0; d < nd; ++d) {
      L[d] = lo[(size_t)d * n + i];
      W[d] = len[(size_t)d * n + i];
    }
    orc_result res;
    orc_eval_region(r, f, L, W, NULL, NULL, 0, &res);
    double q = res.err / max_err(res.avg, epsrel, epsabs);
    avg[i] = res.avg;
    err[i] = res.err;
    axis[i] = res.axis;
    active[i] = q > 1;
    if (margin) margin[i] = res.axis_margin;
    if (ratio) ratio[i] = q;
    if (mag) mag[i] = res.mag;
  }
  (void)nthreads;
}

size_t orc_split(int ndim, size_t n, const double* lo, const double* len, const int* active,
                 const int* axis, double* out_lo, double* out_len)
{
  size_t m = 0;
  for (size_t i = 0; i < n; ++i) m += active[i] == 1;
  size_t j = 0;
  for (size_t i = 0; i < n; ++i) {
    if (active[i] != 1) continue;
    for (int d = 0; d < ndim; ++d) {
      double l = lo[(size_t)d * n + i], w = len[(size_t)d * n + i];
      if (d == axis[i]) {
        double h = w / 2;
        out_lo[(size_t)d * 2 * m + j] = l;
        out_lo[(size_t)d * 2 * m + m + j] = l + 1 * h;
        out_len[(size_t)d * 2 * m + j] = h;
        out_len[(size_t)d * 2 * m + m + j] = h;
      } else {
        out_lo[(size_t)d * 2 * m + j] = l;
        out_lo[(size_t)d * 2 * m + m + j] = l;
        out_len[(size_t)d * 2 * m + j] = w;
        out_len[(size_t)d * 2 * m + m + j] = w;
      }
    }
    ++j;
  }
  return 2 * m;
}

/* Divisions per axis of the initial grid, GPUKernelquad.cu:300-311. */
static int grid_divisions(int ndim)
{
  if (ndim > 10) return 1;
  if (ndim >= 5) return 2;
  return 4;
}

size_t orc_initial_grid(int ndim, double* lo, double* len)
{
  const int dv = grid_divisions(ndim);
  size_t count = 1;
  for (int d = 0; d < ndim; ++d) count *= (size_t)dv;
  if (!lo) return count;
  const double w = 1.0 / dv;
  for (size_t i = 0; i < count; ++i) {
    size_t rem = i;
    for (int d = 0; d < ndim; ++d) {
      size_t id = rem % (size_t)dv;
      rem /= (size_t)dv;
      lo[(size_t)d * count + i] = 0 + id * w;
      len[(size_t)d * count + i] = w;
    }
  }
  return count;
}

size_t orc_initial_grid_box(const orc_integrand* f, double* lo, double* len)
{
  const int ndim = f->ndim;
  if (!f->has_box) return orc_initial_grid(ndim, lo, len);
  const int dv = grid_divisions(ndim);
  size_t count = 1;
  for (int d = 0; d < ndim; ++d) count *= (size_t)dv;
  if (!lo) return count;
  for (size_t i = 0; i < count; ++i) {
    size_t rem = i;
    for (int d = 0; d < ndim; ++d) {
      const double w = (f->box_hi[d] - f->box_lo[d]) / dv;
      size_t id = rem % (size_t)dv;
      rem /= (size_t)dv;
      lo[(size_t)d * count + i] = f->box_lo[d] + id * w;
      len[(size_t)d * count + i] = w;
    }
  }
  return count;
}

/* pairwise sum: the reductions only need to be accurate, not ordered */
static double psum(const double* v, size_t n)
{
  if (n <= 16) {
    double s = 0;
    for (size_t i = 0; i < n; ++i) s += v[i];
    return s;
  }
  size_t h = n / 2;
  return psum(v, h) + psum(v + h, n - h);
}

/* ------------------------------------------------------------------------
 * Phase 2 on one leftover box: serial Cuhre with a local tolerance and a
 * region cap (GPUQuadPhases.cu:424-536).  Regions live in local [0,1]^n
 * coordinates of the box; a max-heap on the error picks the next region.
 * ---------------------------------------------------------------------- */
typedef struct {
  double avg, err;
  int axis, div;
  double lo[ORC_MAXDIM], hi[ORC_MAXDIM];
} p2_region;

static void heap_push(p2_region* pool, int* heap, int* hn, int idx)
{
  int i = (*hn)++;
  heap[i] = idx;
  while (i > 0) {
    int p = (i - 1) / 2;
    if (pool[heap[p]].err >= pool[heap[i]].err) break;
    int t = heap[p]; heap[p] = heap[i]; heap[i] = t;
    i = p;
  }
}

static int heap_pop(p2_region* pool, int* heap, int* hn)
{
  int top = heap[0];
  heap[0] = heap[--(*hn)];
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, rr = l + 1, m = i;
    if (l < *hn && pool[heap[l]].err > pool[heap[m]].err) m = l;
    if (rr < *hn && pool[heap[rr]].err > pool[heap[m]].err) m = rr;
    if (m == i) break;
    int t = heap[m]; heap[m] = heap[i]; heap[i] = t;
    i = m;
  }
  return top;
}

int orc_phase2_box(const orc_rule* r, const orc_integrand* f, const double* L,
                   const double* W, double epsrel, double epsabs, int max_regions,
                   double* result, double* error, int* failed)
{
  const int n = r->ndim;
  const int cap = max_regions + 2;
  p2_region* pool = (p2_region*)malloc(sizeof(p2_region) * (size_t)cap);
  int* heap = (int*)malloc(sizeof(int) * (size_t)cap);
  int hn = 0, used = 0;
  orc_result res;

  p2_region* r0 = &pool[used++];
  for (int d = 0; d < n; ++d) { r0->lo[d] = 0; r0->hi[d] = 1; }
  r0->div = 0;
  orc_eval_region(r, f, L, W, r0->lo, r0->hi, 0, &res);
  r0->avg = res.avg; r0->err = res.err; r0->axis = res.axis;
  heap_push(pool, heap, &hn, 0);
  double ERR = r0->err, RESULT = r0->avg;

  int nregions = 1;
  for (; nregions <= max_regions &&
         (nregions == 1 || ERR > max_err(RESULT, epsrel, epsabs));
       ++nregions) {
    int pi = heap_pop(pool, heap, &hn);
    p2_region parent = pool[pi];
    p2_region* left = &pool[pi];
    p2_region* right = &pool[used++];
    int ax = parent.axis;
    left->div = right->div = parent.div + 1;
    memcpy(right->lo, parent.lo, sizeof(double) * n);
    memcpy(right->hi, parent.hi, sizeof(double) * n);
    double mid = 0.5 * (parent.lo[ax] + parent.hi[ax]);
    left->hi[ax] = mid;
    right->lo[ax] = mid;
    orc_eval_region(r, f, L, W, left->lo, left->hi, left->div, &res);
    left->avg = res.avg; left->err = res.err; left->axis = res.axis;
    orc_eval_region(r, f, L, W, right->lo, right->hi, right->div, &res);
    right->avg = res.avg; right->err = res.err; right->axis = res.axis;
    /* Cuhre error refinement, GPUQuadPhases.cu:498-511 */
    double diff = fabs(.25 * (left->avg + right->avg - parent.avg));
    double e = left->err + right->err;
    if (e > 0) {
      double c = 1 + 2 * diff / e;
      left->err *= c;
      right->err *= c;
    }
    left->err += diff;
    right->err += diff;
    ERR += left->err + right->err - parent.err;
    RESULT += left->avg + right->avg - parent.avg;
    heap_push(pool, heap, &hn, pi);
    heap_push(pool, heap, &hn, (int)(right - pool));
  }
  int active = ERR > max_err(RESULT, epsrel, epsabs);
  if (ERR > 1e10) { /* GPUQuadPhases.cu:519-527 */
    RESULT = 0;
    ERR = 0;
    active = 1;
  }
  *result = RESULT;
  *error = ERR;
  *failed = active;
  free(pool);
  free(heap);
  return nregions;
}

/* ------------------------------------------------------------------------
 * Two-phase integration with the reference policy (GPUquad.h:611-727,
 * GPUKernelquad.cu:509-668 and :672-911).
 * ---------------------------------------------------------------------- */
/* The two phases with the second one restricted to a contiguous share of
 * the leftover boxes: share `rank` of `world`, cut as the reference cuts
 * its leftover list across devices (GPUKernelquad.cu:759-768: world equal
 * parts, the last one taking the remainder).  p1 receives the first
 * phase's result (its finished sums, or the converged result when no box
 * is left; phase2_regions = leftover boxes), part the share's boxes (their
 * value and error sums, regions, evaluations; status = failed boxes, or
 * ORC_STATUS_NONFINITE).  Every rank computes the same first phase. */
int orc_integrate_reference_shard(const orc_rule* r, const orc_integrand* f, double epsrel,
                                  double epsabs, int phase1_cap, int phase2_max, int nthreads,
                                  int rank, int world, orc_out* p1, orc_out* part)
{
  if (phase2_max <= 0) phase2_max = 2048; /* MAX_GLOBALPOOL_SIZE, quad.h:9 */
  if (world < 1 || rank < 0 || rank >= world) return -1;
  orc_out scratch;
  orc_out* out = &scratch;
  const int nd = r->ndim;
  const size_t fe = (size_t)r->npts;
  if (phase1_cap <= 0) phase1_cap = 1 << 14; /* FIRST_PHASE_MAXREGIONS, quad.h:21 */
  memset(out, 0, sizeof(*out));

  size_t n = orc_initial_grid_box(f, NULL, NULL);
  double* lo = (double*)malloc(sizeof(double) * n * nd);
  double* len = (double*)malloc(sizeof(double) * n * nd);
  orc_initial_grid_box(f, lo, len);

  double integral = 0, error = 0;
  size_t nregions = 0, neval = 0;
  int iters = 0, nonfinite = 0;
  for (int it = 0; it < 100; ++it) {
    double* avg = (double*)malloc(sizeof(double) * n);
    double* err = (double*)malloc(sizeof(double) * n);
    int* axis = (int*)malloc(sizeof(int) * n);
    int* act = (int*)malloc(sizeof(int) * n);
    orc_phase1_eval(r, f, n, lo, len, epsrel, epsabs, avg, err, axis, act, NULL, NULL, NULL,
                    nthreads);
    ++iters;
    nregions += n;
    neval += n * fe;
    double sum_avg = psum(avg, n), sum_err = psum(err, n);
    for (size_t i = 0; i < n; ++i)
      if (act[i]) { avg[i] = 0; err[i] = 0; }
    double fin_avg = psum(avg, n), fin_err = psum(err, n);
    double rG = integral + sum_avg, errG = error + sum_err;
    integral += fin_avg;
    error += fin_err;
    if (!isfinite(sum_avg) || !isfinite(sum_err)) {
      /* a NaN or infinite integrand value: stop with the sums as they are */
      integral = rG;
      error = errG;
      nonfinite = 1;
      n = 0;
      free(avg); free(err); free(axis); free(act);
      break;
    }
    if (errG <= max_err(rG, epsrel, epsabs)) {
      integral = rG;
      error = errG;
      n = 0;
      free(avg); free(err); free(axis); free(act);
      break;
    }
    size_t m = 0;
    for (size_t i = 0; i < n; ++i) m += act[i];
    double* nlo = (double*)malloc(sizeof(double) * (2 * m + 1) * nd);
    double* nlen = (double*)malloc(sizeof(double) * (2 * m + 1) * nd);
    size_t nn = orc_split(nd, n, lo, len, act, axis, nlo, nlen);
    free(lo); free(len);
    lo = nlo; len = nlen;
    n = nn;
    free(avg); free(err); free(axis); free(act);
    if (n < 1) break;
    if (n >= (size_t)phase1_cap) break;
  }
  memset(p1, 0, sizeof(*p1));
  memset(part, 0, sizeof(*part));
  p1->value = integral;
  p1->error = error;
  p1->nregions = nregions;
  p1->neval = neval;
  p1->phase1_iters = iters;
  p1->phase2_regions = n;
  p1->status = nonfinite ? ORC_STATUS_NONFINITE : 0;
  out->phase1_iters = iters;
  out->phase2_regions = n;

  int status = 0;
  size_t first = 0, last = n;
  if (world > 1) {
    const size_t each = n / (size_t)world;
    first = (size_t)rank * each;
    last = rank == world - 1 ? n : first + each;
  }
  if (n > 0) {
    double* res = (double*)malloc(sizeof(double) * n);
    double* er = (double*)malloc(sizeof(double) * n);
    int* cnt = (int*)malloc(sizeof(int) * n);
    int* fail = (int*)malloc(sizeof(int) * n);
#ifdef _OPENMP
    int nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
#endif
    for (long long i = 0; i < (long long)n; ++i) {
      if ((size_t)i < first || (size_t)i >= last) {
        res[i] = 0;
        er[i] = 0;
        cnt[i] = 0;
        fail[i] = 0;
        continue;
      }
      double L[ORC_MAXDIM], W[ORC_MAXDIM];
      for (int d = 0; d < nd; ++d) {
        L[d] = lo[(size_t)d * n + i];
        W[d] = len[(size_t)d * n + i];
      }
      cnt[i] = orc_phase2_box(r, f, L, W, epsrel, epsabs, phase2_max, &res[i], &er[i], &fail[i]);
    }
    size_t total = 0, failed = 0;
    int part_nonfinite = 0;
    for (size_t i = 0; i < n; ++i) {
      total += (size_t)cnt[i];
      failed += (size_t)fail[i];
      if (!isfinite(res[i]) || !isfinite(er[i])) part_nonfinite = 1;
    }
    const size_t nb = last - first;
    part->value = psum(res, n);
    part->error = psum(er, n);
    part->nregions = total;
    part->neval = (total - nb) * fe * 2 + nb * fe;
    part->phase2_regions = nb;
    part->phase2_failed = failed;
    part->status = part_nonfinite ? ORC_STATUS_NONFINITE : (int)failed;
    nonfinite |= part_nonfinite;
    integral += part->value;
    error += part->error;
    nregions += total;
    neval += part->neval;
    status = (int)failed;
    out->phase2_failed = failed;
    free(res); free(er); free(cnt); free(fail);
  }
  if (error <= max_err(integral, epsrel, epsabs)) status = 0;
  if (nonfinite) status = ORC_STATUS_NONFINITE;
  free(lo);
  free(len);
  (void)status;
  return 0;
}

/* The shares of all ranks combined: value, error, regions, evaluations
 * and failed boxes summed, and the reference's final status test
 * (GPUquad.h:713). */
void orc_combine_shards(const orc_out* p1, const orc_out* parts, int world, double epsrel,
                        double epsabs, orc_out* out)
{
  *out = *p1;
  size_t failed = 0;
  int nonfinite = p1->status == ORC_STATUS_NONFINITE;
  for (int k = 0; k < world; ++k) {
    out->value += parts[k].value;
    out->error += parts[k].error;
    out->nregions += parts[k].nregions;
    out->neval += parts[k].neval;
    failed += parts[k].phase2_failed;
    nonfinite |= parts[k].status == ORC_STATUS_NONFINITE;
  }
  out->phase2_failed = failed;
  int status = (int)failed;
  if (out->error <= max_err(out->value, epsrel, epsabs)) status = 0;
  out->status = nonfinite ? ORC_STATUS_NONFINITE : status;
}

int orc_integrate_reference(const orc_rule* r, const orc_integrand* f, double epsrel,
                            double epsabs, int phase1_cap, int phase2_max, int nthreads,
                            orc_out* out)
{
  orc_out p1, part;
  if (orc_integrate_reference_shard(r, f, epsrel, epsabs, phase1_cap, phase2_max, nthreads, 0,
                                    1, &p1, &part))
    return -1;
  orc_combine_shards(&p1, &part, 1, epsrel, epsabs, out);
  return out->status;
}

/* ------------------------------------------------------------------------
 * Breadth-first integration with the global-budget policy: a region is
 * finished when its error is below its volume share of the global budget
 * max(epsrel |I|, epsabs), with I the previous iteration's estimate.
 * ---------------------------------------------------------------------- */
int orc_integrate_global(const orc_rule* r, const orc_integrand* f, double epsrel,
                         double epsabs, size_t max_regions, int max_iters, int nthreads,
                         orc_out* out)
{
  const int nd = r->ndim;
  const size_t fe = (size_t)r->npts;
  memset(out, 0, sizeof(*out));
  if (max_iters <= 0) max_iters = 200;
  size_t n = orc_initial_grid_box(f, NULL, NULL);
  double* lo = (double*)malloc(sizeof(double) * n * nd);
  double* len = (double*)malloc(sizeof(double) * n * nd);
  orc_initial_grid_box(f, lo, len);
  double fin_value = 0, fin_error = 0, estimate = 0;
  int have_estimate = 0, status = 1, iters = 0;
  size_t nregions = 0, neval = 0;
  while (n > 0 && iters < max_iters) {
    double* avg = (double*)malloc(sizeof(double) * n);
    double* err = (double*)malloc(sizeof(double) * n);
    int* axis = (int*)malloc(sizeof(int) * n);
    int* act = (int*)malloc(sizeof(int) * n);
    orc_phase1_eval(r, f, n, lo, len, 0, 0, avg, err, axis, act, NULL, NULL, NULL, nthreads);
    ++iters;
    nregions += n;
    neval += n * fe;
    double rG = fin_value + psum(avg, n), eG = fin_error + psum(err, n);
    if (!have_estimate) { estimate = rG; have_estimate = 1; }
    if (eG <= max_err(rG, epsrel, epsabs)) {
      fin_value = rG;
      fin_error = eG;
      status = 0;
      free(avg); free(err); free(axis); free(act);
      n = 0;
      break;
    }
    double budget = max_err(estimate, epsrel, epsabs);
    size_t m = 0;
    for (size_t i = 0; i < n; ++i) {
      double vol = 1;
      for (int d = 0; d < nd; ++d) vol *= len[(size_t)d * n + i];
      act[i] = err[i] > budget * vol;
      m += (size_t)act[i];
    }
    for (size_t i = 0; i < n; ++i)
      if (act[i]) { avg[i] = 0; err[i] = 0; }
    fin_value += psum(avg, n);
    fin_error += psum(err, n);
    estimate = rG;
    if (m == 0 || nregions + 2 * m > max_regions) {
      /* out of regions: report the current totals, not converged */
      fin_value = rG;
      fin_error = eG;
      free(avg); free(err); free(axis); free(act);
      n = 0;
      break;
    }
    double* nlo = (double*)malloc(sizeof(double) * 2 * m * nd);
    double* nlen = (double*)malloc(sizeof(double) * 2 * m * nd);
    size_t nn = orc_split(nd, n, lo, len, act, axis, nlo, nlen);
    free(lo); free(len);
    lo = nlo; len = nlen;
    n = nn;
    free(avg); free(err); free(axis); free(act);
  }
  free(lo);
  free(len);
  out->value = fin_value;
  out->error = fin_error;
  out->nregions = nregions;
  out->neval = neval;
  out->status = status;
  out->phase1_iters = iters;
  return status;
}

/* ------------------------------------------------------------------------
 * Sequential global-heap Cuhre: one region list for the whole cube, always
 * bisect the worst region (the classic algorithm of Berntsen, Espelid and
 * Genz 1991 as used by Hahn's Cuhre), same rule and refinement as above.
 * ---------------------------------------------------------------------- */
int orc_cuhre_sequential(const orc_rule* r, const orc_integrand* f, double epsrel,
                         double epsabs, size_t max_regions, orc_out* out)
{
  const int n = r->ndim;
  memset(out, 0, sizeof(*out));
  if (max_regions < 3) max_regions = 3;
  p2_region* pool = (p2_region*)malloc(sizeof(p2_region) * (max_regions + 2));
  int* heap = (int*)malloc(sizeof(int) * (max_regions + 2));
  int hn = 0;
  size_t used = 0;
  double Lz[ORC_MAXDIM], W1[ORC_MAXDIM];
  for (int d = 0; d < n; ++d) {
    Lz[d] = f->has_box ? f->box_lo[d] : 0;
    W1[d] = f->has_box ? f->box_hi[d] - f->box_lo[d] : 1;
  }
  orc_result res;
  p2_region* r0 = &pool[used++];
  for (int d = 0; d < n; ++d) { r0->lo[d] = 0; r0->hi[d] = 1; }
  r0->div = 0;
  orc_eval_region(r, f, Lz, W1, r0->lo, r0->hi, 0, &res);
  r0->avg = res.avg; r0->err = res.err; r0->axis = res.axis;
  heap_push(pool, heap, &hn, 0);
  double ERR = r0->err, RESULT = r0->avg;
  size_t nregions = 1;
  int status = 1;
  while (used + 1 < max_regions) {
    if (ERR <= max_err(RESULT, epsrel, epsabs)) { status = 0; break; }
    int pi = heap_pop(pool, heap, &hn);
    p2_region parent = pool[pi];
    p2_region* left = &pool[pi];
    p2_region* right = &pool[used++];
    int ax = parent.axis;
    left->div = right->div = parent.div + 1;
    memcpy(right->lo, parent.lo, sizeof(double) * n);
    memcpy(right->hi, parent.hi, sizeof(double) * n);
    double mid = 0.5 * (parent.lo[ax] + parent.hi[ax]);
    left->hi[ax] = mid;
    right->lo[ax] = mid;
    orc_eval_region(r, f, Lz, W1, left->lo, left->hi, left->div, &res);
    left->avg = res.avg; left->err = res.err; left->axis = res.axis;
    orc_eval_region(r, f, Lz, W1, right->lo, right->hi, right->div, &res);
    right->avg = res.avg; right->err = res.err; right->axis = res.axis;
    double diff = fabs(.25 * (left->avg + right->avg - parent.avg));
    double e = left->err + right->err;
    if (e > 0) {
      double c = 1 + 2 * diff / e;
      left->err *= c;
      right->err *= c;
    }
    left->err += diff;
    right->err += diff;
    ERR += left->err + right->err - parent.err;
    RESULT += left->avg + right->avg - parent.avg;
    heap_push(pool, heap, &hn, pi);
    heap_push(pool, heap, &hn, (int)(right - pool));
    nregions += 2;
  }
  if (status && ERR <= max_err(RESULT, epsrel, epsabs)) status = 0;
  /* recompute the totals from the leaves to shed the running-sum drift */
  double* av = (double*)malloc(sizeof(double) * used);
  double* er = (double*)malloc(sizeof(double) * used);
  for (size_t i = 0; i < used; ++i) { av[i] = pool[i].avg; er[i] = pool[i].err; }
  out->value = psum(av, used);
  out->error = psum(er, used);
  free(av); free(er);
  out->nregions = nregions;
  out->neval = nregions * (size_t)r->npts;
  out->status = status;
  free(pool);
  free(heap);
  return status;
}
