/*
 * cuhre_oracle.h -- CPU oracle for the adaptive cubature hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * engine's algorithm (marcpaterno/old-gpuintegration, quad/GPUquad), used
 * as the checker for the CUDA path and as the timed CPU baseline.  Only the
 * tests, __graft_entry__.smoke() and bench.py's CPU legs may load it; the
 * product library never links or calls it.
 *
 * Parity pinning: the restatement is checked (tests/test_oracle.py) against
 *   - the rule's own algebra (degree-9 exactness, point counts, weights);
 *   - analytic integrals of the Genz families;
 *   - golden outputs of the reference engine itself, compiled from its own
 *     sources by oracle/ref_driver and run on a B200 (tests/golden/).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef CUHRE_ORACLE_H
#define CUHRE_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXDIM 16
#define ORC_NSETS 9
#define ORC_NRULES 5
/* Status of an integral whose integrand gave a NaN or an infinite value:
 * the value and error sums stopped being finite (an extension of the
 * engine, which the reference does not detect). */
#define ORC_STATUS_NONFINITE (1 << 30)

/* Integrand families.  The numbering is shared with include/cubature.h. */
enum {
  ORC_GAUSSIAN = 1,      /* exp(-sum a_i^2 (x_i-u_i)^2)                    */
  ORC_OSCILLATORY = 2,   /* cos(2 pi u_0 + sum a_i x_i)                    */
  ORC_CORNER_PEAK = 3,   /* (1 + sum a_i x_i)^-(n+1)                       */
  ORC_PRODUCT_PEAK = 4,  /* prod 1/(a_i^-2 + (x_i-u_i)^2)                  */
  ORC_CONTINUOUS = 5,    /* exp(-sum a_i |x_i-u_i|)                        */
  ORC_DISCONTINUOUS = 6, /* 0 if x_0>u_0 or x_1>u_1 else exp(sum a_i x_i)  */
  ORC_COSSUM = 7,        /* -sum cos(10 x_i)/0.054402111088937 / 2
                            (cudaCuhre.cu:11-22, function.cu:111-117)      */
  ORC_LCLT = 8,          /* LC_LT over (lt, zt, lc) from five 2-D tables
                            (lc_lt_t.h:18-52)                              */
  ORC_TABLE7 = 9         /* spline(x0) bilinear(x1,x2)
                            exp(-(4 x3 - mu)^2 / 2 sigma^2),
                            mu = offset + 2 x4 + 0.1 (x5 + x6)            */
};

/* Rectilinear 2-D table, row-major zs[i * ny + j] at (xs[i], ys[j]); the
 * reference's Interp2D (GPUQuadInterp2D.cu:50-106) in FP64. */
typedef struct orc_interp2d {
  const double* xs;
  const double* ys;
  const double* zs;
  int nx, ny;
} orc_interp2d;

/* Natural cubic spline: knots, values, second derivatives. */
typedef struct orc_spline1d {
  const double* xs;
  const double* ys;
  const double* y2;
  int n;
} orc_spline1d;

/* Tables of the table integrands (host memory, owned by the caller). */
typedef struct orc_tables {
  orc_interp2d lclt[5];  /* tau, mu, sigma, fmsk, fprj on one grid         */
  orc_spline1d spline;   /* TABLE7 */
  orc_interp2d grid;     /* TABLE7 */
  double sigma;          /* TABLE7 kernel width */
  double offset;         /* TABLE7 mu offset */
} orc_tables;

/* Policy for classifying regions as finished. */
enum {
  ORC_POLICY_REFERENCE = 0, /* err_r <= max(epsrel |avg_r|, epsabs)
                               (GPUQuadPhases.cu:63-74)                    */
  ORC_POLICY_GLOBAL = 1     /* err_r <= max(epsrel |I|, epsabs) * vol_r    */
};

typedef struct orc_integrand {
  int family;
  int ndim;
  double a[ORC_MAXDIM];
  double u[ORC_MAXDIM];
  /* integration box [box_lo, box_hi] when has_box, else the unit cube
   * (the reference's Volume, GPUQuadVolume.cu:4-25, here in FP64) */
  int has_box;
  double box_lo[ORC_MAXDIM];
  double box_hi[ORC_MAXDIM];
  const orc_tables* tables;  /* ORC_LCLT, ORC_TABLE7 */
} orc_integrand;

typedef struct orc_rule orc_rule;

typedef struct orc_result {
  double avg;
  double err;
  int axis;             /* split axis from the fourth divided difference  */
  double axis_margin;   /* relative gap between the best and second-best
                           fourth difference; 0 on an exact tie           */
  double mag;           /* jac * sum_k |w_k0| sum_p |f_p|: the scale of the
                           rounding error of avg (cancellation-aware)     */
} orc_result;

typedef struct orc_out {
  double value;
  double error;
  size_t nregions;
  size_t neval;
  int status;           /* reference errorFlag (GPUquad.h:713)             */
  int phase1_iters;
  size_t phase2_regions; /* leftover regions handed to phase 2            */
  size_t phase2_failed;
} orc_out;

/* ---- tables ---- */
int orc_table_cell(const double* xs, int n, double t);
double orc_interp2d_eval(const orc_interp2d* t, double x, double y);
double orc_spline_eval(const orc_spline1d* s, double t);
/* Natural cubic spline second derivatives (tridiagonal solve). */
void orc_spline_second_derivs(int n, const double* xs, const double* ys, double* y2);

/* ---- rule (GPUQuadRule.cu:31-390) ---- */
orc_rule* orc_rule_new(int ndim);
void orc_rule_free(orc_rule* r);
int orc_rule_ndim(const orc_rule* r);
int orc_rule_npoints(const orc_rule* r);
/* gen[9*ndim], wt[45], scale[45], norm[45], count[9] */
void orc_rule_tables(const orc_rule* r, double* gen, double* wt, double* scale,
                     double* norm, int* count);
/* g[npts*ndim] point offsets, set[npts] generator set of each point */
void orc_rule_points(const orc_rule* r, double* g, int* set);
int orc_npoints_formula(int ndim);

/* ---- integrands ---- */
double orc_eval_integrand(const orc_integrand* f, const double* x);
double orc_exact(const orc_integrand* f);

/* ---- one region (GPUQuadSample.cu:35-220) ----
 * Box [L, L+W] (global coordinates) with the region's local bounds
 * [llo, lhi] inside it and bisection depth div; phase 1 uses llo=0, lhi=1,
 * div=0.  llo/lhi may be NULL for the unit local box. */
void orc_eval_region(const orc_rule* r, const orc_integrand* f,
                     const double* L, const double* W, const double* llo,
                     const double* lhi, int div, orc_result* out);

/* ---- phase-1 rule + classify over an SoA list (GPUQuadPhases.cu:38-79) ----
 * lo/len are [ndim][n]; outputs avg/err/axis/active are [n].  margin (may
 * be NULL) receives axis_margin; ratio (may be NULL) receives
 * err / max(epsrel |avg|, epsabs). */
void orc_phase1_eval(const orc_rule* r, const orc_integrand* f, size_t n,
                     const double* lo, const double* len, double epsrel,
                     double epsabs, double* avg, double* err, int* axis,
                     int* active, double* margin, double* ratio, double* mag,
                     int nthreads);

/* ---- scan + compact + bisect (GPUKernelquad.cu:63-149,357-505) ----
 * Children are written [ndim][2m]: child 0 of the j-th active region at
 * column j, child 1 at column m+j.  Returns 2m. */
size_t orc_split(int ndim, size_t n, const double* lo, const double* len,
                 const int* active, const int* axis, double* out_lo,
                 double* out_len);

/* ---- the initial grid (GPUKernelquad.cu:24-61,272-354) ----
 * Writes d^ndim regions [ndim][count]; returns count.  If lo is NULL only
 * the count is returned. */
size_t orc_initial_grid(int ndim, double* lo, double* len);
/* The same grid laid over f's box (the unit cube when f has none). */
size_t orc_initial_grid_box(const orc_integrand* f, double* lo, double* len);

/* ---- phase 2 for one leftover box (GPUQuadPhases.cu:424-536), exact
 * max-error selection.  Returns the region count of the box. */
int orc_phase2_box(const orc_rule* r, const orc_integrand* f, const double* L,
                   const double* W, double epsrel, double epsabs,
                   int max_regions, double* result, double* error,
                   int* failed);

/* ---- full two-phase integration (GPUquad.h:611-727) ---- */
/* The second phase restricted to share `rank` of `world` of the leftover
 * boxes (GPUKernelquad.cu:759-768); see cuhre_oracle.c. */
int orc_integrate_reference_shard(const orc_rule* r, const orc_integrand* f, double epsrel,
                                  double epsabs, int phase1_cap, int phase2_max, int nthreads,
                                  int rank, int world, orc_out* p1, orc_out* part);
void orc_combine_shards(const orc_out* p1, const orc_out* parts, int world, double epsrel,
                        double epsabs, orc_out* out);
int orc_integrate_reference(const orc_rule* r, const orc_integrand* f,
                            double epsrel, double epsabs, int phase1_cap,
                            int phase2_max, int nthreads, orc_out* out);

/* ---- breadth-first integration with the global-budget policy ---- */
int orc_integrate_global(const orc_rule* r, const orc_integrand* f,
                         double epsrel, double epsabs, size_t max_regions,
                         int max_iters, int nthreads, orc_out* out);

/* ---- sequential global-heap Cuhre (Berntsen-Espelid-Genz / Hahn Cuhre,
 * same rule and the same error refinement as GPUQuadPhases.cu:498-515) */
int orc_cuhre_sequential(const orc_rule* r, const orc_integrand* f,
                         double epsrel, double epsabs, size_t max_regions,
                         orc_out* out);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
