/*
 * cubature.h -- C ABI of the B200 adaptive cubature engine.
 *
 * The reference engine (marcpaterno/old-gpuintegration) is a header-only
 * C++ template, quad::GPUcuhre<T>, with one entry point:
 *
 *   GPUcuhre(int argc, char** argv, int dim, int key = 0, int verbose = 0,
 *            int numDevices = 1)                     quad/GPUquad/GPUquad.h:46-63
 *   template <class F> int integrate(T epsrel, T epsabs, T& integral,
 *            T& error, size_t& nregions, size_t& neval, F* f,
 *            Volume* vol = NULL)                      quad/GPUquad/GPUquad.h:611-727
 *
 * This ABI is what a foreign-language binding of that path binds: plain
 * pointers and sizes, no C++ or torch types.  Built-in integrand families
 * are selected by id with a parameter block (arbitrary device functors go
 * through the C++ template front end, include/cubature/gpucuhre.cuh).
 *
 * Error handling: every function returns an int; negative values are API or
 * CUDA errors (message in cub_last_error()), positive values are numerical
 * statuses.  Nothing calls exit(), resets a device or uses device malloc.
 *
 * Threading: one cub_ctx per host thread (a context owns its stream and
 * its device pools); distinct contexts may be used concurrently.
 */
#ifndef CUBATURE_H
#define CUBATURE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUB_MAXDIM 16
#define CUB_MIN_NDIM 2
#define CUB_MAX_NDIM 8 /* dimensions instantiated in the prebuilt library */

/* Integrand families (Genz test families + the reference driver's own). */
enum cub_family {
  CUB_GAUSSIAN = 1,      /* exp(-sum a_i^2 (x_i-u_i)^2)                    */
  CUB_OSCILLATORY = 2,   /* cos(2 pi u_0 + sum a_i x_i)                    */
  CUB_CORNER_PEAK = 3,   /* (1 + sum a_i x_i)^-(n+1)                       */
  CUB_PRODUCT_PEAK = 4,  /* prod 1/(a_i^-2 + (x_i-u_i)^2)                  */
  CUB_CONTINUOUS = 5,    /* exp(-sum a_i |x_i-u_i|)                        */
  CUB_DISCONTINUOUS = 6, /* 0 if x_0>u_0 or x_1>u_1, else exp(sum a_i x_i) */
  CUB_COSSUM = 7         /* -sum cos(10 x_i)/0.054402111088937/2
                            (reference cudaCuhre.cu:9-23)                  */
};

/* Region classification / phase structure. */
enum cub_policy {
  /* The reference's two phases: breadth-first until 2^14 children or 100
   * iterations, then each leftover box refined depth-first with its own
   * tolerance and at most 2048 bisections (GPUKernelquad.cu:609-911). */
  CUB_POLICY_REFERENCE = 0,
  /* Breadth-first only, with the reference's per-region classification,
   * until convergence or the region capacity. */
  CUB_POLICY_BREADTH = 1
};

/* Result status values (cub_result.status). */
#define CUB_STATUS_OK 0 /* converged (reference errorFlag == 0)         */
/* > 0: not converged; for the reference policy the number of failed
 * phase-2 boxes (GPUKernelquad.cu:891,910), for the breadth policy 1.  */
/* The integrand returned a NaN or an infinite value: the integral stopped
 * at the iteration whose sums met it (value and error are those sums).
 * The reference does not detect this (a NaN region error fails no test
 * there, GPUQuadPhases.cu:63-74, and its value enters the sum).          */
#define CUB_STATUS_NONFINITE (1 << 30)

/* Error codes (negative return values). */
#define CUB_ERR_INVALID -1
#define CUB_ERR_CUDA -2
#define CUB_ERR_CAPACITY -3
#define CUB_ERR_UNSUPPORTED -4
#define CUB_ERR_TIMEOUT -5 /* a bounded device-side wait gave up          */

typedef struct cub_ctx cub_ctx;

typedef struct cub_genz_params {
  double a[CUB_MAXDIM]; /* per-axis parameters a_i */
  double u[CUB_MAXDIM]; /* per-axis offsets u_i    */
} cub_genz_params;

typedef struct cub_result {
  double value;                 /* integral estimate                       */
  double error;                 /* error estimate                          */
  unsigned long long nregions;  /* regions evaluated (GPUKernelquad.cu:558,884) */
  unsigned long long neval;     /* integrand evaluations (:559,887-888)    */
  int status;                   /* CUB_STATUS_OK or > 0                    */
  int iterations;               /* breadth-first iterations                */
  int state;                    /* 1 done, 3 stopped at capacity           */
  int reserved;
} cub_result;

typedef struct cub_options {
  int policy;              /* enum cub_policy                              */
  int phase1_cap;          /* children that end phase 1 (default 16384)    */
  int max_iters;           /* breadth-first iteration limit (default 100)  */
  int phase2_max_regions;  /* bisections per leftover box (default 2048)   */
  long long max_slots;     /* region-list capacity; 0 (default) = the
                              slots that fit in 40% of free device memory */
  int lanes;               /* lanes per region in the multi-launch rule
                              kernel (1, 8 or 32); 0 = automatic          */
  int no_persistent;       /* 1: never use the persistent kernel           */
  int persistent_max_n;    /* list length above which the persistent
                              kernel hands over to one launch per step;
                              0 = automatic                               */
  int persistent_max_r;    /* most regions a block of the persistent kernel
                              evaluates at once (1, 2, 4 or 8; a region
                              gets 256/R threads); 0 = 8                  */
  int no_replicated;       /* 1: batches of at most 32 integrals on short
                              lists use the persistent kernel instead of
                              the replicated-decision kernel (same
                              results, bit for bit)                       */
  long long barrier_spins; /* polls of a device-side grid barrier before
                              it gives up (CUB_ERR_TIMEOUT); 0 = default
                              (a few seconds)                             */
  int test_hold_block;     /* failure-detection tests only: b + 1 keeps
                              block b of the persistent kernels from
                              arriving at their grid barriers, so every
                              wait runs out; 0 = off                      */
  int no_device_loop;      /* 1: the host launches each iteration on long
                              lists instead of one graph launch with a
                              conditional loop running them (same results,
                              bit for bit)                                */
} cub_options;

/* Library version, (major << 16) | minor. */
int cub_version(void);

/* Message of the last error on this host thread ("" if none). */
const char* cub_last_error(void);

/* Fill *opt with the reference's defaults. */
void cub_default_options(cub_options* opt);

/* Context on a CUDA device: owns a stream and device pools, grown on demand
 * and reused across calls.  Replaces the GPUcuhre constructor
 * (GPUquad.h:46-63), which resets every visible device and parses argv.
 * Returns NULL on failure. */
cub_ctx* cub_create(int device);
void cub_destroy(cub_ctx* ctx);

/* Device bytes currently held by the context's pools. */
size_t cub_ctx_bytes(const cub_ctx* ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events against the engine's. */
void* cub_ctx_stream(cub_ctx* ctx);

/* Counters of the work a context launched since the last reset.  With
 * timing on, CUDA events bracket every rule-kernel and phase-2 launch and
 * their device times are summed (adds one event pair per launch). */
typedef struct cub_stats {
  double ms_eval;             /* device time of the multi-launch rule kernel
                                 (timing on)                                */
  double ms_phase2;           /* device time of the phase-2 kernel          */
  long long eval_launches;    /* rule-kernel launches                       */
  long long launches;         /* all kernel launches                        */
  long long regions_evaluated;/* regions through the rule kernel           */
  long long iterations;       /* breadth-first iterations                   */
  long long phase2_boxes;     /* leftover boxes refined depth-first         */
  long long h2d_bytes;        /* host-to-device bytes copied                */
  long long d2h_bytes;        /* device-to-host bytes copied                */
  double ms_persistent;       /* device time of the persistent kernel       */
  long long persistent_launches;
  long long persistent_iterations; /* iterations run inside it          */
  long long replicated_launches; /* of those, launches of the replicated-
                                    decision kernel (small batches)     */
  long long persistent_regions;  /* regions evaluated by both persistent
                                    kernels                             */
  long long device_loops;        /* launches of the device-driven loop of
                                    long-list iterations                */
} cub_stats;

int cub_ctx_stats(const cub_ctx* ctx, cub_stats* out);
void cub_ctx_reset_stats(cub_ctx* ctx);

/* Return the context's device pools to the driver (the next call reserves
 * what it needs again). */
void cub_ctx_release(cub_ctx* ctx);

/* Diagnostics: device timestamps (ns, %globaltimer) of the first 8
 * iterations of the last persistent-kernel launch on this context, 8 per
 * iteration: 0 start, 1 next list assigned, 2 grid barrier passed,
 * 3 deciding warp read its integral state, 4 block 0's evaluations done,
 * 5 last chunk summed, 6 integrals decided, 7 chunk sums combined (3, 6
 * and 7 for batches of up to 32 integrals); zero where not reached.  out
 * must hold 64 values. */
int cub_ctx_trace(const cub_ctx* ctx, unsigned long long* out);
void cub_ctx_set_timing(cub_ctx* ctx, int on);

/* One integral over [0,1]^ndim: the body of GPUcuhre::integrate
 * (GPUquad.h:611-727) for a built-in family.  Unlike the reference, results
 * are written (not accumulated with +=) into *out.  Returns 0, or a
 * negative error code; the numerical status is out->status. */
int cub_integrate(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                  double epsrel, double epsabs, const cub_options* opt, cub_result* out);

/* `count` independent integrals of one family and dimension, integrated
 * together (one shared region list).  params/epsrel/epsabs/out have
 * `count` entries; epsrel/epsabs may be NULL to use epsrel0/epsabs0.  The
 * reference has no batched form; it would loop over integrate(). */
int cub_integrate_batch(cub_ctx* ctx, int family, int ndim, int count,
                        const cub_genz_params* params, const double* epsrel,
                        const double* epsabs, double epsrel0, double epsabs0,
                        const cub_options* opt, cub_result* out);

/* `count` integrals of possibly different families (families[k]) and one
 * dimension, integrated together on one region list -- e.g. the 8-D
 * oscillatory and corner peak in one persistent launch.  Results are those
 * of cub_integrate_batch per family (the same arithmetic). */
int cub_integrate_mixed_batch(cub_ctx* ctx, int ndim, int count, const int* families,
                              const cub_genz_params* params, const double* epsrel,
                              const double* epsabs, double epsrel0, double epsabs0,
                              const cub_options* opt, cub_result* out);

/* One integral with its second phase split over `world` processes (the
 * reference's multi-device path, GPUquad.h:430-609 and
 * GPUKernelquad.cu:729-906).  Every caller runs the same first phase (it is
 * deterministic, so all agree on the leftover boxes without exchanging
 * them) and refines share `rank` of the leftover boxes: world contiguous
 * parts of the leftover list, the last taking the remainder
 * (GPUKernelquad.cu:759-768).  *phase1 receives the first phase's result
 * (its finished sums, regions and evaluations; the whole result when no box
 * was left, with *part zeroed); *part the share's value and error sums,
 * regions, evaluations, and its failed boxes in `status` (or
 * CUB_STATUS_NONFINITE).  The combined result is phase1 plus the sum of all
 * parts, with status = the summed failed boxes unless
 * error <= max(epsrel |value|, epsabs) (GPUquad.h:713); the Python binding
 * does that with one all-reduce (cubature.parallel.integrate_split). */
int cub_integrate_shard(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                        double epsrel, double epsabs, const cub_options* opt, int rank,
                        int world, cub_result* phase1, cub_result* part);

/* cub_integrate over the box [lo, hi] (ndim values each, host memory,
 * finite, hi > lo) instead of the unit cube: the reference's Volume
 * argument (GPUQuadVolume.cu:4-25, GPUQuadSample.cu:44-56,174-179), here in
 * FP64.  The initial grid is laid over the box, so every region is held in
 * the integrand's own coordinates. */
int cub_integrate_box(cub_ctx* ctx, int family, int ndim, const cub_genz_params* params,
                      const double* lo, const double* hi, double epsrel, double epsabs,
                      const cub_options* opt, cub_result* out);

/* cub_integrate_batch with a box per integral: lo and hi are [count][ndim]
 * host arrays. */
int cub_integrate_batch_box(cub_ctx* ctx, int family, int ndim, int count,
                            const cub_genz_params* params, const double* lo, const double* hi,
                            const double* epsrel, const double* epsabs, double epsrel0,
                            double epsabs0, const cub_options* opt, cub_result* out);

/* Autotuner: integrate the batch (or its first `sample` integrals when
 * sample > 0) with each candidate tiling -- regions per block of the
 * persistent kernel (persistent_max_r 1, 2, 4, 8), lanes per region of the
 * multi-launch rule kernel (1, 8, 32), the persistent kernel on or off and
 * its hand-over length -- starting from *opt (or the defaults), and write
 * the fastest to *best; *best_ms receives its time (may be NULL).  Each
 * candidate runs twice and keeps the faster run. */
int cub_autotune_batch(cub_ctx* ctx, int family, int ndim, int count,
                       const cub_genz_params* params, double epsrel, double epsabs, int sample,
                       const cub_options* opt, cub_options* best, double* best_ms);

/* ---- replayable batches (CUDA graph) ---------------------------------- */

/* Repeated integrations of the same shape -- the same families,
 * dimensions and counts, new parameters and tolerances each call -- as one
 * captured CUDA graph.  Entry i is a batch of counts[i] integrals of
 * families[i] in ndims[i] dimensions over the unit cube.  The graph records
 * per entry the parameter and state uploads, one cooperative persistent
 * launch (initial grid and every breadth-first iteration while the list
 * stays within the persistent kernel's limit) and the state download; each
 * entry has its own region lists, so the recorded pointers never change.
 * The initial grid of each entry must fit the persistent limit
 * (CUB_ERR_UNSUPPORTED otherwise).  No counterpart in the reference: its
 * integrate (GPUquad.h:611-727) drives every iteration from the host,
 * with device-to-host copies in between (GPUKernelquad.cu:565-598). */
typedef struct cub_graph cub_graph;

int cub_graph_create(cub_ctx* ctx, int nentries, const int* families, const int* ndims,
                     const int* counts, const cub_options* opt, cub_graph** out);

/* One replay: params, epsrel, epsabs and out hold every entry's integrals
 * in entry order (sum of counts).  Parameters and starting states are
 * written to pinned buffers, the graph is launched on the context's stream
 * and waited for once.  An entry that the launch did not finish (its list
 * outgrew the persistent limit, or boxes went to phase 2) is integrated
 * again by cub_integrate_batch, so every result equals that call's.
 * Returns 0, CUB_ERR_CAPACITY (as cub_integrate_batch) or an error. */
int cub_graph_launch(cub_graph* g, const cub_genz_params* params, const double* epsrel,
                     const double* epsabs, cub_result* out);

/* Replays so far, and entries that needed cub_integrate_batch after one. */
int cub_graph_info(const cub_graph* g, long long* replays, long long* reruns);

/* Free the graph and its buffers; call it before cub_destroy of its context. */
void cub_graph_destroy(cub_graph* g);

/* ---- integrands on device tables ------------------------------------- */

/* Rectilinear 2-D table in device memory, row-major zs[i * ny + j] at
 * (xs[i], ys[j]), knots ascending, nx, ny >= 2: the reference's Interp2D
 * (GPUQuadInterp2D.cu:50-106), evaluated in FP64 with a binary search for
 * the cell (the reference reads FP32 textures and searches linearly).
 * Points outside the knots extrapolate linearly from the end cells. */
typedef struct cub_interp2d {
  const double* xs;
  const double* ys;
  const double* zs;
  int nx, ny;
} cub_interp2d;

/* Natural cubic spline in device memory: knots xs (ascending), values ys,
 * second derivatives y2 (cub_spline_second_derivatives), n >= 2. */
typedef struct cub_spline1d {
  const double* xs;
  const double* ys;
  const double* y2;
  int n;
} cub_spline1d;

/* The five tables of the LC_LT integrand (tau, mu, sigma, fmsk, fprj) over
 * (lt, zt); all five share xs, ys, nx, ny of the first. */
typedef struct cub_lclt_tables {
  cub_interp2d t[5];
} cub_lclt_tables;

/* The 7-D table integrand: spline(x0) * bilinear(x1, x2) *
 * exp(-(4 x3 - mu)^2 / (2 sigma^2)), mu = offset + 2 x4 + 0.1 (x5 + x6). */
typedef struct cub_table7 {
  cub_spline1d spline;
  cub_interp2d grid;
  double sigma;
} cub_table7;

/* Natural cubic spline second derivatives for n knots (host memory). */
int cub_spline_second_derivatives(int n, const double* xs, const double* ys, double* y2);

/* The reference's LC_LT integrand (lc_lt_t.h:18-52) over the box [lo, hi]
 * in (lt, zt, lc), in FP64; tables in device memory, owned by the caller. */
int cub_integrate_lclt(cub_ctx* ctx, const cub_lclt_tables* tables, const double* lo,
                       const double* hi, double epsrel, double epsabs, const cub_options* opt,
                       cub_result* out);

/* `count` integrals of the 7-D table integrand over [0,1]^7, one mu offset
 * each (host array), on one shared region list.  epsrel/epsabs as in
 * cub_integrate_batch. */
int cub_integrate_table7_batch(cub_ctx* ctx, const cub_table7* tables, int count,
                               const double* offsets, const double* epsrel, const double* epsabs,
                               double epsrel0, double epsabs0, const cub_options* opt,
                               cub_result* out);

/* ---- control-variate network (BF16 tensor cores, tcgen05) ------------ */

/* D[e] = A[e] * B[e]^T on the tensor cores for e < batch: A is m x k, B is
 * n x k, both bf16 and K-major (row-major with leading dimensions lda, ldb,
 * multiples of 8), D is m x n fp32 (ldd); FP32 accumulation.  m a multiple
 * of 128, k of 16, n = 16 or 128.  Device pointers; consecutive batch
 * entries are lda * m, ldb * n and ldd * m elements apart.  The building
 * block of the network's training and inference; no counterpart in the
 * reference. */
int cub_mlp_gemm_bf16(int batch, int m, int n, int k, const void* d_a, long long lda,
                      const void* d_b, long long ldb, float* d_d, long long ldd, void* stream);

/* The control-variate networks: `count` independent MLPs g: [0,1]^7 -> R,
 * 7 -> 128 -> 128 -> 128 -> 1 with SiLU, BF16 weights and activations,
 * FP32 accumulation on the tensor cores, FP32 master parameters and Adam.
 * Each network has `samples` training points (a multiple of `batch`, itself
 * a multiple of 128).  Parameters are initialised from `seed`.  No
 * counterpart in the reference. */
#define CUB_MLP_PARAMS 35336 /* fp32 parameters per network (with padding) */
typedef struct cub_mlp cub_mlp;
cub_mlp* cub_mlp_create(int device, int count, int samples, int batch, unsigned long long seed);
void cub_mlp_destroy(cub_mlp* m);
/* Training data on the device: x [count][samples][7] in [0,1] and
 * y [count][samples] (fp64).  Targets are scaled by 1 / max|y| per network;
 * inputs are mapped to 2 x - 1. */
int cub_mlp_set_data(cub_mlp* m, const double* d_x, const double* d_y);
/* Host copy of the parameters [count][CUB_MLP_PARAMS]: read (set = 0) or
 * write (set = 1). */
int cub_mlp_params(cub_mlp* m, float* h_params, int set);
/* Forward and backward pass of minibatch b without an update: loss
 * [count] (mean squared error of the scaled targets) and gradients
 * [count][CUB_MLP_PARAMS] (host; either may be NULL). */
int cub_mlp_grad(cub_mlp* m, int b, float* h_loss, float* h_grads);
/* `epochs` passes of Adam over the data; loss [count] of the last
 * minibatch (host, may be NULL). */
int cub_mlp_train(cub_mlp* m, int epochs, float lr, float* h_loss);
/* g at n points per network: d_x [count][n][7] in [0,1] -> d_g [count][n]
 * (device, fp64, in the units of the targets). */
int cub_mlp_eval(cub_mlp* m, long long n, const double* d_x, double* d_g);

/* Learned control variate (7-D): for each integral, a coarse plain run
 * (epsrel coarse_epsrel; it checks the result), a network trained on f at `samples`
 * rule nodes of the initial grid, then the integral of (f - g) and of g,
 * each adaptively to half the absolute tolerance max(epsrel |I|, epsabs).
 * The plain method takes over for an integral whose training residual
 * |f - g| / |f| exceeds rho_max, or whose control-variate result is not
 * converged or disagrees with the coarse run beyond three times their
 * error estimates.  Breadth-first refinement throughout.  No counterpart in
 * the reference. */
typedef struct cub_cv_options {
  int samples;           /* training points per integral (default 8192) */
  int batch;             /* minibatch (default 1024)                     */
  int epochs;            /* Adam epochs (default 30)                     */
  float lr;              /* Adam step (default 2e-3)                     */
  double rho_max;        /* residual ratio above which the plain method
                            runs instead (default 0.5)                   */
  double coarse_epsrel;  /* tolerance of the judging plain run (1e-3)    */
  unsigned long long seed;
} cub_cv_options;

typedef struct cub_cv_stats {
  double ms_coarse, ms_train, ms_integrate;  /* wall time of the stages   */
  int fallbacks;          /* integrals done by the plain method          */
  int rejected;           /* of which the check rejected the CV result   */
  double mean_residual_ratio;
  unsigned long long regions_residual;  /* regions of the (f - g) runs  */
  unsigned long long regions_network;   /* regions of the g runs        */
} cub_cv_stats;

void cub_cv_default_options(cub_cv_options* opt);
int cub_cv_integrate_batch(cub_ctx* ctx, int family, int count, const cub_genz_params* params,
                           double epsrel, double epsabs, const cub_cv_options* opt,
                           cub_result* out, cub_cv_stats* stats);

/* ---- per-step entry points on caller device buffers ------------------ */

/* Rule tables of the degree-9 rule for ndim (GPUQuadRule.cu:31-228):
 * wt/scale/norm are [9][5], count is [9].  Host memory; any may be NULL. */
int cub_rule_tables(int ndim, double* wt, double* scale, double* norm, int* count);

/* Phase-1 rule + classification over an SoA region list
 * (INTEGRATE_GPU_PHASE1, GPUQuadPhases.cu:38-79).  Regions are
 * [lo, lo+len], lo/len laid out [ndim][ld] on the device.  Writes per
 * region: avg, err, split axis, active (err > max(epsrel|avg|, epsabs)).
 * params is host memory.  stream may be NULL (default stream). */
int cub_rule_eval(int family, int ndim, const cub_genz_params* params, long long n,
                  const double* d_lo, const double* d_len, long long ld, double epsrel,
                  double epsabs, double* d_avg, double* d_err, int* d_axis, int* d_active,
                  void* stream);

/* Scratch bytes cub_split / cub_reduce need for n regions. */
size_t cub_split_scratch_bytes(long long n);
size_t cub_reduce_scratch_bytes(long long n);

/* Scan + compact + bisect (GenerateActiveIntervals, alignRegions,
 * divideIntervalsGPU; GPUKernelquad.cu:63-149,357-505).  Every region with
 * active == 1 yields two children halved on its axis, written [ndim][out_ld]:
 * layout 0 = the reference's (child 0 of the j-th active region at column j,
 * child 1 at column m+j); layout 1 = adjacent (2j, 2j+1).  The number of
 * children 2m is written to *d_count (device).  d_scratch must hold
 * cub_split_scratch_bytes(n); out_ld must be >= 2m. */
int cub_split(int ndim, long long n, const double* d_lo, const double* d_len, long long ld,
              const int* d_active, const int* d_axis, double* d_out_lo, double* d_out_len,
              long long out_ld, int layout, long long* d_count, void* d_scratch,
              size_t scratch_bytes, void* stream);

/* cub_split for callers that cannot allocate device memory at call time
 * (their memory belongs to another allocator, or a cudaMalloc/cudaFree --
 * which can synchronise the device -- is not allowed on their path).  It
 * allocates nothing: its scratch is a fixed 1 MiB device array in the
 * library, so n is limited to 2^22 regions (larger n returns
 * CUB_ERR_INVALID).  The array is shared by every call on a device: calls
 * that overlap on the GPU race and must be serialised.  The first call on
 * each device looks up the array's address; make it before any stream
 * capture.  The address is kept for the process's lifetime: after a
 * cudaDeviceReset of that device, the next call would use a stale address,
 * so do not reset a device between calls.  Same arguments and results as
 * cub_split, minus the scratch.  No counterpart in the reference. */
int cub_split_noalloc(int ndim, long long n, const double* d_lo, const double* d_len,
                      long long ld, const int* d_active, const int* d_axis, double* d_out_lo,
                      double* d_out_len, long long out_ld, int layout, long long* d_count,
                      void* stream);

/* The four sums of a phase-1 iteration (GPUKernelquad.cu:565-577):
 * d_out[0] = sum avg, [1] = sum err, [2] = sum avg over active == 0,
 * [3] = sum err over active == 0.  Device output; fixed-order tree. */
int cub_reduce(long long n, const double* d_avg, const double* d_err, const int* d_active,
               double* d_out, void* d_scratch, size_t scratch_bytes, void* stream);

/* Measured FP64 throughput of the CUDA cores of `device` (DFMA loop,
 * TFLOP/s, FMA = 2 flops) into *tflops: the roofline denominator of the
 * rule kernels, whose FP64 work is DFMA/DMUL/DADD on the CUDA cores.  A
 * measurement utility with no counterpart in the reference; it launches on
 * the device's legacy default stream and waits for it. */
int cub_fp64_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* CUBATURE_H */
