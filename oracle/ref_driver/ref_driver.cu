// ref_driver.cu -- runs the reference engine (quad::GPUcuhre, compiled from
// the reference's own headers) on Genz integrands and prints its outputs,
// to produce golden vectors for the tests.  Test infrastructure only.
//
//   ref_driver integrate <family> <ndim> <epsrel> <epsabs> a_0..a_{n-1} u_0..u_{n-1}
//       -> "RESULT {json}" with integral, error, nregions, neval, errorFlag, ms
//   ref_driver interp2d <tables.bin> <out.bin>
//       quad::Interp2D (GPUQuadInterp2D.cu:50-106) at query points
//   ref_driver lclt <tables.bin> <epsrel> <epsabs> lo.. hi..
//       LC_LT (lc_lt_t.h:18-52) on quad::Interp2D tables, integrated
//   ref_driver bench <family> <ndim> <epsrel> <epsabs> <warmup> <reps> a.. u..
//       -> "BENCH {json}": warm median ms per integrate call on one object
//   ref_driver phase1 <family> <ndim> <epsrel> <epsabs> <in.bin> <out.bin> a.. u..
//       runs INTEGRATE_GPU_PHASE1 (GPUQuadPhases.cu:38-79) on the region list
//       in in.bin ([int64 n][n*ndim lo][n*ndim len], dimension-major) and
//       writes [n avg][n err][n int32 active][n int32 axis] to out.bin.
//
// The integration volume is always the unit cube (vol = NULL): the
// reference's Volume path skips the volume map for the middle sample pass
// (GPUQuadSample.cu:174-179) and reads bounds through float textures.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "quad/GPUquad/GPUquad.h"
#include "quad/GPUquad/GPUQuadInterp2D.cu"

struct GenzRef {
  int family;
  int ndim;
  double a[8];
  double u[8];

  __device__ double operator()(double x[], int dim) {
    double s = 0, p = 1;
    switch (family) {
      case 1:  // Gaussian
        for (int i = 0; i < dim; ++i) {
          const double t = a[i] * (x[i] - u[i]);
          s += t * t;
        }
        return exp(-s);
      case 2:  // oscillatory
        s = 2 * M_PI * u[0];
        for (int i = 0; i < dim; ++i) s += a[i] * x[i];
        return cos(s);
      case 3:  // corner peak
        s = 1;
        for (int i = 0; i < dim; ++i) s += a[i] * x[i];
        for (int k = 0; k <= dim; ++k) p *= s;
        return 1 / p;
      case 4:  // product peak
        for (int i = 0; i < dim; ++i) {
          const double t = x[i] - u[i];
          p *= 1 / (1 / (a[i] * a[i]) + t * t);
        }
        return p;
      case 5:  // continuous
        for (int i = 0; i < dim; ++i) s += a[i] * fabs(x[i] - u[i]);
        return exp(-s);
      case 6:  // discontinuous
        if (x[0] > u[0] || (dim > 1 && x[1] > u[1])) return 0;
        for (int i = 0; i < dim; ++i) s += a[i] * x[i];
        return exp(s);
      case 7:  // the reference driver's own integrand (cudaCuhre.cu:11-22)
        for (int i = 0; i < dim; ++i) s = s - cos(10.0 * x[i]) / 0.054402111088937;
        return s / 2.0;
    }
    return 0;
  }
};

// The reference's LC_LT integrand (lc_lt_t.h:18-52, with gaussian and
// erfc_scaled as in CuhreInteface.h:19-31) on five quad::Interp2D tables
// over (lt, zt), restated here because lc_lt_t.h pulls in GSL headers.  The
// engine integrates over the unit cube (vol = NULL), so the functor maps x
// to the box [lo, hi] and carries its volume: its integral is that of
// LC_LT over the box.
struct LcLtRef {
  quad::Interp2D tau_interp, mu_interp, sigma_interp, fmsk_interp, fprj_interp;
  double lo[3], width[3], volume;

  __device__ double operator()(double xx[], int) {
    const double lt = lo[0] + xx[0] * width[0];
    const double zt = lo[1] + xx[1] * width[1];
    const double lc = lo[2] + xx[2] * width[2];
    const float tau = tau_interp(lt, zt);
    const float mu = mu_interp(lt, zt);
    const float sigma = sigma_interp(lt, zt);
    const float fmsk = fmsk_interp(lt, zt);
    const float fprj = fprj_interp(lt, zt);
    const double exptau = exp(tau * (2.0 * mu + tau * sigma * sigma - 2.0 * lc) / 2.0);
    const double root_two_sigma = sqrt(2.0) * sigma;
    const double mu_tau_sig_sqr = mu + tau * sigma * sigma;
    const double z = (lc - mu) / sigma;
    const double gauss = exp(-z * z / 2.) * 0.3989422804014327 / sigma;
    const double f =
        (1.0 - fmsk) * (1.0 - fprj) * gauss +
        0.5 * ((1.0 - fmsk) * fprj * tau + fmsk * fprj / lt) * exptau *
            erfc((mu_tau_sig_sqr - lc) / root_two_sigma) +
        0.5 * fmsk / lt *
            (erfc((lc - mu) / root_two_sigma) - erfc((lc + lt - mu) / root_two_sigma)) -
        0.5 * fmsk * fprj / lt *
            (exp(-tau * lt) * exptau * erfc((mu_tau_sig_sqr - lc - lt) / root_two_sigma));
    return f * volume;
  }
};

// Table file: [int32 rows][int32 cols][int32 ntables][rows float xs]
// [cols float ys][ntables x rows*cols float z, row-major: z[i*cols+j] at
// (xs[i], ys[j])].  quad::Interp2D reads its values through a rows-wide
// texture, so value (i, j) sits at j*rows + i (allocText,
// cudaMemoryUtil.h:5-30): the tables are transposed on load.
struct TableFile {
  int rows = 0, cols = 0, ntab = 0;
  std::vector<float> xs, ys;
  std::vector<std::vector<float>> z;  // texture layout
};

static bool read_tables(FILE* in, TableFile& t) {
  int hdr[3];
  if (std::fread(hdr, sizeof(int), 3, in) != 3) return false;
  t.rows = hdr[0];
  t.cols = hdr[1];
  t.ntab = hdr[2];
  if (t.rows < 2 || t.cols < 2 || t.ntab < 1 || t.ntab > 8) return false;
  t.xs.resize(t.rows);
  t.ys.resize(t.cols);
  if (std::fread(t.xs.data(), sizeof(float), t.rows, in) != (size_t)t.rows ||
      std::fread(t.ys.data(), sizeof(float), t.cols, in) != (size_t)t.cols)
    return false;
  std::vector<float> rm((size_t)t.rows * t.cols);
  for (int q = 0; q < t.ntab; ++q) {
    if (std::fread(rm.data(), sizeof(float), rm.size(), in) != rm.size()) return false;
    std::vector<float> tex(rm.size());
    for (int i = 0; i < t.rows; ++i)
      for (int j = 0; j < t.cols; ++j) tex[(size_t)j * t.rows + i] = rm[(size_t)i * t.cols + j];
    t.z.push_back(tex);
  }
  return true;
}

__global__ void k_interp_points(quad::Interp2D t, const double* qx, const double* qy, int nq,
                                double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nq) out[i] = t(qx[i], qy[i]);
}

// ref_driver interp2d <in.bin> <out.bin>: quad::Interp2D (first table of
// the file) at nq query points appended to the file as [int64 nq]
// [nq double x][nq double y]; writes nq doubles (the float results).
static int run_interp2d(int argc, char** argv) {
  if (argc < 4) return 2;
  FILE* in = std::fopen(argv[2], "rb");
  if (!in) return 3;
  TableFile t;
  long long nq = 0;
  if (!read_tables(in, t) || std::fread(&nq, sizeof(nq), 1, in) != 1 || nq <= 0) return 3;
  std::vector<double> qx(nq), qy(nq), out(nq);
  if (std::fread(qx.data(), sizeof(double), nq, in) != (size_t)nq ||
      std::fread(qy.data(), sizeof(double), nq, in) != (size_t)nq)
    return 3;
  std::fclose(in);
  quad::Interp2D interp;
  interp.Initialize(t.xs.data(), t.ys.data(), t.z[0].data(), t.rows, t.cols);
  double *dx, *dy, *dout;
  cudaMalloc(&dx, sizeof(double) * nq);
  cudaMalloc(&dy, sizeof(double) * nq);
  cudaMalloc(&dout, sizeof(double) * nq);
  cudaMemcpy(dx, qx.data(), sizeof(double) * nq, cudaMemcpyHostToDevice);
  cudaMemcpy(dy, qy.data(), sizeof(double) * nq, cudaMemcpyHostToDevice);
  k_interp_points<<<(unsigned)((nq + 127) / 128), 128>>>(interp, dx, dy, (int)nq, dout);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "interp2d kernel: %s\n", cudaGetErrorString(e));
    return 4;
  }
  cudaMemcpy(out.data(), dout, sizeof(double) * nq, cudaMemcpyDeviceToHost);
  FILE* o = std::fopen(argv[3], "wb");
  if (!o) return 3;
  std::fwrite(out.data(), sizeof(double), nq, o);
  std::fclose(o);
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(dout);
  std::printf("INTERP2D %lld points\n", nq);
  return 0;
}

// ref_driver lclt <in.bin> <epsrel> <epsabs> lo0 lo1 lo2 hi0 hi1 hi2: the
// LC_LT integrand on the file's five tables (tau, mu, sigma, fmsk, fprj)
// over the box, through GPUcuhre::integrate -> "RESULT {json}".
static int run_lclt(int argc, char** argv) {
  if (argc < 11) return 2;
  FILE* in = std::fopen(argv[2], "rb");
  if (!in) return 3;
  TableFile t;
  if (!read_tables(in, t) || t.ntab != 5) return 3;
  std::fclose(in);
  const double epsrel = std::atof(argv[3]), epsabs = std::atof(argv[4]);
  LcLtRef f;
  f.volume = 1;
  for (int d = 0; d < 3; ++d) {
    f.lo[d] = std::atof(argv[5 + d]);
    f.width[d] = std::atof(argv[8 + d]) - f.lo[d];
    f.volume *= f.width[d];
  }
  char* fake[] = {argv[0], nullptr};
  quad::GPUcuhre<double> cuhre(1, fake, 3, 0, 0, 1);
  // the engine's constructor resets the device, so the tables' textures
  // are made after it
  f.tau_interp.Initialize(t.xs.data(), t.ys.data(), t.z[0].data(), t.rows, t.cols);
  f.mu_interp.Initialize(&f.tau_interp, t.z[1].data());
  f.sigma_interp.Initialize(&f.tau_interp, t.z[2].data());
  f.fmsk_interp.Initialize(&f.tau_interp, t.z[3].data());
  f.fprj_interp.Initialize(&f.tau_interp, t.z[4].data());
  double integral = 0, error = 0;
  size_t nregions = 0, neval = 0;
  cudaDeviceSynchronize();
  const int flag = cuhre.integrate(epsrel, epsabs, integral, error, nregions, neval, &f);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "lclt integrate: %s\n", cudaGetErrorString(e));
    return 4;
  }
  std::printf("RESULT {\"epsrel\": %.17g, \"epsabs\": %.17g, \"integral\": %.17g, "
              "\"error\": %.17g, \"nregions\": %zu, \"neval\": %zu, \"errorFlag\": %d}\n",
              epsrel, epsabs, integral, error, nregions, neval, flag);
  return 0;
}

static GenzRef parse_integrand(int family, int ndim, char** v) {
  GenzRef f;
  std::memset(&f, 0, sizeof(f));
  f.family = family;
  f.ndim = ndim;
  for (int i = 0; i < ndim; ++i) f.a[i] = std::atof(v[i]);
  for (int i = 0; i < ndim; ++i) f.u[i] = std::atof(v[ndim + i]);
  return f;
}

static int run_integrate(int argc, char** argv) {
  if (argc < 6) return 2;
  const int family = std::atoi(argv[2]), ndim = std::atoi(argv[3]);
  const double epsrel = std::atof(argv[4]), epsabs = std::atof(argv[5]);
  if (ndim < 2 || ndim > 8 || argc < 6 + 2 * ndim) return 2;
  GenzRef f = parse_integrand(family, ndim, argv + 6);
  char* fake[] = {argv[0], nullptr};
  quad::GPUcuhre<double> cuhre(1, fake, ndim, 0, 0, 1);
  double integral = 0, error = 0;
  size_t nregions = 0, neval = 0;
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  const int flag = cuhre.integrate(epsrel, epsabs, integral, error, nregions, neval, &f);
  cudaDeviceSynchronize();
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::printf("RESULT {\"family\": %d, \"ndim\": %d, \"epsrel\": %.17g, \"epsabs\": %.17g, "
              "\"integral\": %.17g, \"error\": %.17g, \"nregions\": %zu, \"neval\": %zu, "
              "\"errorFlag\": %d, \"ms\": %.3f}\n",
              family, ndim, epsrel, epsabs, integral, error, nregions, neval, flag, ms);
  return 0;
}

// ref_driver bench <family> <ndim> <epsrel> <epsabs> <warmup> <reps> a.. u..
// One GPUcuhre object, `warmup` untimed integrate calls, then `reps` timed
// ones (steady clock around each call, device synchronised on both sides);
// prints "BENCH {json}" with the median and minimum ms per call and the last
// call's outputs.  integrate() accumulates into its outputs
// (GPUKernelquad.cu:558-559), so each call starts from zeroed variables.
static int run_bench(int argc, char** argv) {
  if (argc < 6) return 2;
  const int family = std::atoi(argv[2]), ndim = std::atoi(argv[3]);
  const double epsrel = std::atof(argv[4]), epsabs = std::atof(argv[5]);
  if (argc < 8) return 2;
  const int warmup = std::atoi(argv[6]), reps = std::atoi(argv[7]);
  if (ndim < 2 || ndim > 8 || argc < 8 + 2 * ndim || reps < 1) return 2;
  GenzRef f = parse_integrand(family, ndim, argv + 8);
  char* fake[] = {argv[0], nullptr};
  quad::GPUcuhre<double> cuhre(1, fake, ndim, 0, 0, 1);
  double integral = 0, error = 0;
  size_t nregions = 0, neval = 0;
  int flag = 0;
  std::vector<double> ms;
  for (int i = 0; i < warmup + reps; ++i) {
    integral = error = 0;
    nregions = neval = 0;
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    flag = cuhre.integrate(epsrel, epsabs, integral, error, nregions, neval, &f);
    cudaDeviceSynchronize();
    const double t =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (i >= warmup) ms.push_back(t);
  }
  std::vector<double> sorted = ms;
  std::sort(sorted.begin(), sorted.end());
  std::printf("BENCH {\"family\": %d, \"ndim\": %d, \"epsrel\": %.17g, \"reps\": %d, "
              "\"median_ms\": %.6f, \"min_ms\": %.6f, \"integral\": %.17g, \"error\": %.17g, "
              "\"nregions\": %zu, \"neval\": %zu, \"errorFlag\": %d}\n",
              family, ndim, epsrel, reps, sorted[sorted.size() / 2], sorted[0], integral, error,
              nregions, neval, flag);
  return 0;
}

static int run_phase1(int argc, char** argv) {
  if (argc < 6) return 2;
  const int family = std::atoi(argv[2]), ndim = std::atoi(argv[3]);
  const double epsrel = std::atof(argv[4]), epsabs = std::atof(argv[5]);
  if (ndim < 2 || ndim > 8 || argc < 8 + 2 * ndim) return 2;
  FILE* in = std::fopen(argv[6], "rb");
  if (!in) return 3;
  long long n = 0;
  if (std::fread(&n, sizeof(n), 1, in) != 1 || n <= 0) return 3;
  std::vector<double> lo(n * ndim), len(n * ndim);
  if (std::fread(lo.data(), sizeof(double), lo.size(), in) != lo.size() ||
      std::fread(len.data(), sizeof(double), len.size(), in) != len.size())
    return 3;
  std::fclose(in);
  GenzRef f = parse_integrand(family, ndim, argv + 8);

  // the rule tables go to __constant__ memory here (GPUKernelquad.cu:237-257)
  quad::GPUKernelCuhre<double> kernel;
  kernel.InitGPUKernelCuhre(ndim, 0, 0, 1);
  const int fEval = 1 + 2 * ndim + 2 * ndim + 2 * ndim + 2 * ndim + 2 * ndim * (ndim - 1) +
                    4 * ndim * (ndim - 1) + 4 * ndim * (ndim - 1) * (ndim - 2) / 3 + (1 << ndim);
  double *dlo, *dlen, *dint, *derr;
  int *dact, *dax;
  GenzRef* dtest;
  cudaMalloc(&dlo, sizeof(double) * n * ndim);
  cudaMalloc(&dlen, sizeof(double) * n * ndim);
  cudaMalloc(&dint, sizeof(double) * n * 2);
  cudaMalloc(&derr, sizeof(double) * n * 2);
  cudaMalloc(&dact, sizeof(int) * n);
  cudaMalloc(&dax, sizeof(int) * n);
  cudaMalloc(&dtest, sizeof(GenzRef));
  cudaMemcpy(dlo, lo.data(), sizeof(double) * n * ndim, cudaMemcpyHostToDevice);
  cudaMemcpy(dlen, len.data(), sizeof(double) * n * ndim, cudaMemcpyHostToDevice);
  cudaMemcpy(dtest, &f, sizeof(GenzRef), cudaMemcpyHostToDevice);
  quad::INTEGRATE_GPU_PHASE1<double><<<(unsigned)n, BLOCK_SIZE>>>(
      dlo, dlen, (size_t)n, dint, derr, dact, dax, epsrel, epsabs, fEval, ndim, dtest,
      (Volume*)nullptr);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "phase1 kernel: %s\n", cudaGetErrorString(e));
    return 4;
  }
  std::vector<double> avg(n), err(n);
  std::vector<int> act(n), ax(n);
  cudaMemcpy(avg.data(), dint + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(err.data(), derr + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(act.data(), dact, sizeof(int) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(ax.data(), dax, sizeof(int) * n, cudaMemcpyDeviceToHost);
  FILE* out = std::fopen(argv[7], "wb");
  if (!out) return 3;
  std::fwrite(avg.data(), sizeof(double), n, out);
  std::fwrite(err.data(), sizeof(double), n, out);
  std::fwrite(act.data(), sizeof(int), n, out);
  std::fwrite(ax.data(), sizeof(int), n, out);
  std::fclose(out);
  cudaFree(dlo);
  cudaFree(dlen);
  cudaFree(dint);
  cudaFree(derr);
  cudaFree(dact);
  cudaFree(dax);
  cudaFree(dtest);
  std::printf("PHASE1 %lld regions\n", n);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: ref_driver integrate|phase1|bench|interp2d|lclt ...\n");
    return 2;
  }
  if (std::strcmp(argv[1], "integrate") == 0) return run_integrate(argc, argv);
  if (std::strcmp(argv[1], "phase1") == 0) return run_phase1(argc, argv);
  if (std::strcmp(argv[1], "bench") == 0) return run_bench(argc, argv);
  if (std::strcmp(argv[1], "interp2d") == 0) return run_interp2d(argc, argv);
  if (std::strcmp(argv[1], "lclt") == 0) return run_lclt(argc, argv);
  return 2;
}
