// ref_driver.cu -- runs the reference engine (quad::GPUcuhre, compiled from
// the reference's own headers) on Genz integrands and prints its outputs,
// to produce golden vectors for the tests.  Test infrastructure only.
//
//   ref_driver integrate <family> <ndim> <epsrel> <epsabs> a_0..a_{n-1} u_0..u_{n-1}
//       -> "RESULT {json}" with integral, error, nregions, neval, errorFlag, ms
//   ref_driver phase1 <family> <ndim> <epsrel> <epsabs> <in.bin> <out.bin> a.. u..
//       runs INTEGRATE_GPU_PHASE1 (GPUQuadPhases.cu:38-79) on the region list
//       in in.bin ([int64 n][n*ndim lo][n*ndim len], dimension-major) and
//       writes [n avg][n err][n int32 active][n int32 axis] to out.bin.
//
// The integration volume is always the unit cube (vol = NULL): the
// reference's Volume path skips the volume map for the middle sample pass
// (GPUQuadSample.cu:174-179) and reads bounds through float textures.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "quad/GPUquad/GPUquad.h"

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

static int run_phase1(int argc, char** argv) {
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
  if (argc < 6) {
    std::fprintf(stderr, "usage: ref_driver integrate|phase1 ...\n");
    return 2;
  }
  if (std::strcmp(argv[1], "integrate") == 0) return run_integrate(argc, argv);
  if (std::strcmp(argv[1], "phase1") == 0) return run_phase1(argc, argv);
  return 2;
}
