// ref_api_example.cu -- an integrand written the reference's way (a device
// functor taking double x[] and int dim, held and passed by pointer) and
// integrated through the reference-shaped C++ front end
// (cubature/gpucuhre.cuh): the code change a caller of quad::GPUcuhre
// makes is the include line.
//
//   ref_api_example <epsrel> <lo> <hi>
//
// prints one JSON line per integration: the unit cube, then the box
// [lo, hi]^3.
#include <cstdio>
#include <cstdlib>

#include "cubature/gpucuhre.cuh"

// prod_i 1/(a_i^-2 + (x_i - u_i)^2), parameters held by value as the
// reference's functors hold theirs (they are copied to the device).
struct PeakFunctor {
  double a[3] = {8.0, 12.0, 6.0};
  double u[3] = {0.3, 0.6, 0.5};
  __device__ double operator()(double x[], int dim) {
    double den = 1;
    for (int i = 0; i < dim; ++i) {
      const double t = x[i] - u[i];
      den *= 1 / (a[i] * a[i]) + t * t;
    }
    return 1 / den;
  }
};

int main(int argc, char** argv) {
  const double epsrel = argc > 1 ? atof(argv[1]) : 1e-6;
  const double lo = argc > 2 ? atof(argv[2]) : -0.5;
  const double hi = argc > 3 ? atof(argv[3]) : 1.5;
  PeakFunctor f;
  quad::GPUcuhre<double> cuhre(argc, argv, 3);
  const double los[3] = {lo, lo, lo}, his[3] = {hi, hi, hi};
  quad::Volume<double> vol(los, his, 3);
  for (int pass = 0; pass < 2; ++pass) {
    double integral = 0, error = 0;
    size_t nregions = 0, neval = 0;
    const int flag = cuhre.integrate(epsrel, 1e-14, integral, error, nregions, neval, &f,
                                     pass ? &vol : nullptr);
    printf("{\"box\": %s, \"flag\": %d, \"integral\": %.17g, \"error\": %.17g, "
           "\"nregions\": %zu, \"neval\": %zu}\n",
           pass ? "true" : "false", flag, integral, error, nregions, neval);
    if (flag < 0) {
      fprintf(stderr, "error %d: %s\n", flag, cuhre.last_error().c_str());
      return 1;
    }
  }
  return 0;
}
