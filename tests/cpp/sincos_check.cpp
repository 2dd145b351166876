// Error of pxp::sincos_cw against long-double sinl/cosl over [0, xmax]:
// prints the largest error in units of the double ulp of the exact value
// (1 ulp of 1.0 used below it, since the results feed a product with values
// of modulus about one).  Arguments: samples xmax.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../paxpro_b200/csrc/pxp_sincos.h"

int main(int argc, char **argv) {
  const long n = argc > 1 ? std::atol(argv[1]) : 200000;
  const double xmax = argc > 2 ? std::atof(argv[2]) : 2000.0;
  std::mt19937_64 rng(12345);
  std::uniform_real_distribution<double> u(0.0, xmax);
  const long double eps = std::ldexp(1.0L, -52);
  long double worst = 0.0L;
  double worst_x = 0.0;
  for (long i = 0; i < n; ++i) {
    double x = i < 64 ? i * 0.78539816339744830962 : u(rng);  // include multiples of pi/4
    double s, c;
    pxp::sincos_cw(x, &s, &c);
    long double es = sinl((long double)x), ec = cosl((long double)x);
    long double e = std::fmax(std::fabs((long double)s - es), std::fabs((long double)c - ec)) / eps;
    if (e > worst) {
      worst = e;
      worst_x = x;
    }
  }
  std::printf("%.3Lf %.17g\n", worst, worst_x);
  return 0;
}
