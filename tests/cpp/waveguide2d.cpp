// The reference's Examples/waveguide2D.cpp usage pattern, written against the
// B200 solver API (include/paxpro/paxpro.hpp): a planar waveguide material
// function, a Gaussian beam source, a solver handed to ParaxialSimulation,
// solve(), then the last solution.  Arguments: solver (fft | cn), Nx, steps,
// output file (binary complex128 exit field, then the saved column at
// step steps/2), transparent (0 | 1).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "paxpro/paxpro.hpp"

class Waveguide2D : public MaterialFunction {
 public:
  Waveguide2D(double xmin, double dx, unsigned n) : xmin(xmin), dx(dx), n(n) {}
  void getXrayMatProp(double x, double y, double z, double &delta, double &beta) const override {
    long ix = (long)std::floor((x - xmin) / dx + 0.5);
    long d = ix < (long)n - 1 - ix ? ix : (long)n - 1 - ix;
    if (d < 25) {
      delta = 7.5e-6;
      beta = 1e-7 + (1e-4 - 1e-7) * (double)(25 - d) / 25.0;
    } else if (std::fabs(x) <= 25.0) {
      delta = 0.0;
      beta = 0.0;
    } else {
      delta = 7.5e-6;
      beta = 1e-7;
    }
  }
  bool zInvariant() const override { return zinv; }
  bool zinv{true};

 private:
  double xmin, dx;
  unsigned n;
};

int main(int argc, char **argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s fft|cn Nx steps out.bin transparent [zvary]\n", argv[0]);
    return 2;
  }
  const std::string kind = argv[1];
  const unsigned n = std::atoi(argv[2]);
  const unsigned steps = std::atoi(argv[3]);
  const bool transparent = std::atoi(argv[5]) != 0;
  const bool zvary = argc > 6 && std::atoi(argv[6]) != 0;
  const double xmin = -250.0, xmax = 250.0;
  double dx = (xmax - xmin) / (n - 1);
  while (pxp_node_count(xmin, xmax, dx) != n) dx = std::nextafter(dx, pxp_node_count(xmin, xmax, dx) < n ? 0.0 : 1e9);
  const double dz = kind == "cn" ? 500.0 : 1000.0;

  Waveguide2D wg(xmin, dx, n);
  wg.zinv = !zvary;
  ParaxialSimulation sim("Wg2D");
  sim.setTransverseDiscretization(xmin, xmax, dx);
  sim.setLongitudinalDiscretization(0.0, steps * dz, dz);
  GaussianBeam gbeam;
  gbeam.setWaist(15.0);
  gbeam.setCenter(kind == "cn" ? 40.0 : 0.0, 0.0);
  gbeam.setWavelength(0.1);

  FFTSolver2D fft;
  CrankNicholson cn;
  Solver2D &solver = kind == "cn" ? static_cast<Solver2D &>(cn) : static_cast<Solver2D &>(fft);
  if (transparent) solver.setBoundaryCondition(Solver2D::BC_t::TRANSPARENT);
  try {
    sim.setSolver(solver);
    sim.material = &wg;
    sim.setBoundaryConditions(gbeam);
    sim.solve();
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const arma::cx_vec &last = solver.getLastSolution();
  const arma::cx_mat &sol = solver.getSolution();
  FILE *f = std::fopen(argv[4], "wb");
  if (!f) return 1;
  std::fwrite(last.memptr(), sizeof(cdouble), last.n_elem, f);
  std::fwrite(&sol(0, steps / 2), sizeof(cdouble), sol.n_rows, f);
  std::fwrite(&sol(0, 0), sizeof(cdouble), sol.n_rows, f);
  std::fclose(f);
  std::printf("%s Nx=%u steps=%u solution %zu x %zu\n", kind.c_str(), n, steps,
              (size_t)sol.n_rows, (size_t)sol.n_cols);
  return 0;
}
