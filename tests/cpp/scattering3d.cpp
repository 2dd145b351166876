// GenericScattering usage (the reference's Examples/sphere.cpp pattern): a
// Gaussian beam through a sphere with the vacuum reference run, then the far
// field through the B200 solver API (include/paxpro/paxpro.hpp).
// Arguments: solver (fft | adi), N, steps, pad length, max angle, export N,
// output file: N, then rows, cols (as doubles), the initial field, the
// reference run's exit field, the exit field (complex128, column-major) and
// the far field (rows x cols doubles, column-major).
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "paxpro/paxpro.hpp"

int main(int argc, char **argv) {
  if (argc < 8) return 2;
  const std::string kind = argv[1];
  const unsigned n = std::atoi(argv[2]);
  const unsigned steps = std::atoi(argv[3]);
  const double L = 1000.0;
  double dx = L / (n - 1);
  while (pxp_node_count(-L / 2, L / 2, dx) != n) dx = std::nextafter(dx, pxp_node_count(-L / 2, L / 2, dx) < n ? 0.0 : 1e9);
  SphereMaterial sphere;
  sphere.addSphere(20.0, -10.0, 0.0, 200.0, 8.9e-6, 7e-7);
  GenericScattering sim("sphere");
  sim.setBeamWaist(300.0);
  sim.setMaxScatteringAngle(std::atof(argv[5]));
  sim.xmin = -L / 2;
  sim.xmax = L / 2;
  sim.ymin = -L / 2;
  sim.ymax = L / 2;
  sim.zmin = -300.0;
  sim.zmax = 300.0;
  sim.dx = dx;
  sim.dy = dx;
  sim.dz = 600.0 / steps;
  sim.wavelength = 0.1569;
  sim.FFTPadLength = std::atoi(argv[4]);
  sim.exportNx = sim.exportNy = std::atoi(argv[6]);
  sim.propagator = kind == "adi" ? GenericScattering::SolverType_t::ADI : GenericScattering::SolverType_t::FFT;
  sim.setMaterial(sphere);
  arma::mat ff;
  try {
    sim.solve();
    sim.getFarField(ff);
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const arma::cx_cube &cube = sim.getSolver().getSolution3D();
  const arma::cx_mat &exitField = sim.getSolver().getLastSolution3D();
  const arma::cx_mat &ref = sim.getReference();
  FILE *f = std::fopen(argv[7], "wb");
  if (!f) return 1;
  const double hdr[3] = {(double)n, (double)ff.n_rows, (double)ff.n_cols};
  std::fwrite(hdr, sizeof(double), 3, f);
  std::fwrite(&cube(0, 0, 0), sizeof(cdouble), (size_t)n * n, f);
  std::fwrite(ref.memptr(), sizeof(cdouble), ref.n_elem, f);
  std::fwrite(exitField.memptr(), sizeof(cdouble), exitField.n_elem, f);
  std::fwrite(ff.memptr(), sizeof(double), ff.n_elem, f);
  std::fclose(f);
  std::printf("%s N=%u far field %zu x %zu\n", kind.c_str(), n, (size_t)ff.n_rows, (size_t)ff.n_cols);
  return 0;
}
