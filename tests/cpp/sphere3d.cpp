// 3-D usage: a plane wave through spheres with FFTSolver3D or ADI, through
// the B200 solver API (include/paxpro/paxpro.hpp).  Arguments: solver
// (fft3d | adi), N, steps, save ratio, output file (binary complex128: the
// last solution, then slice 1 of the saved cube).
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "paxpro/paxpro.hpp"

int main(int argc, char **argv) {
  if (argc < 6) return 2;
  const std::string kind = argv[1];
  const unsigned n = std::atoi(argv[2]);
  const unsigned steps = std::atoi(argv[3]);
  const unsigned ratio = std::atoi(argv[4]);
  const double L = 1000.0;
  double dx = L / (n - 1);
  while (pxp_node_count(-L / 2, L / 2, dx) != n) dx = std::nextafter(dx, pxp_node_count(-L / 2, L / 2, dx) < n ? 0.0 : 1e9);
  const double dz = 1000.0;
  SphereMaterial spheres;
  spheres.addSphere(40.0, -30.0, 3000.0, 150.0, 4.5e-5, 9e-7);
  spheres.addSphere(-120.0, 90.0, 6500.0, 100.0, 2e-5, 4e-7);
  ParaxialSimulation sim("spheres");
  sim.setTransverseDiscretization(-L / 2, L / 2, dx);
  sim.setVerticalDiscretization(-L / 2, L / 2, dx);
  sim.setLongitudinalDiscretization(0.0, steps * dz, dz, ratio);
  PlaneWave pw;
  pw.setWavelength(0.1);
  pw.setDim(ParaxialSource::Dim_t::THREE_D);
  FFTSolver3D fft;
  ADI adi;
  adi.useTBC = false;
  Solver3D &solver = kind == "adi" ? static_cast<Solver3D &>(adi) : static_cast<Solver3D &>(fft);
  try {
    sim.setSolver(solver);
    sim.material = &spheres;
    sim.setBoundaryConditions(pw);
    sim.solve();
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const arma::cx_mat &last = solver.getLastSolution3D();
  const arma::cx_cube &cube = solver.getSolution3D();
  FILE *f = std::fopen(argv[5], "wb");
  if (!f) return 1;
  std::fwrite(last.memptr(), sizeof(cdouble), last.n_elem, f);
  std::fwrite(&cube(0, 0, 1), sizeof(cdouble), (size_t)cube.n_rows * cube.n_cols, f);
  std::fclose(f);
  std::printf("%s N=%u steps=%u cube %zu x %zu x %zu\n", kind.c_str(), n, steps,
              (size_t)cube.n_rows, (size_t)cube.n_cols, (size_t)cube.n_slices);
  return 0;
}
