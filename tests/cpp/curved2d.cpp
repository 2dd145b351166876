// CurvedWaveGuideFD usage: a Gaussian beam entering a bent waveguide, the
// transmittivity computed at every step (post::Transmittivity), through the
// B200 solver API.  Arguments: solver (fft | cn), N, steps, smoothed (0|1),
// output file: Nx, Nz, intensity at zero, the transmission (Nz-1 doubles),
// then the solution matrix (Nx x Nz complex128, column-major).
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "paxpro/paxpro.hpp"

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  const std::string kind = argv[1];
  if (kind == "material") {
    // curved2d material <smoothed> <out>: delta, beta of the guide below on
    // a 61 x 41 grid of (x, z), x in [-400, 200], z in [0, 2e5]
    Cladding c;
    c.setRefractiveIndex(4.14e-5, 3.45e-6);
    Cladding inside;
    inside.setRefractiveIndex(1e-6, 2e-8);
    CurvedWaveGuideFD g;
    g.setRadiusOfCurvature(40e6);
    g.setWidth(100.0);
    g.setCladding(c);
    g.setInsideMaterial(inside);
    g.setWaveguideLength(1.5e5);
    if (std::atoi(argv[2])) g.useSmoothedWG();
    g.setTransverseDiscretization(-400.0, 200.0, 10.0);
    g.setLongitudinalDiscretization(0.0, 2e5, 5000.0);
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    for (int iz = 0; iz <= 40; ++iz)
      for (int ix = 0; ix <= 60; ++ix) {
        double d, b;
        g.getXrayMatProp(-400.0 + 10.0 * ix, 5000.0 * iz, d, b);
        std::fwrite(&d, sizeof(double), 1, f);
        std::fwrite(&b, sizeof(double), 1, f);
      }
    std::fclose(f);
    return 0;
  }
  if (argc < 6) return 2;
  const unsigned n = std::atoi(argv[2]);
  const unsigned steps = std::atoi(argv[3]);
  const double xmin = -400.0, xmax = 200.0;
  double dx = (xmax - xmin) / (n - 1);
  while (pxp_node_count(xmin, xmax, dx) != n) dx = std::nextafter(dx, pxp_node_count(xmin, xmax, dx) < n ? 0.0 : 1e9);
  const double dz = 500.0;
  Cladding clad;
  clad.setRefractiveIndex(4.14e-5, 3.45e-6);
  CurvedWaveGuideFD wg;
  wg.setRadiusOfCurvature(40e6);
  wg.setWidth(100.0);
  wg.setCladding(clad);
  if (std::atoi(argv[4])) wg.useSmoothedWG();
  wg.setTransverseDiscretization(xmin, xmax, dx);
  wg.setLongitudinalDiscretization(0.0, steps * dz, dz);
  GaussianBeam gb;
  gb.setWavelength(0.1569);
  gb.setWaist(20.0);
  gb.setCenter(50.0, 0.0);
  gb.setDim(ParaxialSource::Dim_t::TWO_D);
  FFTSolver2D fft;
  CrankNicholson cn;
  Solver2D &solver = kind == "cn" ? static_cast<Solver2D &>(cn) : static_cast<Solver2D &>(fft);
  try {
    wg.setSolver(solver);
    wg.setBoundaryConditions(gb);
    wg.solve();
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const std::vector<double> &t = wg.getTransmittivity().get();
  const arma::cx_mat &sol = solver.getSolution();
  FILE *f = std::fopen(argv[5], "wb");
  if (!f) return 1;
  const double hdr[3] = {(double)sol.n_rows, (double)sol.n_cols, wg.getTransmittivity().getIntensityAtZero()};
  std::fwrite(hdr, sizeof(double), 3, f);
  std::fwrite(t.data(), sizeof(double), t.size(), f);
  std::fwrite(sol.memptr(), sizeof(cdouble), sol.n_elem, f);
  std::fclose(f);
  std::printf("%s N=%u steps=%u T(end)=%.6f\n", kind.c_str(), n, steps, t.empty() ? 0.0 : t.back());
  return 0;
}
