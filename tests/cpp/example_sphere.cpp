// The reference's 3-D example (Examples/sphere.cpp) through the B200 solver
// API: a user MaterialFunction subclass (a sphere of radius 500 nm at the
// origin), GenericScattering with the example's domain, steps, beam waist
// and wavelength (513 transverse nodes, 257 longitudinal), the far field of
// the exit field minus the vacuum reference.  Real-time visualisation and
// the HDF5 save are left out.  Arguments: output file (N, rows, cols as
// doubles; the reference run's exit field, the exit field (complex128,
// column-major); the far field (rows x cols doubles, column-major)), then
// optionally the propagator: fft (GenericScattering's default, as in the
// example) or adi.
#include <cstdio>
#include <iostream>
#include <string>

#include "paxpro/paxpro.hpp"

/** Sphere centered at (0,0,0), as in the reference example */
class Sphere : public MaterialFunction {
 public:
  explicit Sphere(double rad) : radius(rad) {}
  void getXrayMatProp(double x, double y, double z, double &delta, double &beta) const override {
    double rSq = x * x + y * y + z * z;
    if (rSq < radius * radius) {
      delta = 8.9E-6;
      beta = 7E-7;
      return;
    }
    delta = 0.0;
    beta = 0.0;
  }

 private:
  double radius{0.0};
};

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  double r = 500.0;
  double xmin = -1.5 * r;
  double xmax = 1.5 * r;
  double zmin = -1.05 * r;
  double zmax = 1.05 * r;
  double dx = (xmax - xmin) / 512;
  double dz = (zmax - zmin) / 256;
  GenericScattering simulation("sphere");
  simulation.setBeamWaist(400.0 * r);
  simulation.setMaxScatteringAngle(0.05);
  simulation.xmin = xmin;
  simulation.xmax = xmax;
  simulation.ymin = xmin;
  simulation.ymax = xmax;
  simulation.zmin = zmin;
  simulation.zmax = zmax;
  simulation.dx = dx;
  simulation.dy = dx;
  simulation.dz = dz;
  simulation.wavelength = 0.1569;
  if (argc > 2 && std::string(argv[2]) == "adi")
    simulation.propagator = GenericScattering::SolverType_t::ADI;
  Sphere sphere(r);
  simulation.setMaterial(sphere);
  arma::mat ff;
  try {
    simulation.solve();
    simulation.getFarField(ff);
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const arma::cx_mat &exitField = simulation.getSolver().getLastSolution3D();
  const arma::cx_mat &ref = simulation.getReference();
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 1;
  const double hdr[3] = {(double)exitField.n_rows, (double)ff.n_rows, (double)ff.n_cols};
  std::fwrite(hdr, sizeof(double), 3, f);
  std::fwrite(ref.memptr(), sizeof(cdouble), ref.n_elem, f);
  std::fwrite(exitField.memptr(), sizeof(cdouble), exitField.n_elem, f);
  std::fwrite(ff.memptr(), sizeof(double), ff.n_elem, f);
  std::fclose(f);
  std::printf("N=%u far field %zu x %zu\n", (unsigned)exitField.n_rows, (size_t)ff.n_rows,
              (size_t)ff.n_cols);
  return 0;
}
