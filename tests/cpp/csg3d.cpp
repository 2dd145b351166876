// 3-D usage with constructive solid geometry: geom::Shape / Part / Module
// joined into a CSGMaterial (the reference's Examples pattern), propagated by
// FFTSolver3D or ADI through the B200 solver API
// (include/paxpro/paxpro.hpp).  The geometry is the one of
// tests/csg_geometry.py.
//   csg3d material <points file> <out>  -- CSGMaterial::getXrayMatProp at
//       the points (x y z triples, binary float64), out = (delta, beta) pairs
//   csg3d fft3d|adi N steps <out>       -- last solution then saved slice 1
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "paxpro/paxpro.hpp"

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  const std::string kind = argv[1];
  using geom::Axis_t;
  geom::Box slab(300.0, 200.0, 150.0);
  slab.rotate(30.0, Axis_t::Z);
  slab.translate(0.0, 0.0, 3000.0);
  geom::Sphere bore(60.0);
  bore.translate(20.0, 0.0, 3000.0);
  geom::Cylinder cone(40.0, 80.0, 400.0);
  cone.rotate(90.0, Axis_t::X);
  cone.translate(-150.0, 50.0, 5000.0);
  geom::Sphere ball(120.0);
  ball.translate(100.0, -100.0, 4000.0);
  geom::Sphere far(50.0);
  far.scale(2.0, Axis_t::Z);
  far.translate(-300.0, 300.0, 6000.0);
  geom::Box hole(50.0, 50.0, 50.0);
  hole.translate(100.0, -100.0, 4000.0);

  geom::Part p1("slab"), p2("cone"), p3("ball"), p5("far"), p4("hole");
  p1.delta = 3e-5; p1.beta = 6e-7;
  p1.add(slab);
  p1.difference(bore);
  p2.delta = 1e-5; p2.beta = 2e-7;
  p2.add(cone);
  p3.delta = 2e-5; p3.beta = 4e-7;
  p3.add(ball);
  p5.delta = 5e-6; p5.beta = 1e-7;
  p5.add(far);
  p4.delta = 9e-5; p4.beta = 9e-7;
  p4.add(hole);
  geom::Module lens("lens"), shell("shell");
  lens.add(p1);
  lens.add(p2);
  shell.add(p3);
  shell.add(p5);
  shell.difference(p4);
  CSGMaterial material;
  material.addModule(lens);
  material.addModule(shell);

  if (kind == "material") {
    FILE *in = std::fopen(argv[2], "rb");
    if (!in) return 1;
    std::vector<double> pts;
    double v;
    while (std::fread(&v, sizeof(double), 1, in) == 1) pts.push_back(v);
    std::fclose(in);
    std::vector<double> out;
    for (size_t i = 0; i + 2 < pts.size(); i += 3) {
      double d, b;
      material.getXrayMatProp(pts[i], pts[i + 1], pts[i + 2], d, b);
      out.push_back(d);
      out.push_back(b);
    }
    FILE *f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    std::fwrite(out.data(), sizeof(double), out.size(), f);
    std::fclose(f);
    return 0;
  }
  if (argc < 5) return 2;
  const unsigned n = std::atoi(argv[2]);
  const unsigned steps = std::atoi(argv[3]);
  const double L = 1000.0;
  double dx = L / (n - 1);
  while (pxp_node_count(-L / 2, L / 2, dx) != n) dx = std::nextafter(dx, pxp_node_count(-L / 2, L / 2, dx) < n ? 0.0 : 1e9);
  const double dz = 1000.0;
  ParaxialSimulation sim("csg");
  sim.setTransverseDiscretization(-L / 2, L / 2, dx);
  sim.setVerticalDiscretization(-L / 2, L / 2, dx);
  sim.setLongitudinalDiscretization(0.0, steps * dz, dz, 1);
  PlaneWave pw;
  pw.setWavelength(0.1);
  pw.setDim(ParaxialSource::Dim_t::THREE_D);
  FFTSolver3D fft;
  ADI adi;
  adi.useTBC = false;
  Solver3D &solver = kind == "adi" ? static_cast<Solver3D &>(adi) : static_cast<Solver3D &>(fft);
  try {
    sim.setSolver(solver);
    sim.material = &material;
    sim.setBoundaryConditions(pw);
    sim.solve();
  } catch (std::exception &e) {
    std::cerr << e.what() << std::endl;
    return 1;
  }
  const arma::cx_mat &last = solver.getLastSolution3D();
  const arma::cx_cube &cube = solver.getSolution3D();
  FILE *f = std::fopen(argv[4], "wb");
  if (!f) return 1;
  std::fwrite(last.memptr(), sizeof(cdouble), last.n_elem, f);
  std::fwrite(&cube(0, 0, 1), sizeof(cdouble), (size_t)cube.n_rows * cube.n_cols, f);
  std::fclose(f);
  return 0;
}
