// ref_pin.cpp -- the reference's own propagation path, compiled from its
// sources, behind a C interface for pinning the oracle.  TEST INFRASTRUCTURE
// ONLY: loaded by tests/ (and bench.py's reference arm), never by the
// product.
//
// oracle/Makefile compiles the reference's sources where they lie (never
// copied) against oracle/refshim/, which stands in for the third-party
// headers the build lacks: the Armadillo containers, FFTW3's basic
// interface (transforms by the oracle's FFT), and declarations of HDF5,
// jsoncpp and VISA that the solver classes name but the stepping path never
// reaches.  Compiled reference files: src/crancNicholson.cpp,
// src/alternatingDirectionSolver.cpp, src/fftSolver2D.cpp,
// src/fftSolver3D.cpp, src/solver.cpp, src/solver2D.cpp, src/solver3D.cpp,
// src/paraxialSimulation.cpp, src/absorber.cpp, src/paraxialEquation.cpp,
// src/gaussianBeam.cpp, src/planeWave.cpp, src/paraxialSource.cpp,
// src/materialFunction.cpp, src/geometry.cpp, src/shape.cpp.
//
// The runs below drive the reference classes exactly as a user program does
// (Examples/waveguide2D.cpp:57-75, Examples/sphere.cpp:28-75): a
// ParaxialSimulation with its discretisations, wavenumber and material, a
// solver passed to setSolver, setInitialConditions, then Solver::step().
// The material is a MaterialFunction whose getXrayMatProp evaluates the
// oracle's material description (orc_material_eval), so the oracle and the
// reference see the same medium and differ only in the code under test.
#include <omp.h>

#include <algorithm>
#include <complex>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#include "alternatingDirectionSolver.hpp"
#include "crankNicholson.hpp"
#include "fftSolver2D.hpp"
#include "fftSolver3D.hpp"
#include "gaussianBeam.hpp"
#include "geometry.hpp"
#include "materialFunction.hpp"
#include "paraxialEquation.hpp"
#include "paraxialSimulation.hpp"
#include "planeWave.hpp"
#include "postProcessMod.hpp"
#include "shapes.hpp"
#include "thomasAlgorithm.hpp"

#include "paxpro_oracle.h"

namespace {

class OracleMaterial : public MaterialFunction {
 public:
  OracleMaterial(const orc_material *m, const orc_grid *g) : m_(m), g_(g) {}
  void getXrayMatProp(double x, double y, double z, double &delta, double &beta) const override {
    orc_material_eval(m_, g_, x, y, z, &delta, &beta);
  }

 private:
  const orc_material *m_;
  const orc_grid *g_;
};

// Every run here uses `threads` OpenMP threads and restores the caller's
// setting.  The ADI matrix build runs an OpenMP loop whose (delta, beta)
// temporaries are shared between threads (src/alternatingDirectionSolver.cpp:
// 22-37), so only a single-threaded ADI run is deterministic: parity runs
// pass 1, timing runs may pass more.
struct OmpThreads {
  int saved;
  explicit OmpThreads(int n) : saved(omp_get_max_threads()) { omp_set_num_threads(n > 0 ? n : 1); }
  ~OmpThreads() { omp_set_num_threads(saved); }
};

void copy_out(const std::complex<double> *src, size_t n, double *dst) {
  std::memcpy(dst, src, sizeof(double) * 2 * n);
}

}  // namespace

extern "C" {

// diag, subdiag, rhs: interleaved complex doubles; solution lands in diag.
void ref_thomas_solve(double *diag, const double *subdiag, double *rhs, int n) {
  ThomasAlgorithm solver;
  solver.solve(reinterpret_cast<std::complex<double> *>(diag),
               reinterpret_cast<const std::complex<double> *>(subdiag),
               reinterpret_cast<std::complex<double> *>(rhs), (unsigned)n);
}

// F, G, H, J at (x, z) and the phase factor exp(i k z).
void ref_paraxial_equation(double x, double z, double k, double out[6]) {
  ParaxialEquation eq;
  out[0] = eq.F(x, z);
  out[1] = eq.G(x, z);
  out[2] = eq.H(x, z);
  out[3] = eq.J(x, z);
  std::complex<double> p = eq.phaseFactor(k, z);
  out[4] = p.real();
  out[5] = p.imag();
}

// ParaxialSimulation::nodeNumberTransverse of a discretisation.
unsigned ref_node_count(double mn, double mx, double step) {
  ParaxialSimulation sim("refpin");
  sim.setTransverseDiscretization(mn, mx, step);
  return sim.nodeNumberTransverse();
}

// FFTSolver2D (kind 1) or CrankNicholson (kind 2) on the grid g (x and z),
// from u0 (Nx complex), nsteps calls of Solver::step().  After every step
// that is a multiple of save_every (> 0) the field (getLastSolution) goes to
// saves[(step / save_every - 1) * Nx]; the last field to u_out.  transparent:
// Solver2D::BC_t::TRANSPARENT (CrankNicholson).  Returns 0, or -1 for bad
// arguments (nsteps must stay below nodeNumberLongitudinal, whose columns
// the reference's solution matrix holds), -2 when the reference threw.
int ref_run2d(int kind, const orc_grid *g, const orc_material *m, int transparent,
              const double *u0, int nsteps, int save_every, double *saves, double *u_out,
              int threads) {
  try {
    OmpThreads omp(threads);
    ParaxialSimulation sim("refpin");
    sim.setTransverseDiscretization(g->xmin, g->xmax, g->dx);
    sim.setLongitudinalDiscretization(g->zmin, g->zmax, g->dz);
    sim.setWavenumber(g->wavenumber);
    OracleMaterial mat(m, g);
    sim.material = &mat;
    std::unique_ptr<Solver2D> solver;
    if (kind == 1)
      solver.reset(new FFTSolver2D());
    else if (kind == 2)
      solver.reset(new CrankNicholson());
    else
      return -1;
    if (nsteps < 0 || (unsigned)nsteps >= sim.nodeNumberLongitudinal()) return -1;
    // FFTSolver2D's destructor destroys its FFTW plans unconditionally
    // (src/fftSolver2D.cpp:9-13), and they exist only after the first step
    if (kind == 1 && nsteps == 0) return -1;
    solver->disableLongitudinalFilter();
    if (transparent) solver->setBoundaryCondition(Solver2D::BC_t::TRANSPARENT);
    sim.setSolver(*solver);
    const unsigned nx = sim.nodeNumberTransverse();
    arma::cx_vec v(nx);
    std::memcpy(v.memptr(), u0, sizeof(double) * 2 * nx);
    solver->setInitialConditions(v);
    for (int step = 1; step <= nsteps; ++step) {
      solver->step();
      if (save_every > 0 && step % save_every == 0 && saves)
        copy_out(solver->getLastSolution().memptr(), nx,
                 saves + 2L * (step / save_every - 1) * nx);
    }
    copy_out(solver->getLastSolution().memptr(), nx, u_out);
    return 0;
  } catch (...) {
    return -2;
  }
}

// FFTSolver3D (kind 3) or ADI (kind 4) on the grid g, from u0 (Ny x Nx
// column-major, Ny = Nx as Solver3D::setSimulator forces), nsteps calls of
// Solver::step().  Saves as ref_run2d (getLastSolution3D, Nx*Ny values
// each).  use_tbc: ADI::useTBC.  absorber_damping > 0: FFTSolver3D::
// absorbingBC(absorber_width, absorber_damping).  threads: OpenMP threads
// (1 for a deterministic ADI run, see OmpThreads).  The longitudinal
// downsampling ratio is set to nsteps so that the reference's saved-slice
// cube (src/solver3D.cpp:36) stays two slices.
int ref_run3d(int kind, const orc_grid *g, const orc_material *m, int use_tbc,
              double absorber_width, double absorber_damping, const double *u0, int nsteps,
              int save_every, double *saves, double *u_out, int threads) {
  try {
    OmpThreads omp(threads);
    ParaxialSimulation sim("refpin");
    sim.setTransverseDiscretization(g->xmin, g->xmax, g->dx);
    sim.setVerticalDiscretization(g->ymin, g->ymax, g->dy);
    sim.setLongitudinalDiscretization(g->zmin, g->zmax, g->dz,
                                      (unsigned)std::max(nsteps, 1));
    sim.setWavenumber(g->wavenumber);
    OracleMaterial mat(m, g);
    sim.material = &mat;
    if (nsteps < 0 || (unsigned)nsteps >= sim.nodeNumberLongitudinal()) return -1;
    std::unique_ptr<Solver3D> solver;
    ADI *adi = nullptr;
    FFTSolver3D *fft = nullptr;
    if (kind == 3) {
      fft = new FFTSolver3D();
      solver.reset(fft);
    } else if (kind == 4) {
      adi = new ADI();
      solver.reset(adi);
    } else {
      return -1;
    }
    sim.setSolver(*solver);
    if (adi) adi->useTBC = use_tbc != 0;
    if (fft && absorber_damping > 0.0) fft->absorbingBC(absorber_width, absorber_damping);
    const unsigned nx = sim.nodeNumberTransverse();
    const size_t npts = (size_t)nx * nx;
    arma::cx_mat v(nx, nx);
    std::memcpy(v.memptr(), u0, sizeof(double) * 2 * npts);
    solver->setInitialConditions(v);
    for (int step = 1; step <= nsteps; ++step) {
      solver->step();
      if (save_every > 0 && step % save_every == 0 && saves)
        copy_out(solver->getLastSolution3D().memptr(), npts,
                 saves + 2L * (step / save_every - 1) * npts);
    }
    copy_out(solver->getLastSolution3D().memptr(), npts, u_out);
    return 0;
  } catch (...) {
    return -2;
  }
}

// The saved-slice cube of a 3-D run (Solver3D::getSolution3D,
// src/solver3D.cpp:36, 78-125): kind 3 or 4 as ref_run3d (Dirichlet ADI, no
// absorber), transverse downsampling ratio ratio_x and longitudinal ratio
// ratio_z, nsteps steps; the cube (m x m x slices, m = Nx / ratio_x,
// slices = Nz / ratio_z + 1, Nz = nodeNumberLongitudinal) goes to out, its
// sizes to dims[0..2].  out must hold m*m*slices complex values; pass
// out = NULL to read the sizes only.
int ref_run3d_saved(int kind, const orc_grid *g, const orc_material *m, unsigned ratio_x,
                    unsigned ratio_z, const double *u0, int nsteps, double *out, unsigned *dims,
                    int threads) {
  try {
    OmpThreads omp(kind == 4 ? 1 : threads);
    ParaxialSimulation sim("refpin");
    sim.setTransverseDiscretization(g->xmin, g->xmax, g->dx, ratio_x);
    sim.setVerticalDiscretization(g->ymin, g->ymax, g->dy);
    sim.setLongitudinalDiscretization(g->zmin, g->zmax, g->dz, ratio_z);
    sim.setWavenumber(g->wavenumber);
    OracleMaterial mat(m, g);
    sim.material = &mat;
    if (nsteps < 0 || (unsigned)nsteps >= sim.nodeNumberLongitudinal()) return -1;
    std::unique_ptr<Solver3D> solver;
    if (kind == 3) {
      solver.reset(new FFTSolver3D());
    } else if (kind == 4) {
      ADI *adi = new ADI();
      adi->useTBC = false;
      solver.reset(adi);
    } else {
      return -1;
    }
    sim.setSolver(*solver);
    const arma::cx_cube &cube = solver->getSolution3D();
    dims[0] = (unsigned)cube.n_rows;
    dims[1] = (unsigned)cube.n_cols;
    dims[2] = (unsigned)cube.n_slices;
    if (out == nullptr) return 0;
    const unsigned nx = sim.nodeNumberTransverse();
    arma::cx_mat v(nx, nx);
    std::memcpy(v.memptr(), u0, sizeof(double) * 2 * (size_t)nx * nx);
    solver->setInitialConditions(v);
    for (int step = 1; step <= nsteps; ++step) solver->step();
    copy_out(solver->getSolution3D().memptr(), cube.n_elem, out);
    return 0;
  } catch (...) {
    return -2;
  }
}

// A CSGMaterial (src/materialFunction.cpp:3-13) built from the reference's
// own geometry classes (geom::Sphere / Box / Cylinder, Part, Module:
// src/shape.cpp, src/geometry.cpp) and evaluated at npts points xyz[3*i..];
// delta and beta of point i go to out[2*i], out[2*i + 1].  A shape is built
// from its kind and sizes (sphere: radius; box: Lx, Ly, Lz; cylinder: r1,
// r2, height), then its ops replayed in order: type 0 translate(a, b, c),
// 1 rotate(a degrees, axis b), 2 scale(a, axis b) (axis 0/1/2 = X/Y/Z).
// Shapes join their part by add (operation 0) or difference (1), parts
// their module likewise; modules are added in order.  Returns 0, or -2 when
// the reference threw (e.g. a difference before any add).
typedef struct {
  int kind, operation, first_op, num_ops;
  double size[3];
} ref_csg_shape;
typedef struct {
  int type;
  double a, b, c;
} ref_csg_op;
typedef struct {
  int operation, first_shape, num_shapes;
  double delta, beta;
} ref_csg_part;
typedef struct {
  int first_part, num_parts;
} ref_csg_module;

int ref_csg_eval(const ref_csg_module *modules, int nmodules, const ref_csg_part *parts,
                 const ref_csg_shape *shapes, const ref_csg_op *ops, const double *xyz, int npts,
                 double *out) {
  try {
    std::vector<std::unique_ptr<geom::Shape>> keep_shapes;
    std::vector<std::unique_ptr<geom::Part>> keep_parts;
    std::vector<std::unique_ptr<geom::Module>> keep_modules;
    CSGMaterial mat;
    const geom::Axis_t axes[3] = {geom::Axis_t::X, geom::Axis_t::Y, geom::Axis_t::Z};
    for (int mi = 0; mi < nmodules; ++mi) {
      keep_modules.emplace_back(new geom::Module("module"));
      geom::Module &mod = *keep_modules.back();
      for (int pi = 0; pi < modules[mi].num_parts; ++pi) {
        const ref_csg_part &pd = parts[modules[mi].first_part + pi];
        keep_parts.emplace_back(new geom::Part("part"));
        geom::Part &part = *keep_parts.back();
        part.delta = pd.delta;
        part.beta = pd.beta;
        for (int si = 0; si < pd.num_shapes; ++si) {
          const ref_csg_shape &sd = shapes[pd.first_shape + si];
          geom::Shape *sh = nullptr;
          if (sd.kind == 0)
            sh = new geom::Sphere(sd.size[0]);
          else if (sd.kind == 1)
            sh = new geom::Box(sd.size[0], sd.size[1], sd.size[2]);
          else
            sh = new geom::Cylinder(sd.size[0], sd.size[1], sd.size[2]);
          keep_shapes.emplace_back(sh);
          for (int oi = 0; oi < sd.num_ops; ++oi) {
            const ref_csg_op &op = ops[sd.first_op + oi];
            if (op.type == 0)
              sh->translate(op.a, op.b, op.c);
            else if (op.type == 1)
              sh->rotate(op.a, axes[(int)op.b]);
            else
              sh->scale(op.a, axes[(int)op.b]);
          }
          if (sd.operation == 0)
            part.add(*sh);
          else
            part.difference(*sh);
        }
        if (pd.operation == 0)
          mod.add(part);
        else
          mod.difference(part);
      }
      mat.addModule(mod);
    }
    for (int i = 0; i < npts; ++i)
      mat.getXrayMatProp(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], out[2 * i], out[2 * i + 1]);
    return 0;
  } catch (...) {
    return -2;
  }
}

// The initial field ParaxialSimulation::setBoundaryConditions(const
// ParaxialSource&) hands a solver (src/paraxialSimulation.cpp:356-399) on the
// grid g: a GaussianBeam (source 0: wavelength, waist, centre (cx, cy),
// amplitude, origin z0; src/gaussianBeam.cpp:29-63) or a PlaneWave (source
// 1: wavelength, amplitude, angle_deg, z0; src/planeWave.cpp:5-19), in 2-D
// (dim 2: Nx values, through a CrankNicholson solver) or 3-D (dim 3: Ny x Nx
// column-major, through an FFTSolver3D), read back with getLastSolution /
// getLastSolution3D.  Returns 0, -1 for bad arguments, -2 when the reference
// threw.
int ref_source_field(int dim, const orc_grid *g, int source, double wavelength, double waist,
                     double cx, double cy, double amplitude, double angle_deg, double z0,
                     double *out) {
  try {
    ParaxialSimulation sim("refpin");
    sim.setTransverseDiscretization(g->xmin, g->xmax, g->dx);
    sim.setVerticalDiscretization(g->ymin, g->ymax, g->dy);
    sim.setLongitudinalDiscretization(g->zmin, g->zmax, g->dz);
    GaussianBeam gauss;
    PlaneWave plane;
    ParaxialSource *src = nullptr;
    if (source == 0) {
      gauss.setWaist(waist);
      gauss.setCenter(cx, cy);
      src = &gauss;
    } else if (source == 1) {
      plane.setAngleDeg(angle_deg);
      src = &plane;
    } else {
      return -1;
    }
    src->setWavelength(wavelength);
    src->setAmplitude(amplitude);
    src->setOrigin(0.0, z0);
    const unsigned nx = sim.nodeNumberTransverse();
    if (dim == 2) {
      // any Solver2D takes the field; CrankNicholson holds no FFTW plans
      // (FFTSolver2D's destructor frees plans made only by a first step)
      CrankNicholson solver;
      sim.setSolver(solver);
      sim.setBoundaryConditions(*src);
      copy_out(solver.getLastSolution().memptr(), nx, out);
    } else if (dim == 3) {
      src->setDim(ParaxialSource::Dim_t::THREE_D);
      FFTSolver3D solver;
      sim.setSolver(solver);
      sim.setBoundaryConditions(*src);
      copy_out(solver.getLastSolution3D().memptr(), (size_t)nx * nx, out);
    } else {
      return -1;
    }
    return 0;
  } catch (...) {
    return -2;
  }
}

}  // extern "C"
