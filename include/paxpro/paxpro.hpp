// paxpro.hpp -- the reference's C++ solver API (ParaxialSimulation, Solver,
// Solver2D/3D, FFTSolver2D, CrankNicholson, FFTSolver3D, ADI, sources and the
// material hook) backed by the B200 solvers through the C ABI of
// paxpro_b200.h.  Header only; link with libpaxpro_b200.so.
//
// Class names, members and call order follow the reference
// (include/paraxialSimulation.hpp, include/solver.hpp, include/solver2D.hpp,
// include/solver3D.hpp, include/fftSolver2D.hpp, include/crankNicholson.hpp,
// include/fftSolver3D.hpp, include/alternatingDirectionSolver.hpp,
// include/paraxialSource.hpp, include/gaussianBeam.hpp, include/planeWave.hpp,
// include/materialFunction.hpp) so that user code written against them
// (e.g. Examples/waveguide2D.cpp) builds against this header instead.
// Errors surface as std::runtime_error, as in the reference
// (src/solver.cpp:5-28).
//
// Also here: post::FarField (computed on the device), Cladding,
// WaveGuideFDSimulation, CurvedWaveGuideFD with post::Transmittivity (its
// per-step integrals fused into the step kernels) and GenericScattering.
//
// Not provided (no counterpart on the GPU path, or a third-party dependency
// this build does not have): HDF5 save (save() throws), the other
// post-processing modules (the Python package has them), VISA visualisation
// and the VISA longitudinal low-pass filter (solve() requires
// disableLongitudinalFilter() when the longitudinal downsampling ratio is
// above 1), the waveguides' border tracker, control files and eigenmode
// projections, the projection solver.  The 3-D solvers take any
// MaterialFunction: a SphereMaterial or a CSGMaterial over geom::Module /
// Part / Shape is evaluated on the device; any other material (a user
// subclass, as in the reference's examples) is sampled on the host at the
// planes the reference's solvers sample and handed over per block of steps.
#pragma once
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../paxpro_b200.h"
#include "arma_lite.hpp"

typedef std::complex<double> cdouble;

/** Discretisation record (include/paraxialSimulation.hpp:20-26). */
struct Disctretization {
  double min{0.0};
  double max{0.0};
  double step{1.0};
  unsigned int downsamplingRatio{1};
};

// ------------------------------------------------------------ material ----
/** Material hook (include/materialFunction.hpp:6-10). */
class MaterialFunction {
 public:
  virtual ~MaterialFunction() {}
  virtual void getXrayMatProp(double x, double y, double z, double &delta,
                              double &beta) const = 0;
  /** Extension without a reference counterpart: return true when delta and
   * beta do not depend on z, so the CUDA solvers sample the medium once
   * instead of once per step.  The default (false) is always correct. */
  virtual bool zInvariant() const { return false; }
};

/** First-hit list of spheres, r^2 < R^2 as Examples/sphere.cpp:13-14; the
 * 3-D CUDA solvers evaluate it on the device. */
class SphereMaterial : public MaterialFunction {
 public:
  struct Sphere {
    double cx, cy, cz, radius, delta, beta;
  };
  void addSphere(double cx, double cy, double cz, double radius, double delta, double beta) {
    spheres.push_back({cx, cy, cz, radius, delta, beta});
  }
  void getXrayMatProp(double x, double y, double z, double &delta,
                      double &beta) const override {
    for (const Sphere &s : spheres) {
      double dx = x - s.cx, dy = y - s.cy, dz = z - s.cz;
      if (dx * dx + dy * dy + dz * dz < s.radius * s.radius) {
        delta = s.delta;
        beta = s.beta;
        return;
      }
    }
    delta = 0.0;
    beta = 0.0;
  }
  std::vector<Sphere> spheres;
};

// ------------------------------------------------------------ geometry ----
/** include/shapes.hpp, include/geometry.hpp, src/shape.cpp, src/geometry.cpp:
 * shapes with a world-to-shape 4x4 transformation (row-major here), parts
 * (shapes joined by union / difference, with a material) and modules (parts
 * joined by union / difference). */
namespace geom {
enum class Axis_t { X, Y, Z };
enum class Operation_t { UNION, DIFFERENCE };

class Shape {
 public:
  explicit Shape(const char *name) : name(name) {
    for (int i = 0; i < 16; ++i) transformation[i] = (i % 5 == 0) ? 1.0 : 0.0;
  }
  virtual ~Shape() {}
  /** src/shape.cpp:16-26: transformation = transformation * T(-x, -y, -z) */
  void translate(double x, double y, double z) {
    double m[16];
    identity(m);
    m[3] = -x;
    m[7] = -y;
    m[11] = -z;
    rightMultiply(m);
  }
  /** src/shape.cpp:28-57 */
  void rotate(double angleDeg, Axis_t axis) {
    const double PI = std::acos(-1.0);
    const double angle = angleDeg * PI / 180.0;
    double m[16];
    identity(m);
    switch (axis) {
      case Axis_t::X: m[5] = std::cos(angle); m[6] = std::sin(angle); m[9] = -std::sin(angle); m[10] = std::cos(angle); break;
      case Axis_t::Y: m[0] = std::cos(angle); m[2] = -std::sin(angle); m[8] = std::sin(angle); m[10] = std::cos(angle); break;
      case Axis_t::Z: m[0] = std::cos(angle); m[1] = std::sin(angle); m[4] = -std::sin(angle); m[5] = std::cos(angle); break;
    }
    rightMultiply(m);
  }
  /** src/shape.cpp:128-144: transformation = S(1/factor) * transformation */
  void scale(double factor, Axis_t axis) {
    double m[16];
    identity(m);
    const int a = axis == Axis_t::X ? 0 : (axis == Axis_t::Y ? 1 : 2);
    m[a * 5] = 1.0 / factor;
    double out[16];
    multiply(m, transformation, out);
    std::memcpy(transformation, out, sizeof(out));
  }
  /** src/shape.cpp:59-70 */
  void transform(double &x, double &y, double &z) const {
    const double x0 = x, y0 = y, z0 = z;
    const double *T = transformation;
    x = T[0] * x0 + T[1] * y0 + T[2] * z0 + T[3] * 1.0;
    y = T[4] * x0 + T[5] * y0 + T[6] * z0 + T[7] * 1.0;
    z = T[8] * x0 + T[9] * y0 + T[10] * z0 + T[11] * 1.0;
  }
  virtual bool isInside(double x, double y, double z) const = 0;
  virtual int kind() const = 0;
  virtual void size(double out[3]) const = 0;
  std::string name;
  double transformation[16];

 private:
  static void identity(double *m) {
    for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.0 : 0.0;
  }
  static void multiply(const double *a, const double *b, double *out) {
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        double acc = 0.0;
        for (int k = 0; k < 4; ++k) acc += a[i * 4 + k] * b[k * 4 + j];
        out[i * 4 + j] = acc;
      }
  }
  void rightMultiply(const double *m) {
    double out[16];
    multiply(transformation, m, out);
    std::memcpy(transformation, out, sizeof(out));
  }
};

/** geom::Sphere (src/shape.cpp:146-151) */
class Sphere : public Shape {
 public:
  explicit Sphere(double radius) : Shape("sphere"), radius(radius) {}
  bool isInside(double x, double y, double z) const override {
    transform(x, y, z);
    double r = std::sqrt(x * x + y * y + z * z);
    return r < radius;
  }
  int kind() const override { return PXP_SHAPE_SPHERE; }
  void size(double out[3]) const override { out[0] = radius; out[1] = out[2] = 0.0; }
  double radius;
};

/** geom::Box (src/shape.cpp:160-164) */
class Box : public Shape {
 public:
  Box(double Lx, double Ly, double Lz) : Shape("Cube"), Lx(Lx), Ly(Ly), Lz(Lz) {}
  bool isInside(double x, double y, double z) const override {
    transform(x, y, z);
    return (x > -Lx / 2.0) && (x < Lx / 2.0) && (y > -Ly / 2.0) && (y < Ly / 2.0) &&
           (z > -Lz / 2.0) && (z < Lz / 2.0);
  }
  int kind() const override { return PXP_SHAPE_BOX; }
  void size(double out[3]) const override { out[0] = Lx; out[1] = Ly; out[2] = Lz; }
  double Lx, Ly, Lz;
};

/** geom::Cylinder (src/shape.cpp:175-187) */
class Cylinder : public Shape {
 public:
  Cylinder(double radius, double height) : Shape("Cylinder"), r1(radius), r2(radius), height(height) {}
  Cylinder(double r1, double r2, double height) : Shape("Cylinder"), r1(r1), r2(r2), height(height) {}
  bool isInside(double x, double y, double z) const override {
    transform(x, y, z);
    bool zIsInside = (z < height / 2.0) && (z > -height / 2.0);
    if (!zIsInside) return false;
    double slope = (r2 - r1) / height;
    double radius = slope * (z + height / 2.0) + r1;
    double r = std::sqrt(x * x + y * y);
    return r < radius;
  }
  int kind() const override { return PXP_SHAPE_CYLINDER; }
  void size(double out[3]) const override { out[0] = height; out[1] = r1; out[2] = r2; }
  double r1, r2, height;
};

/** geom::Part (src/geometry.cpp:53-108): non-owning shape pointers. */
class Part {
 public:
  explicit Part(const char *name) : name(name) {}
  void add(Shape &shape) {
    shapes.push_back(&shape);
    operations.push_back(Operation_t::UNION);
  }
  void difference(Shape &shape) {
    if (shapes.empty())
      throw std::runtime_error("There is no shape to make difference with. You have to add at least one shape before...");
    shapes.push_back(&shape);
    operations.push_back(Operation_t::DIFFERENCE);
  }
  bool isInside(double x, double y, double z) const {
    for (size_t i = 0; i < shapes.size(); ++i)
      if (shapes[shapes.size() - 1 - i]->isInside(x, y, z))
        return operations[operations.size() - 1 - i] == Operation_t::UNION;
    return false;
  }
  void translate(double x, double y, double z) { for (Shape *s : shapes) s->translate(x, y, z); }
  void rotate(double deg, Axis_t axis) { for (Shape *s : shapes) s->rotate(deg, axis); }
  void scale(double f, Axis_t axis) { for (Shape *s : shapes) s->scale(f, axis); }
  std::string name;
  double delta{0.0};
  double beta{0.0};
  std::vector<Shape *> shapes;
  std::vector<Operation_t> operations;
};

/** geom::Module (src/geometry.cpp:195-234): non-owning part pointers. */
class Module {
 public:
  explicit Module(const char *name) : name(name) {}
  void add(Part &part) {
    parts.push_back(&part);
    operations.push_back(Operation_t::UNION);
  }
  void difference(Part &part) {
    if (parts.size() <= 1)
      throw std::runtime_error("There have to be at least one part present before making difference!");
    parts.push_back(&part);
    operations.push_back(Operation_t::DIFFERENCE);
  }
  bool getXrayMatProp(double x, double y, double z, double &delta, double &beta) const {
    delta = 0.0;
    beta = 0.0;
    for (size_t i = 0; i < parts.size(); ++i) {
      const Part *p = parts[parts.size() - i - 1];
      if (p->isInside(x, y, z)) {
        if (operations[parts.size() - i - 1] == Operation_t::UNION) {
          delta = p->delta;
          beta = p->beta;
        }
        return true;
      }
    }
    return false;
  }
  void translate(double x, double y, double z) { for (Part *p : parts) p->translate(x, y, z); }
  void rotate(double deg, Axis_t axis) { for (Part *p : parts) p->rotate(deg, axis); }
  void scale(double f, Axis_t axis) { for (Part *p : parts) p->scale(f, axis); }
  std::string name;
  std::vector<Part *> parts;
  std::vector<Operation_t> operations;
};
}  // namespace geom

/** CSGMaterial (include/materialFunction.hpp, src/materialFunction.cpp:3-18):
 * the first module that claims a point gives its material; evaluated on the
 * device by the CUDA 3-D solvers. */
class CSGMaterial : public MaterialFunction {
 public:
  void getXrayMatProp(double x, double y, double z, double &delta, double &beta) const override {
    delta = 0.0;
    beta = 0.0;
    if (isReferenceRun) return;
    for (const geom::Module *m : modules)
      if (m->getXrayMatProp(x, y, z, delta, beta)) return;
  }
  void addModule(const geom::Module &module) { modules.push_back(&module); }
  void setReferenceRun(bool ref) { isReferenceRun = ref; }
  std::vector<const geom::Module *> modules;
  bool isReferenceRun{false};
};

// ------------------------------------------------------------- sources ----
/** include/paraxialSource.hpp:10-59, src/paraxialSource.cpp. */
class ParaxialSource {
 public:
  enum class Dim_t { TWO_D, THREE_D };
  explicit ParaxialSource(const char *name) : name(name) {}
  virtual ~ParaxialSource() {}
  virtual cdouble get(double x, double z) const {
    throw std::runtime_error("2D version of the ParaxialSorce get function is not implemented!");
  }
  virtual cdouble get(double x, double y, double z) const {
    throw std::runtime_error("3D version of the ParaxialSource get function is not implemented!");
  }
  void setWavenumber(double k) { wavenumber = k; }
  double getWavenumber() const { return wavenumber; }
  void setWavelength(double lambda) { wavenumber = 2.0 * pi() / lambda; }
  double getWavelength() const { return 2.0 * pi() / wavenumber; }
  void setOrigin(double, double zOrig) { z0 = zOrig; }
  void setAmplitude(double amp) { amplitude = amp; }
  void setDim(Dim_t d) { dim = d; }
  Dim_t getDim() const { return dim; }
  std::string getName() const { return name; }

 protected:
  static double pi() { return std::acos(-1.0); }
  double wavenumber{0.0};
  double z0{0.0};
  double x0{0.0};
  double amplitude{1.0};
  Dim_t dim{Dim_t::TWO_D};

 private:
  std::string name;
};

/** include/gaussianBeam.hpp:6-66, src/gaussianBeam.cpp:7-63. */
class GaussianBeam : public ParaxialSource {
 public:
  GaussianBeam() : ParaxialSource("gaussianBeam") {}
  cdouble get(double x, double z) const override {
    x -= centerX;
    cdouble im(0.0, 1.0);
    double waistRatio = waist / spotSize(z - z0);
    double gaussianFactor = std::exp(-std::pow(x / spotSize(z - z0), 2));
    cdouble phaseFactor = std::exp(-im * wavenumber * z0 +
                                   0.5 * im * wavenumber * x * x * invR(z - z0) -
                                   im * guoy(z - z0));
    return amplitude * waistRatio * gaussianFactor * phaseFactor * angleFactor(angleX, x);
  }
  cdouble get(double x, double y, double z) const override {
    y -= centerY;
    double gaussY = std::exp(-std::pow(y / spotSize(z - z0), 2));
    return get(x, z) * gaussY * angleFactor(angleY, y);
  }
  void setWaist(double w) { waist = w; }
  void setCenter(double xc, double yc) {
    centerX = xc;
    centerY = yc;
  }
  void setAngleX(double a) { angleX = a; }
  void setAngleY(double a) { angleY = a; }
  double getWaist() const { return waist; }

 private:
  double waist{1.0}, centerX{0.0}, centerY{0.0}, angleX{0.0}, angleY{0.0};
  double zR() const { return pi() * waist * waist / getWavelength(); }
  double guoy(double z) const { return std::atan(z / zR()); }
  double invR(double z) const {
    double r = zR();
    return z / (z * z + r * r);
  }
  double spotSize(double z) const { return waist * std::sqrt(1.0 + std::pow(z / zR(), 2)); }
  cdouble angleFactor(double angDeg, double x) const {
    double a = angDeg * pi() / 180.0;
    cdouble im(0.0, 1.0);
    return std::exp(im * getWavenumber() * std::sin(a) * x);
  }
};

/** include/planeWave.hpp:7-25, src/planeWave.cpp:5-14. */
class PlaneWave : public ParaxialSource {
 public:
  PlaneWave() : ParaxialSource("planeWave") {}
  cdouble get(double x, double z) const override {
    cdouble im(0.0, 1.0);
    return amplitude * std::exp(im * wavenumber * x * std::sin(angleWithZAxis) - im * wavenumber * z0);
  }
  cdouble get(double x, double y, double z) const override { return get(x, z); }
  void setAngleDeg(double angle) { angleWithZAxis = angle * pi() / 180.0; }

 private:
  double angleWithZAxis{0.0};
};

/** include/arraySource.hpp: the values must match the transverse grid. */
class ArraySource : public ParaxialSource {
 public:
  ArraySource() : ParaxialSource("arraySource") {}
  void setData(const arma::cx_vec *data) { values = data; }
  const arma::cx_vec &getVec() const { return *values; }

 private:
  const arma::cx_vec *values{nullptr};
};

class ParaxialSimulation;

// -------------------------------------------------------------- solvers ----
/** include/solver.hpp:10-74 */
class Solver {
 public:
  enum class Dimension_t { TWO_D, THREE_D };
  Solver(const char *name, Dimension_t dim) : dim(dim), name(name) {}
  virtual ~Solver() { release(); }
  Dimension_t getDim() const { return dim; }
  std::string getName() const { return name; }
  virtual void setSimulator(ParaxialSimulation &g) { guide = &g; }
  const ParaxialSimulation &getSimulator() const { return *guide; }
  virtual void reset() {
    currentStep = 1;
    if (handle) pxp_reset(handle);
  }
  virtual const arma::cx_cube &getSolution3D() const {
    throw std::runtime_error("The 3D version of getSolution() is not implemented!");
  }
  virtual const arma::cx_mat &getSolution() const {
    throw std::runtime_error("The 2D version of getSolution() is not implemented!");
  }
  virtual const arma::cx_vec &getLastSolution() const {
    throw std::runtime_error("The 2D version of getLastSolution() is not implemented!");
  }
  virtual const arma::cx_mat &getLastSolution3D() const {
    throw std::runtime_error("The 3D version of getLastSolution3D() is not implemented!");
  }
  virtual void solve() {}
  virtual void step() = 0;
  virtual void setInitialConditions(const arma::cx_vec &) {}
  virtual void setInitialConditions(const arma::cx_mat &) {}
  virtual void filterInLongitudinalDirection() {}
  virtual void downSampleLongitudinalDirection() {}
  virtual void updateDimensionsOfArrays() {}
  /** Precision of the CUDA solver: PXP_FP64 (plain) or PXP_FP32 (served). */
  void setPrecision(int p) { precision = p; }
  /** The C-ABI handle behind this solver (null before the first step). */
  pxp_solver nativeHandle() const { return handle; }

 protected:
  Dimension_t dim;
  std::string name;
  ParaxialSimulation *guide{nullptr};
  unsigned int currentStep{1};
  pxp_solver handle{nullptr};
  int precision{PXP_FP64};

  void release() {
    if (handle) pxp_solver_destroy(handle);
    handle = nullptr;
  }
  void check(int status) const {
    if (status != PXP_OK) {
      char msg[1024];
      pxp_last_error(handle, msg, sizeof(msg));
      throw std::runtime_error(std::string(name) + ": " + msg + " (" +
                               pxp_status_string(status) + ")");
    }
  }
};

/** include/paraxialSimulation.hpp:28-236 (minus HDF5 and post-processing). */
class ParaxialSimulation {
 public:
  enum class Boundary_t { TOP, BOTTOM, LEFT, RIGHT };
  explicit ParaxialSimulation(const char *name) : name(name) {}
  ParaxialSimulation(const ParaxialSimulation &) = delete;
  ParaxialSimulation &operator=(const ParaxialSimulation &) = delete;
  virtual ~ParaxialSimulation() {}

  void setTransverseDiscretization(double xmin, double xmax, double step) {
    setTransverseDiscretization(xmin, xmax, step, 1);
  }
  void setTransverseDiscretization(double xmin, double xmax, double step, unsigned int ratio) {
    xDisc = {xmin, xmax, step, ratio};
    yDisc.downsamplingRatio = ratio;
  }
  void setLongitudinalDiscretization(double zmin, double zmax, double step) {
    setLongitudinalDiscretization(zmin, zmax, step, 1);
  }
  void setLongitudinalDiscretization(double zmin, double zmax, double step, unsigned int ratio) {
    zDisc = {zmin, zmax, step, ratio};
  }
  void setVerticalDiscretization(double ymin, double ymax, double step) {
    yDisc.min = ymin;
    yDisc.max = ymax;
    yDisc.step = step;
  }
  unsigned int nodeNumberTransverse() const { return pxp_node_count(xDisc.min, xDisc.max, xDisc.step); }
  unsigned int nodeNumberLongitudinal() const { return pxp_node_count(zDisc.min, zDisc.max, zDisc.step); }
  unsigned int nodeNumberVertical() const { return pxp_node_count(yDisc.min, yDisc.max, yDisc.step); }
  const Disctretization &transverseDiscretization() const { return xDisc; }
  const Disctretization &longitudinalDiscretization() const { return zDisc; }
  const Disctretization &verticalDiscretization() const { return yDisc; }

  double getWavenumber() const { return wavenumber; }
  void setWavenumber(double k) { wavenumber = k; }
  double getWavelength() const { return 2.0 * std::acos(-1.0) / wavenumber; }
  void setWaveLength(double lambda) { wavenumber = 2.0 * std::acos(-1.0) / lambda; }

  void setSolver(Solver &s) {
    solver = &s;
    solver->setSimulator(*this);
  }
  std::string getName() const { return name; }
  void step() { solver->step(); }
  virtual void solve() { solver->solve(); }
  void reset() {
    if (solver) solver->reset();
  }

  double getZ(unsigned int iz) const { return zDisc.min + iz * zDisc.step; }
  double getX(int ix) const { return xDisc.min + ix * xDisc.step; }
  double getY(int iy) const { return yDisc.min + iy * yDisc.step; }

  /** src/paraxialSimulation.cpp:356-399 */
  virtual void setBoundaryConditions(const ParaxialSource &source) {
    if (solver == nullptr) throw std::runtime_error("Solver needs to be set before boundary conditions!");
    src = &source;
    unsigned Nx = nodeNumberTransverse();
    if (source.getDim() == ParaxialSource::Dim_t::TWO_D) {
      arma::cx_vec values(Nx, 1.0);
      for (unsigned i = 0; i < Nx; ++i) values[i] = src->get(getX(i), 0.0);
      solver->setInitialConditions(values);
    } else {
      unsigned Ny = nodeNumberVertical();
      arma::cx_mat values(Nx, Ny);
      for (unsigned indx = 0; indx < Nx * Ny; ++indx) {
        unsigned i = indx / Ny, j = indx % Ny;
        values(j, i) = src->get(getX(i), getY(j), 0.0);
      }
      solver->setInitialConditions(values);
    }
    setWaveLength(source.getWavelength());
  }
  void setBoundaryConditions(const ArraySource &source) {
    src = &source;
    if (source.getVec().n_elem != nodeNumberTransverse())
      throw std::runtime_error("The size of the given array does not match the number of transverse nodes!");
    solver->setInitialConditions(source.getVec());
  }

  /** src/paraxialSimulation.cpp:513-537 */
  virtual void getXrayMatProp(double x, double z, double &delta, double &beta) const {
    if (material) {
      material->getXrayMatProp(x, 0.0, z, delta, beta);
    } else {
      delta = 0.0;
      beta = 0.0;
    }
  }
  virtual void getXrayMatProp(double x, double y, double z, double &delta, double &beta) const {
    if (material) {
      material->getXrayMatProp(x, y, z, delta, beta);
    } else {
      delta = 0.0;
      beta = 0.0;
    }
  }
  void save(const char *) {
    throw std::runtime_error("HDF5 export is not available in this build");
  }
  const Solver &getSolver() const { return *solver; }
  Solver &getSolver() { return *solver; }

  /** True when getXrayMatProp describes a medium (a material function, or
   * a simulation that overrides getXrayMatProp). */
  virtual bool hasMaterial() const { return material != nullptr; }
  /** True when delta and beta do not depend on z. */
  virtual bool materialZInvariant() const { return material == nullptr || material->zInvariant(); }

  /** src/paraxialSimulation.cpp:215-219 (conversions truncate). */
  void closestIndex(double x, double z, unsigned int &ix, unsigned int &iz) const {
    ix = (unsigned int)((x - xDisc.min) / xDisc.step);
    iz = (unsigned int)((z - zDisc.min) / zDisc.step);
  }
  /** Far-field parameters (include/farFieldParameters.hpp). */
  void setFarFieldPadValue(double padValue) { farPadValue = padValue; }
  void setFarFieldAngleRange(double phiMin, double phiMax) {
    farPhiMin = phiMin;
    farPhiMax = phiMax;
  }
  /** Value of the padded entries of the 2-D far field
   * (include/paraxialSimulation.hpp:174). */
  virtual double padExitField(double, double) const { return farPadValue; }

  std::string description{""};
  const MaterialFunction *material{nullptr};

 protected:
  Solver *solver{nullptr};
  Disctretization xDisc, zDisc, yDisc;
  double wavenumber{1.0};
  std::string name;
  const ParaxialSource *src{nullptr};
  double farPadValue{0.0}, farPhiMin{-90.0}, farPhiMax{90.0};
};

/** Base of the 2-D (one transverse dimension) solvers, include/solver2D.hpp. */
class Solver2D : public Solver {
 public:
  enum class Comp_t { REAL, IMAG };
  enum class BC_t { DIRICHLET, TRANSPARENT };
  Solver2D(const char *name, int kind) : Solver(name, Dimension_t::TWO_D), kind(kind) {}
  Solver2D(const Solver2D &) = delete;

  void setSimulator(ParaxialSimulation &g) override {
    Solver::setSimulator(g);
    release();
    Nx = g.nodeNumberTransverse();
    Nz = g.nodeNumberLongitudinal();
    unsigned ds = Nx / g.transverseDiscretization().downsamplingRatio;
    solution = arma::cx_mat(ds, Nz);
    prevSolution = arma::cx_vec(Nx);
    currentSolution = arma::cx_vec(Nx);
    currentStep = 1;
  }
  const arma::cx_mat &getSolution() const override { return solution; }
  const arma::cx_vec &getLastSolution() const override { return prevSolution; }
  void setInitialConditions(const arma::cx_vec &vec) override {
    for (unsigned i = 0; i < Nx; ++i) currentSolution(i) = vec(i);
    copyCurrentSolution(0);
    icPending = true;
  }
  void setBoundaryCondition(BC_t bc) { boundaryCondition = bc; }
  void disableLongitudinalFilter() { longitudinalFilterDisabled = true; }

  /** Per-step flux windows (pxp_set_flux_windows): the step kernels sum
   * |u|^2 with trapezoid weights over [start[k], end[k]] after step
   * first + k. */
  void setFluxWindows(unsigned first, const std::vector<unsigned> &start,
                      const std::vector<unsigned> &end) {
    initDevice();
    if (start.size() != end.size()) throw std::invalid_argument("flux windows: sizes differ");
    check(pxp_set_flux_windows(handle, (int)first, (int)start.size(), start.data(), end.data()));
  }
  std::vector<double> getFlux(unsigned first, unsigned count) const {
    std::vector<double> out(count);
    check(pxp_get_flux(handle, (int)first, (int)count, out.data()));
    return out;
  }
  /** The same sum over the current field. */
  double fieldFlux(unsigned start, unsigned end) {
    initDevice();
    double v = 0.0;
    check(pxp_field_flux(handle, start, end, &v));
    return v;
  }

  /** Solver2D::step (src/solver2D.cpp:243-250): one step, field copied back. */
  void step() override {
    initDevice();
    runSteps(currentStep, 1);
    check(pxp_get_last_solution(handle, reinterpret_cast<double *>(currentSolution.memptr())));
    copyCurrentSolution(currentStep);
    currentStep++;
  }

  /** Solver2D::solve (src/solver2D.cpp:224-241): all steps on the device,
   * the saved columns copied back once at the end. */
  void solve() override {
    initDevice();
    const unsigned first = currentStep, last = Nz - 1;
    if (first > last) return;
    runSteps(first, last - first + 1);
    int nsaved = 0;
    check(pxp_num_saved(handle, &nsaved));
    for (unsigned s = first; s <= last && (int)(s - 1) < nsaved; ++s) {
      check(pxp_get_saved(handle, (int)(s - 1), reinterpret_cast<double *>(currentSolution.memptr())));
      copyCurrentSolution(s);
    }
    currentStep = last + 1;
    if (!longitudinalFilterDisabled && guide->longitudinalDiscretization().downsamplingRatio > 1)
      throw std::runtime_error(
          "the longitudinal low-pass filter (VISA) is not available: call "
          "disableLongitudinalFilter() or use a longitudinal downsampling ratio of 1");
    if (!longitudinalFilterDisabled) downSampleLongitudinalDirection();
  }

  /** src/solver2D.cpp:267-282 */
  void downSampleLongitudinalDirection() override {
    unsigned nz = Nz / guide->longitudinalDiscretization().downsamplingRatio;
    arma::cx_mat copy(solution.n_rows, nz);
    double delta = static_cast<double>(solution.n_cols) / static_cast<double>(nz);
    for (unsigned iz = 0; iz < nz; ++iz) {
      unsigned indx = iz * delta + delta / 2.0;
      for (unsigned ix = 0; ix < copy.n_rows; ++ix) copy(ix, iz) = solution(ix, indx);
    }
    solution = copy;
  }

 protected:
  int kind;
  unsigned Nx{0}, Nz{0};
  arma::cx_mat solution;
  arma::cx_vec prevSolution, currentSolution;
  BC_t boundaryCondition{BC_t::DIRICHLET};
  bool longitudinalFilterDisabled{false};
  bool icPending{false};
  bool materialPlanes{false};

  /** src/solver2D.cpp:173-193 with a transverse ratio of 1 or a plain
   * middle-sample downsampling (the VISA filter is not applied). */
  void copyCurrentSolution(unsigned step) {
    for (unsigned i = 0; i < currentSolution.n_elem; ++i) prevSolution(i) = currentSolution(i);
    double delta = static_cast<double>(currentSolution.n_elem) / static_cast<double>(solution.n_rows);
    if (step < solution.n_cols)
      for (unsigned i = 0; i < solution.n_rows; ++i)
        solution(i, step) = currentSolution((unsigned)(delta * i + delta / 2.0));
  }

  void initDevice() {
    if (guide == nullptr) throw std::runtime_error("No waveguide specified!");
    if (handle == nullptr) {
      const ParaxialSimulation &g = *guide;
      pxp_problem p{};
      p.kind = kind;
      p.precision = precision;
      p.x = {g.transverseDiscretization().min, g.transverseDiscretization().max,
             g.transverseDiscretization().step, 1};
      p.y = p.x;
      p.z = {g.longitudinalDiscretization().min, g.longitudinalDiscretization().max,
             g.longitudinalDiscretization().step, 1};
      p.wavenumber = g.getWavenumber();
      p.transparent_bc = boundaryCondition == BC_t::TRANSPARENT;
      p.save_every = 1;
      check(pxp_solver_create(&p, &handle));
      materialPlanes = g.hasMaterial() && !g.materialZInvariant();
      if (g.hasMaterial() && !materialPlanes) {
        std::vector<double> d(Nx), b(Nx);
        for (unsigned i = 0; i < Nx; ++i) g.getXrayMatProp(g.getX(i), 0.0, d[i], b[i]);
        check(pxp_set_material_table(handle, d.data(), b.data(), Nx));
      }
    }
    if (icPending) {
      check(pxp_set_initial_conditions(handle, reinterpret_cast<const double *>(currentSolution.memptr())));
      icPending = false;
    }
  }

  /** The planes the reference samples (FFTSolver2D: z = getZ(s) + dz/2,
   * src/fftSolver2D.cpp:38; CrankNicholson: z and z - dz,
   * src/crancNicholson.cpp:29-38) for steps s = first .. first+n-1, in
   * chunks, then the steps. */
  void runSteps(unsigned first, unsigned n) {
    const ParaxialSimulation &g = *guide;
    const double dz = g.longitudinalDiscretization().step;
    const unsigned chunk = 256;
    for (unsigned s0 = first; s0 < first + n;) {
      unsigned cnt = std::min(chunk, first + n - s0);
      if (materialPlanes) {
        const unsigned per = kind == PXP_CRANK_NICHOLSON ? 2 : 1;
        std::vector<double> d((size_t)cnt * per * Nx), b(d.size());
        for (unsigned k = 0; k < cnt; ++k) {
          const unsigned s = s0 + k;
          for (unsigned pl = 0; pl < per; ++pl) {
            double z;
            if (kind == PXP_CRANK_NICHOLSON) {
              z = g.longitudinalDiscretization().min + static_cast<double>(s) * dz;
              if (pl == 1) z = z - dz;
            } else {
              z = g.getZ(s) + 0.5 * dz;
            }
            size_t off = ((size_t)k * per + pl) * Nx;
            for (unsigned i = 0; i < Nx; ++i) g.getXrayMatProp(g.getX(i), z, d[off + i], b[off + i]);
          }
        }
        check(pxp_set_material_planes(handle, d.data(), b.data(), (int)s0, (int)cnt));
      } else if (!materialPlanes && s0 == first && n > chunk) {
        cnt = n;  // z-invariant: one launch
      }
      check(pxp_step(handle, (int)cnt));
      s0 += cnt;
    }
  }
};

/** include/fftSolver2D.hpp */
class FFTSolver2D : public Solver2D {
 public:
  FFTSolver2D() : Solver2D("FFTSolver2D", PXP_FFT_SOLVER_2D) {}
};

/** include/crankNicholson.hpp */
class CrankNicholson : public Solver2D {
 public:
  CrankNicholson() : Solver2D("CrankNicholson", PXP_CRANK_NICHOLSON) {}
};

/** Base of the 3-D (two transverse dimension) solvers, include/solver3D.hpp. */
class Solver3D : public Solver {
 public:
  Solver3D(const char *name, int kind) : Solver(name, Dimension_t::THREE_D), kind(kind) {}

  /** src/solver3D.cpp:19-44 (Ny is forced to Nx) */
  void setSimulator(ParaxialSimulation &g) override {
    Solver::setSimulator(g);
    release();
    Nx = g.nodeNumberTransverse();
    Nz = g.nodeNumberLongitudinal();
    Ny = Nx;
    unsigned dx = Nx / g.transverseDiscretization().downsamplingRatio;
    unsigned dzs = Nz / g.longitudinalDiscretization().downsamplingRatio;
    prevSolution = arma::cx_mat(Ny, Nx);
    currentSolution = arma::cx_mat(Ny, Nx);
    solution = arma::cx_cube(dx, dx, dzs + 1);
    currentStep = 1;
  }
  void updateDimensionsOfArrays() override { setSimulator(*guide); }
  const arma::cx_cube &getSolution3D() const override { return solution; }
  const arma::cx_mat &getLastSolution3D() const override { return prevSolution; }

  /** src/solver3D.cpp:127-146 */
  void setInitialConditions(const arma::cx_mat &values) override {
    if (values.n_rows != currentSolution.n_rows || values.n_cols != currentSolution.n_cols)
      throw std::runtime_error("Dimension of matrices does not match!");
    std::memcpy(currentSolution.memptr(), values.memptr(), sizeof(cdouble) * values.n_elem);
    copyCurrentSolution(0);
    icPending = true;
  }

  void step() override {
    initDevice();
    runSteps(currentStep, 1);
    check(pxp_get_last_solution(handle, reinterpret_cast<double *>(currentSolution.memptr())));
    copyCurrentSolution(currentStep++);
  }

  /** src/solver3D.cpp:168-199: all steps on the device; the saved slices
   * (every longitudinal downsampling ratio steps) copied back at the end. */
  void solve() override {
    initDevice();
    const unsigned first = currentStep, last = Nz - 1;
    if (first > last) return;
    runSteps(first, last - first + 1);
    const unsigned ratio = guide->longitudinalDiscretization().downsamplingRatio;
    int nsaved = 0;
    check(pxp_num_saved(handle, &nsaved));
    for (int k = 0; k < nsaved; ++k) {
      const unsigned s = (unsigned)(k + 1) * ratio;
      if (s < first) continue;
      check(pxp_get_saved(handle, k, reinterpret_cast<double *>(currentSolution.memptr())));
      storeSlice(s / ratio);
    }
    check(pxp_get_last_solution(handle, reinterpret_cast<double *>(currentSolution.memptr())));
    std::memcpy(prevSolution.memptr(), currentSolution.memptr(), sizeof(cdouble) * currentSolution.n_elem);
    currentStep = last + 1;
  }

 protected:
  int kind;
  unsigned Nx{0}, Ny{0}, Nz{0};
  arma::cx_cube solution;
  arma::cx_mat prevSolution, currentSolution;
  bool icPending{false};
  double absorberWidth{0.0}, absorberDamping{0.0};
  bool tbc{false};
  bool materialPlanes{false};  // a user MaterialFunction, sampled per step

  /** FFTSolver3D::refraction's material at (x, y) for the step from z0 to
   * z1 (src/fftSolver3D.cpp:138-149): the value at z1, or, where it differs
   * from the value at z0 by more than 1e-10, refractionIntegral (:253-273,
   * the endpoints once, interior samples 1..8 of 10 twice, over 2*10). */
  static void refractionMaterial(const ParaxialSimulation &g, double x, double y, double z0,
                                 double z1, double &delta, double &beta) {
    const double ZERO = 1E-10;
    const unsigned nSteps = 10;
    double deltaPrev, betaPrev;
    g.getXrayMatProp(x, y, z1, delta, beta);
    g.getXrayMatProp(x, y, z0, deltaPrev, betaPrev);
    if ((std::abs(delta - deltaPrev) > ZERO) || (std::abs(beta - betaPrev) > ZERO)) {
      double deltaTemp = 0.0, betaTemp = 0.0;
      g.getXrayMatProp(x, y, z0, delta, beta);
      g.getXrayMatProp(x, y, z1, deltaTemp, betaTemp);
      delta += deltaTemp;
      beta += betaTemp;
      const double dz = (z1 - z0) / nSteps;
      for (unsigned i = 1; i < nSteps - 1; ++i) {
        g.getXrayMatProp(x, y, z0 + i * dz, deltaTemp, betaTemp);
        delta += 2.0 * deltaTemp;
        beta += 2.0 * betaTemp;
      }
      delta /= (2.0 * nSteps);
      beta /= (2.0 * nSteps);
    }
  }

  /** Steps first .. first+n-1 on the device.  With a user MaterialFunction
   * the medium is sampled on the host, per block of steps, at the planes
   * the reference samples -- FFTSolver3D: the refraction material of each
   * step (refractionMaterial); ADI: getZ(s) for the x half step and
   * getZ(s) + dz/2 for the y half step (src/alternatingDirectionSolver.cpp:
   * 21, 91) -- and handed over with pxp_set_material_planes.  Like the
   * reference's OpenMP loops, this calls the material from several threads
   * when OpenMP is enabled, so getXrayMatProp must be thread-safe. */
  void runSteps(unsigned first, unsigned n) {
    if (!materialPlanes) {
      check(pxp_step(handle, (int)n));
      return;
    }
    const ParaxialSimulation &g = *guide;
    const long long npts = (long long)Nx * Ny;
    const unsigned per = kind == PXP_ADI ? 2 : 1;
    const double dz = g.longitudinalDiscretization().step;
    // blocks of up to about 256 MB of planes
    const unsigned cap = (unsigned)std::max<long long>(1, (256ll << 20) / (16 * per * npts));
    for (unsigned s0 = first; s0 < first + n;) {
      const unsigned cnt = std::min(cap, first + n - s0);
      std::vector<double> d((size_t)cnt * per * npts), b(d.size());
      for (unsigned k = 0; k < cnt; ++k) {
        const unsigned s = s0 + k;
        for (unsigned pl = 0; pl < per; ++pl) {
          double *dp = d.data() + ((size_t)k * per + pl) * npts;
          double *bp = b.data() + ((size_t)k * per + pl) * npts;
#ifdef _OPENMP
#pragma omp parallel for
#endif
          for (long long i = 0; i < npts; ++i) {
            const unsigned col = (unsigned)(i / Ny), row = (unsigned)(i % Ny);
            const double x = g.getX((int)col), y = g.getY((int)row);
            if (kind == PXP_FFT_SOLVER_3D)
              refractionMaterial(g, x, y, g.getZ(s - 1), g.getZ(s), dp[i], bp[i]);
            else
              g.getXrayMatProp(x, y, pl == 0 ? g.getZ(s) : g.getZ(s) + dz / 2.0, dp[i], bp[i]);
          }
        }
      }
      check(pxp_set_material_planes(handle, d.data(), b.data(), (int)s0, (int)cnt));
      check(pxp_step(handle, (int)cnt));
      s0 += cnt;
    }
  }

  /** src/solver3D.cpp:78-125: block average into the saved slice. */
  void storeSlice(unsigned currZ) {
    if (currZ >= solution.n_slices) return;
    double deltaX = static_cast<double>(currentSolution.n_rows) / static_cast<double>(solution.n_rows);
    double deltaY = static_cast<double>(currentSolution.n_cols) / static_cast<double>(solution.n_cols);
    for (unsigned i = 0; i < solution.n_rows * solution.n_cols; ++i) {
      unsigned row = i % solution.n_rows, col = i / solution.n_rows;
      // submat bounds [row*deltaX, row*deltaX + deltaX - 1], truncated
      const unsigned r0 = (unsigned)(row * deltaX), r1 = (unsigned)(row * deltaX + deltaX - 1);
      const unsigned c0 = (unsigned)(col * deltaY), c1 = (unsigned)(col * deltaY + deltaY - 1);
      cdouble sum = 0.0;
      for (unsigned c = c0; c <= c1; ++c) {
        cdouble colsum = 0.0;
        for (unsigned r = r0; r <= r1; ++r) colsum += currentSolution(r, c);
        sum += colsum;
      }
      solution(row, col, currZ) = sum / (deltaX * deltaY);
    }
  }
  void copyCurrentSolution(unsigned step) {
    std::memcpy(prevSolution.memptr(), currentSolution.memptr(), sizeof(cdouble) * currentSolution.n_elem);
    if (step % guide->longitudinalDiscretization().downsamplingRatio == 0)
      storeSlice(step / guide->longitudinalDiscretization().downsamplingRatio);
  }

  /** Flattens a CSGMaterial for pxp_set_material_csg. */
  void setCsg(const CSGMaterial &cm) {
    std::vector<pxp_csg_module> mods;
    std::vector<pxp_csg_part> parts;
    std::vector<pxp_csg_shape> shapes;
    for (const geom::Module *m : cm.modules) {
      mods.push_back({(int)parts.size(), (int)m->parts.size()});
      for (size_t i = 0; i < m->parts.size(); ++i) {
        const geom::Part *p = m->parts[i];
        pxp_csg_part cp{};
        cp.operation = m->operations[i] == geom::Operation_t::UNION ? PXP_CSG_UNION : PXP_CSG_DIFFERENCE;
        cp.first_shape = (int)shapes.size();
        cp.num_shapes = (int)p->shapes.size();
        cp.delta = p->delta;
        cp.beta = p->beta;
        parts.push_back(cp);
        for (size_t k = 0; k < p->shapes.size(); ++k) {
          pxp_csg_shape cs{};
          cs.kind = p->shapes[k]->kind();
          cs.operation = p->operations[k] == geom::Operation_t::UNION ? PXP_CSG_UNION : PXP_CSG_DIFFERENCE;
          std::memcpy(cs.transform, p->shapes[k]->transformation, sizeof(cs.transform));
          p->shapes[k]->size(cs.size);
          shapes.push_back(cs);
        }
      }
    }
    check(pxp_set_material_csg(handle, mods.data(), (int)mods.size(), parts.data(), (int)parts.size(),
                               shapes.data(), (int)shapes.size()));
  }

  void initDevice() {
    if (guide == nullptr) throw std::runtime_error("No waveguide specified!");
    if (handle == nullptr) {
      const ParaxialSimulation &g = *guide;
      pxp_problem p{};
      p.kind = kind;
      p.precision = precision;
      p.x = {g.transverseDiscretization().min, g.transverseDiscretization().max,
             g.transverseDiscretization().step, 1};
      p.y = {g.verticalDiscretization().min, g.verticalDiscretization().max,
             g.verticalDiscretization().step, 1};
      p.z = {g.longitudinalDiscretization().min, g.longitudinalDiscretization().max,
             g.longitudinalDiscretization().step, 1};
      p.wavenumber = g.getWavenumber();
      p.transparent_bc = tbc ? 1 : 0;
      p.absorber_width = absorberWidth;
      p.absorber_damping = absorberDamping;
      p.save_every = (int)g.longitudinalDiscretization().downsamplingRatio;
      check(pxp_solver_create(&p, &handle));
      materialPlanes = false;
      if (g.material != nullptr) {
        const SphereMaterial *sm = dynamic_cast<const SphereMaterial *>(g.material);
        const CSGMaterial *cm = dynamic_cast<const CSGMaterial *>(g.material);
        if (sm != nullptr) {
          std::vector<pxp_sphere> sp;
          for (const auto &s : sm->spheres) sp.push_back({s.cx, s.cy, s.cz, s.radius, s.delta, s.beta});
          check(pxp_set_material_spheres(handle, sp.data(), (int)sp.size()));
        } else if (cm != nullptr) {
          if (!cm->isReferenceRun) setCsg(*cm);
        } else if (g.material->zInvariant()) {
          // any z: the table serves every step and both half steps
          std::vector<double> d((size_t)Nx * Ny), b(d.size());
          for (unsigned col = 0; col < Nx; ++col)
            for (unsigned row = 0; row < Ny; ++row)
              g.getXrayMatProp(g.getX((int)col), g.getY((int)row), g.getZ(1),
                               d[(size_t)col * Ny + row], b[(size_t)col * Ny + row]);
          check(pxp_set_material_table(handle, d.data(), b.data(), d.size()));
        } else {
          materialPlanes = true;  // sampled per step (runSteps)
        }
      }
    }
    if (icPending) {
      check(pxp_set_initial_conditions(handle, reinterpret_cast<const double *>(currentSolution.memptr())));
      icPending = false;
    }
  }
};

/** include/fftSolver3D.hpp */
class FFTSolver3D : public Solver3D {
 public:
  FFTSolver3D() : Solver3D("FFTSolver3D", PXP_FFT_SOLVER_3D) {}
  /** src/fftSolver3D.cpp:327-349 */
  void absorbingBC(double width, double dampingLength) {
    if (guide == nullptr)
      throw std::runtime_error("No waveguide set! The solver needs first to be passed to a waveguide object. Then call this function!");
    if (handle != nullptr)
      throw std::runtime_error("absorbingBC must be called before the first step");
    absorberWidth = width;
    absorberDamping = dampingLength;
  }
  void reset() override { Solver::reset(); }
};

/** include/alternatingDirectionSolver.hpp */
class ADI : public Solver3D {
 public:
  ADI() : Solver3D("ADI", PXP_ADI) {}
  /** If true transparent boundary conditions are used, otherwise Dirichlet. */
  bool useTBC{true};
  void step() override {
    syncTbc();
    Solver3D::step();
  }
  void solve() override {
    syncTbc();
    Solver3D::solve();
  }

 private:
  void syncTbc() {
    if (handle == nullptr)
      tbc = useTBC;
    else if (tbc != useTBC)
      throw std::runtime_error("useTBC changed after the first step");
  }
};

// ---------------------------------------------------- post-processing ----
namespace post {

/** post::FarField (include/postProcessMod.hpp:68-123, src/farFieldPost.cpp),
 * computed on the device by pxp_farfield. */
class FarField {
 public:
  enum class Pad_t { ZERO, LINEAR_FIT, CONSTANT };
  void setPadding(Pad_t padType) { padding = padType; }
  void setPadLength(unsigned int pad) { signalLength = pad; }
  void setReference(const arma::cx_mat &ref) { reference = &ref; }
  void setAngleRange(double angMin, double angMax) {
    phiMin = angMin;
    phiMax = angMax;
  }
  void linkParaxialSim(const ParaxialSimulation &simulation) { sim = &simulation; }
  double getMaxScatteringAngle() const { return phiMax; }
  double getMinScatteringAngle() const { return phiMin; }
  /** PostProcessingModule::setExportDimensions (src/postProcessing.cpp:51-56) */
  void setExportDimensions(unsigned int nrows, unsigned int ncols) {
    exportRows = nrows;
    exportCols = ncols;
    resizeMatrices = true;
  }
  /** src/farFieldPost.cpp:323-333 */
  void verifyConsistentAngles(double dx, double dy, double wavenumber) const {
    double d = dx > dy ? dy : dx;
    double PI = std::acos(-1.0);
    double qmax = PI / d;
    double alphaMax = 2.0 * std::asin(qmax / wavenumber);
    if (alphaMax * 180.0 / PI < phiMax)
      throw std::runtime_error("The specified scattering angle is to large. Increase the spatial resolution!");
  }
  /** Amplitude of the far field of a 2-D solver (:22-62). */
  void result(const Solver &solver, arma::vec &res) {
    pxp_farfield_params p = params();
    p.pad_value_re = sim ? sim->padExitField(0.0, 0.0) : 0.0;
    run(solver, p, res);
  }
  /** Far field of a 3-D solver (:141-247). */
  void result(const Solver &solver, arma::mat &res) {
    pxp_farfield_params p = params();
    pxp_solver h = solver.nativeHandle();
    if (h == nullptr) throw std::runtime_error("FarField: the solver has not run");
    if (reference != nullptr) {
      if (pxp_set_reference(h, reinterpret_cast<const double *>(reference->memptr())) != PXP_OK)
        throw std::runtime_error("FarField: the reference does not match the solver's grid");
      p.subtract_reference = 1;
    }
    run(solver, p, res);
  }

 private:
  unsigned int signalLength{0};
  double phiMin{-90.0};
  double phiMax{90.0};
  const ParaxialSimulation *sim{nullptr};
  Pad_t padding{Pad_t::ZERO};
  const arma::cx_mat *reference{nullptr};
  unsigned int exportRows{0}, exportCols{0};
  bool resizeMatrices{false};

  pxp_farfield_params params() const {
    pxp_farfield_params p;
    pxp_farfield_defaults(&p);
    p.pad_length = signalLength;
    p.phi_min = phiMin;
    p.phi_max = phiMax;
    p.padding = padding == Pad_t::ZERO ? PXP_PAD_ZERO
                                       : (padding == Pad_t::CONSTANT ? PXP_PAD_CONSTANT : PXP_PAD_LINEAR_FIT);
    if (resizeMatrices) {
      p.export_rows = exportRows;
      p.export_cols = exportCols;
    }
    return p;
  }
  void run(const Solver &solver, const pxp_farfield_params &p, arma::Mat<double> &res) const {
    pxp_solver h = solver.nativeHandle();
    if (h == nullptr) throw std::runtime_error("FarField: the solver has not run");
    unsigned rows = 0, cols = 0;
    int rc = pxp_farfield_shape(h, &p, &rows, &cols);
    if (rc == PXP_OK) {
      res.set_size(rows, cols);
      rc = pxp_farfield(h, &p, res.memptr());
    }
    if (rc != PXP_OK) {
      char msg[512];
      pxp_last_error(h, msg, sizeof(msg));
      throw std::runtime_error(std::string("FarField: ") + msg);
    }
  }
};

class Transmittivity;
}  // namespace post

// ------------------------------------------------------------ waveguides ----
/** Cladding (include/cladding.hpp, src/cladding.cpp): a refractive index. */
class Cladding {
 public:
  void setRefractiveIndex(double newdelta, double newbeta) {
    delta = newdelta;
    beta = newbeta;
  }
  /** src/cladding.cpp:7-16 */
  void setElectronDensity(double eDensity) {
    electronDensity = eDensity;
    potential = 4.0 * std::acos(-1.0) * thomsonScatteringLength * electronDensity;
  }
  double getDelta() const { return delta; }
  double getBeta() const { return beta; }
  double getPotential() const { return potential; }
  double delta{0.0};
  double beta{0.0};
  double thomsonScatteringLength{2.8179403267E-6};
  double electronDensity{0.0};

 private:
  double potential{0.0};
};

/** WaveGuideFDSimulation (include/waveGuideFDSimulation.hpp,
 * src/waveGuideFDSimulation.cpp:219-265): a 2-D simulation whose medium is a
 * waveguide in a cladding, sampled per step (it depends on z).  The border
 * tracker, the HDF5 datasets and the control-file set-up are not provided. */
class WaveGuideFDSimulation : public ParaxialSimulation {
 public:
  explicit WaveGuideFDSimulation(const char *name) : ParaxialSimulation(name) {}
  void setCladding(const Cladding &clad) { cladding = &clad; }
  void setInsideMaterial(const Cladding &mat) { insideMaterial = &mat; }
  void setWaveguideLength(double wgl) { wglength = wgl; }
  virtual bool isInsideGuide(double x, double z) const = 0;
  virtual bool waveguideEnded(double, double z) const { return z > wglength; }
  bool hasMaterial() const override { return true; }
  bool materialZInvariant() const override { return false; }
  void getXrayMatProp(double x, double z, double &delta, double &beta) const override {
    if (cladding == nullptr) throw std::runtime_error("No cladding set!");
    const double dx = xDisc.step, dz = zDisc.step;
    if (waveguideEnded(x, z)) {
      beta = 0.0;
      delta = 0.0;
      return;
    }
    bool isInside = isInsideGuide(x, z);
    bool neighboursAreInside = isInsideGuide(x + dx, z) && isInsideGuide(x - dx, z) &&
                               isInsideGuide(x, z + dz) && isInsideGuide(x, z - dz);
    double betaInside = 0.0, deltaInside = 0.0;
    if (insideMaterial != nullptr) {
      betaInside = insideMaterial->getBeta();
      deltaInside = insideMaterial->getDelta();
    }
    if (isInside && neighboursAreInside) {
      beta = betaInside;
      delta = deltaInside;
      return;
    } else if (isInside && !neighboursAreInside) {
      delta = 0.5 * (cladding->getDelta() + deltaInside);
      beta = 0.5 * (cladding->getBeta() + betaInside);
      return;
    }
    delta = cladding->getDelta();
    beta = cladding->getBeta();
  }
  void getXrayMatProp(double x, double, double z, double &delta, double &beta) const override {
    getXrayMatProp(x, z, delta, beta);
  }

 protected:
  const Cladding *cladding{nullptr};
  const Cladding *insideMaterial{nullptr};
  double wglength{1E10};
};

class CurvedWaveGuideFD;

namespace post {
/** post::Transmittivity (include/transmittivity.hpp, src/transmittivity.cpp):
 * |u|^2 integrated over the waveguide after every step, relative to the
 * integral over [0, width] after the first step.  The step kernels compute
 * the per-step trapezoid sums (pxp_set_flux_windows); the dx/2 factors and
 * the ratio are applied here. */
class Transmittivity {
 public:
  const std::vector<double> &get() const { return transmission; }
  double getIntensityAtZero() const { return intensityAtZero; }

 private:
  friend class ::CurvedWaveGuideFD;
  std::vector<double> transmission;
  double intensityAtZero{1E80};
};
}  // namespace post

/** CurvedWaveGuideFD (include/curvedWaveGuide2D.hpp, src/curvedWaveGuide2D.cpp):
 * a waveguide of width `width` bent with radius R, inner wall
 * x = -z^2/(2R).  solve() steps it on the device with the transmittivity
 * fused into the step kernels. */
class CurvedWaveGuideFD : public WaveGuideFDSimulation {
 public:
  CurvedWaveGuideFD() : CurvedWaveGuideFD("CurvedWaveGuide2D") {}
  explicit CurvedWaveGuideFD(const char *name) : WaveGuideFDSimulation(name) {}
  void setRadiusOfCurvature(double newR) { R = newR; }
  void setWidth(double newWidth) { width = newWidth; }
  double getWidth() const { return width; }
  double getRadiusOfCurvature() const { return R; }
  void useSmoothedWG() { useSmoothed = true; }
  /** src/curvedWaveGuide2D.cpp:49-52 */
  bool isInsideGuide(double x, double z) const override {
    return (2.0 * x * R + z * z > 0.0) && (2.0 * x * R + z * z < 2.0 * width * R);
  }
  /** src/curvedWaveGuide2D.cpp:61-69 */
  double waveGuideStartX(double z) const { return -0.5 * z * z / R; }
  double waveGuideEndX(double z) const { return waveGuideStartX(z) + width; }
  /** src/curvedWaveGuide2D.cpp:178-193 */
  double smoothedWG(double x, double z) const {
    double w = 0.1 * width;
    double d = 2.0 * R * x + z * z;
    double f1 = 1.0 / (1.0 + std::exp(-d / w));
    double f2 = 1.0 / (1.0 + std::exp((2 * R * width - d) / w));
    return 1.0 - (f1 - f2);
  }
  /** src/curvedWaveGuide2D.cpp:195-205 */
  void getXrayMatProp(double x, double z, double &delta, double &beta) const override {
    if (!useSmoothed) {
      WaveGuideFDSimulation::getXrayMatProp(x, z, delta, beta);
      return;
    }
    delta = cladding->getDelta() * smoothedWG(x, z);
    beta = cladding->getBeta() * smoothedWG(x, z);
  }
  using WaveGuideFDSimulation::getXrayMatProp;
  const post::Transmittivity &getTransmittivity() const { return transmittivity; }

  /** src/curvedWaveGuide2D.cpp:207-219 with Transmittivity::compute
   * (src/transmittivity.cpp:43-83) at every step. */
  void solve() override {
    Solver2D *s2 = dynamic_cast<Solver2D *>(solver);
    if (s2 == nullptr) throw std::runtime_error("CurvedWaveGuideFD needs a 2-D solver");
    const unsigned Nz = nodeNumberLongitudinal(), Nx = nodeNumberTransverse();
    if (Nz < 2) return;
    std::vector<unsigned> a(Nz - 1), b(Nz - 1);
    unsigned iz;
    for (unsigned n = 1; n < Nz; ++n) {
      const double z = getZ(n);
      closestIndex(waveGuideStartX(z), z, a[n - 1], iz);
      closestIndex(waveGuideEndX(z), z, b[n - 1], iz);
      if (waveGuideStartX(z) < xDisc.min || a[n - 1] > b[n - 1] || b[n - 1] >= Nx)
        throw std::runtime_error("the waveguide leaves the transverse grid at z = " + std::to_string(z));
    }
    s2->setFluxWindows(1, a, b);
    s2->step();
    unsigned z0, z1;
    closestIndex(0.0, 0.0, z0, iz);
    closestIndex(width, 0.0, z1, iz);
    if (z0 > z1 || z1 >= Nx) throw std::runtime_error("the waveguide's entrance is outside the grid");
    transmittivity.intensityAtZero = integral(s2->fieldFlux(z0, z1), z0, z1);
    s2->solve();
    const std::vector<double> sums = s2->getFlux(1, Nz - 1);
    transmittivity.transmission.resize(Nz - 1);
    for (unsigned n = 1; n < Nz; ++n)
      transmittivity.transmission[n - 1] =
          integral(sums[n - 1], a[n - 1], b[n - 1]) / transmittivity.intensityAtZero;
  }

 private:
  double R{1.0};
  double width{1.0};
  bool useSmoothed{false};
  post::Transmittivity transmittivity;

  /** trapezoidalIntegrateIntensityZ (src/transmittivity.cpp:30-41) from
   * the weighted sum. */
  double integral(double sum, unsigned ixStart, unsigned ixEnd) const {
    double dx = (getX(ixEnd) - getX(ixStart)) / static_cast<double>(ixEnd - ixStart);
    return sum * dx * 0.5;
  }
};

// -------------------------------------------------------------- scattering ----
/** GenericScattering (include/genericScattering.hpp, src/genericScattering.cpp):
 * a Gaussian beam through a 3-D object, first in vacuum with three steps
 * (the reference run whose exit field the far field subtracts), then through
 * the material.  Any MaterialFunction works: a SphereMaterial or a
 * CSGMaterial is evaluated on the device, other materials are sampled on the
 * host at the planes the reference samples (Solver3D::runSteps);
 * real-time visualisation, image export and the projection solver are not
 * provided. */
class GenericScattering : public ParaxialSimulation {
 public:
  enum class SolverType_t { ADI, FFT, PROJ };
  explicit GenericScattering(const char *name) : ParaxialSimulation(name) {
    gbeam.setDim(ParaxialSource::Dim_t::THREE_D);
  }
  void setMaterial(const MaterialFunction &mat) { userMaterial = &mat; }
  void setBeamWaist(double w) { gbeam.setWaist(w); }
  void setMaxScatteringAngle(double anglemax) { ff.setAngleRange(-anglemax, anglemax); }
  /** GenericScattering::getFarField (src/genericScattering.cpp:235-238) */
  void getFarField(arma::mat &farF) { ff.result(*solver, farF); }
  const arma::cx_mat &getReference() const { return reference; }

  /** src/genericScattering.cpp:21-135 */
  void init() {
    reset();
    ff.setPadLength(FFTPadLength);
    ff.setExportDimensions(exportNx, exportNy);
    setTransverseDiscretization(xmin, xmax, dx, downSampleX);
    setVerticalDiscretization(ymin, ymax, dy);
    setLongitudinalDiscretization(zmin, zmax, (zmax - zmin) / 3.0, 1);
    setWaveLength(wavelength);
    gbeam.setWavelength(wavelength);
    switch (propagator) {
      case SolverType_t::ADI: setSolver(adisolver); break;
      case SolverType_t::FFT: setSolver(fft3Dsolver); break;
      case SolverType_t::PROJ: throw std::runtime_error("the projection solver is not provided");
    }
    material = nullptr;  // reference run: vacuum
    setBoundaryConditions(gbeam);
    ff.linkParaxialSim(*this);
    ff.verifyConsistentAngles(dx, dy, wavenumber);
  }

  /** src/genericScattering.cpp:148-213 */
  void solve() override {
    if (userMaterial == nullptr) throw std::runtime_error("No material set!");
    init();
    ParaxialSimulation::solve();
    reference = solver->getLastSolution3D();
    if (subtract_reference) ff.setReference(reference);
    reset();
    material = userMaterial;
    setLongitudinalDiscretization(zmin, zmax, dz, downSampleZ);
    solver->updateDimensionsOfArrays();
    setBoundaryConditions(gbeam);
    ParaxialSimulation::solve();
  }

  unsigned int exportNx{512};
  unsigned int exportNy{512};
  unsigned int FFTPadLength{1024};
  double xmin{-1.0};
  double xmax{1.0};
  double ymin{-1.0};
  double ymax{1.0};
  double zmin{-1.0};
  double zmax{1.0};
  double dx{0.1};
  double dy{0.1};
  double dz{0.1};
  unsigned int downSampleX{1};
  unsigned int downSampleY{1};
  unsigned int downSampleZ{1};
  double wavelength{0.1569};
  bool subtract_reference{true};
  SolverType_t propagator{SolverType_t::FFT};
  bool supressMessages{false};

 private:
  const MaterialFunction *userMaterial{nullptr};
  post::FarField ff;
  GaussianBeam gbeam;
  FFTSolver3D fft3Dsolver;
  ADI adisolver;
  arma::cx_mat reference;
};
