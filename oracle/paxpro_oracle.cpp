// paxpro_oracle.cpp -- CPU oracle for the paraxial propagation step.
//
// TEST INFRASTRUCTURE ONLY (see paxpro_oracle.h).  Never linked into or
// called by the product path.
//
// The reference computes in std::complex<double> with GCC at -O3, no -march
// flag (CMakeLists.txt:4-7), so no FMA contraction.  This file restates each
// step with the same std::complex operations in the same order, built with
// -ffp-contract=off, so that for identical inputs the oracle's coefficients
// match the reference's bit for bit wherever the reference's arithmetic does
// not pass through FFTW.  Each function cites the reference lines it follows.
// The FFT itself is our own radix-2 transform (a direct DFT for other
// lengths; FFTW3 is not available), so
// FFT-based results agree with the reference to rounding, not bit for bit.

#include "paxpro_oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// geom::Shape::transform (src/shape.cpp:59-70): the 4x4 matrix times
// (x, y, z, 1), each row summed left to right.
void csg_transform(const double *T, double &x, double &y, double &z) {
  const double x0 = x, y0 = y, z0 = z;
  x = T[0] * x0 + T[1] * y0 + T[2] * z0 + T[3] * 1.0;
  y = T[4] * x0 + T[5] * y0 + T[6] * z0 + T[7] * 1.0;
  z = T[8] * x0 + T[9] * y0 + T[10] * z0 + T[11] * 1.0;
}

// Sphere / Box / Cylinder::isInside (src/shape.cpp:146-187).
bool csg_shape_inside(const orc_csg_shape &s, double x, double y, double z) {
  csg_transform(s.transform, x, y, z);
  if (s.kind == 0) {
    double r = std::sqrt(x * x + y * y + z * z);
    return r < s.size[0];
  }
  if (s.kind == 1) {
    const double Lx = s.size[0], Ly = s.size[1], Lz = s.size[2];
    return (x > -Lx / 2.0) && (x < Lx / 2.0) && (y > -Ly / 2.0) && (y < Ly / 2.0) &&
           (z > -Lz / 2.0) && (z < Lz / 2.0);
  }
  const double height = s.size[0], r1 = s.size[1], r2 = s.size[2];
  bool zIsInside = (z < height / 2.0) && (z > -height / 2.0);
  if (!zIsInside) return false;
  double slope = (r2 - r1) / height;
  double radius = slope * (z + height / 2.0) + r1;
  double r = std::sqrt(x * x + y * y);
  return r < radius;
}

// geom::Part::isInside (src/geometry.cpp:91-108): shapes from the last to
// the first; the first containing the point decides by its operation.
bool csg_part_inside(const orc_csg_shape *shapes, const orc_csg_part &p, double x,
                            double y, double z) {
  for (int i = p.num_shapes - 1; i >= 0; --i) {
    const orc_csg_shape &s = shapes[p.first_shape + i];
    if (csg_shape_inside(s, x, y, z)) return s.operation == 0;
  }
  return false;
}


using cd = std::complex<double>;
const double PI = std::acos(-1.0);  // src/fftSolver2D.cpp:7

int g_threads = 0;

int nthreads() {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------------------------- grid --
// src/paraxialSimulation.cpp:107-120 (node count), :250-263 (coordinates)
unsigned node_count(double mn, double mx, double st) {
  return (unsigned)((mx - mn) / st + 1.0);
}
double get_x(const orc_grid &g, int ix) { return g.xmin + ix * g.dx; }
double get_y(const orc_grid &g, int iy) { return g.ymin + iy * g.dy; }
double get_z(const orc_grid &g, unsigned iz) { return g.zmin + iz * g.dz; }

// ------------------------------------------------------------ material --
// Config materials (the build's own definitions; the reference supplies
// materials through MaterialFunction::getXrayMatProp, include/
// materialFunction.hpp:9).  Waveguide: index-based absorbing ramp, then a
// vacuum core |x| <= w, cladding elsewhere.  Spheres: first sphere with
// dx^2+dy^2+dz^2 < R^2 wins (Examples/sphere.cpp:13-14 form).
void material_eval(const orc_material *m, const orc_grid &g, double x, double y,
                   double z, double &delta, double &beta) {
  delta = 0.0;
  beta = 0.0;
  if (m == nullptr) return;
  switch (m->kind) {
    case ORC_MAT_WAVEGUIDE: {
      double fidx = std::floor((x - g.xmin) / g.dx + 0.5);
      long ix = (long)fidx;
      long n = m->n_transverse;
      long d = ix < (n - 1 - ix) ? ix : (n - 1 - ix);
      if (d < m->ramp_points) {
        delta = m->delta_clad;
        beta = m->beta_clad + (m->ramp_beta - m->beta_clad) *
                                  (double)(m->ramp_points - d) /
                                  (double)m->ramp_points;
      } else if (std::fabs(x) <= m->core_half_width) {
        delta = 0.0;
        beta = 0.0;
      } else {
        delta = m->delta_clad;
        beta = m->beta_clad;
      }
      return;
    }
    case ORC_MAT_SPHERES: {
      for (int s = 0; s < m->n_spheres; ++s) {
        const orc_sphere &sp = m->spheres[s];
        double dx = x - sp.cx, dy = y - sp.cy, dz = z - sp.cz;
        double rsq = dx * dx + dy * dy + dz * dz;
        if (rsq < sp.radius * sp.radius) {
          delta = sp.delta;
          beta = sp.beta;
          return;
        }
      }
      return;
    }
    case ORC_MAT_CSG: {
      // CSGMaterial::getXrayMatProp: the first module that claims the point
      for (int mi = 0; mi < m->n_csg_modules; ++mi) {
        const orc_csg_module &mod = m->csg_modules[mi];
        // geom::Module::getXrayMatProp (src/geometry.cpp:212-234): parts
        // from the last to the first
        for (int pi = mod.num_parts - 1; pi >= 0; --pi) {
          const orc_csg_part &part = m->csg_parts[mod.first_part + pi];
          if (csg_part_inside(m->csg_shapes, part, x, y, z)) {
            if (part.operation == 0) {
              delta = part.delta;
              beta = part.beta;
            }
            return;
          }
        }
      }
      return;
    }
    case ORC_MAT_XTABLE: {
      double fidx = std::floor((x - g.xmin) / g.dx + 0.5);
      long ix = (long)fidx;
      if (ix >= 0 && ix < m->n_transverse) {
        delta = m->delta_table[ix];
        beta = m->beta_table[ix];
      }
      return;
    }
    default:
      return;
  }
}

// ----------------------------------------------------------------- FFT --
// Radix-2 decimation-in-time FFT with twiddles computed in long double.
// Stands in for FFTW3 (fftw_plan_dft_1d/2d, FFTW_ESTIMATE,
// src/fftSolver2D.cpp:68-69, src/fftSolver3D.cpp:61-62): same sign
// convention (FORWARD = exp(-i...)), unnormalised.
struct Twiddles {
  std::vector<cd> w;  // exp(-2 pi i k / n), k < n/2
};
std::mutex g_tw_mutex;
std::map<int, Twiddles> g_tw;

const Twiddles &twiddles(int n) {
  std::lock_guard<std::mutex> lk(g_tw_mutex);
  auto it = g_tw.find(n);
  if (it != g_tw.end()) return it->second;
  Twiddles t;
  t.w.resize(n / 2 > 0 ? n / 2 : 1);
  const long double pi_l = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n / 2; ++k) {
    long double a = -2.0L * pi_l * (long double)k / (long double)n;
    t.w[k] = cd((double)cosl(a), (double)sinl(a));
  }
  return g_tw.emplace(n, std::move(t)).first->second;
}

bool is_pow2(long n) { return n >= 1 && (n & (n - 1)) == 0; }

// Strided in-place FFT over n elements at data[i*stride].
void fft_strided(cd *data, int n, long stride, int sign, cd *scratch) {
  for (int i = 0; i < n; ++i) scratch[i] = data[(long)i * stride];
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  for (int i = 0; i < n; ++i) {
    unsigned r = 0;
    for (int b = 0; b < lg; ++b)
      if (i & (1 << b)) r |= 1u << (lg - 1 - b);
    if ((int)r > i) std::swap(scratch[i], scratch[r]);
  }
  const Twiddles &tw = twiddles(n);
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1;
    int step = n / len;
    for (int s = 0; s < n; s += len) {
      for (int j = 0; j < half; ++j) {
        cd w = tw.w[(long)j * step];
        if (sign > 0) w = std::conj(w);
        cd a = scratch[s + j];
        cd b = scratch[s + j + half] * w;
        scratch[s + j] = a + b;
        scratch[s + j + half] = a - b;
      }
    }
  }
  for (int i = 0; i < n; ++i) data[(long)i * stride] = scratch[i];
}

// A length that is not a power of two: the plain DFT sum_j x_j w^(j k),
// w = exp(sign 2 pi i / n), each factor taken from an n-entry table built
// in extended precision at the exact index (j k) mod n (O(n^2); the lengths
// the tests use are a few thousand at most).
void dft_direct(cd *data, int n, int sign) {
  std::vector<cd> w(n), out(n);
  const long double pi_l = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < n; ++m) {
    const long double a = (long double)sign * 2.0L * pi_l * (long double)m / (long double)n;
    w[m] = cd((double)cosl(a), (double)sinl(a));
  }
  for (int k = 0; k < n; ++k) {
    cd acc(0.0, 0.0);
    long idx = 0;
    for (int j = 0; j < n; ++j) {
      acc += data[j] * w[idx];
      idx += k;
      if (idx >= n) idx -= n;
    }
    out[k] = acc;
  }
  std::copy(out.begin(), out.end(), data);
}

void fft_1d(cd *data, int n, int sign) {
  if (!is_pow2(n)) {
    dft_direct(data, n, sign);
    return;
  }
  std::vector<cd> scratch(n);
  fft_strided(data, n, 1, sign, scratch.data());
}

// 2-D transform of a column-major nrows x ncols buffer (both dims), as
// fftw_plan_dft_2d on the same buffer (src/fftSolver3D.cpp:61-62).  The
// reference never enables FFTW threads, so by default this runs on one
// thread; g_fft_parallel lets the best-effort CPU baseline use OpenMP.
int g_fft_parallel = 0;

void fft_2d(cd *data, int nrows, int ncols, int sign) {
  int th = g_fft_parallel ? nthreads() : 1;
  if (!is_pow2(nrows) || !is_pow2(ncols)) {
    // other lengths: the direct DFT per line, contiguous lines first, then
    // each strided line gathered, transformed and scattered back
#pragma omp parallel num_threads(th)
    {
      std::vector<cd> line(nrows > ncols ? nrows : ncols);
#pragma omp for
      for (int c = 0; c < ncols; ++c) fft_1d(data + (long)c * nrows, nrows, sign);
#pragma omp for
      for (int r = 0; r < nrows; ++r) {
        for (int c = 0; c < ncols; ++c) line[c] = data[(long)c * nrows + r];
        fft_1d(line.data(), ncols, sign);
        for (int c = 0; c < ncols; ++c) data[(long)c * nrows + r] = line[c];
      }
    }
    return;
  }
#pragma omp parallel num_threads(th)
  {
    std::vector<cd> scratch(nrows > ncols ? nrows : ncols);
#pragma omp for
    for (int c = 0; c < ncols; ++c)
      fft_strided(data + (long)c * nrows, nrows, 1, sign, scratch.data());
#pragma omp for
    for (int r = 0; r < nrows; ++r)
      fft_strided(data + r, ncols, nrows, sign, scratch.data());
  }
}

// -------------------------------------------------------------- Thomas --
// include/thomasAlgorithm.tpp:2-32.  Symmetric off-diagonals; solution in
// diag, rhs modified.
void thomas(cd *diag, const cd *subdiag, cd *rhs, unsigned n) {
  std::vector<cd> sup(subdiag, subdiag + (n - 1));
  sup[0] /= diag[0];
  rhs[0] /= diag[0];
  for (unsigned i = 1; i < n; ++i) {
    if (i < n - 1) sup[i] /= (diag[i] - subdiag[i - 1] * sup[i - 1]);
    rhs[i] = (rhs[i] - subdiag[i - 1] * rhs[i - 1]) /
             (diag[i] - subdiag[i - 1] * sup[i - 1]);
  }
  diag[n - 1] = rhs[n - 1];
  for (int i = (int)n - 2; i >= 0; --i) diag[i] = rhs[i] - sup[i] * diag[i + 1];
}

// The ADI half step's Thomas solve (src/alternatingDirectionSolver.cpp:60,
// 124): the reference runs include/thomasAlgorithm.tpp over one chain of
// nsys*len unknowns whose sub-diagonal is exactly zero between systems.  At a
// system's first row the chain's terms sub*sup and sub*rhs are then complex
// zeros, so its divisions equal a fresh solve's; at a system's last row sup
// is 0/den and the back substitution leaves rhs as it is.  Solving each
// system on its own therefore gives the chain's values (pinned bit for bit
// against the reference's own ADI in the tests), and the systems run in
// parallel.
void thomas_systems(cd *diag, const cd *subdiag, cd *rhs, unsigned nsys, unsigned len, int th) {
#pragma omp parallel for num_threads(th)
  for (long s = 0; s < (long)nsys; ++s)
    thomas(diag + s * len, subdiag + s * len, rhs + s * len, len);
}

// --------------------------------------------------------- FFTSolver2D --
// src/fftSolver2D.cpp:15-19 (kernel), :52-59 (spatialFreq)
double spatial_freq(unsigned indx, unsigned size, double step) {
  if (indx > size / 2) indx = size - indx;
  return 2.0 * PI * indx / (step * size);
}

cd kernel_2d(double kx, double dz, double k) {
  cd A(0.0, 0.5 * dz / k);
  return std::exp(-A * kx * kx);
}

// src/fftSolver3D.cpp:24-30
cd kernel_3d(double kx, double ky, double dz, double k) {
  cd A(0.0, 0.5 * dz / k);
  return std::exp(-A * (kx * kx + ky * ky));
}

[[maybe_unused]] cd transmission(double k, double beta, double delta, double dz) {
  cd im(0.0, 1.0);
  return std::exp(-k * (beta + im * delta) * dz);
}

void save_field(const cd *field, long n, int step, int save_every,
                double *saves) {
  if (save_every <= 0 || saves == nullptr) return;
  if (step % save_every != 0) return;
  long slot = step / save_every - 1;
  std::memcpy(saves + 2 * slot * n, field, sizeof(cd) * n);
}

}  // namespace

// The (delta, beta) FFTSolver3D::refraction applies at (x, y) for the step
// from z0 to z1 (src/fftSolver3D.cpp:122-156): the material at z1, or, where
// it differs from the material at z0 by more than 1e-10, refractionIntegral
// (:253-273): endpoints once, the interior samples i = 1..8 of 10 twice (the
// ninth is skipped), divided by 2*10.
void fft3d_point_material(const orc_material *m, const orc_grid &g, double x, double y, double z0,
                          double z1, double &delta, double &beta) {
  const double ZERO = 1E-10;
  const unsigned nStepsInRefrIntegral = 10;
  double deltaPrev, betaPrev;
  material_eval(m, g, x, y, z1, delta, beta);
  material_eval(m, g, x, y, z0, deltaPrev, betaPrev);
  if ((std::abs(delta - deltaPrev) > ZERO) || (std::abs(beta - betaPrev) > ZERO)) {
    double deltaTemp = 0.0, betaTemp = 0.0;
    material_eval(m, g, x, y, z0, delta, beta);
    material_eval(m, g, x, y, z1, deltaTemp, betaTemp);
    delta += deltaTemp;
    beta += betaTemp;
    double dzz = (z1 - z0) / nStepsInRefrIntegral;
    for (unsigned i = 1; i < nStepsInRefrIntegral - 1; ++i) {
      double zz = z0 + i * dzz;
      material_eval(m, g, x, y, zz, deltaTemp, betaTemp);
      delta += 2.0 * deltaTemp;
      beta += 2.0 * betaTemp;
    }
    delta /= (2.0 * nStepsInRefrIntegral);
    beta /= (2.0 * nStepsInRefrIntegral);
  }
}

// ================================================================= API ==
extern "C" {

unsigned orc_node_count(double mn, double mx, double step) {
  return node_count(mn, mx, step);
}

void orc_set_threads(int n) { g_threads = n; }
void orc_set_fft_parallel(int on) { g_fft_parallel = on; }
int orc_get_threads(void) { return nthreads(); }

int orc_material_planes(const orc_grid *gp, const orc_material *m, int kind, int first_step,
                        int nsteps, double *delta, double *beta) {
  const orc_grid &g = *gp;
  const unsigned n = node_count(g.xmin, g.xmax, g.dx);
  const long npts = (long)n * n;
  const int per = kind == 4 ? 2 : 1;
  if ((kind != 3 && kind != 4) || nsteps < 0 || first_step < 1) return -1;
  const int th = nthreads();
  for (int k = 0; k < nsteps; ++k) {
    const unsigned step = (unsigned)(first_step + k);
    for (int pl = 0; pl < per; ++pl) {
      double *d = delta + ((long)k * per + pl) * npts, *b = beta + ((long)k * per + pl) * npts;
#pragma omp parallel for num_threads(th)
      for (long i = 0; i < npts; ++i) {
        const unsigned col = (unsigned)(i / n), row = (unsigned)(i % n);
        const double x = get_x(g, (int)col), y = get_y(g, (int)row);
        if (kind == 3)
          fft3d_point_material(m, g, x, y, get_z(g, step - 1), get_z(g, step), d[i], b[i]);
        else
          material_eval(m, g, x, y, get_z(g, step) + (pl ? g.dz / 2.0 : 0.0), d[i], b[i]);
      }
    }
  }
  return 0;
}

int orc_fft1d(double *data, int n, int sign) {
  if (n < 1) return -1;
  fft_1d(reinterpret_cast<cd *>(data), n, sign);
  return 0;
}

void orc_material_eval(const orc_material *m, const orc_grid *g, double x,
                       double y, double z, double *delta, double *beta) {
  material_eval(m, *g, x, y, z, *delta, *beta);
}

void orc_thomas(double *diag, const double *subdiag, double *rhs, int n) {
  thomas(reinterpret_cast<cd *>(diag), reinterpret_cast<const cd *>(subdiag),
         reinterpret_cast<cd *>(rhs), (unsigned)n);
}


// FFTSolver2D::solveStep (src/fftSolver2D.cpp:61-73): propagate (:21-34) then
// refraction (:36-50, midpoint plane z = getZ(step) + dz/2, 1/N applied after
// the transmission multiply); Solver2D::step / copyCurrentSolution
// (src/solver2D.cpp:243-250, 173-193) copy curr into prev after each step.
int orc_fft2d_run(const orc_grid *gp, const orc_material *m, const double *u0,
                  int nsteps, int save_every, double *saves, double *u_out) {
  const orc_grid &g = *gp;
  unsigned n = node_count(g.xmin, g.xmax, g.dx);
  if (n < 2 || nsteps < 0) return -1;
  const cd *in = reinterpret_cast<const cd *>(u0);
  std::vector<cd> prev(in, in + n), curr(prev), ker(n);
  const double stepX = g.dx, stepZ = g.dz, wavenumber = g.wavenumber;
  cd im(0.0, 1.0);
  for (unsigned i = 0; i < n; ++i)
    ker[i] = kernel_2d(spatial_freq(i, n, stepX), stepZ, wavenumber);
  for (int step = 1; step <= nsteps; ++step) {
    // propagate: FFT(prev) -> curr, curr *= kernel, IFFT(curr) -> prev
    curr = prev;
    fft_1d(curr.data(), (int)n, -1);
    for (unsigned i = 0; i < n; ++i) curr[i] *= ker[i];
    prev = curr;
    fft_1d(prev.data(), (int)n, +1);
    // refraction
    double z = get_z(g, step) + 0.5 * stepZ;
    for (unsigned i = 0; i < n; ++i) {
      double delta, beta;
      double x = get_x(g, (int)i);
      material_eval(m, g, x, 0.0, z, delta, beta);
      double normalization = n;
      curr[i] = prev[i] * std::exp(-wavenumber * (beta + im * delta) * stepZ) /
                normalization;
    }
    prev = curr;  // copyCurrentSolution
    save_field(curr.data(), n, step, save_every, saves);
  }
  std::memcpy(u_out, curr.data(), sizeof(cd) * n);
  return 0;
}

// CrankNicholson::solveStep (src/crancNicholson.cpp:17-105) with the default
// ParaxialEquation coefficients F = G = H = 1, J = 0
// (src/paraxialEquation.cpp:3-21), kept as named values so the expression
// order is the reference's.  Transparent BC: applyTBC/applyTBCOneSide
// (:121-148), using the previous field and the coefficient values left over
// from the last grid point of the build loop.
int orc_cn2d_run(const orc_grid *gp, const orc_material *m, int transparent_bc,
                 const double *u0, int nsteps, int save_every, double *saves,
                 double *u_out) {
  const orc_grid &g = *gp;
  unsigned Nx = node_count(g.xmin, g.xmax, g.dx);
  if (Nx < 3 || nsteps < 0) return -1;
  const cd IMAG_UNIT(0.0, 1.0);
  const cd *in = reinterpret_cast<const cd *>(u0);
  std::vector<cd> prev(in, in + Nx), curr(prev);
  std::vector<cd> subdiag(Nx - 1), rhs(Nx), diag(Nx);
  const double stepX = g.dx, stepZ = g.dz, wavenumber = g.wavenumber,
               zmin = g.zmin;
  for (int iz = 1; iz <= nsteps; ++iz) {
    double rho = stepZ / (wavenumber * stepX * stepX);
    double r = wavenumber * stepZ;
    double z = zmin + static_cast<double>(iz) * stepZ;
    double Hpluss = 1.0, Hminus = 1.0, gval = 1.0, HplussPrev = 1.0,
           HminusPrev = 1.0, gvalPrev = 1.0;
    for (unsigned ix = 0; ix < Nx; ++ix) {
      double x = get_x(g, (int)ix);
      double delta, beta, deltaPrev, betaPrev;
      material_eval(m, g, x, 0.0, z, delta, beta);
      material_eval(m, g, x, 0.0, z - stepZ, deltaPrev, betaPrev);
      Hpluss = 1.0;
      Hminus = 1.0;
      gval = 1.0;
      double fval = 1.0, jval = 0.0, jvalPrev = 0.0;
      delta -= jval;
      deltaPrev -= jvalPrev;
      diag[ix] = fval * 1.0 + 0.25 * (Hpluss + Hminus) * gval * IMAG_UNIT * rho +
                 0.5 * (beta * r + IMAG_UNIT * delta * r);
      if (ix < Nx - 1) subdiag[ix] = -0.25 * IMAG_UNIT * rho * Hminus * gval;
      HplussPrev = 1.0;
      HminusPrev = 1.0;
      gvalPrev = 1.0;
      double fvalPrev = 1.0;
      cd left = ix > 0 ? prev[ix - 1] : cd(0.0);
      cd center = prev[ix];
      cd right = ix < Nx - 1 ? prev[ix + 1] : cd(0.0);
      rhs[ix] = left * HminusPrev * gvalPrev;
      rhs[ix] += right * HplussPrev * gvalPrev;
      rhs[ix] *= (0.25 * IMAG_UNIT * rho);
      rhs[ix] -= 0.25 * center * IMAG_UNIT * rho * (HplussPrev + HminusPrev) * gval;
      rhs[ix] += (1.0 * fvalPrev - 0.5 * (betaPrev * r + IMAG_UNIT * deltaPrev * r)) *
                 center;
    }
    if (transparent_bc) {
      const double ZERO = 1E-16;
      auto one_side = [&](unsigned outer, unsigned inner) {
        cd ratio = prev[outer] / prev[inner];
        cd kdx = std::log(ratio) / IMAG_UNIT;
        if (kdx.real() < 0.0) kdx.real(0.0);
        diag[outer] -= 0.25 * IMAG_UNIT * rho * Hminus * gval * std::exp(IMAG_UNIT * kdx);
        rhs[outer] += 0.25 * IMAG_UNIT * rho * HminusPrev * gvalPrev *
                      std::exp(IMAG_UNIT * kdx) * prev[outer];
      };
      if (std::abs(prev[1]) > ZERO) one_side(0, 1);
      if (std::abs(prev[Nx - 2]) > ZERO) one_side(Nx - 1, Nx - 2);
    }
    thomas(diag.data(), subdiag.data(), rhs.data(), Nx);
    for (unsigned ix = 0; ix < Nx; ++ix) curr[ix] = diag[ix];
    prev = curr;
    save_field(curr.data(), Nx, iz, save_every, saves);
  }
  std::memcpy(u_out, curr.data(), sizeof(cd) * Nx);
  return 0;
}

// FFTSolver3D::solveStep (src/fftSolver3D.cpp:52-85): propagate (:87-120),
// refraction (:122-156, end plane z1 = getZ(step), refraction integral
// :253-273 when the material changes between z0 and z1 by more than 1e-10),
// applyAbsorbingBC (:351-374, Absorber::apply src/absorber.cpp:3-12: first
// every column's y-edge band, then every row's x-edge band).
// Solver3D::step / copyCurrentSolution (src/solver3D.cpp:148-166, 78-125).
int orc_fft3d_run(const orc_grid *gp, const orc_material *m,
                  double absorber_width, double absorber_damping,
                  const double *u0, int nsteps, int save_every, double *saves,
                  double *u_out) {
  const orc_grid &g = *gp;
  unsigned Nx = node_count(g.xmin, g.xmax, g.dx);
  unsigned Ny = Nx;  // Solver3D::setSimulator forces Ny = Nx (solver3D.cpp:24)
  if (Nx < 2 || nsteps < 0) return -1;
  const long npts = (long)Nx * Ny;
  const cd *in = reinterpret_cast<const cd *>(u0);
  std::vector<cd> prev(in, in + npts), curr(prev);
  const unsigned n_rows = Ny, n_cols = Nx;
  const double stepX = g.dx, stepY = g.dy, dz = g.dz, k = g.wavenumber;
  const cd im(0.0, 1.0);
  // Absorber set-up (FFTSolver3D::absorbingBC, src/fftSolver3D.cpp:327-349)
  unsigned thickX = 0, thickY = 0;
  double invDampX = 0.0, invDampY = 0.0;
  if (absorber_damping > 0.0) {
    thickX = absorber_width / stepX + 1;
    thickY = absorber_width / stepY + 1;
    invDampX = stepX / absorber_damping;
    invDampY = stepY / absorber_damping;
  }
  // Kernel table (identical every step: depends on dz, k, kx, ky only).
  std::vector<double> kxs(n_cols), kys(n_rows);
  for (unsigned c = 0; c < n_cols; ++c) kxs[c] = spatial_freq(c, n_cols, stepX);
  for (unsigned r = 0; r < n_rows; ++r) kys[r] = spatial_freq(r, n_rows, stepY);
  const int th = nthreads();

  for (int step = 1; step <= nsteps; ++step) {
    curr = prev;
    fft_2d(curr.data(), n_rows, n_cols, -1);
#pragma omp parallel for num_threads(th)
    for (long i = 0; i < npts; ++i) {
      unsigned row = i % n_rows, col = i / n_rows;
      curr[i] *= kernel_3d(kxs[col], kys[row], dz, k);
    }
    prev = curr;
    fft_2d(prev.data(), n_rows, n_cols, +1);
    double z1 = get_z(g, step), z0 = get_z(g, step - 1);
    double normalization = (double)(n_rows * n_cols);
#pragma omp parallel for num_threads(th)
    for (long i = 0; i < npts; ++i) {
      unsigned row = i % n_rows, col = i / n_rows;
      double x = get_x(g, (int)col), y = get_y(g, (int)row);
      double delta, beta;
      fft3d_point_material(m, g, x, y, z0, z1, delta, beta);
      curr[i] = prev[i] * std::exp(-k * (beta + im * delta) * dz) / normalization;
    }
    // absorbY on every column (rows 0..t-1 and their mirrors), then absorbX on
    // every row.
    for (unsigned c = 0; c < n_cols && thickY > 0; ++c)
      for (unsigned i = 0; i < thickY; ++i) {
        double f = std::exp(-static_cast<double>(thickY - i - 1) * invDampY);
        curr[(long)c * n_rows + i] *= f;
        curr[(long)c * n_rows + (n_rows - i - 1)] *= f;
      }
    for (unsigned r = 0; r < n_rows && thickX > 0; ++r)
      for (unsigned i = 0; i < thickX; ++i) {
        double f = std::exp(-static_cast<double>(thickX - i - 1) * invDampX);
        curr[(long)i * n_rows + r] *= f;
        curr[(long)(n_cols - i - 1) * n_rows + r] *= f;
      }
    prev = curr;
    save_field(curr.data(), npts, step, save_every, saves);
  }
  std::memcpy(u_out, curr.data(), sizeof(cd) * npts);
  return 0;
}

// ADI::solveStep (src/alternatingDirectionSolver.cpp:136-155): xImplicit
// (:8-76), prev = curr, yImplicit (:78-134, including the reference's
// parenthesisation of the y-implicit diagonal at :103).  The reference's
// Thomas chain of Nx*Ny unknowns has a zero sub-diagonal at every system
// start, so it is solved system by system (thomas_systems).  The reference's
// OpenMP build loop shares delta/beta between threads (:22, :92); the oracle
// uses per-point values, i.e. the single-thread result.  TBC: ADI::applyTBC
// (:157-234).
int orc_adi3d_run(const orc_grid *gp, const orc_material *m, int use_tbc,
                  const double *u0, int nsteps, int save_every, double *saves,
                  double *u_out) {
  const orc_grid &g = *gp;
  unsigned Nx = node_count(g.xmin, g.xmax, g.dx);
  unsigned Ny = Nx;
  if (Nx < 3 || nsteps < 0) return -1;
  const long npts = (long)Nx * Ny;
  const cd *in = reinterpret_cast<const cd *>(u0);
  std::vector<cd> prev(in, in + npts), curr(prev);
  std::vector<cd> diag(npts), subdiag(npts - 1), rhs(npts);
  const cd im(0.0, 1.0);
  const double dx = g.dx, dy = g.dy, k = g.wavenumber;
  const int th = nthreads();
  // column-major (row = y index i, col = x index j)
  auto P = [&](unsigned i, unsigned j) -> cd & { return prev[(long)j * Ny + i]; };
  auto C = [&](unsigned i, unsigned j) -> cd & { return curr[(long)j * Ny + i]; };

  auto tbc = [&](bool xdir) {
    double zero = 1E-6;
    if (xdir) {
      for (unsigned i = 0; i < Ny; ++i) {
        cd kdx = -im * std::log(P(i, Nx - 1) / P(i, Nx - 2));
        if (kdx.real() < 0.0) kdx.real(0.0);
        long indx = (long)i * Nx + Nx - 1;
        if (std::abs(P(i, Nx - 2)) > zero) diag[indx] -= 0.5 * im * std::exp(im * kdx) / (k * dx * dx);
        indx = (long)i * Nx;
        kdx = -im * std::log(P(i, 0) / P(i, 1));
        if (kdx.real() < 0.0) kdx.real(0.0);
        if (std::abs(P(i, 1)) > zero) diag[indx] -= 0.5 * im * std::exp(im * kdx) / (k * dx * dx);
      }
      for (unsigned i = 0; i < Nx; ++i) {
        cd kdy = -im * std::log(P(Ny - 1, i) / P(Ny - 2, i));
        if (kdy.real() < 0.0) kdy.real(0.0);
        long indx = (long)(Ny - 1) * Nx + i;
        if (std::abs(P(Ny - 2, i)) > zero) rhs[indx] += 0.5 * im * std::exp(im * kdy) * P(Ny - 1, i) / (k * dy * dy);
        indx = i;
        kdy = -im * std::log(P(0, i) / P(1, i));
        if (kdy.real() < 0.0) kdy.real(0.0);
        if (std::abs(P(1, i)) > zero) rhs[indx] += 0.5 * im * std::exp(im * kdy) * P(0, i) / (k * dy * dy);
      }
    } else {
      for (unsigned i = 0; i < Nx; ++i) {
        cd kdy = -im * std::log(P(Ny - 1, i) / P(Ny - 2, i));
        if (kdy.real() < 0.0) kdy.real(0.0);
        long indx = (long)i * Ny + Ny - 1;
        if (std::abs(P(Ny - 2, i)) > zero) diag[indx] -= 0.5 * im * std::exp(im * kdy) / (k * dy * dy);
        indx = (long)i * Ny;
        kdy = -im * std::log(P(0, i) / P(1, i));
        if (kdy.real() < 0.0) kdy.real(0.0);
        if (std::abs(P(1, i)) > zero) diag[indx] -= 0.5 * im * std::exp(im * kdy) / (k * dy * dy);
      }
      for (unsigned i = 0; i < Ny; ++i) {
        cd kdx = -im * std::log(P(i, Nx - 1) / P(i, Nx - 2));
        if (kdx.real() < 0.0) kdx.real(0.0);
        long indx = (long)(Nx - 1) * Ny + i;
        if (std::abs(P(i, Nx - 2)) > zero) rhs[indx] += 0.5 * im * std::exp(im * kdx) * P(i, Nx - 1) / (k * dx * dx);
        indx = i;
        kdx = -im * std::log(P(i, 0) / P(i, 1));
        if (kdx.real() < 0.0) kdx.real(0.0);
        if (std::abs(P(i, 1)) > zero) rhs[indx] += 0.5 * im * std::exp(im * kdx) * P(i, 0) / (k * dx * dx);
      }
    }
  };

  for (int step = 1; step <= nsteps; ++step) {
    // ---- x implicit
    {
      double dz = g.dz / 2.0;
      double z = get_z(g, step);
      std::fill(subdiag.begin(), subdiag.end(), cd(0.0, 0.0));
#pragma omp parallel for num_threads(th)
      for (long indx = 0; indx < npts; ++indx) {
        unsigned j = indx % Nx, i = indx / Nx;
        double x = get_x(g, (int)j), y = get_y(g, (int)i);
        double delta, beta;
        material_eval(m, g, x, y, z, delta, beta);
        diag[indx] = 1.0 / dz + im / (k * dx * dx) + beta * k + im * delta * k;
        rhs[indx] = (1.0 / dz - im / (k * dy * dy)) * P(i, j);
        if (j > 0) subdiag[indx - 1] = -0.5 * im / (k * dx * dx);
        if (i > 0) rhs[indx] += 0.5 * im * P(i - 1, j) / (k * dy * dy);
        if (i < Ny - 1) rhs[indx] += 0.5 * im * P(i + 1, j) / (k * dy * dy);
      }
      if (use_tbc) tbc(true);
      thomas_systems(diag.data(), subdiag.data(), rhs.data(), Ny, Nx, th);
#pragma omp parallel for num_threads(th)
      for (long indx = 0; indx < npts; ++indx) {
        unsigned i = indx / Nx, j = indx % Nx;
        C(i, j) = diag[indx];
      }
    }
    prev = curr;
    // ---- y implicit
    {
      double dz = g.dz / 2.0;
      double z = get_z(g, step) + dz;
      std::fill(subdiag.begin(), subdiag.end(), cd(0.0, 0.0));
#pragma omp parallel for num_threads(th)
      for (long indx = 0; indx < npts; ++indx) {
        unsigned i = indx / Ny, j = indx % Ny;
        double x = get_x(g, (int)i), y = get_y(g, (int)j);
        double delta, beta;
        material_eval(m, g, x, y, z, delta, beta);
        diag[indx] = 1.0 / dz + im / (k * dy * dy + beta * k + im * delta * k);
        rhs[indx] = (-im / (k * dx * dx) + 1.0 / dz) * P(j, i);
        if (j > 0) subdiag[indx - 1] = -0.5 * im / (k * dy * dy);
        if (i > 0) rhs[indx] += 0.5 * im * P(j, i - 1) / (k * dx * dx);
        if (i < Ny - 1) rhs[indx] += 0.5 * im * P(j, i + 1) / (k * dx * dx);
      }
      if (use_tbc) tbc(false);
      thomas_systems(diag.data(), subdiag.data(), rhs.data(), Nx, Ny, th);
#pragma omp parallel for num_threads(th)
      for (long indx = 0; indx < npts; ++indx) {
        unsigned i = indx / Ny, j = indx % Ny;
        C(j, i) = diag[indx];
      }
    }
    prev = curr;  // Solver3D::copyCurrentSolution
    save_field(curr.data(), npts, step, save_every, saves);
  }
  std::memcpy(u_out, curr.data(), sizeof(cd) * npts);
  return 0;
}

// GaussianBeam::get (src/gaussianBeam.cpp:7-63), origin z0 = 0, no tilt.
namespace {
struct Gauss {
  double waist, wavenumber, centerX, centerY, amplitude, z0 = 0.0;
  double angleX = 0.0, angleY = 0.0;
  double wavelength() const { return 2.0 * PI / wavenumber; }
  double zR() const { return PI * waist * waist / wavelength(); }
  double guoy(double z) const { return std::atan(z / zR()); }
  double invR(double z) const {
    double r = zR();
    return z / (z * z + r * r);
  }
  double spot(double z) const { return waist * std::sqrt(1.0 + std::pow(z / zR(), 2)); }
  cd angX(double x) const {
    double a = angleX * PI / 180.0;
    cd im(0.0, 1.0);
    return std::exp(im * wavenumber * std::sin(a) * x);
  }
  cd angY(double y) const {
    double a = angleY * PI / 180.0;
    cd im(0.0, 1.0);
    return std::exp(im * wavenumber * std::sin(a) * y);
  }
  cd get2(double x, double z) const {
    x -= centerX;
    cd im(0.0, 1.0);
    double waistRatio = waist / spot(z - z0);
    double gaussianFactor = std::exp(-std::pow(x / spot(z - z0), 2));
    cd phaseFactor = std::exp(-im * wavenumber * z0 +
                              0.5 * im * wavenumber * x * x * invR(z - z0) -
                              im * guoy(z - z0));
    cd ax = angX(x);
    return amplitude * waistRatio * gaussianFactor * phaseFactor * ax;
  }
  cd get3(double x, double y, double z) const {
    y -= centerY;
    double gy = std::exp(-std::pow(y / spot(z - z0), 2));
    cd ay = angY(y);
    return get2(x, z) * gy * ay;
  }
};
}  // namespace

void orc_gaussian_beam_2d(const orc_grid *g, double wavelength, double waist,
                          double center, double amplitude, double z,
                          double *out) {
  Gauss b{waist, 2.0 * PI / wavelength, center, 0.0, amplitude};
  unsigned n = node_count(g->xmin, g->xmax, g->dx);
  cd *o = reinterpret_cast<cd *>(out);
  for (unsigned i = 0; i < n; ++i) o[i] = b.get2(get_x(*g, (int)i), z);
}

// ParaxialSimulation::setBoundaryConditions, THREE_D branch
// (src/paraxialSimulation.cpp:378-392): values(j, i) = src->get(x_i, y_j, 0).
void orc_gaussian_beam_3d(const orc_grid *g, double wavelength, double waist,
                          double cx, double cy, double amplitude, double z,
                          double *out) {
  Gauss b{waist, 2.0 * PI / wavelength, cx, cy, amplitude};
  unsigned nx = node_count(g->xmin, g->xmax, g->dx);
  unsigned ny = node_count(g->ymin, g->ymax, g->dy);
  cd *o = reinterpret_cast<cd *>(out);
  for (unsigned i = 0; i < nx; ++i)
    for (unsigned j = 0; j < ny; ++j)
      o[(long)i * ny + j] = b.get3(get_x(*g, (int)i), get_y(*g, (int)j), z);
}

// PlaneWave::get (src/planeWave.cpp:5-14) at normal incidence and z0 = 0 is
// the constant amplitude; callers pass the value.
void orc_plane_wave(int n, double value_re, double value_im, double *out) {
  for (int i = 0; i < n; ++i) {
    out[2 * i] = value_re;
    out[2 * i + 1] = value_im;
  }
}

// Solver3D::copyCurrentSolution's block average (src/solver3D.cpp:94-112).
void orc_block_average(const double *full, int n, int m, double *out) {
  const cd *u = reinterpret_cast<const cd *>(full);
  cd *o = reinterpret_cast<cd *>(out);
  const double delta = static_cast<double>(n) / static_cast<double>(m);
  for (int col = 0; col < m; ++col)
    for (int row = 0; row < m; ++row) {
      const unsigned r0 = static_cast<unsigned>(row * delta);
      const unsigned r1 = static_cast<unsigned>(row * delta + delta - 1);
      const unsigned c0 = static_cast<unsigned>(col * delta);
      const unsigned c1 = static_cast<unsigned>(col * delta + delta - 1);
      cd total(0.0, 0.0);
      for (unsigned c = c0; c <= c1; ++c) {
        cd colsum(0.0, 0.0);
        for (unsigned r = r0; r <= r1; ++r) colsum += u[(size_t)c * n + r];
        total += colsum;
      }
      o[(size_t)col * m + row] = total / (delta * delta);
    }
}

}  // extern "C"
