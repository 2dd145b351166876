// ref_pin.cpp -- exposes the parts of the reference that compile from their
// own sources here, for pinning the oracle.  TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/Makefile against the reference tree (REF_DIR); the
// reference sources are compiled where they lie and never copied.  Only two
// pieces of the propagation path build without third-party libraries:
//   * ThomasAlgorithm::solve<T> (include/thomasAlgorithm.tpp:2-32), header
//     only, needs OpenMP;
//   * ParaxialEquation's default coefficients (src/paraxialEquation.cpp:3-27).
// Everything else on the path needs Armadillo / FFTW3 / HDF5 / jsoncpp /
// VISA, which are absent.
#include <complex>

#include "paraxialEquation.hpp"
#include "thomasAlgorithm.hpp"

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
}
