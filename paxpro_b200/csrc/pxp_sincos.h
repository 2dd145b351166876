// pxp_sincos.h -- sin and cos of a double for the propagator phases.
//
// The FFTSolver3D propagator needs exp(-i phi) with phi = a (kx^2 + ky^2) up
// to about 1.5e3 rad for every grid point of every step.  This is a
// compact FP64 sin/cos for |x| < 2^20, written from two published methods:
//   * Cody-Waite argument reduction (W. J. Cody and W. Waite, "Software
//     Manual for the Elementary Functions", 1980): q = nearest integer to
//     x * 2/pi, r = x - q*(pi/2) with pi/2 split into three doubles
//     (P1 + P2 + P3; each product formed exactly inside an FMA), so r keeps
//     full precision;
//   * the Taylor series of sin and cos on |r| <= pi/4, truncated after the
//     r^19 / r^18 terms (remainder below 1e-22), evaluated by Horner's rule
//     in r^2 with coefficients (-1)^k / (2k+1)! and (-1)^k / (2k)!.
// The quadrant q mod 4 selects the signs and the swap of sin and cos.  The
// split constants are the doubles nearest to pi/2, to pi/2 - P1 and to
// pi/2 - P1 - P2.  Host and device share this code; tests check it against
// long-double sinl/cosl.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define PXP_HD __host__ __device__ __forceinline__
#else
#define PXP_HD inline
#endif

namespace pxp {

PXP_HD void sincos_cw(double x, double *s, double *c) {
  const double two_over_pi = 0x1.45f306dc9c883p-1;
  const double P1 = 0x1.921fb54442d18p+0;
  const double P2 = 0x1.1a62633145c07p-54;
  const double P3 = -0x1.f1976b7ed8fbcp-110;
  const double q = std::rint(x * two_over_pi);
  double r = std::fma(-q, P1, x);
  r = std::fma(-q, P2, r);
  r = std::fma(-q, P3, r);
  const double r2 = r * r;
  // sin r = r + r^3 * (-1/3! + r^2 (1/5! - r^2 (1/7! - ...)))
  double ps = -1.0 / 121645100408832000.0;          // -1/19!
  ps = std::fma(ps, r2, 1.0 / 355687428096000.0);   //  1/17!
  ps = std::fma(ps, r2, -1.0 / 1307674368000.0);    // -1/15!
  ps = std::fma(ps, r2, 1.0 / 6227020800.0);        //  1/13!
  ps = std::fma(ps, r2, -1.0 / 39916800.0);         // -1/11!
  ps = std::fma(ps, r2, 1.0 / 362880.0);            //  1/9!
  ps = std::fma(ps, r2, -1.0 / 5040.0);             // -1/7!
  ps = std::fma(ps, r2, 1.0 / 120.0);               //  1/5!
  ps = std::fma(ps, r2, -1.0 / 6.0);                // -1/3!
  const double sn = std::fma(r * r2, ps, r);
  // cos r = 1 - r^2/2 + r^4 * (1/4! - r^2 (1/6! - ...))
  double pc = 1.0 / 6402373705728000.0;             //  1/18!
  pc = std::fma(pc, r2, -1.0 / 20922789888000.0);   // -1/16!
  pc = std::fma(pc, r2, 1.0 / 87178291200.0);       //  1/14!
  pc = std::fma(pc, r2, -1.0 / 479001600.0);        // -1/12!
  pc = std::fma(pc, r2, 1.0 / 3628800.0);           //  1/10!
  pc = std::fma(pc, r2, -1.0 / 40320.0);            // -1/8!
  pc = std::fma(pc, r2, 1.0 / 720.0);               //  1/6!
  pc = std::fma(pc, r2, -1.0 / 24.0);               // -1/4!
  const double h = 0.5 * r2;
  const double cs = std::fma(r2 * r2, -pc, 1.0 - h) ;
  const long long quad = (long long)q & 3;
  double ss = sn, cc = cs;
  if (quad == 1) {
    ss = cs;
    cc = -sn;
  } else if (quad == 2) {
    ss = -sn;
    cc = -cs;
  } else if (quad == 3) {
    ss = -cs;
    cc = sn;
  }
  *s = ss;
  *c = cc;
}

}  // namespace pxp
