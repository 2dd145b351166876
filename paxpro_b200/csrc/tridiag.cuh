// tridiag.cuh -- parallel complex tridiagonal solve used by the CN and ADI
// kernels (replacing the serial ThomasAlgorithm::solve sweep,
// include/thomasAlgorithm.tpp:2-32).
//
// Systems have a symmetric, constant off-diagonal `sub` (CN: -i rho/4,
// ADI: -i/(2 k d^2)) and per-row diagonals / right-hand sides.  A system of L
// unknowns is split into P chunks of M consecutive rows, one chunk per
// thread.  Each thread eliminates its chunk interior in registers (partition
// method: interior x_i = y_i + p_i x_first + q_i x_last, three right-hand
// sides through one Thomas factorisation) and emits the two boundary rows of
// its chunk; those 2P rows form a tridiagonal reduced system that the
// threads solve by cyclic reduction in shared memory.  All arithmetic is
// FP64; each pivot is inverted once (complex reciprocal) and applied by
// multiplication.
#pragma once
#include "pxp_complex.cuh"

namespace pxp {

struct ReducedRows {
  double2 ea, eb, ec, ed;  // first row of the chunk: a x_{s-1} + b x_s + c x_e = d
  double2 fa, fb, fc, fd;  // last row: a x_s + b x_e + c x_{e+1} = d
};

// dg/rh: the M rows of the chunk.  has_left / has_right: whether the chunk's
// first / last row couples to a neighbouring chunk (false at the system ends).
template <int M>
__device__ __forceinline__ ReducedRows chunk_eliminate(const double2 (&dg)[M], const double2 (&rh)[M],
                                                       double2 sub, bool has_left, bool has_right,
                                                       double2 (&y)[M > 2 ? M - 2 : 1],
                                                       double2 (&p)[M > 2 ? M - 2 : 1],
                                                       double2 (&q)[M > 2 ? M - 2 : 1]) {
  ReducedRows o;
  const double2 zero = mk(0.0, 0.0);
  if constexpr (M > 2) {
    double2 cp[M - 2];
#pragma unroll
    for (int m = 1; m <= M - 2; ++m) {
      const int j = m - 1;
      double2 den = dg[m];
      if (j > 0) den = csub(den, cmul(sub, cp[j - 1]));
      const double2 inv = crecip(den);
      if (m < M - 2) cp[j] = cmul(sub, inv);
      double2 ry = rh[m];
      double2 rp = (m == 1) ? csub(zero, sub) : zero;
      double2 rq = (m == M - 2) ? csub(zero, sub) : zero;
      if (j > 0) {
        ry = csub(ry, cmul(sub, y[j - 1]));
        rp = csub(rp, cmul(sub, p[j - 1]));
        if (m == M - 2) rq = csub(rq, cmul(sub, q[j - 1]));
      }
      y[j] = cmul(ry, inv);
      p[j] = cmul(rp, inv);
      q[j] = (m == M - 2) ? cmul(rq, inv) : zero;
    }
#pragma unroll
    for (int j = M - 4; j >= 0; --j) {
      y[j] = csub(y[j], cmul(cp[j], y[j + 1]));
      p[j] = csub(p[j], cmul(cp[j], p[j + 1]));
      q[j] = csub(q[j], cmul(cp[j], q[j + 1]));
    }
    o.ea = has_left ? sub : zero;
    o.eb = cadd(dg[0], cmul(sub, p[0]));
    o.ec = cmul(sub, q[0]);
    o.ed = csub(rh[0], cmul(sub, y[0]));
    o.fa = cmul(sub, p[M - 3]);
    o.fb = cadd(dg[M - 1], cmul(sub, q[M - 3]));
    o.fc = has_right ? sub : zero;
    o.fd = csub(rh[M - 1], cmul(sub, y[M - 3]));
  } else {
    o.ea = has_left ? sub : zero;
    o.eb = dg[0];
    o.ec = sub;
    o.ed = rh[0];
    o.fa = sub;
    o.fb = dg[M - 1];
    o.fc = has_right ? sub : zero;
    o.fd = rh[M - 1];
  }
  return o;
}

// Interior values of a chunk once its first (xf) and last (xl) are known.
template <int M>
__device__ __forceinline__ double2 chunk_value(int m, double2 xf, double2 xl,
                                               const double2 (&y)[M > 2 ? M - 2 : 1],
                                               const double2 (&p)[M > 2 ? M - 2 : 1],
                                               const double2 (&q)[M > 2 ? M - 2 : 1]) {
  if (m == 0) return xf;
  if (m == M - 1) return xl;
  return cadd(cadd(y[m - 1], cmul(p[m - 1], xf)), cmul(q[m - 1], xl));
}

// Cyclic reduction on n = 2^L >= 4 equations (a: coupling to x_{i-1},
// b: diagonal, c: coupling to x_{i+1}, d: rhs -> solution).  `tid` runs over
// the `nt` threads that share this system; every thread of the CTA must call
// with the same n, because the levels are separated by __syncthreads().
__device__ __forceinline__ void cyclic_reduction(double2 *a, double2 *b, double2 *c, double2 *d,
                                                 int n, int tid, int nt) {
  const double2 zero = mk(0.0, 0.0);
  int s = 1;
  for (; 4 * s <= n; s <<= 1) {
    const int cnt = n / (2 * s);
    for (int k = tid; k < cnt; k += nt) {
      const int i = 2 * s * k + 2 * s - 1;
      const int il = i - s, ir = i + s;
      double2 k1 = cmul(a[i], crecip(b[il]));
      double2 ai = csub(zero, cmul(a[il], k1));
      double2 bi = csub(b[i], cmul(c[il], k1));
      double2 di = csub(d[i], cmul(d[il], k1));
      double2 ci = zero;
      if (ir < n) {
        double2 k2 = cmul(c[i], crecip(b[ir]));
        ci = csub(zero, cmul(c[ir], k2));
        bi = csub(bi, cmul(a[ir], k2));
        di = csub(di, cmul(d[ir], k2));
      }
      a[i] = ai;
      b[i] = bi;
      c[i] = ci;
      d[i] = di;
    }
    __syncthreads();
  }
  if (tid == 0) {
    const int i1 = n / 2 - 1, i2 = n - 1;
    double2 det = cx_sub_rn(cx_mul_rn(b[i1], b[i2]), cx_mul_rn(c[i1], a[i2]));
    double2 x1 = cx_div_rn(cx_sub_rn(cx_mul_rn(b[i2], d[i1]), cx_mul_rn(c[i1], d[i2])), det);
    double2 x2 = cx_div_rn(cx_sub_rn(cx_mul_rn(b[i1], d[i2]), cx_mul_rn(a[i2], d[i1])), det);
    d[i1] = x1;
    d[i2] = x2;
  }
  __syncthreads();
  for (s >>= 1; s >= 1; s >>= 1) {
    const int cnt = n / (2 * s);
    for (int k = tid; k < cnt; k += nt) {
      const int i = 2 * s * k + s - 1;
      double2 acc = d[i];
      if (i - s >= 0) acc = csub(acc, cmul(a[i], d[i - s]));
      if (i + s < n) acc = csub(acc, cmul(c[i], d[i + s]));
      d[i] = cmul(acc, crecip(b[i]));
    }
    __syncthreads();
  }
}

}  // namespace pxp
