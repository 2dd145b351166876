/* fftw3.h -- the part of FFTW3's basic interface that the reference's
 * solvers call (src/fftSolver2D.cpp:9-13, 25, 33, 64-71;
 * src/fftSolver3D.cpp:14-22, 52-85).  TEST INFRASTRUCTURE ONLY: the reference
 * pin (oracle/Makefile) compiles the reference's solver sources against this
 * header.  FFTW itself (the apt libfftw3-dev of the reference's CI, version
 * unpinned) is absent here; its published semantics are restated:
 *
 *   fftw_plan_dft_1d(n, in, out, sign, flags): out[k] = sum_j in[j]
 *     exp(sign * 2 pi i j k / n), unnormalised, FFTW_FORWARD = -1,
 *     FFTW_BACKWARD = +1, in and out may alias;
 *   fftw_plan_dft_2d(n0, n1, ...): the same along both dimensions of a
 *     row-major n0 x n1 array (element (i0, i1) at i0*n1 + i1).
 *
 * The 1-D transforms are the oracle's (orc_fft1d: radix-2 for powers of two,
 * a direct DFT with an extended-precision table otherwise), and the 2-D plan
 * transforms the contiguous dimension first, as the oracle's FFTSolver3D
 * restatement does, so the pinned reference and the oracle share every FFT
 * rounding.  The flags (FFTW_ESTIMATE, ...) do not change results here. */
#ifndef PXP_REFSHIM_FFTW3_H
#define PXP_REFSHIM_FFTW3_H
#include <stdlib.h>
#include <string.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct pxp_refshim_fftw_plan_s {
  int rank, n0, n1, sign;
  fftw_complex *in, *out;
} *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

int orc_fft1d(double *data, int n, int sign); /* oracle/paxpro_oracle.cpp */

static inline fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign,
                                         unsigned flags) {
  (void)flags;
  fftw_plan p = (fftw_plan)malloc(sizeof(*p));
  p->rank = 1;
  p->n0 = n;
  p->n1 = 1;
  p->sign = sign;
  p->in = in;
  p->out = out;
  return p;
}

static inline fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                                         int sign, unsigned flags) {
  fftw_plan p = fftw_plan_dft_1d(n0, in, out, sign, flags);
  p->rank = 2;
  p->n1 = n1;
  return p;
}

static inline void fftw_execute(const fftw_plan p) {
  const long n = (long)p->n0 * p->n1;
  double *o = (double *)p->out;
  if (p->out != p->in) memmove(o, p->in, sizeof(fftw_complex) * n);
  if (p->rank == 1) {
    orc_fft1d(o, p->n0, p->sign);
    return;
  }
  /* contiguous dimension (i1) first, then the strided one (i0) */
  for (int i0 = 0; i0 < p->n0; ++i0) orc_fft1d(o + 2L * i0 * p->n1, p->n1, p->sign);
  double *line = (double *)malloc(sizeof(fftw_complex) * p->n0);
  for (int i1 = 0; i1 < p->n1; ++i1) {
    for (int i0 = 0; i0 < p->n0; ++i0) {
      line[2 * i0] = o[2L * ((long)i0 * p->n1 + i1)];
      line[2 * i0 + 1] = o[2L * ((long)i0 * p->n1 + i1) + 1];
    }
    orc_fft1d(line, p->n0, p->sign);
    for (int i0 = 0; i0 < p->n0; ++i0) {
      o[2L * ((long)i0 * p->n1 + i1)] = line[2 * i0];
      o[2L * ((long)i0 * p->n1 + i1) + 1] = line[2 * i0 + 1];
    }
  }
  free(line);
}

static inline void fftw_destroy_plan(fftw_plan p) { free(p); }

#ifdef __cplusplus
}
#endif
#endif
