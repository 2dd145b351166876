// fft_r16.cuh -- pieces of the register-resident radix-16 line transforms
// shared by the FFTSolver2D kernel (fft1d_r16.cu) and the FFTSolver3D line
// passes (fft3d_r16.cu).
//
// A line of n = R0 * 16^k points (R0 = 16, 8, 4 or 2) belongs to n/16
// threads; thread j holds the points j + s*n/16 (s = 0..15) in registers.
// A transform is a first pass of radix R0 over the thread's own points
// (16/R0 butterflies: butterfly b = j + u*n/16 takes points
// s = u + r*(16/R0), no twiddles, outputs to Stockham position b*R0 + r)
// and k radix-16 Stockham passes in which thread j owns butterfly j (inputs
// j + r*n/16, twiddles W_{16 NS}^(r k) with k = j mod NS, outputs to
// (j - k)*16 + k + r*NS).  The last pass's outputs j + r*n/16 are in natural
// order: exactly the thread's points of the next transform.
#pragma once
#include "fft_smem.cuh"

namespace pxp {
namespace r16c {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

// Radix of the first pass, number of radix-16 passes, twiddle-table entries.
template <int N> struct Plan {
  static constexpr int LOG = ilog2c(N);
  static constexpr int R0 = 1 << (LOG % 4 == 0 ? 4 : LOG % 4);
  static constexpr int NP16 = (LOG - ilog2c(R0)) / 4;
  static constexpr int TWN = R0 * ((1 << (4 * NP16)) - 1);
  static constexpr int TL = N / 16;
};

// Exchange-buffer positions.  16-byte elements: every access of 8
// consecutive threads (reads at stride 1, first-pass writes at stride 16, 8,
// 4 or 2, radix-16 writes) lands on 8 different 16-byte bank groups.
// 8-byte elements: every access of 16 consecutive threads lands on 16
// different 8-byte bank pairs.  Both permute each aligned block of 8 (16)
// elements, so positions stay below n.
__device__ __forceinline__ int xsw16(int i) { return i ^ (((i >> 3) ^ (i >> 4)) & 7); }
__device__ __forceinline__ int xsw8(int i) { return i ^ ((i >> 4) & 15); }
template <int BYTES> __device__ __forceinline__ int xsw(int i) {
  return BYTES == 16 ? xsw16(i) : xsw8(i);
}

// Offset of the twiddles of radix-16 pass P (NS = R0 * 16^P) in the table.
template <int R0, int P> __host__ __device__ constexpr int tw_offset() {
  int off = 0, ns = R0;
  for (int p = 0; p < P; ++p, ns *= 16) off += 15 * ns;
  return off;
}

// The twiddle table of every radix-16 pass, entry off + (r-1)*NS + k =
// W_{16 NS}^(r k), from the table wn[m] = exp(-2 pi i m / N) (complex128, or
// its split form for complex64 data); threads tid = 0 .. nthreads-1.
template <int N, typename W>
__device__ __forceinline__ void load_twiddles(W *tws, const W *__restrict__ wn, int tid,
                                              int nthreads) {
  int off = 0;
  for (int ns = Plan<N>::R0; ns < N; off += 15 * ns, ns *= 16)
    for (int i = tid; i < 15 * ns; i += nthreads) {
      const int r = i / ns + 1, k = i % ns;
      tws[off + i] = wn[r * k * (N / (16 * ns))];
    }
}

// First pass on the thread's 16 points (in place: point s of butterfly u,
// input r, holds its output r afterwards).
template <int SIGN, int R0, typename C>
__device__ __forceinline__ void first_pass(C (&v)[16]) {
  if constexpr (R0 == 16) {
    dft16<SIGN>(v);
  } else {
#pragma unroll
    for (int u = 0; u < 16 / R0; ++u) {
      C w[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) w[r] = v[u + r * (16 / R0)];
      dft_r<R0, SIGN>(w);
#pragma unroll
      for (int r = 0; r < R0; ++r) v[u + r * (16 / R0)] = w[r];
    }
  }
}

}  // namespace r16c
}  // namespace pxp
