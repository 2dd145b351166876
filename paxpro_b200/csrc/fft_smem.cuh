// fft_smem.cuh -- power-of-two complex FFT held in shared memory.
//
// Stockham autosort passes, radix 8 while it divides the remaining length,
// then one radix-4 or radix-2 pass.  Each pass: every thread loads its
// butterflies' R inputs into registers, the CTA synchronises, then every
// thread applies twiddles and an R-point DFT and stores in place.  Twiddles
// come from a table in pass order: for the pass with sub-transform length NS
// and radix R, entry stockham_offset(N, NS) + (r-1)*NS + k holds
// exp(-2 pi i r k / (NS R)), r = 1..R-1, k < NS, so that the threads of a
// warp read consecutive entries.  Values are FP64, computed on the host in
// extended precision; the inverse transform uses their conjugates.  With
// complex64 data (served mode) every product with a twiddle or with
// 1/sqrt(2) is formed in FP64 and rounded once to FP32: an FP32 complex
// product (ac - bd with a rounded factor and cancellation) leaves a bias that
// the same transform, applied to a slowly changing field thousands of times,
// would accumulate coherently.
// SIGN = -1 is the forward transform exp(-2 pi i jk/N), +1 the backward one,
// both unnormalised (the FFTW convention the reference relies on,
// src/fftSolver2D.cpp:68-69).
#pragma once
#include "pxp_complex.cuh"

namespace pxp {

// Shared-memory layout of a transform line: 16-byte chunks are XOR-swizzled,
// chunk' = chunk ^ ((chunk >> 3) & 7), so that the eight threads of every
// access phase hit eight different 16-byte bank groups in every Stockham pass
// (stride-R stores of the first passes included).  sw() maps an element index
// to its slot; every access to a line in shared memory goes through it.
template <typename C> __device__ __forceinline__ int sw(int i);
template <> __device__ __forceinline__ int sw<double2>(int i) { return i ^ ((i >> 3) & 7); }
template <> __device__ __forceinline__ int sw<float2>(int i) {
  const int c = i >> 1;
  return ((c ^ ((c >> 3) & 7)) << 1) | (i & 1);
}

// v * w and v * conj(w) with FP64 twiddles.
__device__ __forceinline__ double2 tw_mul(double2 v, double2 w) { return cmul(v, w); }
__device__ __forceinline__ double2 tw_mulc(double2 v, double2 w) { return cmulc(v, w); }
__device__ __forceinline__ float2 tw_mul(float2 v, double2 w) {
  double x = v.x, y = v.y;
  return make_float2((float)fma(x, w.x, -y * w.y), (float)fma(x, w.y, y * w.x));
}
__device__ __forceinline__ float2 tw_mulc(float2 v, double2 w) {
  double x = v.x, y = v.y;
  return make_float2((float)fma(x, w.x, y * w.y), (float)fma(y, w.x, -x * w.y));
}
// (a, b) * 1/sqrt(2), the product formed in FP64 for complex64 data.
__device__ __forceinline__ double2 scale_h(double a, double b) {
  const double h = 0.70710678118654752440084436210484903928;
  return make_double2(a * h, b * h);
}
__device__ __forceinline__ float2 scale_h(float a, float b) {
  const double h = 0.70710678118654752440084436210484903928;
  return make_float2((float)((double)a * h), (float)((double)b * h));
}

// In-register R-point DFT, R in {2, 4, 8}.
template <int SIGN, typename C>
__device__ __forceinline__ void dft2(C &a, C &b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft4(C &v0, C &v1, C &v2, C &v3) {
  C a0 = cadd(v0, v2), a1 = csub(v0, v2);
  C a2 = cadd(v1, v3), a3 = mul_i<SIGN>(csub(v1, v3));
  v0 = cadd(a0, a2);
  v2 = csub(a0, a2);
  v1 = cadd(a1, a3);
  v3 = csub(a1, a3);
}

template <int SIGN, typename C>
__device__ __forceinline__ void dft8(C *v) {
  C a0 = cadd(v[0], v[4]), b0 = csub(v[0], v[4]);
  C a1 = cadd(v[1], v[5]), b1 = csub(v[1], v[5]);
  C a2 = cadd(v[2], v[6]), b2 = csub(v[2], v[6]);
  C a3 = cadd(v[3], v[7]), b3 = csub(v[3], v[7]);
  // b_r *= W8^(r) (forward) or its conjugate (inverse)
  if (SIGN < 0) {
    b1 = scale_h(b1.x + b1.y, b1.y - b1.x);
    b2 = mk(b2.y, -b2.x);
    b3 = scale_h(b3.y - b3.x, -(b3.x + b3.y));
  } else {
    b1 = scale_h(b1.x - b1.y, b1.x + b1.y);
    b2 = mk(-b2.y, b2.x);
    b3 = scale_h(-(b3.x + b3.y), b3.x - b3.y);
  }
  dft4<SIGN>(a0, a1, a2, a3);
  dft4<SIGN>(b0, b1, b2, b3);
  v[0] = a0; v[2] = a1; v[4] = a2; v[6] = a3;
  v[1] = b0; v[3] = b1; v[5] = b2; v[7] = b3;
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft_r(C *v) {
  if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
  else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else dft8<SIGN>(v);
}

// One Stockham pass over x (length N, swizzled layout) with T threads; NS =
// length of the sub-transforms already done.  `lane` is this thread's index
// in [0, T).
// Number of twiddle entries of all passes of a length-N transform, and the
// offset of the pass with sub-transform length NS.
__host__ __device__ constexpr int stockham_radix(int n, int ns) { return n / ns >= 8 ? 8 : n / ns; }
__host__ __device__ constexpr int stockham_offset(int n, int ns) {
  int off = 0;
  for (int s = 1; s < ns; s *= stockham_radix(n, s)) off += (stockham_radix(n, s) - 1) * s;
  return off;
}
__host__ __device__ constexpr int stockham_twiddle_count(int n) { return stockham_offset(n, n); }

template <typename C, int N, int T, int SIGN, int R, int NS>
__device__ __forceinline__ void stockham_pass(C *x, const double2 *tw, int lane) {
  constexpr int OFF = stockham_offset(N, NS);
  constexpr int NB = N / R;
  constexpr int PER = (NB + T - 1) / T;
  C v[PER][R];
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    int j = lane + b * T;
    if (NB % T == 0 || j < NB) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[b][r] = x[sw<C>(j + r * NB)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    int j = lane + b * T;
    if (NB % T == 0 || j < NB) {
      int k = j & (NS - 1);
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          double2 w = tw[OFF + (r - 1) * NS + k];
          v[b][r] = SIGN < 0 ? tw_mul(v[b][r], w) : tw_mulc(v[b][r], w);
        }
      }
      dft_r<R, SIGN>(v[b]);
      int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) x[sw<C>(base + r * NS)] = v[b][r];
    }
  }
  __syncthreads();
}

template <typename C, int N, int T, int SIGN, int NS = 1>
__device__ __forceinline__ void fft_smem(C *x, const double2 *tw, int lane) {
  if constexpr (NS < N) {
    constexpr int REM = N / NS;
    constexpr int R = REM >= 8 ? 8 : REM;
    stockham_pass<C, N, T, SIGN, R, NS>(x, tw, lane);
    fft_smem<C, N, T, SIGN, NS * R>(x, tw, lane);
  }
}

}  // namespace pxp
