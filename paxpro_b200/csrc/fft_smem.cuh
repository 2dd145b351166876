// fft_smem.cuh -- power-of-two complex FFT held in shared memory.
//
// Stockham autosort passes, radix 8 while it divides the remaining length,
// then one radix-4 or radix-2 pass.  Each pass: every thread loads its
// butterflies' R inputs into registers, the CTA synchronises, then every
// thread applies twiddles and an R-point DFT and stores in place.  Twiddles
// come from a table in pass order: for the pass with sub-transform length NS
// and radix R, entry stockham_offset(N, NS) + (r-1)*NS + k holds
// exp(-2 pi i r k / (NS R)), r = 1..R-1, k < NS, so that the threads of a
// warp read consecutive entries.  Values are computed on the host in
// extended precision; the inverse transform uses their conjugates.  FP64
// data use FP64 twiddles.  Complex64 data (served mode) compute in FP32
// throughout, with every constant factor -- table twiddles, the 1/sqrt(2)
// and W16 constants of the small DFTs, propagator and transmission tables --
// held as an unevaluated sum of two complex64 values, hi = fl32(w) and
// lo = fl32(w - hi), and each product formed by one chain of FP32 FMAs
// (tw_mul): the factor is then exact to about 2^-48 and the product is
// rounded once at the end of the chain.  A factor rounded to FP32 instead
// errs by the same amount at every step, and on a field that changes little
// between steps that error accumulates linearly with the step count (to
// 3e-4 relative intensity at 4000 steps of the 2048-point waveguide); with
// split factors the error stays at the level of the data rounding (about
// 1e-6 at 5000 steps, as with products formed in FP64).
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

// Table entry type for data of complex type C: complex128 for FP64 data,
// the split (hi.re, hi.im, lo.re, lo.im) for complex64 data.  Both are 16
// bytes, so a table has the same size and layout in both precisions.
template <typename C> struct TwOf;
template <> struct TwOf<double2> { using T = double2; };
template <> struct TwOf<float2> { using T = float4; };
template <typename C> using Tw = typename TwOf<C>::T;

// v * w and v * conj(w).
__device__ __forceinline__ double2 tw_mul(double2 v, double2 w) { return cmul(v, w); }
__device__ __forceinline__ double2 tw_mulc(double2 v, double2 w) { return cmulc(v, w); }
// Split factor w = hi + lo: (x + iy)(hi + lo) with the lo products first
// and one rounding per FMA of the chain.
__device__ __forceinline__ float2 tw_mul(float2 v, float4 w) {
  const float x = v.x, y = v.y;
  return make_float2(__fmaf_rn(x, w.x, __fmaf_rn(-y, w.y, __fmaf_rn(x, w.z, __fmul_rn(-y, w.w)))),
                     __fmaf_rn(x, w.y, __fmaf_rn(y, w.x, __fmaf_rn(x, w.w, __fmul_rn(y, w.z)))));
}
__device__ __forceinline__ float2 tw_mulc(float2 v, float4 w) {
  const float x = v.x, y = v.y;
  return make_float2(__fmaf_rn(x, w.x, __fmaf_rn(y, w.y, __fmaf_rn(x, w.z, __fmul_rn(y, w.w)))),
                     __fmaf_rn(-x, w.y, __fmaf_rn(y, w.x, __fmaf_rn(-x, w.w, __fmul_rn(y, w.z)))));
}
// Complex64 data times a factor computed in FP64 on the device (the 3-D
// propagator and transmission): product formed in FP64, rounded once.
__device__ __forceinline__ float2 tw_mul(float2 v, double2 w) {
  double x = v.x, y = v.y;
  return make_float2((float)fma(x, w.x, -y * w.y), (float)fma(x, w.y, y * w.x));
}
__device__ __forceinline__ float2 tw_mulc(float2 v, double2 w) {
  double x = v.x, y = v.y;
  return make_float2((float)fma(x, w.x, y * w.y), (float)fma(y, w.x, -x * w.y));
}
// A real constant c as hi + lo (FP32) for complex64 data.
struct SplitF {
  float hi, lo;
};
__host__ __device__ constexpr SplitF split_f(double c) {
  return SplitF{(float)c, (float)(c - (double)(float)c)};
}
__device__ __forceinline__ float mul_split(float a, SplitF c) {
  return __fmaf_rn(a, c.hi, __fmul_rn(a, c.lo));
}
// (a, b) * 1/sqrt(2).
__device__ __forceinline__ double2 scale_h(double a, double b) {
  const double h = 0.70710678118654752440084436210484903928;
  return make_double2(a * h, b * h);
}
__device__ __forceinline__ float2 scale_h(float a, float b) {
  constexpr SplitF h = split_f(0.70710678118654752440084436210484903928);
  return make_float2(mul_split(a, h), mul_split(b, h));
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

// v * W16^m (forward) or v * conj(W16^m) (inverse), W16 = exp(-2 pi i / 16),
// for the internal twiddles of the 16-point DFT (split constants for
// complex64 data).
template <int SIGN, int M>
__device__ __forceinline__ double2 w16(double2 v) {
  constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
  constexpr double h = 0.70710678118654752440;
  constexpr double c = M == 1 ? c1 : M == 2 ? h : M == 3 ? s1 : M == 6 ? -h : -c1;
  constexpr double sf = M == 1 ? -s1 : M == 2 ? -h : M == 3 ? -c1 : M == 6 ? -h : s1;
  constexpr double sn = SIGN < 0 ? sf : -sf;
  return make_double2(fma(v.x, c, -v.y * sn), fma(v.x, sn, v.y * c));
}
template <int SIGN, int M>
__device__ __forceinline__ float2 w16(float2 v) {
  constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
  constexpr double h = 0.70710678118654752440;
  constexpr double c = M == 1 ? c1 : M == 2 ? h : M == 3 ? s1 : M == 6 ? -h : -c1;
  constexpr double sf = M == 1 ? -s1 : M == 2 ? -h : M == 3 ? -c1 : M == 6 ? -h : s1;
  constexpr double sn = SIGN < 0 ? sf : -sf;
  constexpr SplitF cs = split_f(c), ss = split_f(sn);
  return tw_mul(v, make_float4(cs.hi, ss.hi, cs.lo, ss.lo));
}

// 16-point DFT as 4 x 4: DFTs over the stride-4 subsequences, internal
// twiddles W16^(n2 k1), DFTs over n2, then the 4 x 4 transpose of the
// output order.
template <int SIGN, typename C>
__device__ __forceinline__ void dft16(C *v) {
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) dft4<SIGN>(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
  // v[n2 + 4 k1] *= W16^(n2 k1)
  v[5] = w16<SIGN, 1>(v[5]);
  v[9] = w16<SIGN, 2>(v[9]);
  v[13] = w16<SIGN, 3>(v[13]);
  v[6] = w16<SIGN, 2>(v[6]);
  v[10] = mul_i<SIGN>(v[10]);
  v[14] = w16<SIGN, 6>(v[14]);
  v[7] = w16<SIGN, 3>(v[7]);
  v[11] = w16<SIGN, 6>(v[11]);
  v[15] = w16<SIGN, 9>(v[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<SIGN>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // X[k1 + 4 k2] sits at v[4 k1 + k2]
  C t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
}

template <int R, int SIGN, typename C>
__device__ __forceinline__ void dft_r(C *v) {
  if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
  else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8<SIGN>(v);
  else dft16<SIGN>(v);
}

// One Stockham pass over x (length N, swizzled layout) with T threads; NS =
// length of the sub-transforms already done.  `lane` is this thread's index
// in [0, T).
// Radix of the pass with sub-transform length ns (largest of MAXR, 8 that
// divides the rest, else the rest), the offset of its twiddles, and the
// table size (n - 1 entries: the passes telescope).
__host__ __device__ constexpr int stockham_radix(int n, int ns, int maxr) {
  return n / ns >= maxr ? maxr : (n / ns >= 8 ? 8 : n / ns);
}
__host__ __device__ constexpr int stockham_offset(int n, int ns, int maxr) {
  int off = 0;
  for (int s = 1; s < ns; s *= stockham_radix(n, s, maxr)) off += (stockham_radix(n, s, maxr) - 1) * s;
  return off;
}

template <typename C, int N, int T, int SIGN, int R, int NS, int MAXR>
__device__ __forceinline__ void stockham_pass(C *x, const Tw<C> *tw, int lane) {
  constexpr int OFF = stockham_offset(N, NS, MAXR);
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
          const Tw<C> w = tw[OFF + (r - 1) * NS + k];
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

template <typename C, int N, int T, int SIGN, int MAXR = 8, int NS = 1>
__device__ __forceinline__ void fft_smem(C *x, const Tw<C> *tw, int lane) {
  if constexpr (NS < N) {
    constexpr int R = stockham_radix(N, NS, MAXR);
    stockham_pass<C, N, T, SIGN, R, NS, MAXR>(x, tw, lane);
    fft_smem<C, N, T, SIGN, MAXR, NS * R>(x, tw, lane);
  }
}

// The same transform applied to W lines at once (line w at x + w*LD, LD >=
// N): every pass loads the butterflies of all W lines before one barrier, so
// each thread carries W independent butterfly sets.
template <typename C, int N, int T, int SIGN, int R, int NS, int W, int LD>
__device__ __forceinline__ void stockham_pass_w(C *x, const Tw<C> *tw, int lane) {
  constexpr int OFF = stockham_offset(N, NS, 8);
  constexpr int NB = N / R;
  constexpr int PER = (NB + T - 1) / T;
  C v[W][PER][R];
#pragma unroll
  for (int w = 0; w < W; ++w)
#pragma unroll
    for (int b = 0; b < PER; ++b) {
      const int j = lane + b * T;
      if (NB % T == 0 || j < NB) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[w][b][r] = x[w * LD + sw<C>(j + r * NB)];
      }
    }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < PER; ++b) {
    const int j = lane + b * T;
    if (NB % T == 0 || j < NB) {
      const int k = j & (NS - 1);
      if constexpr (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const Tw<C> t = tw[OFF + (r - 1) * NS + k];
#pragma unroll
          for (int w = 0; w < W; ++w) v[w][b][r] = SIGN < 0 ? tw_mul(v[w][b][r], t) : tw_mulc(v[w][b][r], t);
        }
      }
      const int base = (j - k) * R + k;
#pragma unroll
      for (int w = 0; w < W; ++w) {
        dft_r<R, SIGN>(v[w][b]);
#pragma unroll
        for (int r = 0; r < R; ++r) x[w * LD + sw<C>(base + r * NS)] = v[w][b][r];
      }
    }
  }
  __syncthreads();
}

template <typename C, int N, int T, int SIGN, int W, int LD, int NS = 1>
__device__ __forceinline__ void fft_smem_w(C *x, const Tw<C> *tw, int lane) {
  if constexpr (NS < N) {
    constexpr int R = stockham_radix(N, NS, 8);
    stockham_pass_w<C, N, T, SIGN, R, NS, W, LD>(x, tw, lane);
    fft_smem_w<C, N, T, SIGN, W, LD, NS * R>(x, tw, lane);
  }
}

}  // namespace pxp
