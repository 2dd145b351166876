// pxp_complex.cuh -- complex arithmetic for the propagation kernels.
//
// Two families:
//  * "exact" helpers (cx_mul_rn, ...) use the _rn intrinsics so that no FMA
//    contraction changes the rounding; they reproduce the operation order of
//    std::complex<double> as GCC compiles it for x86-64 without FMA (complex
//    times complex = (ac - bd, ad + bc); complex / complex = Smith's method,
//    R. L. Smith, "Algorithm 116: Complex division", CACM 5(8), 1962).  They
//    are used wherever the step must reproduce the reference's coefficient
//    arithmetic (matrix build, transmission multiply).
//  * plain helpers (cmul, ...) let the compiler fuse; used inside FFT
//    butterflies and in FP32 served mode.
#pragma once
#include <cuda_runtime.h>

namespace pxp {

template <typename R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

// ---- plain (contractible) ----
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return mk(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return mk(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return mk(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
// a * b + c with four FMAs; the chain from c is two FMAs deep
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
  return mk(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return mk(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return mk(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <int SIGN> __device__ __forceinline__ double2 mul_i(double2 a) {
  return SIGN < 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}
template <int SIGN> __device__ __forceinline__ float2 mul_i(float2 a) {
  return SIGN < 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

// ---- exact (no contraction), FP64 ----
__device__ __forceinline__ double2 cx_add_rn(double2 a, double2 b) {
  return mk(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 cx_sub_rn(double2 a, double2 b) {
  return mk(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y));
}
// (a.x*b.x - a.y*b.y, a.x*b.y + a.y*b.x), each product rounded.
__device__ __forceinline__ double2 cx_mul_rn(double2 a, double2 b) {
  return mk(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
            __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cx_scale_rn(double2 a, double s) {
  return mk(__dmul_rn(a.x, s), __dmul_rn(a.y, s));
}
__device__ __forceinline__ double2 cx_div_real_rn(double2 a, double s) {
  return mk(__ddiv_rn(a.x, s), __ddiv_rn(a.y, s));
}
// Smith's complex division (a / b) with the branch on |b.x| vs |b.y|.
__device__ __forceinline__ double2 cx_div_rn(double2 a, double2 b) {
  if (fabs(b.x) < fabs(b.y)) {
    double ratio = __ddiv_rn(b.x, b.y);
    double denom = __dadd_rn(__dmul_rn(b.x, ratio), b.y);
    return mk(__ddiv_rn(__dadd_rn(__dmul_rn(a.x, ratio), a.y), denom),
              __ddiv_rn(__dsub_rn(__dmul_rn(a.y, ratio), a.x), denom));
  } else {
    double ratio = __ddiv_rn(b.y, b.x);
    double denom = __dadd_rn(__dmul_rn(b.y, ratio), b.x);
    return mk(__ddiv_rn(__dadd_rn(__dmul_rn(a.y, ratio), a.x), denom),
              __ddiv_rn(__dsub_rn(a.y, __dmul_rn(a.x, ratio)), denom));
  }
}

// Complex reciprocal conj(b)/|b|^2: one real division.  Used inside the
// tridiagonal solves, where the operands are O(1e-3..1e3) and well away from
// overflow or underflow.
__device__ __forceinline__ double2 crecip(double2 b) {
  double m = fma(b.x, b.x, b.y * b.y);
  double r = 1.0 / m;
  return mk(b.x * r, -b.y * r);
}

// Plain complex division for FP32 served mode (Smith, contractible).
__device__ __forceinline__ float2 cdiv(float2 a, float2 b) {
  if (fabsf(b.x) < fabsf(b.y)) {
    float ratio = b.x / b.y;
    float denom = b.x * ratio + b.y;
    return mk((a.x * ratio + a.y) / denom, (a.y * ratio - a.x) / denom);
  } else {
    float ratio = b.y / b.x;
    float denom = b.y * ratio + b.x;
    return mk((a.y * ratio + a.x) / denom, (a.y - a.x * ratio) / denom);
  }
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cx_div_rn(a, b); }

// Padded shared-memory position for arrays read in chunks of 8 consecutive
// rows per thread: chunk c starts at 9c, so the eight threads of an access
// phase (c .. c+7) hit eight different 16-byte bank groups.
__host__ __device__ __forceinline__ int pad8(int p) { return p + (p >> 3); }

// Conversions between storage precisions.
__device__ __forceinline__ double2 to_d(float2 a) { return mk((double)a.x, (double)a.y); }
__device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <typename R> __device__ __forceinline__ typename Cx<R>::T from_d(double2 a);
template <> __device__ __forceinline__ double2 from_d<double>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 from_d<float>(double2 a) {
  return mk((float)a.x, (float)a.y);
}

}  // namespace pxp
