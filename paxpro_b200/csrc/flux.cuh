// flux.cuh -- per-step flux integrals fused into the 2-D step kernels.
//
// post::Transmittivity (src/transmittivity.cpp:30-83) integrates |u|^2 over
// the waveguide after every step with the trapezoid rule
// (trapezoidalIntegrateIntensityZ, :30-41): |u_a|^2 + |u_b|^2 + 2 sum_{a<i<b}
// |u_i|^2, times dx/2.  The step kernels add the weighted terms of the new
// field as they store it (no extra pass over the field).  A thread adds its
// few terms (at most N/T, all positive: relative error below N/T ulps),
// warps add their threads' sums by a shuffle tree, and after the step's
// closing barrier warp 0 adds the warp totals the same way (pairwise sums:
// error growth log2 of the count).  The host applies the dx/2 factor.  |u|^2 is fma(x, x, y*y),
// within two ulps of the reference's pow(abs(u), 2) (the kernels are single
// SMs per field, where hypot per point would cost as much as the step).
#pragma once
#include "pxp_kernels.h"

namespace pxp {

// Window (a, b) of this step, when the job integrates it.
__device__ __forceinline__ bool flux_window(const FluxSpec &f, int step, int2 &w) {
  const int k = step - f.step0;
  if (f.out == nullptr || k < 0 || k >= f.count) return false;
  w = f.win[k];
  return true;
}

// Trapezoid weight of point i in window (a, b): 1 at each end, 2 between
// (a single-point window counts its point twice, as the reference does).
__device__ __forceinline__ void flux_add(double &acc, int i, int2 w, double2 u) {
  if (i < w.x || i > w.y) return;
  const double wt = (i > w.x && i < w.y) || w.x == w.y ? 2.0 : 1.0;
  acc = fma(wt, fma(u.x, u.x, u.y * u.y), acc);
}

// Slots of the per-step partial sums: one per warp, or one per thread when
// the CTA is smaller than a warp.
template <int T> __host__ __device__ constexpr int flux_slots() { return T >= 32 ? T / 32 : T; }

// Before the step's closing barrier: each warp's total (each thread's sum
// in a CTA of fewer than 32 threads) into row.
template <int T>
__device__ __forceinline__ void flux_warp_total(double acc, double *row) {
  double v = acc;
  if constexpr (T >= 32) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) row[threadIdx.x >> 5] = v;
  } else {
    row[threadIdx.x] = v;
  }
}

// After the barrier: warp 0 adds the partial sums by a shuffle tree (thread
// 0 alone in a CTA smaller than a warp) and stores the total.
template <int T>
__device__ __forceinline__ void flux_store(const FluxSpec &f, int step, const double *row) {
  if constexpr (T >= 32) {
    if (threadIdx.x >= 32) return;
    double v = (int)threadIdx.x < flux_slots<T>() ? row[threadIdx.x] : 0.0;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if (threadIdx.x == 0) f.out[step - f.step0] = v;
  } else {
    if (threadIdx.x != 0) return;
    double v = 0.0;
    for (int w = 0; w < flux_slots<T>(); ++w) v += row[w];
    f.out[step - f.step0] = v;
  }
}

}  // namespace pxp
