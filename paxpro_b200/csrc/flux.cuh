// flux.cuh -- per-step flux integrals fused into the 2-D step kernels.
//
// post::Transmittivity (src/transmittivity.cpp:30-83) integrates |u|^2 over
// the waveguide after every step with the trapezoid rule
// (trapezoidalIntegrateIntensityZ, :30-41): |u_a|^2 + |u_b|^2 + 2 sum_{a<i<b}
// |u_i|^2, times dx/2.  The step kernels add the weighted terms of the new
// field as they store it (no extra pass over the field): each thread keeps a
// compensated (Neumaier) sum of its points, warps add their threads' sums,
// and thread 0 adds the warp totals after the step's closing barrier.  The
// host applies the dx/2 factor.  |u|^2 is pow(abs(u), 2) as in the
// reference: hypot, then squared.
#pragma once
#include "pxp_kernels.h"

namespace pxp {

struct FluxSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    const double t = s + v;
    c += fabs(s) >= fabs(v) ? (s - t) + v : (v - t) + s;
    s = t;
  }
  __device__ __forceinline__ double total() const { return s + c; }
};

// Window (a, b) of this step, when the job integrates it.
__device__ __forceinline__ bool flux_window(const FluxSpec &f, int step, int2 &w) {
  const int k = step - f.step0;
  if (f.out == nullptr || k < 0 || k >= f.count) return false;
  w = f.win[k];
  return true;
}

__device__ __forceinline__ void flux_add(FluxSum &acc, int i, int2 w, double2 u) {
  if (i < w.x || i > w.y) return;
  const double a = hypot(u.x, u.y);
  const double wt = (i == w.x ? 1.0 : 0.0) + (i == w.y ? 1.0 : 0.0) + ((i > w.x && i < w.y) ? 2.0 : 0.0);
  acc.add(wt * (a * a));
}

// Slots of the per-step partial sums: one per warp, or one per thread when
// the CTA is smaller than a warp.
template <int T> __host__ __device__ constexpr int flux_slots() { return T >= 32 ? T / 32 : T; }

// Before the step's closing barrier: each warp's total (each thread's sum
// in a CTA of fewer than 32 threads) into row.
template <int T>
__device__ __forceinline__ void flux_warp_total(const FluxSum &acc, double *row) {
  double v = acc.total();
  if constexpr (T >= 32) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) row[threadIdx.x >> 5] = v;
  } else {
    row[threadIdx.x] = v;
  }
}

// After the barrier: thread 0 adds the partial sums and stores the total.
template <int T>
__device__ __forceinline__ void flux_store(const FluxSpec &f, int step, const double *row) {
  if (threadIdx.x != 0) return;
  FluxSum t;
  for (int w = 0; w < flux_slots<T>(); ++w) t.add(row[w]);
  f.out[step - f.step0] = t.total();
}

}  // namespace pxp
