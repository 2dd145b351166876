// scan_solve.cuh -- tridiagonal solve with a step-invariant matrix as two
// parallel linear-recurrence scans.
//
// When the system matrix does not change between steps (CrankNicholson with a
// z-invariant medium and Dirichlet ends; an ADI half step whose plane holds
// no material), its Thomas factorisation (include/thomasAlgorithm.tpp:2-32)
// is computed once on the host:
//   den_0 = b_0,  den_i = b_i - s * c'_{i-1},  c'_i = s / den_i,
// and stored per position as g_i = 1/den_i and h_i = -s * g_i (s = the
// constant symmetric off-diagonal; h_i is zero at the last position).  Each
// step then needs only the two substitutions, both first-order linear
// recurrences:
//   forward   y_i = g_i r_i + h_i y_{i-1}          (h_{-1} term absent)
//   backward  x_i = y_i + h_i x_{i+1}
// (with symmetric off-diagonals the forward multiplier -s g_i equals the
// backward one -c'_i).  A system of L rows is split into P chunks of M rows,
// one chunk per thread: each thread runs its chunk with a zero carry-in and
// records the chunk's transfer (A, B) (y_out = A y_in + B); a scan of the
// transfers across the P chunks (warp shuffles, then one shared-memory step
// across warps) gives every chunk its carry-in, and a second sweep adds the
// carry-in times the running product of multipliers.  No division occurs in
// the step.  The scan reassociates the products, a rounding-level difference
// from the serial sweep; the multipliers have modulus below one for these
// diagonally dominant systems, so the products stay bounded.
#pragma once
#include "pxp_complex.cuh"

namespace pxp {

struct Affine {
  double2 a, b;  // y_out = a * y_in + b
};

// after(first, second): apply `first`, then `second`.
__device__ __forceinline__ Affine compose(Affine first, Affine second) {
  return {cmul(second.a, first.a), cadd(cmul(second.a, first.b), second.b)};
}

template <bool DOWN>
__device__ __forceinline__ Affine shfl(Affine v, int d) {
  Affine o;
  if (DOWN) {
    o.a.x = __shfl_down_sync(0xffffffffu, v.a.x, d);
    o.a.y = __shfl_down_sync(0xffffffffu, v.a.y, d);
    o.b.x = __shfl_down_sync(0xffffffffu, v.b.x, d);
    o.b.y = __shfl_down_sync(0xffffffffu, v.b.y, d);
  } else {
    o.a.x = __shfl_up_sync(0xffffffffu, v.a.x, d);
    o.a.y = __shfl_up_sync(0xffffffffu, v.a.y, d);
    o.b.x = __shfl_up_sync(0xffffffffu, v.b.x, d);
    o.b.y = __shfl_up_sync(0xffffffffu, v.b.y, d);
  }
  return o;
}

__device__ __forceinline__ Affine shfl_idx(Affine v, int src) {
  Affine o;
  o.a.x = __shfl_sync(0xffffffffu, v.a.x, src);
  o.a.y = __shfl_sync(0xffffffffu, v.a.y, src);
  o.b.x = __shfl_sync(0xffffffffu, v.b.x, src);
  o.b.y = __shfl_sync(0xffffffffu, v.b.y, src);
  return o;
}

// Exclusive scan of chunk transfers over the P threads of each system (the
// P threads are contiguous in the CTA, chunk c at thread offset c, P a power
// of two).  REVERSE = false scans in increasing chunk order (forward
// substitution), true in decreasing order (back substitution).  Returns the
// composition of the transfers of all chunks that precede this one in scan
// order (identity for the first).  `scratch` holds one Affine per warp of the
// CTA; every thread of the CTA must call with the same P.
template <int P, bool REVERSE>
__device__ __forceinline__ Affine exclusive_scan(Affine v, Affine *scratch) {
  const int lane = threadIdx.x & 31;
  constexpr int SEG = P < 32 ? P : 32;  // lanes per system inside a warp
  const int seg_lane = lane & (SEG - 1);
  const Affine ident = {mk(1.0, 0.0), mk(0.0, 0.0)};
  Affine inc = v;
#pragma unroll
  for (int d = 1; d < SEG; d <<= 1) {
    Affine o = shfl<REVERSE>(inc, d);
    const bool take = REVERSE ? (seg_lane + d < SEG) : (seg_lane >= d);
    if (take) inc = compose(o, inc);
  }
  Affine ex = shfl<REVERSE>(inc, 1);
  if (REVERSE ? seg_lane == SEG - 1 : seg_lane == 0) ex = ident;
  if constexpr (P > 32) {
    constexpr int W = P / 32;  // warps per system
    const int warp = threadIdx.x >> 5;
    const int chunk_warp = (threadIdx.x % P) >> 5;  // warp index inside the system
    const int first_warp = warp - chunk_warp;
    __syncthreads();
    // a warp's total is the inclusive value of its last lane in scan order
    if (lane == (REVERSE ? 0 : 31)) scratch[warp] = inc;
    __syncthreads();
    Affine pre = ident;
    if constexpr (W <= 2) {
      if (REVERSE) {
        for (int w = W - 1; w > chunk_warp; --w) pre = compose(pre, scratch[first_warp + w]);
      } else {
        for (int w = 0; w < chunk_warp; ++w) pre = compose(pre, scratch[first_warp + w]);
      }
    } else {
      // every warp scans its system's W warp totals with shuffles (lanes < W)
      // and takes the exclusive value at its own position
      Affine t = lane < W ? scratch[first_warp + lane] : ident;
#pragma unroll
      for (int d = 1; d < W; d <<= 1) {
        Affine o = shfl<REVERSE>(t, d);
        const bool take = REVERSE ? (lane + d < W) : (lane >= d && lane < W);
        if (take) t = compose(o, t);
      }
      const Affine x = shfl_idx(t, REVERSE ? (chunk_warp + 1) & 31 : (chunk_warp + 31) & 31);
      if (REVERSE ? chunk_warp < W - 1 : chunk_warp > 0) pre = x;
    }
    ex = compose(pre, ex);
  }
  return ex;
}

// Solve one system whose chunk rows this thread holds: r[m] is the right-hand
// side of row p0 + m on entry and the solution on exit.  g, h: the factor
// tables in shared memory at padded positions pad8(p).  P threads per
// system, chunk c = thread offset.
template <int M, int P>
__device__ __forceinline__ void const_solve(double2 (&r)[M], const double2 *__restrict__ g,
                                            const double2 *__restrict__ h, int p0,
                                            Affine *scratch) {
  const double2 one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
  // forward, zero carry-in
  double2 prod = one, y = zero;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const double2 hm = h[pad8(p0 + m)];
    y = cadd(cmul(g[pad8(p0 + m)], r[m]), cmul(hm, y));
    prod = cmul(hm, prod);
    r[m] = y;
  }
  Affine ex = exclusive_scan<P, false>(Affine{prod, y}, scratch);
  const double2 y_in = ex.b;
  prod = one;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    prod = cmul(h[pad8(p0 + m)], prod);
    r[m] = cadd(r[m], cmul(prod, y_in));
  }
  // backward, zero carry-in: x_i = y_i + h_i x_{i+1}
  double2 x = zero;
  prod = one;
#pragma unroll
  for (int m = M - 1; m >= 0; --m) {
    const double2 hm = h[pad8(p0 + m)];
    x = cadd(r[m], cmul(hm, x));
    prod = cmul(hm, prod);
    r[m] = x;
  }
  ex = exclusive_scan<P, true>(Affine{prod, x}, scratch);
  const double2 x_in = ex.b;
  prod = one;
#pragma unroll
  for (int m = M - 1; m >= 0; --m) {
    prod = cmul(h[pad8(p0 + m)], prod);
    r[m] = cadd(r[m], cmul(prod, x_in));
  }
}

// Chunk-transposed shared-memory slot of position p (chunk c = p / M, row m =
// p % M) in a length M*P array: slot = m*P + (c ^ (m & 7)).  Threads of a warp
// that read row m of consecutive chunks hit consecutive 16-byte slots, and
// eight consecutive positions (one chunk, rows m..m+7) land in eight
// different 16-byte bank groups, so both the per-chunk reads of the solve and
// the position-order reads and writes of staging are free of bank conflicts
// for 16-byte elements.  P must be a multiple of 8.
template <int M, int P>
__host__ __device__ __forceinline__ int cslot(int c, int m) {
  static_assert(P % 8 == 0, "cslot needs P a multiple of 8");
  return m * P + (c ^ (m & 7));
}
template <int M, int P>
__host__ __device__ __forceinline__ int cslot_pos(int p) {
  return cslot<M, P>(p / M, p % M);
}

// const_solve with the factor tables in chunk-transposed slots (cslot) and
// the step-invariant in-chunk products of the multipliers read from tables:
// pf at a row holds the product of h over the chunk's rows up to and
// including it (forward), pb over the rows from it to the chunk's end
// (backward).  Same recurrences and scans as const_solve.
template <int M, int P>
__device__ __forceinline__ void const_solve_tab(double2 (&r)[M], const double2 *__restrict__ g,
                                                const double2 *__restrict__ h,
                                                const double2 *__restrict__ pf,
                                                const double2 *__restrict__ pb, int c,
                                                Affine *scratch) {
  // forward, zero carry-in: y_i = g_i r_i + h_i y_{i-1}
  double2 y = cmul(g[cslot<M, P>(c, 0)], r[0]);
  r[0] = y;
#pragma unroll
  for (int m = 1; m < M; ++m) {
    const int k = cslot<M, P>(c, m);
    y = cfma(h[k], y, cmul(g[k], r[m]));
    r[m] = y;
  }
  Affine ex = exclusive_scan<P, false>(Affine{pf[cslot<M, P>(c, M - 1)], y}, scratch);
  const double2 y_in = ex.b;
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pf[cslot<M, P>(c, m)], y_in, r[m]);
  // backward, zero carry-in: x_i = y_i + h_i x_{i+1}
  double2 x = r[M - 1];
#pragma unroll
  for (int m = M - 2; m >= 0; --m) {
    x = cfma(h[cslot<M, P>(c, m)], x, r[m]);
    r[m] = x;
  }
  ex = exclusive_scan<P, true>(Affine{pb[cslot<M, P>(c, 0)], x}, scratch);
  const double2 x_in = ex.b;
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pb[cslot<M, P>(c, m)], x_in, r[m]);
}

// const_solve with the factor tables in chunk-transposed slots (cslot) and
// the in-chunk products of the multipliers formed in the sweeps and kept in
// registers for the carry-in fix-ups.
template <int M, int P>
__device__ __forceinline__ void const_solve_reg(double2 (&r)[M], const double2 *__restrict__ g,
                                                const double2 *__restrict__ h, int c,
                                                Affine *scratch) {
  double2 pr[M];
  // forward, zero carry-in: y_i = g_i r_i + h_i y_{i-1}
  double2 y = cmul(g[cslot<M, P>(c, 0)], r[0]);
  pr[0] = h[cslot<M, P>(c, 0)];
  r[0] = y;
#pragma unroll
  for (int m = 1; m < M; ++m) {
    const int k = cslot<M, P>(c, m);
    const double2 hm = h[k];
    y = cfma(hm, y, cmul(g[k], r[m]));
    pr[m] = cmul(hm, pr[m - 1]);
    r[m] = y;
  }
  Affine ex = exclusive_scan<P, false>(Affine{pr[M - 1], y}, scratch);
  const double2 y_in = ex.b;
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pr[m], y_in, r[m]);
  // backward, zero carry-in: x_i = y_i + h_i x_{i+1}
  double2 x = r[M - 1];
  pr[M - 1] = h[cslot<M, P>(c, M - 1)];
#pragma unroll
  for (int m = M - 2; m >= 0; --m) {
    const double2 hm = h[cslot<M, P>(c, m)];
    x = cfma(hm, x, r[m]);
    pr[m] = cmul(hm, pr[m + 1]);
    r[m] = x;
  }
  ex = exclusive_scan<P, true>(Affine{pr[0], x}, scratch);
  const double2 x_in = ex.b;
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pr[m], x_in, r[m]);
}

}  // namespace pxp
