// cn.cu -- K-CN: Crank-Nicolson step with a fused tridiagonal solve.
//
// Replaces CrankNicholson::solveStep (src/crancNicholson.cpp:17-105) with the
// default ParaxialEquation (F = G = H = 1, J = 0, src/paraxialEquation.cpp:
// 3-21) and ThomasAlgorithm::solve (include/thomasAlgorithm.tpp:2-32).
//
// One CTA owns one problem; the field stays in shared memory for every step
// of the launch.  Per step:
//   1. each thread builds the matrix rows of its chunk of M consecutive points
//      (diag, rhs; sub-diagonal constant) with the reference's operation
//      order, rounded op by op, so the coefficients equal the reference's;
//   2. each thread eliminates its chunk interior in registers (a partition
//      method: interior x_i = y_i + p_i x_first + q_i x_last) and writes the
//      two boundary equations of its chunk into a reduced system of 2T
//      unknowns;
//   3. the CTA solves the reduced system by cyclic reduction in shared memory;
//   4. each thread reconstructs its interior.
// The solve runs in FP64 in both storage precisions: with rho = dz/(k dx^2)
// of a few hundred the system is only weakly diagonally dominant.
// The split into chunks changes the rounding relative to the reference's
// serial Thomas sweep; the step matrix is well conditioned (Cayley transform,
// condition ~ rho), so the difference stays near machine precision.
#include "pxp_complex.cuh"
#include "flux.cuh"
#include "pxp_kernels.h"
#include <cooperative_groups.h>

#include "scan_solve.cuh"
#include "tridiag.cuh"

namespace cg = cooperative_groups;

namespace pxp {

// Coefficients of row i (exact FP64, reference operation order).
struct CnRow {
  double2 diag, rhs;
};

__device__ __forceinline__ double2 cn_diag(double delta, double beta, double rho, double r) {
  // fval*1.0 + 0.25*(H+ + H-)*g*i*rho + 0.5*(beta*r + i*delta*r)
  double im_a = __dmul_rn(0.5, rho);              // 0.25*(1+1)*1 = 0.5, *i, *rho
  double br = __dmul_rn(beta, r);
  double dr = __dmul_rn(delta, r);
  double2 t = mk(__dmul_rn(0.5, br), __dmul_rn(0.5, dr));
  return mk(__dadd_rn(1.0, t.x), __dadd_rn(im_a, t.y));
}

__device__ __forceinline__ double2 cn_rhs(double2 left, double2 center, double2 right,
                                          double deltaPrev, double betaPrev, double rho,
                                          double r) {
  // rhs = left*H-'*g' + right*H+'*g'; rhs *= 0.25*i*rho
  double2 s = cx_add_rn(left, right);
  double q = __dmul_rn(0.25, rho);
  double2 rhs = cx_mul_rn(s, mk(0.0, q));
  // rhs -= 0.25*center*i*rho*(H+' + H-')*g
  double2 c4 = cx_scale_rn(center, 0.25);
  double2 t = cx_mul_rn(c4, mk(0.0, 1.0));
  t = cx_scale_rn(t, rho);
  t = cx_scale_rn(t, 2.0);
  rhs = cx_sub_rn(rhs, t);
  // rhs += (1.0*f' - 0.5*(beta'*r + i*delta'*r)) * center
  double2 h = mk(__dmul_rn(0.5, __dmul_rn(betaPrev, r)), __dmul_rn(0.5, __dmul_rn(deltaPrev, r)));
  // libstdc++ evaluates (double - complex) as (-y) + x
  double2 coef = mk(__dadd_rn(-h.x, 1.0), -h.y);
  return cx_add_rn(rhs, cx_mul_rn(coef, center));
}

// Transparent boundary (CrankNicholson::applyTBCOneSide,
// src/crancNicholson.cpp:136-148) with H- = g = 1.
__device__ __forceinline__ void cn_tbc(double2 outer, double2 inner, double rho, double2 &diag,
                                       double2 &rhs) {
  double2 ratio = cx_div_rn(outer, inner);
  double lr = log(hypot(ratio.x, ratio.y));
  double ar = atan2(ratio.y, ratio.x);
  double2 kdx = cx_div_rn(mk(lr, ar), mk(0.0, 1.0));
  if (kdx.x < 0.0) kdx.x = 0.0;
  double2 ik = cx_mul_rn(mk(0.0, 1.0), kdx);
  double e = exp(ik.x);
  double sn, cs;
  sincos(ik.y, &sn, &cs);
  double2 ex = mk(e * cs, e * sn);
  double2 coef = cx_mul_rn(mk(0.0, __dmul_rn(0.25, rho)), ex);
  diag = cx_sub_rn(diag, coef);
  rhs = cx_add_rn(rhs, cx_mul_rn(coef, outer));
}

template <typename R, int M, int T, bool FLUX>
__global__ void __launch_bounds__(T) cn_kernel(const CnJob *__restrict__ jobs, int step0_ov,
                                              int nsteps_ov) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double flux_red[2][flux_slots<T>()];
  CnJob job = jobs[blockIdx.x];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int n = job.n;  // == M * T
  // rows at and beyond nreal pad the system to M * T: diagonal kCnPad, zero
  // right-hand side and zero field, so they decouple from row nreal - 1 to
  // within |sub|^2 / kCnPad (the field beyond the grid is the Dirichlet zero)
  const int nreal = job.n_real > 0 ? job.n_real : n;
  const int nr = 2 * T;
  double2 *ra = reinterpret_cast<double2 *>(smem_raw);
  double2 *rb = ra + nr;
  double2 *rc = rb + nr;
  double2 *rd = rc + nr;
  C *u = reinterpret_cast<C *>(rd + nr);
  const int t = threadIdx.x;
  C *field = reinterpret_cast<C *>(job.field);
  for (int i = t; i < n; i += T) u[i] = i < nreal ? field[i] : C{};
  __syncthreads();
  const double rho = job.rho, r = job.r;
  const double2 sub = mk(-0.0, __dmul_rn(-0.25, rho));  // -0.25*i*rho*H-*g
  C *saves = reinterpret_cast<C *>(job.saves);
  const int s0 = t * M;

  for (int st = 0; st < job.nsteps; ++st) {
    const int step = job.step0 + st;
    // this step's flux window, loaded early so its latency hides behind the step
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    const long long moff = job.mat_stride * (long long)(step - job.mat_step0);
    // ---- 1. rows of this chunk
    double2 dg[M], rh[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      int i = s0 + m;
      if (i >= nreal) {
        dg[m] = mk(kCnPad, 0.0);
        rh[m] = mk(0.0, 0.0);
        continue;
      }
      double2 center = to_d(u[i]);
      double2 left = i > 0 ? to_d(u[i - 1]) : mk(0.0, 0.0);
      double2 right = i < nreal - 1 ? to_d(u[i + 1]) : mk(0.0, 0.0);
      double de = job.delta[moff + i], be = job.beta[moff + i];
      double dp = job.delta_prev[moff + i], bp = job.beta_prev[moff + i];
      dg[m] = cn_diag(de, be, rho, r);
      rh[m] = cn_rhs(left, center, right, dp, bp, rho, r);
    }
    if (job.transparent) {
      const double ZERO = 1e-16;
      if (t == 0) {
        double2 o = to_d(u[0]), in = to_d(u[1]);
        if (hypot(in.x, in.y) > ZERO) cn_tbc(o, in, rho, dg[0], rh[0]);
      }
      if (t == T - 1) {
        double2 o = to_d(u[n - 1]), in = to_d(u[n - 2]);
        if (hypot(in.x, in.y) > ZERO) cn_tbc(o, in, rho, dg[M - 1], rh[M - 1]);
      }
    }
    // ---- 2. interior elimination (partition method)
    double2 y[M > 2 ? M - 2 : 1], p[M > 2 ? M - 2 : 1], q[M > 2 ? M - 2 : 1];
    const ReducedRows rr = chunk_eliminate<M>(dg, rh, sub, s0 > 0, s0 + M < n, y, p, q);
    const double2 ea = rr.ea, eb = rr.eb, ec = rr.ec, ed = rr.ed;
    const double2 fa = rr.fa, fb = rr.fb, fc = rr.fc, fd = rr.fd;
    ra[2 * t] = ea; rb[2 * t] = eb; rc[2 * t] = ec; rd[2 * t] = ed;
    ra[2 * t + 1] = fa; rb[2 * t + 1] = fb; rc[2 * t + 1] = fc; rd[2 * t + 1] = fd;
    __syncthreads();
    // ---- 3. reduced system
    cyclic_reduction(ra, rb, rc, rd, nr, t, T);
    // ---- 4. reconstruct
    const double2 xf = rd[2 * t], xl = rd[2 * t + 1];
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * nreal : nullptr;
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const C v = from_d<R>(chunk_value<M>(m, xf, xl, y, p, q));
      u[s0 + m] = v;
      if (save && s0 + m < nreal) slot[s0 + m] = v;
      if (flux) flux_add(acc, s0 + m, fw, to_d(v));
    }
    if (flux) flux_warp_total<T>(acc, flux_red[st & 1]);
    __syncthreads();
    if (flux) flux_store<T>(job.flux, step, flux_red[st & 1]);
  }
  for (int i = t; i < nreal; i += T) field[i] = u[i];
}

// z-invariant medium, Dirichlet ends: the step matrix is fixed, so the
// factor tables g, h (host-computed) are loaded into shared memory once and
// each step is the right-hand-side stencil plus two substitution scans
// (scan_solve.cuh).  The field stays in registers: thread t owns points
// t*M .. t*M+M-1 and trades its two edge values with its neighbours through
// shared memory.  The right-hand side is regrouped as
// i*q*(left + right) + d*centre, q = rho/4, with the per-point coefficient
// d = (1 - 0.5*(beta'*r + i*delta'*r)) - i*rho/2 formed once (the first part
// with the reference's rounding) and kept in shared memory; the regrouping
// and the FMAs differ from the reference's operation order at rounding level.
// Tables sit in chunk-transposed slots (cslot), free of bank conflicts.
template <typename R, int M, int T, bool FLUX>
__global__ void __launch_bounds__(T) cn_const_kernel(const CnJob *__restrict__ jobs, int step0_ov,
                                                    int nsteps_ov) {
  using C = typename Cx<R>::T;
  constexpr int N = M * T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *gs = reinterpret_cast<double2 *>(smem_raw);
  double2 *hs = gs + N;
  double2 *ds = hs + N;
  double2 *xch = ds + N;  // 2 per thread
  Affine *scratch = reinterpret_cast<Affine *>(xch + 2 * T);
  __shared__ double flux_red[2][flux_slots<T>()];
  CnJob job = jobs[blockIdx.x];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int t = threadIdx.x;
  const double rho = job.rho, r = job.r;
  const double2 *gt = reinterpret_cast<const double2 *>(job.lu_g);
  const double2 *ht = reinterpret_cast<const double2 *>(job.lu_h);
  const double q = __dmul_rn(0.25, rho);
  const int s0 = t * M;
  // rows nreal..N-1 pad the system (their factor-table rows were built with
  // diagonal kCnPad on the host; their right-hand side is zero)
  const int nreal = job.n_real > 0 ? job.n_real : N;
  // each thread fills the slots of its own chunk
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int k = cslot<M, T>(t, m);
    gs[k] = gt[s0 + m];
    hs[k] = ht[s0 + m];
    if (s0 + m < nreal) {
      const double bp = job.beta_prev[s0 + m], dp = job.delta_prev[s0 + m];
      const double2 hh = mk(__dmul_rn(0.5, __dmul_rn(bp, r)), __dmul_rn(0.5, __dmul_rn(dp, r)));
      ds[k] = mk(__dadd_rn(-hh.x, 1.0), __dsub_rn(-hh.y, 0.5 * rho));
    } else {
      ds[k] = mk(0.0, 0.0);
    }
  }
  C *field = reinterpret_cast<C *>(job.field);
  double2 u[M];
#pragma unroll
  for (int m = 0; m < M; ++m) u[m] = s0 + m < nreal ? to_d(field[s0 + m]) : mk(0.0, 0.0);
  C *saves = reinterpret_cast<C *>(job.saves);
  for (int st = 0; st < job.nsteps; ++st) {
    const int step = job.step0 + st;
    // this step's flux window, loaded early so its latency hides behind the step
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    xch[2 * t] = u[0];
    xch[2 * t + 1] = u[M - 1];
    __syncthreads();
    const double2 lft = t > 0 ? xch[2 * t - 1] : mk(0.0, 0.0);
    const double2 rgt = t < T - 1 ? xch[2 * t + 2] : mk(0.0, 0.0);
    double2 rh[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double2 left = m > 0 ? u[m - 1] : lft;
      // the Dirichlet zero beyond the last real row
      const double2 right = s0 + m + 1 >= nreal ? mk(0.0, 0.0) : (m < M - 1 ? u[m + 1] : rgt);
      const double2 sum = cadd(left, right);
      rh[m] = s0 + m < nreal ? cfma(ds[cslot<M, T>(t, m)], u[m], mk(-q * sum.y, q * sum.x))
                             : mk(0.0, 0.0);
    }
    const_solve_reg<M, T>(rh, gs, hs, t, scratch);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * nreal : nullptr;
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const C v = from_d<R>(rh[m]);
      u[m] = to_d(v);
      if (save && s0 + m < nreal) slot[s0 + m] = v;
      if (flux) flux_add(acc, s0 + m, fw, u[m]);
    }
    if (flux) flux_warp_total<T>(acc, flux_red[st & 1]);
    __syncthreads();  // xch is rewritten next step
    if (flux) flux_store<T>(job.flux, step, flux_red[st & 1]);
  }
#pragma unroll
  for (int m = 0; m < M; ++m)
    if (s0 + m < nreal) field[s0 + m] = from_d<R>(u[m]);
}

// The same step for systems of K * M * T rows (8192 and 16384) on a cluster
// of K CTAs, one per SM, CTA k holding rows [k*M*T, (k+1)*M*T) with its
// slice of the factor tables in shared memory.  What crosses CTAs goes
// through distributed shared memory, each behind one cluster barrier:
//   * the stencil halo: the first and last rows of the neighbouring CTAs;
//   * the forward recurrence's carry: each CTA scans its chunks as in the
//     single-CTA kernel, publishes its total transfer (y_end = a y_start +
//     b), and folds the totals of the CTAs before it to get its y_start;
//   * the backward recurrence's carry, likewise from the CTAs after it.
// Every chunk's carry-in is then ex.a * start + ex.b (ex: the in-CTA
// exclusive scan), the single-CTA fix-up with a nonzero CTA start.
template <int M, int P>
__device__ __forceinline__ void const_solve_cluster(double2 (&r)[M], const double2 *__restrict__ g,
                                                    const double2 *__restrict__ h, int c,
                                                    Affine *scratch, Affine *tot_fwd,
                                                    Affine *tot_bwd, cg::cluster_group &cluster,
                                                    int rank, int K) {
  double2 pr[M];
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
  const Affine own_f{pr[M - 1], y};
  Affine ex = exclusive_scan<P, false>(own_f, scratch);
  if (c == P - 1) *tot_fwd = compose(ex, own_f);  // this CTA's total transfer
  cluster.sync();
  double2 start = mk(0.0, 0.0);  // y at the end of the previous CTA's rows
  for (int j = 0; j < rank; ++j) {
    const Affine t = *cluster.map_shared_rank(tot_fwd, j);
    start = cfma(t.a, start, t.b);
  }
  const double2 y_in = cfma(ex.a, start, ex.b);
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pr[m], y_in, r[m]);
  double2 x = r[M - 1];
  pr[M - 1] = h[cslot<M, P>(c, M - 1)];
#pragma unroll
  for (int m = M - 2; m >= 0; --m) {
    const double2 hm = h[cslot<M, P>(c, m)];
    x = cfma(hm, x, r[m]);
    pr[m] = cmul(hm, pr[m + 1]);
    r[m] = x;
  }
  const Affine own_b{pr[0], x};
  ex = exclusive_scan<P, true>(own_b, scratch);
  if (c == 0) *tot_bwd = compose(ex, own_b);
  cluster.sync();
  start = mk(0.0, 0.0);  // x at the first row of the next CTA
  for (int j = K - 1; j > rank; --j) {
    const Affine t = *cluster.map_shared_rank(tot_bwd, j);
    start = cfma(t.a, start, t.b);
  }
  const double2 x_in = cfma(ex.a, start, ex.b);
#pragma unroll
  for (int m = 0; m < M; ++m) r[m] = cfma(pr[m], x_in, r[m]);
}

template <typename R, int M, int T, int K, bool FLUX>
__global__ void __launch_bounds__(T) cn_const_cluster_kernel(const CnJob *__restrict__ jobs,
                                                            int step0_ov, int nsteps_ov) {
  using C = typename Cx<R>::T;
  constexpr int NC = M * T;  // rows of this CTA
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double2 *gs = reinterpret_cast<double2 *>(smem_raw);
  double2 *hs = gs + NC;
  double2 *ds = hs + NC;
  double2 *xch = ds + NC;  // 2 per thread
  Affine *scratch = reinterpret_cast<Affine *>(xch + 2 * T);
  __shared__ Affine tot_fwd, tot_bwd;
  __shared__ double flux_red[2][flux_slots<T>()];
  __shared__ double flux_part[K];
  CnJob job = jobs[blockIdx.x / K];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int t = threadIdx.x;
  const double rho = job.rho, r = job.r;
  const double2 *gt = reinterpret_cast<const double2 *>(job.lu_g);
  const double2 *ht = reinterpret_cast<const double2 *>(job.lu_h);
  const double q = __dmul_rn(0.25, rho);
  const int base = rank * NC;     // first row of this CTA
  const int s0 = base + t * M;    // first row of this thread
  const int nreal = job.n_real > 0 ? job.n_real : K * NC;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int k = cslot<M, T>(t, m);
    gs[k] = gt[s0 + m];
    hs[k] = ht[s0 + m];
    if (s0 + m < nreal) {
      const double bp = job.beta_prev[s0 + m], dp = job.delta_prev[s0 + m];
      const double2 hh = mk(__dmul_rn(0.5, __dmul_rn(bp, r)), __dmul_rn(0.5, __dmul_rn(dp, r)));
      ds[k] = mk(__dadd_rn(-hh.x, 1.0), __dsub_rn(-hh.y, 0.5 * rho));
    } else {
      ds[k] = mk(0.0, 0.0);
    }
  }
  C *field = reinterpret_cast<C *>(job.field);
  double2 u[M];
#pragma unroll
  for (int m = 0; m < M; ++m) u[m] = s0 + m < nreal ? to_d(field[s0 + m]) : mk(0.0, 0.0);
  C *saves = reinterpret_cast<C *>(job.saves);
  const double2 *xch_prev = rank > 0 ? cluster.map_shared_rank(xch, rank - 1) : nullptr;
  const double2 *xch_next = rank < K - 1 ? cluster.map_shared_rank(xch, rank + 1) : nullptr;
  for (int st = 0; st < job.nsteps; ++st) {
    const int step = job.step0 + st;
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    xch[2 * t] = u[0];
    xch[2 * t + 1] = u[M - 1];
    cluster.sync();  // every CTA's edge rows are published
    double2 lft = mk(0.0, 0.0), rgt = mk(0.0, 0.0);
    if (t > 0) lft = xch[2 * t - 1];
    else if (rank > 0) lft = xch_prev[2 * T - 1];
    if (t < T - 1) rgt = xch[2 * t + 2];
    else if (rank < K - 1) rgt = xch_next[0];
    double2 rh[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double2 left = m > 0 ? u[m - 1] : lft;
      const double2 right = s0 + m + 1 >= nreal ? mk(0.0, 0.0) : (m < M - 1 ? u[m + 1] : rgt);
      const double2 sum = cadd(left, right);
      rh[m] = s0 + m < nreal ? cfma(ds[cslot<M, T>(t, m)], u[m], mk(-q * sum.y, q * sum.x))
                             : mk(0.0, 0.0);
    }
    const_solve_cluster<M, T>(rh, gs, hs, t, scratch, &tot_fwd, &tot_bwd, cluster, rank, K);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * nreal : nullptr;
    double acc = 0.0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const C v = from_d<R>(rh[m]);
      u[m] = to_d(v);
      if (save && s0 + m < nreal) slot[s0 + m] = v;
      if (flux) flux_add(acc, s0 + m, fw, u[m]);
    }
    if constexpr (FLUX) {
      if (flux) flux_warp_total<T>(acc, flux_red[st & 1]);
      __syncthreads();
      if (flux && t < 32) {
        double v = t < flux_slots<T>() ? flux_red[st & 1][t] : 0.0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if (t == 0) *cluster.map_shared_rank(&flux_part[rank], 0) = v;
      }
      cluster.sync();  // every CTA's total is in CTA 0's flux_part
      if (flux && rank == 0 && t == 0) {
        double v = 0.0;
        for (int j = 0; j < K; ++j) v += flux_part[j];
        job.flux.out[step - job.flux.step0] = v;
      }
    }
  }
  cluster.sync();  // no CTA leaves while a peer may still address its shared memory
#pragma unroll
  for (int m = 0; m < M; ++m)
    if (s0 + m < nreal) field[s0 + m] = from_d<R>(u[m]);
}

static constexpr int kCnM = 8;

template <typename R, int M, int T, bool FLUX>
static cudaError_t cn_const_launch_f(const CnJob *d_jobs, int nj, int step0, int nsteps,
                                     cudaStream_t s) {
  constexpr int N = M * T;
  constexpr size_t smem = sizeof(double2) * (3 * N + 2 * T) + sizeof(Affine) * (T / 32 + 1);
  auto k = cn_const_kernel<R, M, T, FLUX>;
  {  // the static flux slots count against the 48 KB default too
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  k<<<nj, T, smem, s>>>(d_jobs, step0, nsteps);
  return cudaGetLastError();
}

template <typename R, int M, int T>
static cudaError_t cn_const_launch_t(const CnJob *d_jobs, int nj, int step0, int nsteps,
                                     cudaStream_t s, bool flux) {
  return flux ? cn_const_launch_f<R, M, T, true>(d_jobs, nj, step0, nsteps, s)
              : cn_const_launch_f<R, M, T, false>(d_jobs, nj, step0, nsteps, s);
}

template <typename R, int M, int T, int K, bool FLUX>
static cudaError_t cn_cluster_launch_f(const CnJob *d_jobs, int nj, int step0, int nsteps,
                                       cudaStream_t s) {
  constexpr int NC = M * T;
  constexpr size_t smem = sizeof(double2) * (3 * NC + 2 * T) + sizeof(Affine) * (T / 32 + 1);
  auto k = cn_const_cluster_kernel<R, M, T, K, FLUX>;
  {
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(K * nj);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = K;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, d_jobs, step0, nsteps);
}

template <typename R, int K, int M = 16, int T = 256>
static cudaError_t cn_cluster_launch_t(const CnJob *d_jobs, int nj, int step0, int nsteps,
                                       cudaStream_t s, bool flux) {
  return flux ? cn_cluster_launch_f<R, M, T, K, true>(d_jobs, nj, step0, nsteps, s)
              : cn_cluster_launch_f<R, M, T, K, false>(d_jobs, nj, step0, nsteps, s);
}

// 4096 rows on a cluster of two CTAs (2048 rows each) is variant 1: the
// single-CTA step is bound by one SM's FP64 issue rate (about 36 FP64
// operations a row) and its scans' latency, the pair halves the first and
// adds two cluster barriers a step.
int cn_const_variants(Precision, int n) { return n == 4096 ? 2 : 1; }

bool cn_const_supported(Precision, int n) {
  return n >= 8 * kCnM && !(n & (n - 1)) && n <= 16384;  // 8192, 16384: clusters of 2, 4
}

cudaError_t launch_cn_const(Precision p, const CnJob *d_jobs, int nj, int n, int step0, int nsteps,
                            cudaStream_t s, bool flux, int variant) {
  if (nj <= 0) return cudaSuccess;
  if (n == 8192)
    return p == kFP64 ? cn_cluster_launch_t<double, 2>(d_jobs, nj, step0, nsteps, s, flux)
                      : cn_cluster_launch_t<float, 2>(d_jobs, nj, step0, nsteps, s, flux);
  if (n == 16384)
    return p == kFP64 ? cn_cluster_launch_t<double, 4>(d_jobs, nj, step0, nsteps, s, flux)
                      : cn_cluster_launch_t<float, 4>(d_jobs, nj, step0, nsteps, s, flux);
  // n >= 2048: 16 rows per thread (half the threads of 8 rows: fewer warps
  // in each scan's barriers and shuffles; measured 4.07 -> 3.08 us per step
  // at n = 4096)
  if (n == 4096 && variant == 1)
    return p == kFP64 ? cn_cluster_launch_t<double, 2, 16, 128>(d_jobs, nj, step0, nsteps, s, flux)
                      : cn_cluster_launch_t<float, 2, 16, 128>(d_jobs, nj, step0, nsteps, s, flux);
  if (n == 4096)
    return p == kFP64 ? cn_const_launch_t<double, 16, 256>(d_jobs, nj, step0, nsteps, s, flux)
                      : cn_const_launch_t<float, 16, 256>(d_jobs, nj, step0, nsteps, s, flux);
  if (n == 2048)
    return p == kFP64 ? cn_const_launch_t<double, 16, 128>(d_jobs, nj, step0, nsteps, s, flux)
                      : cn_const_launch_t<float, 16, 128>(d_jobs, nj, step0, nsteps, s, flux);
#define PXP_CC(TT)                                                                     \
  case TT:                                                                             \
    return p == kFP64 ? cn_const_launch_t<double, kCnM, TT>(d_jobs, nj, step0, nsteps, s, flux) \
                      : cn_const_launch_t<float, kCnM, TT>(d_jobs, nj, step0, nsteps, s, flux);
  switch (n / kCnM) {
    PXP_CC(8) PXP_CC(16) PXP_CC(32) PXP_CC(64) PXP_CC(128)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_CC
}

template <typename R, int T, bool FLUX>
static cudaError_t cn_launch_f(const CnJob *d_jobs, int nj, int step0, int nsteps,
                               cudaStream_t s) {
  using C = typename Cx<R>::T;
  size_t smem = sizeof(double2) * 4 * 2 * T + sizeof(C) * kCnM * T;
  auto k = cn_kernel<R, kCnM, T, FLUX>;
  {  // the static flux slots count against the 48 KB default too
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  k<<<nj, T, smem, s>>>(d_jobs, step0, nsteps);
  return cudaGetLastError();
}

template <typename R, int T>
static cudaError_t cn_launch_t(const CnJob *d_jobs, int nj, int step0, int nsteps, cudaStream_t s,
                               bool flux) {
  return flux ? cn_launch_f<R, T, true>(d_jobs, nj, step0, nsteps, s)
              : cn_launch_f<R, T, false>(d_jobs, nj, step0, nsteps, s);
}

int cn_padded_n(int n) {
  int t = 2;
  while (t * kCnM < n) t *= 2;
  return t * kCnM;
}

bool cn_supported(Precision p, int n) {
  if (n < 2 * kCnM) return false;
  const int np = cn_padded_n(n);
  return p == kFP64 ? np <= 4096 : np <= 8192;
}

cudaError_t launch_cn(Precision p, const CnJob *d_jobs, int nj, int n, int step0, int nsteps,
                      cudaStream_t s, bool flux) {
  if (nj <= 0) return cudaSuccess;
  const int T = n / kCnM;
#define PXP_CN(TT)                                                                 \
  case TT:                                                                         \
    return p == kFP64 ? cn_launch_t<double, TT>(d_jobs, nj, step0, nsteps, s, flux) \
                      : cn_launch_t<float, TT>(d_jobs, nj, step0, nsteps, s, flux);
  switch (T) {
    PXP_CN(2) PXP_CN(4) PXP_CN(8) PXP_CN(16) PXP_CN(32) PXP_CN(64) PXP_CN(128) PXP_CN(256)
    PXP_CN(512)
    case 1024:
      if (p == kFP32) return cn_launch_t<float, 1024>(d_jobs, nj, step0, nsteps, s, flux);
      return cudaErrorInvalidValue;
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_CN
}

}  // namespace pxp
