// adi.cu -- K-ADI: one alternating-direction half step with the right-hand
// side stencil fused with a parallel complex tridiagonal solve.
//
// Replaces ADI::xImplicit / ADI::yImplicit / ADI::applyTBC
// (src/alternatingDirectionSolver.cpp:8-234) and the ThomasAlgorithm sweep
// over the chain of n*n unknowns (include/thomasAlgorithm.tpp:2-32), whose
// zero sub-diagonal entries at every system start make the n systems of a
// half step independent.
//
// A CTA owns G consecutive systems.  It stages them, plus one halo system on
// each side for the explicit stencil, in shared memory with loads that are
// coalesced for either layout (systems interleaved in memory for the x half
// step, contiguous for the y half step).  Each system is split into
// P = n/M chunks, one per thread; the chunk rows are built with the
// reference's operation order (matrix coefficients equal the reference's),
// the chunk interior is eliminated in registers, and the 2P-unknown reduced
// system is solved by cyclic reduction in shared memory.  The solution goes
// back through shared memory for coalesced stores.
//
// Materials: a first-hit sphere list evaluated per point with rounded FP64
// operations (the same r^2 < R^2 test as the oracle); the host culls, per
// half step, spheres whose dz^2 alone is >= R^2, which cannot contain any
// point of the plane.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "bulk_copy.cuh"
#include "csg.cuh"
#include "pxp_complex.cuh"
#include "pxp_kernels.h"
#include "scan_solve.cuh"
#include "tridiag.cuh"

namespace pxp {

// kernel waits that ran out on this device (never reset), read by the host
__device__ unsigned int g_wait_timeouts = 0;

// The material of the half step's plane at (x, y); idx: the point's index in
// the field's layout, for a sampled plane.
__device__ __forceinline__ void sphere_material(const AdiHalf &h, double x, double y,
                                                long long idx, double &delta, double &beta) {
  if (h.plane_delta) {
    delta = h.plane_delta[idx];
    beta = h.plane_beta[idx];
    return;
  }
  if (h.csg.active) {
    csg_material(h.csg, x, y, h.z, delta, beta);
    return;
  }
  delta = 0.0;
  beta = 0.0;
  const int n = h.nspheres;
  const Sphere *list = n > kInlineSpheres ? h.spheres_all : h.spheres;
  for (int i = 0; i < n; ++i) {
    const Sphere sp = list[i];
    double ddx = __dsub_rn(x, sp.cx), ddy = __dsub_rn(y, sp.cy), ddz = __dsub_rn(h.z, sp.cz);
    double rsq = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
    if (rsq < __dmul_rn(sp.r, sp.r)) {
      delta = sp.delta;
      beta = sp.beta;
      return;
    }
  }
}

// Transparent-boundary factor 0.5*i*exp(i*kd)/kd2 with kd = -i*log(ratio),
// Re(kd) clamped at 0 (src/alternatingDirectionSolver.cpp:157-234).
__device__ __forceinline__ double2 tbc_factor(double2 num, double2 den) {
  double2 ratio = cx_div_rn(num, den);
  double2 lg = mk(log(hypot(ratio.x, ratio.y)), atan2(ratio.y, ratio.x));
  double2 kd = cx_mul_rn(mk(-0.0, -1.0), lg);
  if (kd.x < 0.0) kd.x = 0.0;
  double2 ik = cx_mul_rn(mk(0.0, 1.0), kd);
  double e = exp(ik.x), sn, cs;
  sincos(ik.y, &sn, &cs);
  return cx_mul_rn(mk(0.0, 0.5), mk(e * cs, e * sn));
}

// Diagonal of the padding rows of a system padded to M times a power of two.
constexpr double kAdiPad = 1e30;

template <typename R, int M, int G>
__global__ void __launch_bounds__(512) adi_half_kernel(const AdiHalf h) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // n: rows of each solved system (h.n, or h.n padded to M times a power of
  // two); nreal: the grid's positions per system and its number of systems.
  // Pad rows get diagonal kAdiPad, zero right-hand side and zero field, so
  // they decouple from the last real row to within |sub|^2 / kAdiPad.
  const int n = h.n_pad > 0 ? h.n_pad : h.n;
  const int nreal = h.n;
  const int P = n / M;        // chunks per system
  const int T = G * P;        // threads
  const int ld = n + n / 8 + 2;  // padded row of the staging tile (pad8)
  C *tile = reinterpret_cast<C *>(smem_raw);                  // (G+2) x ld
  double2 *red = reinterpret_cast<double2 *>(
      smem_raw + ((sizeof(C) * (G + 2) * ld + 15) & ~size_t(15)));  // 4 x G x 2P
  const int nr = 2 * P;
  const int tid = threadIdx.x;
  const int s_base = blockIdx.x * G;  // first system of this CTA
  const C *in = reinterpret_cast<const C *>(h.in);
  C *out = reinterpret_cast<C *>(h.out);
  const bool interleaved = h.stride_sys == 1;

  // ---- stage systems s_base-1 .. s_base+G (out-of-range halo rows zero)
  const int rows = G + 2;
  for (int idx = tid; idx < rows * n; idx += T) {
    int g, p;
    if (interleaved) {
      p = idx / rows;
      g = idx - p * rows;
    } else {
      g = idx / n;
      p = idx - g * n;
    }
    const int s = s_base - 1 + g;
    C v = from_d<R>(mk(0.0, 0.0));
    if (s >= 0 && s < nreal && p < nreal)
      v = in[(long long)p * h.stride_pos + (long long)s * h.stride_sys];
    tile[g * ld + pad8(p)] = v;
  }
  __syncthreads();

  const int g = tid / P;          // system within the CTA
  const int c = tid - g * P;      // chunk
  const int s = s_base + g;       // global system index
  const int p0 = c * M;
  const double2 sub = mk(-0.0, __ddiv_rn(-0.5, h.kd2_impl));  // -0.5*i/(k d^2)
  const double inv_kd2_impl = __ddiv_rn(1.0, h.kd2_impl);
  const double inv_kd2_expl = __ddiv_rn(1.0, h.kd2_expl);
  // y half step diagonal in vacuum: i/(k dy^2 + 0 + i 0) = (0, 1/(k dy^2))
  // exactly (Smith's division with a zero imaginary part).
  const C *ctr = tile + (g + 1) * ld;
  const C *lft = tile + g * ld;
  const C *rgt = tile + (g + 2) * ld;

  double2 dg[M], rh[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int p = p0 + m;
    if (p >= nreal) {
      dg[m] = mk(kAdiPad, 0.0);
      rh[m] = mk(0.0, 0.0);
      continue;
    }
    // coordinates: position runs along x in the x half step, along y in the y half step
    double x, y;
    const double pos_c = (double)p, sys_c = (double)s;
    if (!h.y_implicit) {
      x = __dadd_rn(h.xmin, __dmul_rn(pos_c, h.dx));
      y = __dadd_rn(h.ymin, __dmul_rn(sys_c, h.dy));
    } else {
      x = __dadd_rn(h.xmin, __dmul_rn(sys_c, h.dx));
      y = __dadd_rn(h.ymin, __dmul_rn(pos_c, h.dy));
    }
    double delta, beta;
    sphere_material(h, x, y,
                    h.y_implicit ? (long long)s * h.n + p : (long long)p * h.n + s, delta, beta);
    if (!h.y_implicit) {
      // 1.0/dz + i/(k dx dx) + beta*k + i*delta*k   (reference :38)
      dg[m] = mk(__dadd_rn(h.inv_dzh, __dmul_rn(beta, h.k)),
                 __dadd_rn(inv_kd2_impl, __dmul_rn(delta, h.k)));
    } else {
      // 1.0/dz + i/(k dy dy + beta*k + i*delta*k)   (reference :103, as written)
      double2 q = mk(0.0, inv_kd2_impl);
      if (delta != 0.0 || beta != 0.0)
        q = cx_div_rn(mk(0.0, 1.0), mk(__dadd_rn(h.kd2_impl, __dmul_rn(beta, h.k)),
                                       __dmul_rn(delta, h.k)));
      dg[m] = mk(__dadd_rn(q.x, h.inv_dzh), q.y);
    }
    // rhs = (1/dz - i/(k d_e^2)) u + 0.5 i (u_left + u_right)/(k d_e^2); the
    // reference divides each neighbour term by k d_e^2, here it is one
    // multiplication by the reciprocal (a rounding-level difference).
    const double2 uc = to_d(ctr[pad8(p)]);
    double2 r = cmul(mk(h.inv_dzh, -inv_kd2_expl), uc);
    double2 nb = mk(0.0, 0.0);
    if (s > 0) nb = to_d(lft[pad8(p)]);
    if (s < nreal - 1) nb = cadd(nb, to_d(rgt[pad8(p)]));
    const double hk = 0.5 * inv_kd2_expl;
    r = mk(fma(-hk, nb.y, r.x), fma(hk, nb.x, r.y));
    rh[m] = r;
  }
  if (h.use_tbc) {
    const double zero = 1e-6;
    // along the system (implicit direction): diagonal at both ends (the last
    // real row: row n - 1 of an unpadded system)
    if (p0 <= nreal - 1 && nreal - 1 < p0 + M) {
      double2 inner = to_d(ctr[pad8(nreal - 2)]);
      if (hypot(inner.x, inner.y) > zero) {
        const double2 t = cx_div_real_rn(tbc_factor(to_d(ctr[pad8(nreal - 1)]), inner), h.kd2_impl);
#pragma unroll
        for (int m = 0; m < M; ++m)
          if (p0 + m == nreal - 1) dg[m] = cx_sub_rn(dg[m], t);
      }
    }
    if (c == 0) {
      double2 inner = to_d(ctr[pad8(1)]);
      if (hypot(inner.x, inner.y) > zero)
        dg[0] = cx_sub_rn(dg[0], cx_div_real_rn(tbc_factor(to_d(ctr[pad8(0)]), inner), h.kd2_impl));
    }
    // across systems (explicit direction): rhs of the first and last system
    if (s == nreal - 1 || s == 0) {
      const C *inner_row = (s == nreal - 1) ? lft : rgt;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int p = p0 + m;
        if (p >= nreal) continue;
        double2 inner = to_d(inner_row[pad8(p)]);
        if (hypot(inner.x, inner.y) > zero) {
          double2 edge = to_d(ctr[pad8(p)]);
          double2 f = cx_mul_rn(tbc_factor(edge, inner), edge);
          rh[m] = cx_add_rn(rh[m], cx_div_real_rn(f, h.kd2_expl));
        }
      }
    }
  }

  double2 yv[M > 2 ? M - 2 : 1], pv[M > 2 ? M - 2 : 1], qv[M > 2 ? M - 2 : 1];
  const ReducedRows rr = chunk_eliminate<M>(dg, rh, sub, p0 > 0, p0 + M < n, yv, pv, qv);
  double2 *ra = red + (0 * G + g) * nr;
  double2 *rb = red + (1 * G + g) * nr;
  double2 *rc = red + (2 * G + g) * nr;
  double2 *rd = red + (3 * G + g) * nr;
  ra[2 * c] = rr.ea; rb[2 * c] = rr.eb; rc[2 * c] = rr.ec; rd[2 * c] = rr.ed;
  ra[2 * c + 1] = rr.fa; rb[2 * c + 1] = rr.fb; rc[2 * c + 1] = rr.fc; rd[2 * c + 1] = rr.fd;
  __syncthreads();  // also: every read of the staged tile is done
  cyclic_reduction(ra, rb, rc, rd, nr, c, P);
  const double2 xf = rd[2 * c], xl = rd[2 * c + 1];
  C *dst = tile + (g + 1) * ld;
#pragma unroll
  for (int m = 0; m < M; ++m) dst[pad8(p0 + m)] = from_d<R>(chunk_value<M>(m, xf, xl, yv, pv, qv));
  __syncthreads();
  C *save = reinterpret_cast<C *>(h.save);
  for (int idx = tid; idx < G * n; idx += T) {
    int gg, p;
    if (interleaved) {
      p = idx / G;
      gg = idx - p * G;
    } else {
      gg = idx / n;
      p = idx - gg * n;
    }
    if (p >= nreal || s_base + gg >= nreal) continue;
    const long long off = (long long)p * h.stride_pos + (long long)(s_base + gg) * h.stride_sys;
    const C v = tile[(gg + 1) * ld + pad8(p)];
    out[off] = v;
    if (save) save[off] = v;
  }
}

// Same half step when the matrix is the vacuum one for every system: the
// right-hand side stencil is fused with the two substitution scans of the
// precomputed factorisation (scan_solve.cuh).  No material, no boundary terms.
template <typename R, int N, int M, int G>
__global__ void __launch_bounds__(G *(N / M)) adi_const_kernel(const AdiHalf h,
                                                               const double2 *__restrict__ gtab,
                                                               const double2 *__restrict__ htab) {
  using C = typename Cx<R>::T;
  constexpr int P = N / M;
  constexpr int T = G * P;
  constexpr int ld = N + N / 8 + 2;  // padded row (pad8)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *tile = reinterpret_cast<C *>(smem_raw);
  double2 *gs = reinterpret_cast<double2 *>(smem_raw + ((sizeof(C) * (G + 2) * ld + 15) & ~size_t(15)));
  double2 *hs = gs + (N + N / 8);
  Affine *scratch = reinterpret_cast<Affine *>(hs + (N + N / 8));
  const int tid = threadIdx.x;
  const int s_base = blockIdx.x * G;
  const C *in = reinterpret_cast<const C *>(h.in);
  C *out = reinterpret_cast<C *>(h.out);
  const bool interleaved = h.stride_sys == 1;
  constexpr int rows = G + 2;
  for (int idx = tid; idx < rows * N; idx += T) {
    int g, p;
    if (interleaved) {
      p = idx / rows;
      g = idx - p * rows;
    } else {
      g = idx / N;
      p = idx - g * N;
    }
    const int s = s_base - 1 + g;
    C v = from_d<R>(mk(0.0, 0.0));
    if (s >= 0 && s < N) v = in[(long long)p * h.stride_pos + (long long)s * h.stride_sys];
    tile[g * ld + pad8(p)] = v;
  }
  for (int i = tid; i < N; i += T) {
    gs[pad8(i)] = gtab[i];
    hs[pad8(i)] = htab[i];
  }
  __syncthreads();
  const int g = tid / P, c = tid - g * P;
  const int s = s_base + g;
  const int p0 = c * M;
  const double inv_kd2_expl = __ddiv_rn(1.0, h.kd2_expl);
  const double hk = 0.5 * inv_kd2_expl;
  const C *ctr = tile + (g + 1) * ld;
  const C *lft = tile + g * ld;
  const C *rgt = tile + (g + 2) * ld;
  double2 r[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const int p = p0 + m;
    double2 rr = cmul(mk(h.inv_dzh, -inv_kd2_expl), to_d(ctr[pad8(p)]));
    double2 nb = mk(0.0, 0.0);
    if (s > 0) nb = to_d(lft[pad8(p)]);
    if (s < N - 1) nb = cadd(nb, to_d(rgt[pad8(p)]));
    r[m] = mk(fma(-hk, nb.y, rr.x), fma(hk, nb.x, rr.y));
  }
  const_solve<M, P>(r, gs, hs, p0, scratch);
  __syncthreads();  // every read of the staged tile is done
  C *dst = tile + (g + 1) * ld;
#pragma unroll
  for (int m = 0; m < M; ++m) dst[pad8(p0 + m)] = from_d<R>(r[m]);
  __syncthreads();
  C *save = reinterpret_cast<C *>(h.save);
  for (int idx = tid; idx < G * N; idx += T) {
    int gg, p;
    if (interleaved) {
      p = idx / G;
      gg = idx - p * G;
    } else {
      gg = idx / N;
      p = idx - gg * N;
    }
    const long long off = (long long)p * h.stride_pos + (long long)(s_base + gg) * h.stride_sys;
    const C v = tile[(gg + 1) * ld + pad8(p)];
    out[off] = v;
    if (save) save[off] = v;
  }
}

template <typename R, int N, int G>
static cudaError_t adi_const_launch(const AdiHalf &h, const void *g, const void *hh, cudaStream_t s) {
  using C = typename Cx<R>::T;
  constexpr int M = 8, P = N / M, T = G * P;
  constexpr size_t smem = ((sizeof(C) * (G + 2) * (N + N / 8 + 2) + 15) & ~size_t(15)) +
                          2 * sizeof(double2) * (N + N / 8) + sizeof(Affine) * (T / 32 + 1);
  auto k = adi_const_kernel<R, N, M, G>;
  {
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  k<<<N / G, T, smem, s>>>(h, (const double2 *)g, (const double2 *)hh);
  return cudaGetLastError();
}

// Vacuum half step, FP64, n <= 1024, one wave: G systems per CTA so that
// ceil(n / G) CTAs cover the 148 SMs once (G = 7 at n = 1024: 147 CTAs).
// Systems are solved with N rows, N the smallest of 64, 128, 256, 512, 768
// and 1024 that holds the grid's n (h.n): rows n .. N-1 are decoupled (their
// factors g = 1, h = 0, right-hand sides zero, nothing copied in or out),
// so grids of any size up to 1024 take this path.
// The G + 2 staged rows (G systems and their two stencil halos) arrive by
// coalesced 16-byte cp.async copies, the factor tables (one 64 KB block at
// n = 1024) by one TMA bulk copy counted on an mbarrier; results leave by
// coalesced stores.  (Bulk copies per position run or per chunk -- 32 to 256
// bytes each -- measured slower than per-thread copies: the copy engine's
// per-request cost dominates at these sizes.)
//
// Compute: the CTA's systems form two groups (GS0 = ceil(G/2) and G - GS0
// systems); a thread owns one chunk of M rows of every system of its group.
// Each staged value is read from shared memory once and serves the three
// stencils it enters, each factor-table entry serves all systems of the
// group, and the sweeps run the group's independent recurrences side by
// side.  The chunk-carry scans handle the group's systems together: the
// multiplier product is the same for all of them (one matrix), the carry
// differs per system (multi_exclusive_scan).
//
// Shared-memory layouts keep the per-chunk reads of the solve and the
// copies in memory order free of bank conflicts:
//   XH (x half step, the G + 2 systems of a position adjacent in memory):
//      entry (c, m, g) at c*(M*(G+2) + 1) + m*(G+2) + g, one spare entry after
//      each chunk;
//   YH (y half step, a system is a row): entry (c, m, g) at
//      g*P*(M+1) + c*(M+1) + m, one spare entry after each chunk.
// The tables [g | h | pf | pb] (Thomas factors and the in-chunk products of
// the multipliers) are host-built in chunk-transposed slots
// (adi_const_staged_tables) and copied in as one block.  The same tile holds
// the results (row g + 1 of system g) for the stores.
template <int N, int M, int G, bool XH>
struct AdiWaveTile {
  static constexpr int P = N / M, RW = G + 2;
  static constexpr int SIZE = XH ? N * RW + P : RW * P * (M + 1);
  __device__ static __forceinline__ int at(int c, int m, int g) {
    return XH ? c * (M * RW + 1) + m * RW + g : g * P * (M + 1) + c * (M + 1) + m;
  }
};

__device__ __forceinline__ void adi_cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}


__device__ __forceinline__ void group_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

template <bool DOWN>
__device__ __forceinline__ double2 shfl2(double2 v, int d) {
  if (DOWN) return mk(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d));
  return mk(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}

// Exclusive scan of chunk transfers y_out = a*y_in + b[j] over the P threads
// of a group (P a multiple of 32, the group starting at a warp boundary),
// S systems at once with a common multiplier a.  REV scans in decreasing
// chunk order.  On return (a, b) hold the composition of the transfers of
// the chunks before this one in scan order (identity for the first).
// scratch: (S + 1) * P / 32 entries for this group; bar: its named barrier.
template <int P, int S, bool REV>
__device__ __forceinline__ void multi_exclusive_scan(double2 &a, double2 (&b)[S], double2 *scratch,
                                                     int gtid, int bar) {
  const int lane = threadIdx.x & 31;
  double2 ia = a, ib[S];
#pragma unroll
  for (int j = 0; j < S; ++j) ib[j] = b[j];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const double2 oa = shfl2<REV>(ia, d);
    double2 ob[S];
#pragma unroll
    for (int j = 0; j < S; ++j) ob[j] = shfl2<REV>(ib[j], d);
    if (REV ? lane + d < 32 : lane >= d) {
#pragma unroll
      for (int j = 0; j < S; ++j) ib[j] = cfma(ia, ob[j], ib[j]);
      ia = cmul(ia, oa);
    }
  }
  double2 ea = shfl2<REV>(ia, 1), eb[S];
#pragma unroll
  for (int j = 0; j < S; ++j) eb[j] = shfl2<REV>(ib[j], 1);
  if (REV ? lane == 31 : lane == 0) {
    ea = mk(1.0, 0.0);
#pragma unroll
    for (int j = 0; j < S; ++j) eb[j] = mk(0.0, 0.0);
  }
  if constexpr (P > 32) {
    constexpr int W = P / 32;
    const int w = gtid >> 5;
    group_sync(bar, P);  // the previous scan's readers are done with scratch
    if (lane == (REV ? 0 : 31)) {
      scratch[w * (S + 1)] = ia;
#pragma unroll
      for (int j = 0; j < S; ++j) scratch[w * (S + 1) + 1 + j] = ib[j];
    }
    group_sync(bar, P);
    double2 pa = mk(1.0, 0.0), pb[S];
#pragma unroll
    for (int j = 0; j < S; ++j) pb[j] = mk(0.0, 0.0);
#pragma unroll
    for (int k = 1; k < W; ++k) {
      const int v = REV ? W - k : k - 1;  // warps before this one in scan order
      if (REV ? v > w : v < w) {
        const double2 ta = scratch[v * (S + 1)];
#pragma unroll
        for (int j = 0; j < S; ++j) pb[j] = cfma(ta, pb[j], scratch[v * (S + 1) + 1 + j]);
        pa = cmul(ta, pa);
      }
    }
    // compose(pre, ex): apply the preceding warps, then this warp's lanes
#pragma unroll
    for (int j = 0; j < S; ++j) eb[j] = cfma(ea, pb[j], eb[j]);
    ea = cmul(ea, pa);
  }
  a = ea;
#pragma unroll
  for (int j = 0; j < S; ++j) b[j] = eb[j];
}

// Right-hand sides and solve of systems sys0 .. sys0+SC-1 of this CTA for
// chunk c: r[j][m] holds the solution of row c*M + m of system sys0 + j.
template <int N, int M, int G, bool XH, int SCAP, int S>
__device__ __forceinline__ void adi_group_solve(double2 (&r)[SCAP][M], const AdiHalf &h,
                                                const double2 *tile, const double2 *gs,
                                                const double2 *hs, const double2 *pf,
                                                const double2 *pb, double2 *scratch, int sys0,
                                                int s_base, int c, int gtid, int bar) {
  using L = AdiWaveTile<N, M, G, XH>;
  constexpr int P = N / M;
  const double inv_kd2_expl = __ddiv_rn(1.0, h.kd2_expl);
  const double hk = 0.5 * inv_kd2_expl;
  const double2 coef = mk(h.inv_dzh, -inv_kd2_expl);
  // table chunk: inside the run of identical chunks every thread reads the
  // run's first chunk, so a warp's table reads there are broadcasts
  const int ct = (c > h.tab_c0 && c < h.tab_c1) ? h.tab_c0 : c;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double2 v[S + 2];
#pragma unroll
    for (int k = 0; k < S + 2; ++k) v[k] = tile[L::at(c, m, sys0 + k)];
#pragma unroll
    for (int j = 0; j < S; ++j) {
      const int s = s_base + sys0 + j;  // s >= h.n: padding system, all zero
      const double2 rr = cmul(coef, v[j + 1]);
      double2 nb = mk(0.0, 0.0);
      if (s > 0) nb = v[j];
      if (s < h.n - 1) nb = cadd(nb, v[j + 2]);
      r[j][m] = mk(fma(-hk, nb.y, rr.x), fma(hk, nb.x, rr.y));
    }
  }
  // forward, zero carry-in: y_i = g_i r_i + h_i y_{i-1}
  double2 y[S];
  {
    const double2 g0 = gs[cslot<M, P>(ct, 0)];
#pragma unroll
    for (int j = 0; j < S; ++j) r[j][0] = y[j] = cmul(g0, r[j][0]);
  }
#pragma unroll
  for (int m = 1; m < M; ++m) {
    const int k = cslot<M, P>(ct, m);
    const double2 gm = gs[k], hm = hs[k];
#pragma unroll
    for (int j = 0; j < S; ++j) r[j][m] = y[j] = cfma(hm, y[j], cmul(gm, r[j][m]));
  }
  double2 a = pf[cslot<M, P>(ct, M - 1)];
  multi_exclusive_scan<P, S, false>(a, y, scratch, gtid, bar);
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const double2 f = pf[cslot<M, P>(ct, m)];
#pragma unroll
    for (int j = 0; j < S; ++j) r[j][m] = cfma(f, y[j], r[j][m]);
  }
  // backward, zero carry-in: x_i = y_i + h_i x_{i+1}
  double2 x[S];
#pragma unroll
  for (int j = 0; j < S; ++j) x[j] = r[j][M - 1];
#pragma unroll
  for (int m = M - 2; m >= 0; --m) {
    const double2 hm = hs[cslot<M, P>(ct, m)];
#pragma unroll
    for (int j = 0; j < S; ++j) r[j][m] = x[j] = cfma(hm, x[j], r[j][m]);
  }
  a = pb[cslot<M, P>(ct, 0)];
  multi_exclusive_scan<P, S, true>(a, x, scratch, gtid, bar);
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const double2 f = pb[cslot<M, P>(ct, m)];
#pragma unroll
    for (int j = 0; j < S; ++j) r[j][m] = cfma(f, x[j], r[j][m]);
  }
}

// Systems per group S: a thread owns one chunk of M rows of the S systems of
// its group; NG = ceil(G / S) groups of P = n/M threads each (the last group
// may hold fewer systems).
template <int N, int M, int G, int S, bool XH>
__global__ void __launch_bounds__(((G + S - 1) / S) * (N / M), 1)
    adi_const_wave_kernel(const AdiHalf h, const double2 *__restrict__ tabs) {
  using L = AdiWaveTile<N, M, G, XH>;
  constexpr int P = N / M;
  constexpr int NG = (G + S - 1) / S;
  constexpr int T = NG * P;
  constexpr int RW = G + 2;
  constexpr int SL = G - (NG - 1) * S;  // systems of the last group
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  double2 *gs = reinterpret_cast<double2 *>(smem_raw + 16);
  double2 *hs = gs + N;
  double2 *pf = hs + N;
  double2 *pb = pf + N;
  double2 *scratch = pb + N;  // (S + 1) * P / 32 per group
  double2 *tile = scratch + NG * (S + 1) * (P / 32);
  __shared__ int staged_ok;
  const int tid = threadIdx.x;
  const int group = tid / P, gtid = tid % P;
  const int s_base = blockIdx.x * G;
  const double2 *in = reinterpret_cast<const double2 *>(h.in);
  double2 *out = reinterpret_cast<double2 *>(h.out);
  const int nr = h.n;  // systems, and positions per system (N: rows solved)
  // staged systems s_base - 1 + g exist for g in [g_lo, g_hi)
  const int g_lo = s_base == 0 ? 1 : 0;
  const int g_hi = nr - s_base + 1 < RW ? nr - s_base + 1 : RW;
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, (unsigned)(sizeof(double2) * 4 * N));
  }
  // staged rows outside the grid (first and last CTA) and the padding
  // positions nr .. N-1 are zero
  for (int g = 0; g < RW; ++g)
    for (int p = (g < g_lo || g >= g_hi) ? tid : nr + tid; p < N; p += T)
      tile[L::at(p / M, p % M, g)] = mk(0.0, 0.0);
  __syncthreads();
  if (tid == 0) bulk_load(gs, tabs, (unsigned)(sizeof(double2) * 4 * N), bar);
  // Programmatic dependent launch: everything above (barrier set-up, zero
  // rows, the table copy) does not depend on the previous kernel in the
  // stream, so it may overlap that kernel's tail; the field is read and
  // written only after the previous grid has completed and its writes are
  // visible.  The next kernel may likewise start its own set-up early.
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  if constexpr (XH) {
    // the RW staged systems of a position are adjacent in memory:
    // consecutive threads take consecutive systems
    constexpr int PPI = T / RW;  // positions per pass
    const int g = tid % RW;
    if (tid < PPI * RW && g >= g_lo && g < g_hi) {
      const double2 *src = in + (s_base - 1 + g);
      for (int p = tid / RW; p < nr; p += PPI)
        adi_cp_async16(tile + L::at(p / M, p % M, g), src + (long long)p * h.stride_pos);
    }
  } else {
#pragma unroll 1
    for (int g = g_lo; g < g_hi; ++g) {
      const double2 *src = in + (long long)(s_base - 1 + g) * h.stride_sys;
      for (int p = tid; p < nr; p += T) adi_cp_async16(tile + L::at(p / M, p % M, g), src + p);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  if (tid == 0) {
    const bool ok = mbar_wait_bounded(bar, 0, 2000000000ull);
    if (!ok) {
      atomicAdd(&g_wait_timeouts, 1u);
      mbar_wait_bounded(bar, 0, 2000000000ull);  // the table copy may still be in flight
    }
    staged_ok = ok;
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  if (!staged_ok) return;
  (void)mbar_try_wait(bar, 0);  // completed phase: orders the copied tables for this thread
  double2 r[S][M];
  double2 *gscr = scratch + group * (S + 1) * (P / 32);
  if (SL == S || group < NG - 1)
    adi_group_solve<N, M, G, XH, S, S>(r, h, tile, gs, hs, pf, pb, gscr, group * S, s_base, gtid,
                                       gtid, 1 + group);
  else
    adi_group_solve<N, M, G, XH, S, SL>(r, h, tile, gs, hs, pf, pb, gscr, group * S, s_base, gtid,
                                        gtid, 1 + group);
  __syncthreads();  // every read of the staged tile is done
  const int ns = group < NG - 1 ? S : SL;
#pragma unroll
  for (int j = 0; j < S; ++j)
    if (j < ns) {
#pragma unroll
      for (int m = 0; m < M; ++m) tile[L::at(gtid, m, group * S + j + 1)] = r[j][m];
    }
  __syncthreads();
  double2 *save = reinterpret_cast<double2 *>(h.save);
  const int nsys = nr - s_base < G ? nr - s_base : G;  // the last CTA may hold fewer
  if constexpr (XH) {
    // consecutive threads write consecutive systems of a position
    constexpr int PPI = T / G;
    const int gg = tid % G;
    if (tid < PPI * G && gg < nsys) {
      for (int p = tid / G; p < nr; p += PPI) {
        const double2 v = tile[L::at(p / M, p % M, gg + 1)];
        const long long off = (long long)p * h.stride_pos + s_base + gg;
        out[off] = v;
        if (save) save[off] = v;
      }
    }
  } else {
#pragma unroll 1
    for (int gg = 0; gg < nsys; ++gg) {
      const long long base = (long long)(s_base + gg) * h.stride_sys;
      for (int p = tid; p < nr; p += T) {
        const double2 v = tile[L::at(p / M, p % M, gg + 1)];
        out[base + p] = v;
        if (save) save[base + p] = v;
      }
    }
  }
}

// cp.async completion counted on an mbarrier: when every cp.async this
// thread issued before the instruction has landed, the barrier sees one
// arrival (noinc: the arrival is one of the count the barrier was set up
// with).
__device__ __forceinline__ void cp_async_mbar_arrive(uint64_t *bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

// Bytes before the factor tables in the one-wave kernels' shared memory: the
// mbarriers (one for the tables and, in the pipelined kernel, one per
// system group), rounded up to 16 bytes.
template <int NG> constexpr size_t adi_wave_bar_bytes() { return 16 * ((NG + 2) / 2 + 1); }

// The one-wave vacuum half step with its staging pipelined against the
// solves.  The staged rows are copied in stages, one per system group in
// group order (stage 0: the rows group 0 reads; stage k: the rows group k
// needs that no earlier stage brought); every thread issues its share of a
// stage's copies and then an asynchronous arrival on that stage's mbarrier,
// so a stage completes when all of its copies (and every earlier stage's)
// have landed.  Each group waits for its own stage and the factor tables
// (its leader with the bounded wait, then the group's named barrier),
// solves, and stores its systems straight from registers: group 0 computes
// while later rows are still arriving, and one group's stores overlap the
// others' solves.  Same arithmetic as adi_const_wave_kernel.
template <int N, int M, int G, int S, bool XH>
__global__ void __launch_bounds__(((G + S - 1) / S) * (N / M), 1)
    adi_pipe_wave_kernel(const AdiHalf h, const double2 *__restrict__ tabs) {
  using L = AdiWaveTile<N, M, G, XH>;
  constexpr int P = N / M;
  constexpr int NG = (G + S - 1) / S;
  constexpr int T = NG * P;
  constexpr int RW = G + 2;
  constexpr int SL = G - (NG - 1) * S;  // systems of the last group
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);  // [0]: tables, [1 + k]: stage k
  double2 *gs = reinterpret_cast<double2 *>(smem_raw + adi_wave_bar_bytes<NG>());
  double2 *hs = gs + N;
  double2 *pf = hs + N;
  double2 *pb = pf + N;
  double2 *scratch = pb + N;  // (S + 1) * P / 32 per group
  double2 *tile = scratch + NG * (S + 1) * (P / 32);
  __shared__ int group_ok[NG];
  const int tid = threadIdx.x;
  const int group = tid / P, gtid = tid % P;
  const int s_base = blockIdx.x * G;
  const double2 *in = reinterpret_cast<const double2 *>(h.in);
  double2 *out = reinterpret_cast<double2 *>(h.out);
  double2 *save = reinterpret_cast<double2 *>(h.save);
  const int nr = h.n;  // systems, and positions per system (N: rows solved)
  const int g_lo = s_base == 0 ? 1 : 0;
  const int g_hi = nr - s_base + 1 < RW ? nr - s_base + 1 : RW;
  if (tid == 0) {
    mbar_init(bar, 1);
    for (int k = 0; k < NG; ++k) mbar_init(bar + 1 + k, T);
    mbar_arrive_expect_tx(bar, (unsigned)(sizeof(double2) * 4 * N));
  }
  // rows outside the grid and the padding positions nr .. N-1 are zero
  for (int g = 0; g < RW; ++g)
    for (int p = (g < g_lo || g >= g_hi) ? tid : nr + tid; p < N; p += T)
      tile[L::at(p / M, p % M, g)] = mk(0.0, 0.0);
  __syncthreads();
  if (tid == 0) bulk_load(gs, tabs, (unsigned)(sizeof(double2) * 4 * N), bar);
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  // stage k brings staged rows [lo_k, hi_k); group k reads rows k*S .. k*S + S + 1
#pragma unroll 1
  for (int k = 0; k < NG; ++k) {
    const int lo = k == 0 ? 0 : k * S + 2;
    const int hi = k == NG - 1 ? RW : (k + 1) * S + 2;
    const int rows = hi - lo;
    if constexpr (XH) {
      // the rows of a position are adjacent in memory: consecutive threads
      // take consecutive rows, then the next position
      for (int i = tid; i < nr * rows; i += T) {
        const int p = i / rows, g = lo + i % rows;
        if (g >= g_lo && g < g_hi)
          adi_cp_async16(tile + L::at(p / M, p % M, g),
                         in + (long long)p * h.stride_pos + (s_base - 1 + g));
      }
    } else {
      for (int g = lo; g < hi; ++g) {
        if (g < g_lo || g >= g_hi) continue;
        const double2 *src = in + (long long)(s_base - 1 + g) * h.stride_sys;
        for (int p = tid; p < nr; p += T) adi_cp_async16(tile + L::at(p / M, p % M, g), src + p);
      }
    }
    cp_async_mbar_arrive(bar + 1 + k);
  }
  // this group's rows and the tables
  if (gtid == 0) {
    bool ok = mbar_wait_bounded(bar + 1 + group, 0, 2000000000ull);
    ok = mbar_wait_bounded(bar, 0, 2000000000ull) && ok;
    if (!ok) atomicAdd(&g_wait_timeouts, 1u);
    group_ok[group] = ok;
  }
  group_sync(1 + group, P);
  // a group whose wait ran out skips its solve but still reaches the CTA
  // barriers below (every thread of the CTA passes every barrier); the CTA
  // then leaves without storing
  const bool my_ok = group_ok[group] != 0;
  double2 r[S][M];
  if (my_ok) {
    (void)mbar_try_wait(bar + 1 + group, 0);  // completed phases: order the rows and tables
    (void)mbar_try_wait(bar, 0);
    double2 *gscr = scratch + group * (S + 1) * (P / 32);
    if (SL == S || group < NG - 1)
      adi_group_solve<N, M, G, XH, S, S>(r, h, tile, gs, hs, pf, pb, gscr, group * S, s_base,
                                         gtid, gtid, 1 + group);
    else
      adi_group_solve<N, M, G, XH, S, SL>(r, h, tile, gs, hs, pf, pb, gscr, group * S, s_base,
                                          gtid, gtid, 1 + group);
  }
  // results through the tile to coalesced stores, as in the unpipelined
  // kernel: after every group's reads of the staged rows (one CTA barrier:
  // group 0 waits here for the last group's right-hand sides, while its own
  // solve has already overlapped the later stages' copies), each group
  // writes its systems' rows, and consecutive threads then store
  // consecutive addresses.  (Stores straight from the registers -- each
  // thread's rows strided by the system length -- measured slower than the
  // unpipelined kernel.)
  __syncthreads();  // every group's flag is set and every staged row read
  bool all_ok = true;
#pragma unroll
  for (int k = 0; k < NG; ++k) all_ok = all_ok && group_ok[k] != 0;
  if (!all_ok) {  // the same decision in every thread: nothing writes the flags now
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    return;
  }
  const int ns = group < NG - 1 ? S : SL;
#pragma unroll
  for (int j = 0; j < S; ++j)
    if (j < ns) {
#pragma unroll
      for (int m = 0; m < M; ++m) tile[L::at(gtid, m, group * S + j + 1)] = r[j][m];
    }
  __syncthreads();
  const int nsys = nr - s_base < G ? nr - s_base : G;  // the last CTA may hold fewer
  if constexpr (XH) {
    constexpr int PPI = T / G;
    const int gg = tid % G;
    if (tid < PPI * G && gg < nsys) {
      for (int p = tid / G; p < nr; p += PPI) {
        const double2 v = tile[L::at(p / M, p % M, gg + 1)];
        const long long off = (long long)p * h.stride_pos + s_base + gg;
        out[off] = v;
        if (save) save[off] = v;
      }
    }
  } else {
#pragma unroll 1
    for (int gg = 0; gg < nsys; ++gg) {
      const long long base = (long long)(s_base + gg) * h.stride_sys;
      for (int p = tid; p < nr; p += T) {
        const double2 v = tile[L::at(p / M, p % M, gg + 1)];
        out[base + p] = v;
        if (save) save[base + p] = v;
      }
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");  // copies this thread issued for later groups
}

// The unpipelined one-wave kernel by default; PXP_ADI_PIPE=1 selects the
// pipelined one (measured slower with its stores straight from registers:
// 30.4 against 23.2 us per 1024^2 step).
static bool adi_pipe_enabled() {
  static const bool on = [] {
    const char *e = std::getenv("PXP_ADI_PIPE");
    return e && e[0] == '1';
  }();
  return on;
}

template <int N, int M, int G, int S, bool XH>
static cudaError_t adi_const_wave_launch_x(const AdiHalf &h, const void *tabs, cudaStream_t s) {
  constexpr int P = N / M, NG = (G + S - 1) / S, T = NG * P;
  constexpr size_t smem = adi_wave_bar_bytes<NG>() +
                          sizeof(double2) * (4 * N + NG * (S + 1) * (P / 32)) +
                          sizeof(double2) * AdiWaveTile<N, M, G, XH>::SIZE;
  static_assert(smem + 16 <= 227 * 1024, "staged ADI tile exceeds shared memory");
  static_assert(P % 32 == 0, "whole warps per group");
  static_assert(NG <= 15, "one named barrier per group");
  auto k = adi_pipe_enabled() ? adi_pipe_wave_kernel<N, M, G, S, XH>
                              : adi_const_wave_kernel<N, M, G, S, XH>;
  {
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  // launched as a programmatic dependent of the previous kernel in the
  // stream (the kernel waits for it with griddepcontrol.wait)
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((h.n + G - 1) / G);
  cfg.blockDim = dim3(T);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, h, (const double2 *)tabs);
}

template <int N, int M, int G, int S>
static cudaError_t adi_const_wave_launch(const AdiHalf &h, const void *tabs, cudaStream_t s) {
  if (tabs == nullptr) return cudaErrorInvalidValue;
  return h.stride_sys == 1 ? adi_const_wave_launch_x<N, M, G, S, true>(h, tabs, s)
                           : adi_const_wave_launch_x<N, M, G, S, false>(h, tabs, s);
}

// (M, G) of the one-wave kernel per size: each system group holds whole
// warps (n/M a multiple of 32) and ceil(n / G) CTAs fill the SMs about once.
static bool adi_wave_config(int n, int *m, int *g) {
  switch (n) {
    case 64: *m = 2; *g = 4; return true;
    case 128: *m = 4; *g = 2; return true;
    case 256: *m = 8; *g = 2; return true;
    case 512: *m = 8; *g = 4; return true;
    case 768: *m = 8; *g = 6; return true;
    case 1024: *m = 8; *g = 7; return true;
    default: return false;
  }
}

int adi_wave_n(int n) {
  static const int sizes[] = {64, 128, 256, 512, 768, 1024};
  if (n < 4) return 0;
  for (int w : sizes)
    if (n <= w) return w;
  return 0;
}

bool adi_const_staged_tables(int n, const double *g, const double *h, double *out, int run[2]) {
  int M = 0, G = 0;
  if (!adi_wave_config(n, &M, &G)) return false;
  const int P = n / M;
  auto slot = [&](int c, int m) { return m * P + (c ^ (m & 7)); };
  // the device's cmul: (fma(ax, bx, -ay*by), fma(ax, by, ay*bx))
  auto cmul_h = [](const double *a, const double *b, double *o) {
    const double re = std::fma(a[0], b[0], -(a[1] * b[1]));
    const double im = std::fma(a[0], b[1], a[1] * b[0]);
    o[0] = re;
    o[1] = im;
  };
  double *gs = out, *hs = out + 2 * n, *pf = out + 4 * n, *pb = out + 6 * n;
  for (int c = 0; c < P; ++c) {
    double prod[2] = {1.0, 0.0};
    for (int m = 0; m < M; ++m) {
      const int p = c * M + m, k = slot(c, m);
      gs[2 * k] = g[2 * p];
      gs[2 * k + 1] = g[2 * p + 1];
      hs[2 * k] = h[2 * p];
      hs[2 * k + 1] = h[2 * p + 1];
      cmul_h(h + 2 * p, prod, prod);
      pf[2 * k] = prod[0];
      pf[2 * k + 1] = prod[1];
    }
    prod[0] = 1.0;
    prod[1] = 0.0;
    for (int m = M - 1; m >= 0; --m) {
      const int p = c * M + m, k = slot(c, m);
      cmul_h(h + 2 * p, prod, prod);
      pb[2 * k] = prod[0];
      pb[2 * k + 1] = prod[1];
    }
  }
  // Thomas factors of a constant-coefficient matrix reach their limit to the
  // last bit after a few dozen rows, so most chunks' entries coincide
  auto same_chunk = [&](int c0, int c1) {
    for (int t = 0; t < 4; ++t)
      for (int m = 0; m < M; ++m) {
        const double *e0 = out + 2 * ((size_t)t * n + slot(c0, m));
        const double *e1 = out + 2 * ((size_t)t * n + slot(c1, m));
        if (std::memcmp(e0, e1, 2 * sizeof(double)) != 0) return false;
      }
    return true;
  };
  run[0] = run[1] = 0;
  for (int c = 0; c < P;) {
    int e = c + 1;
    while (e < P && same_chunk(c, e)) ++e;
    if (e - c > run[1] - run[0]) {
      run[0] = c;
      run[1] = e;
    }
    c = e;
  }
  if (run[1] - run[0] < 2) run[0] = run[1] = 0;
  return true;
}

// Self-test of the bounded-wait failure path: one thread arms an mbarrier
// for a 16-byte transaction that no copy ever delivers and waits on it with
// the kernels' bounded wait (mbar_wait_bounded) and the given limit.  The
// wait runs out, the kernel records it in the same counter the propagation
// kernels use, and returns; nothing faults and the context stays usable.
__global__ void wait_selftest_kernel(unsigned long long limit_ns) {
  __shared__ __align__(8) uint64_t bar;
  mbar_init(&bar, 1);
  mbar_arrive_expect_tx(&bar, 16u);
  if (!mbar_wait_bounded(&bar, 0, limit_ns)) atomicAdd(&g_wait_timeouts, 1u);
}

cudaError_t launch_wait_selftest(unsigned long long limit_ns, cudaStream_t s) {
  wait_selftest_kernel<<<1, 1, 0, s>>>(limit_ns);
  return cudaGetLastError();
}

unsigned wait_timeouts(cudaStream_t s) {
  unsigned v = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_wait_timeouts, sizeof(v), 0, cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return 0;
  return v + fft3d_lines_wait_timeouts(s) + fft3d_r16_wait_timeouts(s);
}

cudaError_t launch_adi_half_const(Precision p, const AdiHalf &h, const void *g, const void *hh,
                                  const void *staged, cudaStream_t s) {
#define PXP_AC(NN, GG)                                                                  \
  case NN:                                                                              \
    return p == kFP64 ? adi_const_launch<double, NN, GG>(h, g, hh, s)                   \
                      : adi_const_launch<float, NN, GG>(h, g, hh, s);
  if (p == kFP64) {
    switch (adi_wave_n(h.n)) {
      case 64: return adi_const_wave_launch<64, 2, 4, 2>(h, staged, s);
      case 128: return adi_const_wave_launch<128, 4, 2, 1>(h, staged, s);
      case 256: return adi_const_wave_launch<256, 8, 2, 1>(h, staged, s);
      case 512: return adi_const_wave_launch<512, 8, 4, 2>(h, staged, s);
      case 768: return adi_const_wave_launch<768, 8, 6, 2>(h, staged, s);
      case 1024: return adi_const_wave_launch<1024, 8, 7, 2>(h, staged, s);
      default: break;
    }
  }
  switch (h.n) {
    PXP_AC(64, 4) PXP_AC(128, 4) PXP_AC(256, 4) PXP_AC(512, 4) PXP_AC(1024, 4) PXP_AC(2048, 2)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_AC
}

static constexpr int kAdiM = 8;

template <int G> constexpr int adi_threads(int n) { return G * (n / kAdiM); }

template <typename R, int G>
static cudaError_t adi_launch_g(const AdiHalf &h, cudaStream_t s) {
  using C = typename Cx<R>::T;
  const int n = h.n_pad > 0 ? h.n_pad : h.n;  // solved system length
  const int T = adi_threads<G>(n);
  const size_t tile = (sizeof(C) * (G + 2) * (n + n / 8 + 2) + 15) & ~size_t(15);
  const size_t smem = tile + sizeof(double2) * 4 * G * 2 * (n / kAdiM);
  auto k = adi_half_kernel<R, kAdiM, G>;
  // raise the dynamic shared-memory limit on this device to the largest size
  // the instantiation can need (n = 2048 for G = 2, n = 1024 for G = 4)
  const cudaError_t attr = raise_dynamic_smem(
      (const void *)k,
      (int)(((sizeof(C) * (G + 2) * (G == 2 ? 2048 + 258 : 1024 + 130) + 15) & ~size_t(15)) +
            sizeof(double2) * 4 * G * 2 * ((G == 2 ? 2048 : 1024) / kAdiM)));
  if (attr != cudaSuccess) return attr;
  k<<<(h.n + G - 1) / G, T, smem, s>>>(h);  // one CTA per G of the grid's h.n systems
  return cudaGetLastError();
}

bool adi_supported(Precision p, int n) {
  if (n < 64 || (n & (n - 1))) return false;
  return p == kFP64 ? n <= 2048 : n <= 2048;
}

int adi_padded_n(int n) {
  if (n >= 64 && !(n & (n - 1))) return n;
  int t = 8;
  while (t * kAdiM < n) t *= 2;
  return t * kAdiM;
}

bool adi_padded_supported(Precision p, int n) {
  return n >= 4 && adi_supported(p, adi_padded_n(n));
}

cudaError_t launch_adi_half(Precision p, const AdiHalf &h, cudaStream_t s) {
  const int np = h.n_pad > 0 ? h.n_pad : h.n;
  if (!adi_supported(p, np) || h.n > np) return cudaErrorInvalidValue;
  // G systems per CTA so that G * n/8 <= 512 threads
  if (np <= 1024) return p == kFP64 ? adi_launch_g<double, 4>(h, s) : adi_launch_g<float, 4>(h, s);
  return p == kFP64 ? adi_launch_g<double, 2>(h, s) : adi_launch_g<float, 2>(h, s);
}

}  // namespace pxp
