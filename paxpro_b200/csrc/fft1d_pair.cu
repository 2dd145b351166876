// fft1d_pair.cu -- FFTSolver2D split step for a line too long for one SM's
// shared memory (complex128, n = 16384: 256 KB), on a cluster of two CTAs.
//
// Same step as fft1d.cu (src/fftSolver2D.cpp:21-73): forward FFT,
// propagator, backward FFT, (u * t) / n.  CTA r of the pair keeps the points
// of parity r, u_r[j] = u[2j + r], in its shared memory for the whole launch
// and transforms them with the n/2-point shared-memory FFT; the two halves
// meet through distributed shared memory (each CTA reads its peer's buffer):
//
//   forward:  E = F(u_0), O = F(u_1) (n/2 points each);
//             X[k] = E[k] + w^k O[k], X[k + n/2] = E[k] - w^k O[k]
//   K:        Y[k] = K[k] X[k],      Y[k + n/2] = K[k + n/2] X[k + n/2]
//   backward: a[k] = Y[k] + Y[k + n/2]          -> u_0 = F^-1(a) (even points)
//             b[k] = (Y[k] - Y[k + n/2]) w^-k   -> u_1 = F^-1(b) (odd points)
//
// with w = exp(-2 pi i / n).  Every quantity at index k needs only E[k] and
// O[k], so each CTA computes its own a[k] or b[k] from its value and its
// peer's: two cluster barriers per step (both halves transformed; both
// reads of the peer done before either buffer is overwritten).  The
// refraction of point 2j + r uses the transmission table entry 2j + r, so
// the pointwise arithmetic is the single-CTA kernel's.  Flux sums (when
// windows are set) add each CTA's total through the peer's shared memory.
#include <cooperative_groups.h>

#include "fft_smem.cuh"
#include "flux.cuh"
#include "pxp_kernels.h"

namespace cg = cooperative_groups;

namespace pxp {

template <typename R> __device__ __forceinline__ void pair_refract(typename Cx<R>::T &u, double2 t,
                                                                   R n);
template <> __device__ __forceinline__ void pair_refract<double>(double2 &u, double2 t, double n) {
  u = cx_div_real_rn(cx_mul_rn(u, t), n);  // (u * t) / N as the reference rounds it
}
template <> __device__ __forceinline__ void pair_refract<float>(float2 &u, double2 t, float) {
  u = tw_mul(u, t);  // t / N folded on the host, product in FP64
}
template <typename R> __device__ __forceinline__ typename Cx<R>::T pair_kmul(typename Cx<R>::T u,
                                                                            double2 k);
template <> __device__ __forceinline__ double2 pair_kmul<double>(double2 u, double2 k) {
  return cx_mul_rn(u, k);
}
template <> __device__ __forceinline__ float2 pair_kmul<float>(float2 u, double2 k) {
  return tw_mul(u, k);
}

template <typename R, int NH, int T, bool FLUX>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(T)
    fft1d_pair_kernel(const Fft1dJob *__restrict__ jobs, int step0_ov, int nsteps_ov) {
  using C = typename Cx<R>::T;
  constexpr int N = 2 * NH;
  constexpr int PER = NH / T;
  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();  // 0: even points, 1: odd points
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double flux_red[2][flux_slots<T>()];
  __shared__ double flux_peer[2];
  C *u = reinterpret_cast<C *>(smem_raw);
  const C *peer = cluster.map_shared_rank(u, r ^ 1);
  double *flux_peer_remote = cluster.map_shared_rank(flux_peer, 0);
  Fft1dJob job = jobs[blockIdx.x / 2];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int lane = threadIdx.x;
  const double2 *tw = reinterpret_cast<const double2 *>(job.twiddle);  // n/2-point Stockham
  const double2 *wk = reinterpret_cast<const double2 *>(job.chirp);    // w^k, k < n/2
  const double2 *kern = reinterpret_cast<const double2 *>(job.kern);
  const double2 *trans0 = reinterpret_cast<const double2 *>(job.trans);
  C *field = reinterpret_cast<C *>(job.field);
  C *saves = reinterpret_cast<C *>(job.saves);
  for (int j = lane; j < NH; j += T) u[sw<C>(j)] = field[2 * j + r];
  cluster.sync();  // both CTAs running and loaded before any remote access
  const R nreal = (R)N;
  for (int s = 0; s < job.nsteps; ++s) {
    const int step = job.step0 + s;
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    fft_smem<C, NH, T, -1>(u, tw, lane);  // E (r = 0) or O (r = 1)
    cluster.sync();                       // the peer's half is transformed
    C v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int k = lane + i * T;
      const C mine = u[sw<C>(k)], other = peer[sw<C>(k)];
      const C e = r ? other : mine, o = r ? mine : other;
      const double2 w = wk[k];
      const C wo = tw_mul(o, w);
      const C ylo = pair_kmul<R>(cadd(e, wo), kern[k]);
      const C yhi = pair_kmul<R>(csub(e, wo), kern[k + NH]);
      v[i] = r ? tw_mulc(csub(ylo, yhi), w) : cadd(ylo, yhi);
    }
    cluster.sync();  // every read of the peer's buffer is done
#pragma unroll
    for (int i = 0; i < PER; ++i) u[sw<C>(lane + i * T)] = v[i];
    __syncthreads();
    fft_smem<C, NH, T, +1>(u, tw, lane);  // u[2j + r]
    const double2 *trans = trans0 + job.trans_stride * (long long)(step - job.trans_step0);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * N : nullptr;
    double acc = 0.0;
    for (int j = lane; j < NH; j += T) {
      const int i = 2 * j + r;
      C val = u[sw<C>(j)];
      pair_refract<R>(val, trans[i], nreal);
      u[sw<C>(j)] = val;
      if (save) slot[i] = val;
      if (flux) flux_add(acc, i, fw, to_d(val));
    }
    if (flux) flux_warp_total<T>(acc, flux_red[s & 1]);
    __syncthreads();
    if constexpr (FLUX) {
      // CTA totals: CTA 1 hands its total to CTA 0, which stores the sum
      double t = 0.0;
      if (flux && lane < 32) {
        t = lane < flux_slots<T>() ? flux_red[s & 1][lane] : 0.0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) t += __shfl_down_sync(0xffffffffu, t, d);
        if (lane == 0 && r == 1) flux_peer_remote[s & 1] = t;
      }
      cluster.sync();  // CTA 1's total is in CTA 0's flux_peer
      if (flux && r == 0 && lane == 0) job.flux.out[step - job.flux.step0] = t + flux_peer[s & 1];
    }
  }
  cluster.sync();  // no CTA leaves while its peer may still address its shared memory
  for (int j = lane; j < NH; j += T) field[2 * j + r] = u[sw<C>(j)];
}

template <typename R, int NH, bool FLUX>
static cudaError_t launch_pair_f(const Fft1dJob *d_jobs, int nj, int step0, int nsteps,
                                 cudaStream_t s) {
  using C = typename Cx<R>::T;
  constexpr int T = 512;
  constexpr size_t smem = sizeof(C) * NH;
  auto k = fft1d_pair_kernel<R, NH, T, FLUX>;
  {
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  k<<<2 * nj, T, smem, s>>>(d_jobs, step0, nsteps);
  return cudaGetLastError();
}

cudaError_t launch_fft1d_pair(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                              int nsteps, cudaStream_t s, bool flux) {
  if (nj <= 0) return cudaSuccess;
  if (p != kFP64 || n != 16384) return cudaErrorInvalidValue;
  return flux ? launch_pair_f<double, 8192, true>(d_jobs, nj, step0, nsteps, s)
              : launch_pair_f<double, 8192, false>(d_jobs, nj, step0, nsteps, s);
}

}  // namespace pxp
