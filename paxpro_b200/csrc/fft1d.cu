// fft1d.cu -- K-FFT1: fused split-step kernel for one transverse dimension.
//
// Replaces FFTSolver2D::solveStep (src/fftSolver2D.cpp:61-73): forward FFT,
// propagator multiply (:21-34), backward FFT, transmission multiply and 1/N
// normalisation (:36-50).  One CTA owns one problem and keeps its field in
// shared memory for all steps of the launch, so HBM sees the field once per
// launch plus the save slots; the only per-step global reads are the
// propagator and transmission tables, which stay in L2.
//
// FP64 mode reproduces the reference's pointwise arithmetic exactly:
// curr *= kernel is a rounded complex product and the refraction update is
// (prev * t) / N with t taken from a host table built with std::exp, as the
// reference evaluates it.  FP32 mode computes in FP32 with split
// complex64 tables (fft_smem.cuh): twiddles, the propagator and t/N.
#include "bluestein.cuh"
#include "fft_smem.cuh"
#include "flux.cuh"
#include "persistent.cuh"
#include "pxp_kernels.h"

namespace pxp {

// Per-step factor tables: complex128 in FP64 mode, which reproduces the
// reference's rounding (rounded complex product, then division by N);
// split complex64 pairs of t/N in FP32 served mode (one FMA chain).
__device__ __forceinline__ void refract(double2 &u, double2 t, double n) {
  u = cx_div_real_rn(cx_mul_rn(u, t), n);
}
__device__ __forceinline__ void refract(float2 &u, float4 t, float) { u = tw_mul(u, t); }
__device__ __forceinline__ double2 kmul(double2 u, double2 k) { return cx_mul_rn(u, k); }
__device__ __forceinline__ float2 kmul(float2 u, float4 k) { return tw_mul(u, k); }

template <typename R, int N, int T, bool TW_SMEM, bool FLUX>
__global__ void __launch_bounds__(T) fft1d_kernel(const Fft1dJob *__restrict__ jobs, int step0_ov,
                                                 int nsteps_ov, int njobs, unsigned *queue) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double flux_red[2][flux_slots<T>()];
  __shared__ int s_next;
  C *u = reinterpret_cast<C *>(smem_raw);
  for (int jb = blockIdx.x; jb < njobs; jb = next_job(queue, &s_next)) {
  Fft1dJob job = jobs[jb];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int lane = threadIdx.x;
  using W = Tw<C>;
  const W *gtw = reinterpret_cast<const W *>(job.twiddle);
  const W *tw = gtw;
  if constexpr (TW_SMEM) {
    // twiddles after the field, 16-byte aligned
    W *stw = reinterpret_cast<W *>(smem_raw + ((sizeof(C) * N + 15) & ~size_t(15)));
    for (int i = lane; i < N; i += T) stw[i] = gtw[i];
    tw = stw;
  }
  C *field = reinterpret_cast<C *>(job.field);
  for (int i = lane; i < N; i += T) u[sw<C>(i)] = field[i];
  __syncthreads();
  const W *kern = reinterpret_cast<const W *>(job.kern);
  const W *trans0 = reinterpret_cast<const W *>(job.trans);
  C *saves = reinterpret_cast<C *>(job.saves);
  const R nreal = (R)N;
  for (int s = 0; s < job.nsteps; ++s) {
    const int step = job.step0 + s;
    // this step's flux window, loaded early so its latency hides behind the step
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    fft_smem<C, N, T, -1>(u, tw, lane);
    for (int i = lane; i < N; i += T) u[sw<C>(i)] = kmul(u[sw<C>(i)], kern[i]);
    __syncthreads();
    fft_smem<C, N, T, +1>(u, tw, lane);
    const W *trans = trans0 + job.trans_stride * (long long)(step - job.trans_step0);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * N : nullptr;
    double acc = 0.0;
    for (int i = lane; i < N; i += T) {
      C v = u[sw<C>(i)];
      refract(v, trans[i], nreal);
      u[sw<C>(i)] = v;
      if (save) slot[i] = v;
      if (flux) flux_add(acc, i, fw, to_d(v));
    }
    if (flux) flux_warp_total<T>(acc, flux_red[s & 1]);
    __syncthreads();
    if (flux) flux_store<T>(job.flux, step, flux_red[s & 1]);
  }
  for (int i = lane; i < N; i += T) field[i] = u[sw<C>(i)];
  }
}

template <typename R, int M, int T, bool FLUX>
__global__ void __launch_bounds__(T) fft1d_bluestein_kernel(const Fft1dJob *__restrict__ jobs,
                                                           int step0_ov, int nsteps_ov) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double flux_red[2][flux_slots<T>()];
  C *x = reinterpret_cast<C *>(smem_raw);  // m-point work buffer (swizzled)
  C *u = x + M;                            // the field, n points
  Fft1dJob job = jobs[blockIdx.x];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int n = job.n;
  const int lane = threadIdx.x;
  using W = Tw<C>;
  const W *tw = reinterpret_cast<const W *>(job.twiddle);
  const W *w = reinterpret_cast<const W *>(job.chirp);
  const W *bf = reinterpret_cast<const W *>(job.bconv);
  C *field = reinterpret_cast<C *>(job.field);
  for (int i = lane; i < n; i += T) u[i] = field[i];
  __syncthreads();
  const W *kern = reinterpret_cast<const W *>(job.kern);
  const W *trans0 = reinterpret_cast<const W *>(job.trans);
  C *saves = reinterpret_cast<C *>(job.saves);
  const R nreal = (R)n;
  for (int s = 0; s < job.nsteps; ++s) {
    const int step = job.step0 + s;
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    bluestein_dft<R, M, T>(x, u, n, w, bf, tw, lane, false);
    for (int i = lane; i < n; i += T) u[i] = kmul(u[i], kern[i]);
    __syncthreads();
    bluestein_dft<R, M, T>(x, u, n, w, bf, tw, lane, true);
    const W *trans = trans0 + job.trans_stride * (long long)(step - job.trans_step0);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * n : nullptr;
    double acc = 0.0;
    for (int i = lane; i < n; i += T) {
      C v = u[i];
      refract(v, trans[i], nreal);
      u[i] = v;
      if (save) slot[i] = v;
      if (flux) flux_add(acc, i, fw, to_d(v));
    }
    if (flux) flux_warp_total<T>(acc, flux_red[s & 1]);
    __syncthreads();
    if (flux) flux_store<T>(job.flux, step, flux_red[s & 1]);
  }
  for (int i = lane; i < n; i += T) field[i] = u[i];
}

template <typename R> constexpr int fft1d_threads(int n) {
  return n >= 8192 ? 512 : (n >= 2048 ? 256 : (n >= 512 ? 64 : 32));
}

template <typename R, int N, bool FLUX>
static cudaError_t launch_n(const Fft1dJob *d_jobs, int nj, int step0, int nsteps,
                            cudaStream_t s, unsigned *queue) {
  using C = typename Cx<R>::T;
  constexpr int T = fft1d_threads<R>(N);
  constexpr size_t field_bytes = sizeof(C) * N;
  constexpr size_t tw_bytes = sizeof(Tw<C>) * N;
  constexpr bool tw_smem = field_bytes + tw_bytes <= 200 * 1024;
  constexpr size_t smem = tw_smem ? field_bytes + tw_bytes : field_bytes;
  auto k = fft1d_kernel<R, N, T, tw_smem, FLUX>;
  {  // the static flux slots count against the 48 KB default too
    const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  const int grid = persistent_grid((const void *)k, T, smem, nj, queue);
  k<<<grid, T, smem, s>>>(d_jobs, step0, nsteps, nj, queue);
  return cudaGetLastError();
}

int fft1d_bluestein_m(int n) {
  if (n >= 1 && !(n & (n - 1))) return n;
  int m = 1;
  while (m < 2 * n - 1) m *= 2;
  return m;
}

bool fft1d_supported(Precision p, int n) {
  if (n < 8) return false;
  if (n & (n - 1)) return fft1d_bluestein_m(n) <= (p == kFP64 ? 8192 : 16384);
  return n <= 16384;  // FP64 16384: the two-CTA kernel (fft1d_pair.cu)
}

template <typename R, int M, bool FLUX>
static cudaError_t launch_blu(const Fft1dJob *d_jobs, int nj, int step0, int nsteps,
                              cudaStream_t s, int n) {
  using C = typename Cx<R>::T;
  constexpr int T = M >= 8192 ? 512 : (M >= 2048 ? 256 : (M >= 512 ? 64 : 32));
  auto k = fft1d_bluestein_kernel<R, M, T, FLUX>;
  const cudaError_t attr = raise_dynamic_smem((const void *)k, (int)(sizeof(C) * (M + M / 2)));
  if (attr != cudaSuccess) return attr;
  k<<<nj, T, sizeof(C) * (M + n), s>>>(d_jobs, step0, nsteps);
  return cudaGetLastError();
}

template <typename R, int M>
static cudaError_t launch_bluf(const Fft1dJob *d_jobs, int nj, int step0, int nsteps,
                               cudaStream_t s, int n, bool flux) {
  return flux ? launch_blu<R, M, true>(d_jobs, nj, step0, nsteps, s, n)
              : launch_blu<R, M, false>(d_jobs, nj, step0, nsteps, s, n);
}

static cudaError_t launch_bluestein(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                                    int nsteps, cudaStream_t s, bool flux) {
  const int m = fft1d_bluestein_m(n);
#define PXP_BL(MM)                                                                        \
  case MM:                                                                                \
    return p == kFP64 ? launch_bluf<double, MM>(d_jobs, nj, step0, nsteps, s, n, flux)    \
                      : launch_bluf<float, MM>(d_jobs, nj, step0, nsteps, s, n, flux);
  switch (m) {
    PXP_BL(32) PXP_BL(64) PXP_BL(128) PXP_BL(256) PXP_BL(512) PXP_BL(1024) PXP_BL(2048)
    PXP_BL(4096) PXP_BL(8192)
    case 16384:
      if (p == kFP32) return launch_bluf<float, 16384>(d_jobs, nj, step0, nsteps, s, n, flux);
      return cudaErrorInvalidValue;
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_BL
}

template <typename R, int N>
static cudaError_t launch_nf(const Fft1dJob *d_jobs, int nj, int step0, int nsteps, cudaStream_t s,
                             bool flux, unsigned *queue) {
  return flux ? launch_n<R, N, true>(d_jobs, nj, step0, nsteps, s, queue)
              : launch_n<R, N, false>(d_jobs, nj, step0, nsteps, s, queue);
}

int fft1d_variants(Precision p, int n) {
  return !fft1d_pair_size(p, n) && fft1d_r16_enabled(n) ? 2 : 1;
}

cudaError_t launch_fft1d(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                         int nsteps, cudaStream_t s, bool flux, int variant, unsigned *queue) {
  if (nj <= 0) return cudaSuccess;
  if (n & (n - 1)) return launch_bluestein(p, d_jobs, nj, n, step0, nsteps, s, flux);
  if (fft1d_pair_size(p, n)) return launch_fft1d_pair(p, d_jobs, nj, n, step0, nsteps, s, flux);
  if (variant != 0 && fft1d_r16_enabled(n))
    return launch_fft1d_r16(p, d_jobs, nj, n, step0, nsteps, s, flux, queue);
#define PXP_CASE(NN)                                                              \
  case NN:                                                                        \
    return p == kFP64 ? launch_nf<double, NN>(d_jobs, nj, step0, nsteps, s, flux, queue)     \
                      : launch_nf<float, NN>(d_jobs, nj, step0, nsteps, s, flux, queue);
  switch (n) {
    PXP_CASE(8) PXP_CASE(16) PXP_CASE(32) PXP_CASE(64) PXP_CASE(128) PXP_CASE(256)
    PXP_CASE(512) PXP_CASE(1024) PXP_CASE(2048) PXP_CASE(4096) PXP_CASE(8192)
    case 16384:
      if (p == kFP32) return launch_nf<float, 16384>(d_jobs, nj, step0, nsteps, s, flux, queue);
      return cudaErrorInvalidValue;
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_CASE
}

}  // namespace pxp
