// fft1d_r16.cu -- FFTSolver2D split step with register-resident radix-16
// transforms (n = 512 .. 4096).
//
// Same step as fft1d.cu (src/fftSolver2D.cpp:21-73): forward FFT,
// propagator multiply, backward FFT, transmission and 1/N, one CTA per
// problem for all steps of the launch.  Here the field lives in registers
// between steps: thread j of the n/16 threads holds the points j + s*n/16
// (fft_r16.cuh), every transform crosses shared memory twice (first pass of
// radix R0 on the thread's own points, two radix-16 Stockham passes), and
// the propagator, the transmission, the save and the flux terms are applied
// in registers where the forward and inverse transforms meet.  The two
// crossings of a transform use two buffers alternately, so a transform
// takes two CTA barriers: a thread writing buffer 0 of the next transform
// has passed the barrier that follows every thread's last read of buffer 0,
// and a thread writing buffer 1 has passed the barrier that follows every
// thread's read of buffer 1 in the previous transform.  A step takes four
// barriers (the shared-memory kernel of fft1d.cu takes two per Stockham
// pass plus two for the pointwise products).
//
// Pointwise arithmetic is fft1d.cu's: FP64 rounds (u * kernel) and
// (u * t) / N as the reference does; FP32 multiplies by split complex64
// tables (kernel, t / N) with one FMA chain (fft_smem.cuh).
#include "fft_r16.cuh"
#include "flux.cuh"
#include "persistent.cuh"
#include "pxp_kernels.h"

namespace pxp {
namespace r16_1d {

__device__ __forceinline__ void refract(double2 &u, double2 t, double n) {
  u = cx_div_real_rn(cx_mul_rn(u, t), n);
}
__device__ __forceinline__ void refract(float2 &u, float4 t, float) { u = tw_mul(u, t); }
__device__ __forceinline__ double2 kmul(double2 u, double2 k) { return cx_mul_rn(u, k); }
__device__ __forceinline__ float2 kmul(float2 u, float4 k) { return tw_mul(u, k); }

// One transform of the thread's 16 points (natural order before and after);
// X0, X1: the two exchange buffers (swizzled, elements of the field's type).
template <int SIGN, int N, typename C>
__device__ __forceinline__ void line_fft(C (&v)[16], C *X0, C *X1, const Tw<C> *tws, int j) {
  using P = r16c::Plan<N>;
  constexpr int TL = P::TL, R0 = P::R0, B = (int)sizeof(C);
  static_assert(P::NP16 == 2, "two radix-16 passes");
  r16c::first_pass<SIGN, R0>(v);
#pragma unroll
  for (int u = 0; u < 16 / R0; ++u)
#pragma unroll
    for (int r = 0; r < R0; ++r) X0[r16c::xsw<B>((j + u * TL) * R0 + r)] = v[u + r * (16 / R0)];
  __syncthreads();
  // radix-16 pass 0 (NS = R0): X0 -> X1
  {
    constexpr int NS = R0;
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = X0[r16c::xsw<B>(j + r * TL)];
    const int k = j & (NS - 1);
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      const Tw<C> w = tws[(r - 1) * NS + k];
      v[r] = SIGN < 0 ? tw_mul(v[r], w) : tw_mulc(v[r], w);
    }
    dft16<SIGN>(v);
    const int base = (j - k) * 16 + k;
#pragma unroll
    for (int r = 0; r < 16; ++r) X1[r16c::xsw<B>(base + r * NS)] = v[r];
  }
  __syncthreads();
  // radix-16 pass 1 (NS = 16 R0 = n/16): X1 -> registers, natural order
  {
    constexpr int NS = 16 * R0;
    constexpr int OFF = r16c::tw_offset<R0, 1>();
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = X1[r16c::xsw<B>(j + r * TL)];
#pragma unroll
    for (int r = 1; r < 16; ++r) {
      const Tw<C> w = tws[OFF + (r - 1) * NS + j];
      v[r] = SIGN < 0 ? tw_mul(v[r], w) : tw_mulc(v[r], w);
    }
    dft16<SIGN>(v);
  }
}

template <typename R, int N, bool FLUX>
__global__ void __launch_bounds__(N / 16) fft1d_r16_kernel(const Fft1dJob *__restrict__ jobs,
                                                          int step0_ov, int nsteps_ov, int njobs,
                                                          unsigned *queue) {
  using C = typename Cx<R>::T;
  using W = Tw<C>;
  using P = r16c::Plan<N>;
  constexpr int TL = P::TL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double flux_red[2][flux_slots<TL>()];
  C *X0 = reinterpret_cast<C *>(smem_raw);
  C *X1 = X0 + N;
  W *tws = reinterpret_cast<W *>(X1 + N);
  __shared__ int s_next;
  for (int jb = blockIdx.x; jb < njobs; jb = next_job(queue, &s_next)) {
  Fft1dJob job = jobs[jb];
  if (nsteps_ov >= 0) {
    job.step0 = step0_ov;
    job.nsteps = nsteps_ov;
  }
  const int j = threadIdx.x;
  r16c::load_twiddles<N>(tws, reinterpret_cast<const W *>(job.wn), j, TL);
  C *field = reinterpret_cast<C *>(job.field);
  C v[16];
#pragma unroll
  for (int s = 0; s < 16; ++s) v[s] = field[j + s * TL];
  __syncthreads();
  const W *kern = reinterpret_cast<const W *>(job.kern);
  const W *trans0 = reinterpret_cast<const W *>(job.trans);
  C *saves = reinterpret_cast<C *>(job.saves);
  const R nreal = (R)N;
  for (int st = 0; st < job.nsteps; ++st) {
    const int step = job.step0 + st;
    int2 fw;
    const bool flux = FLUX && flux_window(job.flux, step, fw);
    line_fft<-1, N>(v, X0, X1, tws, j);
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = kmul(v[s], __ldg(kern + j + s * TL));
    line_fft<+1, N>(v, X0, X1, tws, j);
    const W *trans = trans0 + job.trans_stride * (long long)(step - job.trans_step0);
    const bool save = job.save_every > 0 && saves != nullptr && (step % job.save_every) == 0 &&
                      (step / job.save_every - 1) < job.max_slots;
    C *slot = save ? saves + (long long)(step / job.save_every - 1) * N : nullptr;
    double acc = 0.0;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
      const int e = j + s * TL;
      refract(v[s], __ldg(trans + e), nreal);
      if (save) slot[e] = v[s];
      if (flux) flux_add(acc, e, fw, to_d(v[s]));
    }
    if constexpr (FLUX) {
      if (flux) flux_warp_total<TL>(acc, flux_red[st & 1]);
      __syncthreads();
      if (flux) flux_store<TL>(job.flux, step, flux_red[st & 1]);
    }
  }
#pragma unroll
  for (int s = 0; s < 16; ++s) field[j + s * TL] = v[s];
  }
}

template <typename R, int N, bool FLUX>
cudaError_t launch(const Fft1dJob *d_jobs, int nj, int step0, int nsteps, cudaStream_t s,
                   unsigned *queue) {
  using C = typename Cx<R>::T;
  constexpr size_t smem = 2 * sizeof(C) * N + sizeof(Tw<C>) * r16c::Plan<N>::TWN;
  static_assert(smem <= 227 * 1024, "exchange buffers and twiddles exceed shared memory");
  auto k = fft1d_r16_kernel<R, N, FLUX>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const int grid = persistent_grid((const void *)k, N / 16, smem, nj, queue);
  k<<<grid, N / 16, smem, s>>>(d_jobs, step0, nsteps, nj, queue);
  return cudaGetLastError();
}

}  // namespace r16_1d

bool fft1d_r16_enabled(int n) { return n >= 512 && n <= 4096 && !(n & (n - 1)); }

cudaError_t launch_fft1d_r16(Precision p, const Fft1dJob *d_jobs, int nj, int n, int step0,
                             int nsteps, cudaStream_t s, bool flux, unsigned *queue) {
#define PXP_1R(NN)                                                                              \
  case NN:                                                                                      \
    if (p == kFP64)                                                                             \
      return flux ? r16_1d::launch<double, NN, true>(d_jobs, nj, step0, nsteps, s, queue)       \
                  : r16_1d::launch<double, NN, false>(d_jobs, nj, step0, nsteps, s, queue);     \
    return flux ? r16_1d::launch<float, NN, true>(d_jobs, nj, step0, nsteps, s, queue)          \
                : r16_1d::launch<float, NN, false>(d_jobs, nj, step0, nsteps, s, queue);
  switch (n) {
    PXP_1R(512) PXP_1R(1024) PXP_1R(2048) PXP_1R(4096)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_1R
}

}  // namespace pxp
