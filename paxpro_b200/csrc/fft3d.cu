// fft3d.cu -- K-FFT2: FFTSolver3D split step as two HBM line passes.
//
// Replaces FFTSolver3D::solveStep (src/fftSolver3D.cpp:52-85): the 2-D FFTW
// transforms of propagate (:87-120) are split into 1-D transforms along x and
// along y and regrouped so that each step reads and writes the field twice:
//   x pass  (lines of fixed row index, stride n):  F_x, * K(kx, ky), F_x^-1
//   y pass  (contiguous lines of fixed x):          F_y^-1, refraction, F_y
// where the y pass's trailing F_y is the next step's first transform.  A CTA
// keeps L whole lines in shared memory; loads and stores are coalesced in
// runs of L elements for the strided pass and fully for the contiguous one.
//
// FP64 pointwise arithmetic follows the reference op by op: the propagator
// argument fl(a * fl(fl(kx*kx) + fl(ky*ky))) with kx, ky from
// spatialFreqX/Y (:32-50), the refraction (prev * t) / (n*n) with t =
// exp(-k (beta + i delta) dz) (:154), the refraction integral (:253-273) when
// the material at z0 and z1 differs by more than 1e-10, and the absorber
// bands (Absorber::apply, src/absorber.cpp:3-12: y bands, then x bands).
// sin/cos/exp are CUDA's (<= 2 ulp); everything else is rounded as the
// reference rounds it.
#include "fft_smem.cuh"
#include "pxp_kernels.h"

namespace pxp {

__device__ __forceinline__ void sph_eval(const Fft3dPass &q, double x, double y, double z,
                                         double &delta, double &beta) {
  delta = 0.0;
  beta = 0.0;
  const int n = q.nspheres;
  const Sphere *list = n > kInlineSpheres ? q.spheres_all : q.spheres;
  for (int i = 0; i < n; ++i) {
    const Sphere sp = list[i];
    double ddx = __dsub_rn(x, sp.cx), ddy = __dsub_rn(y, sp.cy), ddz = __dsub_rn(z, sp.cz);
    double rsq = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz));
    if (rsq < __dmul_rn(sp.r, sp.r)) {
      delta = sp.delta;
      beta = sp.beta;
      return;
    }
  }
}

// FFTSolver3D::refraction for one point: delta, beta used for the step.
__device__ __forceinline__ void step_material(const Fft3dPass &q, double x, double y,
                                              double &delta, double &beta) {
  double dp, bp;
  sph_eval(q, x, y, q.z1, delta, beta);
  sph_eval(q, x, y, q.z0, dp, bp);
  if (fabs(__dsub_rn(delta, dp)) > 1e-10 || fabs(__dsub_rn(beta, bp)) > 1e-10) {
    // refractionIntegral(x, y, z0, z1): endpoints once, 8 interior samples
    // twice (the 9th is skipped), divided by 2*10
    double dt, bt;
    sph_eval(q, x, y, q.z0, delta, beta);
    sph_eval(q, x, y, q.z1, dt, bt);
    delta = __dadd_rn(delta, dt);
    beta = __dadd_rn(beta, bt);
    const double dzz = __ddiv_rn(__dsub_rn(q.z1, q.z0), 10.0);
    for (int i = 1; i < 9; ++i) {
      const double z = __dadd_rn(q.z0, __dmul_rn((double)i, dzz));
      sph_eval(q, x, y, z, dt, bt);
      delta = __dadd_rn(delta, __dmul_rn(2.0, dt));
      beta = __dadd_rn(beta, __dmul_rn(2.0, bt));
    }
    delta = __ddiv_rn(delta, 20.0);
    beta = __ddiv_rn(beta, 20.0);
  }
}

// spatialFreq: fold, then 2*PI*indx / (step*size)
__device__ __forceinline__ double kfreq(int idx, int n, double two_pi, double stepn) {
  if (idx > n / 2) idx = n - idx;
  return __ddiv_rn(__dmul_rn(two_pi, (double)idx), stepn);
}

template <typename R> __device__ __forceinline__ typename Cx<R>::T mul_k(typename Cx<R>::T u,
                                                                        double2 k);
template <> __device__ __forceinline__ double2 mul_k<double>(double2 u, double2 k) {
  return cx_mul_rn(u, k);
}
template <> __device__ __forceinline__ float2 mul_k<float>(float2 u, double2 k) {
  return tw_mul(u, k);
}

// Refraction, absorber: u = (u * t) / (n*n), then absorber factors.
template <typename R>
__device__ __forceinline__ typename Cx<R>::T refract3(const Fft3dPass &q, typename Cx<R>::T uu,
                                                      int ix, int iy) {
  const double x = __dadd_rn(q.xmin, __dmul_rn((double)ix, q.dx));
  const double y = __dadd_rn(q.ymin, __dmul_rn((double)iy, q.dy));
  double delta = 0.0, beta = 0.0;
  if (q.nspheres > 0) step_material(q, x, y, delta, beta);
  double2 u = to_d(uu);
  if (delta != 0.0 || beta != 0.0) {
    // exp(-k*(beta + i*delta)*dz)
    const double re = __dmul_rn(__dmul_rn(-q.k, beta), q.dz);
    const double im = __dmul_rn(__dmul_rn(-q.k, delta), q.dz);
    const double e = exp(re);
    double sn, cs;
    sincos(im, &sn, &cs);
    const double2 t = mk(__dmul_rn(e, cs), __dmul_rn(e, sn));
    if constexpr (sizeof(R) == 8) {
      u = cx_mul_rn(u, t);
    } else {
      u = cmul(u, t);
    }
  }
  u = cx_div_real_rn(u, q.norm);
  if (q.thick_y > 0) {
    if (iy < q.thick_y) u = cx_scale_rn(u, exp(-(double)(q.thick_y - iy - 1) * q.inv_damp_y));
    if (q.n - 1 - iy < q.thick_y)
      u = cx_scale_rn(u, exp(-(double)(q.thick_y - (q.n - 1 - iy) - 1) * q.inv_damp_y));
  }
  if (q.thick_x > 0) {
    if (ix < q.thick_x) u = cx_scale_rn(u, exp(-(double)(q.thick_x - ix - 1) * q.inv_damp_x));
    if (q.n - 1 - ix < q.thick_x)
      u = cx_scale_rn(u, exp(-(double)(q.thick_x - (q.n - 1 - ix) - 1) * q.inv_damp_x));
  }
  return from_d<R>(u);
}

template <typename R, int N, int L, int TPL>
__global__ void __launch_bounds__(L *TPL) fft3d_pass_kernel(const Fft3dPass q) {
  using C = typename Cx<R>::T;
  constexpr int T = L * TPL;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int tid = threadIdx.x;
  const int line = tid / TPL, lane = tid - line * TPL;
  C *u = buf + line * N;
  const double2 *tw = reinterpret_cast<const double2 *>(q.twiddle);
  C *field = reinterpret_cast<C *>(q.field);
  const int l0 = blockIdx.x * L;  // first line of this CTA
  const bool strided = q.mode == 1;

  // ---- load L lines
  for (int idx = tid; idx < L * N; idx += T) {
    int l, j;
    long long off;
    if (strided) {
      l = idx % L;
      j = idx / L;
      off = (long long)j * N + (l0 + l);
    } else {
      l = idx / N;
      j = idx - l * N;
      off = (long long)(l0 + l) * N + j;
    }
    buf[l * N + j] = field[off];
  }
  __syncthreads();

  if (q.mode == 1) {
    // x pass: row index of these lines is the ky index
    fft_smem<C, N, TPL, -1>(u, tw, lane);
    const double ky = kfreq(l0 + line, N, q.two_pi, q.stepn_y);
    const double ky2 = __dmul_rn(ky, ky);
    for (int j = lane; j < N; j += TPL) {
      const double kx = kfreq(j, N, q.two_pi, q.stepn_x);
      const double phi = __dmul_rn(q.a, __dadd_rn(__dmul_rn(kx, kx), ky2));
      double sn, cs;
      sincos(phi, &sn, &cs);
      u[j] = mul_k<R>(u[j], mk(cs, -sn));
    }
    __syncthreads();
    fft_smem<C, N, TPL, +1>(u, tw, lane);
  } else {
    if (q.mode >= 2) {
      fft_smem<C, N, TPL, +1>(u, tw, lane);
      C *save = reinterpret_cast<C *>(q.save);
      const int ix = l0 + line;
      for (int j = lane; j < N; j += TPL) {
        const C v = refract3<R>(q, u[j], ix, j);
        u[j] = v;
        if (save) save[(long long)ix * N + j] = v;
      }
      __syncthreads();
    }
    if (q.mode != 3) fft_smem<C, N, TPL, -1>(u, tw, lane);
  }

  // ---- store
  for (int idx = tid; idx < L * N; idx += T) {
    int l, j;
    long long off;
    if (strided) {
      l = idx % L;
      j = idx / L;
      off = (long long)j * N + (l0 + l);
    } else {
      l = idx / N;
      j = idx - l * N;
      off = (long long)(l0 + l) * N + j;
    }
    field[off] = buf[l * N + j];
  }
}

// Lines per CTA: about 128 KB of line data; threads per line: N/16 (two
// radix-8 butterflies per thread per pass), at least 16.
template <typename R, int N> constexpr int lines_per_cta() {
  constexpr int per = (int)((128 * 1024) / (sizeof(typename Cx<R>::T) * N));
  return per < 1 ? 1 : (per > 8 ? 8 : per);
}
template <int N> constexpr int threads_per_line() { return N / 16 < 16 ? 16 : (N / 16 > 512 ? 512 : N / 16); }

template <typename R, int N>
static cudaError_t fft3d_launch_n(const Fft3dPass &q, cudaStream_t s) {
  using C = typename Cx<R>::T;
  constexpr int L = lines_per_cta<R, N>();
  constexpr int TPL = threads_per_line<N>();
  constexpr size_t smem = sizeof(C) * L * N;
  auto k = fft3d_pass_kernel<R, N, L, TPL>;
  if (smem > 48 * 1024) {
    static const cudaError_t attr =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr != cudaSuccess) return attr;
  }
  k<<<N / L, L * TPL, smem, s>>>(q);
  return cudaGetLastError();
}

bool fft3d_supported(Precision p, int n) {
  if (n < 64 || (n & (n - 1))) return false;
  return n <= 8192;
}

cudaError_t launch_fft3d_pass(Precision p, const Fft3dPass &q, cudaStream_t s) {
#define PXP_C3(NN)                                                                  \
  case NN:                                                                          \
    return p == kFP64 ? fft3d_launch_n<double, NN>(q, s) : fft3d_launch_n<float, NN>(q, s);
  switch (q.n) {
    PXP_C3(64) PXP_C3(128) PXP_C3(256) PXP_C3(512) PXP_C3(1024) PXP_C3(2048) PXP_C3(4096)
    PXP_C3(8192)
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_C3
}

}  // namespace pxp
