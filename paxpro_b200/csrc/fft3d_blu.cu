// fft3d_blu.cu -- FFTSolver3D line passes for grid sizes that are not powers
// of two (the reference plans FFTW for any n, src/fftSolver3D.cpp:61-62; its
// own example grid has 513 nodes, Examples/sphere.cpp:40).
//
// The same two passes per step as fft3d.cu (x pass: F_x, K, F_x^-1; y pass:
// F_y^-1, refraction, F_y), each line transform a Bluestein chirp-z DFT
// (bluestein.cuh): the n-point DFT as a circular convolution of length m >=
// 2n - 1, two m-point shared-memory FFTs and a product with the filter's
// precomputed transform.  A CTA takes one line at a time (grid-stride),
// keeps it in shared memory beside the m-point work buffer, and applies the
// per-point arithmetic of fft3d_point.cuh between the transforms; the
// refraction divides by n*n (not a power of two here) as the reference
// does.
#include "bluestein.cuh"
#include "fft3d_point.cuh"

namespace pxp {

template <typename R, int M, int T>
__global__ void __launch_bounds__(T) fft3d_blu_kernel(const Fft3dPass q, const double *__restrict__ kx2,
                                                     const Tw<typename Cx<R>::T> *__restrict__ tw,
                                                     const Tw<typename Cx<R>::T> *__restrict__ chirp,
                                                     const Tw<typename Cx<R>::T> *__restrict__ bconv) {
  using C = typename Cx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *x = reinterpret_cast<C *>(smem_raw);  // m-point work buffer (swizzled)
  C *u = x + M;                            // the line, n points
  const int n = q.n;
  const int lane = threadIdx.x;
  C *field = reinterpret_cast<C *>(q.field);
  C *save = reinterpret_cast<C *>(q.save);
  const bool strided = q.mode == 1;  // x lines: fixed row, stride n
  for (int line = blockIdx.x; line < n; line += gridDim.x) {
    for (int j = lane; j < n; j += T)
      u[j] = strided ? field[(long long)j * n + line] : field[(long long)line * n + j];
    __syncthreads();
    if (q.mode == 1) {
      bluestein_dft<R, M, T>(x, u, n, chirp, bconv, tw, lane, false);
      // propagator K = exp(-i a (kx^2 + ky^2)) (src/fftSolver3D.cpp:24-30, 87-120)
      const double ky = kfreq(line, n, q.two_pi, q.stepn_y);
      const double ky2 = __dmul_rn(ky, ky);
      for (int j = lane; j < n; j += T) u[j] = prop3(q, u[j], kx2[j], ky2, j, line);
      __syncthreads();
      bluestein_dft<R, M, T>(x, u, n, chirp, bconv, tw, lane, true);
    } else {
      if (q.mode >= 2) {
        bluestein_dft<R, M, T>(x, u, n, chirp, bconv, tw, lane, true);
        for (int j = lane; j < n; j += T) {
          const C v = refract3<R>(q, u[j], line, j, 0.0);  // 0: divide by n*n
          u[j] = v;
          if (save) save[(long long)line * n + j] = v;
        }
        __syncthreads();
      }
      if (q.mode != 3) bluestein_dft<R, M, T>(x, u, n, chirp, bconv, tw, lane, false);
    }
    for (int j = lane; j < n; j += T) {
      if (strided)
        field[(long long)j * n + line] = u[j];
      else
        field[(long long)line * n + j] = u[j];
    }
    __syncthreads();  // u is reloaded next
  }
}

template <typename R, int M>
static cudaError_t blu_launch(const Fft3dPass &q, const double *kx2, cudaStream_t s) {
  using C = typename Cx<R>::T;
  constexpr int T = M >= 8192 ? 512 : (M >= 2048 ? 256 : (M >= 512 ? 64 : 32));
  const size_t smem = sizeof(C) * (M + (size_t)q.n);
  auto k = fft3d_blu_kernel<R, M, T>;
  {
    const cudaError_t e = raise_dynamic_smem((const void *)k, (int)(sizeof(C) * (M + M / 2)));
    if (e != cudaSuccess) return e;
  }
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, T, smem);
  if (e != cudaSuccess) return e;
  const int cap = sms * (per > 0 ? per : 1);
  using W = Tw<C>;
  k<<<q.n < cap ? q.n : cap, T, smem, s>>>(q, kx2, (const W *)q.twiddle, (const W *)q.chirp,
                                         (const W *)q.bconv);
  return cudaGetLastError();
}

cudaError_t launch_fft3d_bluestein(Precision p, const Fft3dPass &q, const double *kx2,
                                   cudaStream_t s) {
  if (q.chirp == nullptr || q.bconv == nullptr) return cudaErrorInvalidValue;
#define PXP_B3(MM)                                                                  \
  case MM:                                                                          \
    return p == kFP64 ? blu_launch<double, MM>(q, kx2, s) : blu_launch<float, MM>(q, kx2, s);
  switch (q.m) {
    PXP_B3(32) PXP_B3(64) PXP_B3(128) PXP_B3(256) PXP_B3(512) PXP_B3(1024) PXP_B3(2048)
    PXP_B3(4096) PXP_B3(8192)
    case 16384:
      if (p == kFP32) return blu_launch<float, 16384>(q, kx2, s);
      return cudaErrorInvalidValue;
    default:
      return cudaErrorInvalidValue;
  }
#undef PXP_B3
}

}  // namespace pxp
