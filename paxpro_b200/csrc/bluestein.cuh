// bluestein.cuh -- a DFT of any length in shared memory by Bluestein's
// chirp-z identity, shared by the 1-transverse-dim kernel (fft1d.cu) and the
// FFTSolver3D line passes for lengths that are not powers of two
// (fft3d_blu.cu).
#pragma once
#include "fft_smem.cuh"

namespace pxp {

// Lengths that are not powers of two: Bluestein's chirp-z identity
// jk = (j^2 + k^2 - (k - j)^2) / 2 turns the n-point DFT into
//   X_k = w_k sum_j (x_j w_j) conj(w)_{k-j},   w_j = exp(-i pi j^2 / n),
// a circular convolution of length m >= 2n - 1 (a power of two): two
// shared-memory FFTs of length m and a pointwise product with the
// precomputed transform of the filter (1/m folded in).  The inverse
// transform is conj(DFT(conj(X))).  The field stays resident in shared
// memory beside the m-point work buffer, as in the power-of-two kernel.
// Tables (chirp w, filter transform bf, Stockham twiddles tw): complex128
// for FP64 data, split complex64 pairs for complex64 data (fft_smem.cuh).
template <typename R, int M, int T>
__device__ __forceinline__ void bluestein_dft(typename Cx<R>::T *x, typename Cx<R>::T *u, int n,
                                              const Tw<typename Cx<R>::T> *w,
                                              const Tw<typename Cx<R>::T> *bf,
                                              const Tw<typename Cx<R>::T> *tw, int lane,
                                              bool inverse) {
  using C = typename Cx<R>::T;
  for (int j = lane; j < M; j += T) {
    C a{};
    if (j < n) {
      C v = u[j];
      if (inverse) v.y = -v.y;
      a = tw_mul(v, w[j]);
    }
    x[sw<C>(j)] = a;
  }
  __syncthreads();
  fft_smem<C, M, T, -1>(x, tw, lane);
  for (int k = lane; k < M; k += T) x[sw<C>(k)] = tw_mul(x[sw<C>(k)], bf[k]);
  __syncthreads();
  fft_smem<C, M, T, +1>(x, tw, lane);
  for (int k = lane; k < n; k += T) {
    C v = tw_mul(x[sw<C>(k)], w[k]);
    if (inverse) v.y = -v.y;
    u[k] = v;
  }
  __syncthreads();
}

}  // namespace pxp
