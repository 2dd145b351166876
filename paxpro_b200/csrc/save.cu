// save.cu -- transverse downsampling of saved 3-D fields.
//
// Solver3D::copyCurrentSolution (src/solver3D.cpp:94-112) stores, at save
// steps, an m x m slice of the n x n field with m = n / ratio
// (src/solver3D.cpp:26, 36): with delta = n / m (a double), entry (row, col)
// is the sum of the block of rows [row*delta, row*delta + delta - 1] and
// columns [col*delta, col*delta + delta - 1] (bounds truncated to unsigned,
// as the reference's submat arguments are), summed column by column in FP64,
// divided by delta*delta.  One thread per output entry; consecutive threads
// take consecutive rows, so the reads of each block column are coalesced
// across the warp.
#include "pxp_complex.cuh"
#include "pxp_kernels.h"

namespace pxp {

template <typename R>
__global__ void block_average_kernel(const typename Cx<R>::T *__restrict__ full,
                                     typename Cx<R>::T *__restrict__ out, int n, int m,
                                     double delta) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)m * m) return;
  const int row = (int)(idx % m), col = (int)(idx / m);
  const unsigned r0 = (unsigned)(row * delta), r1 = (unsigned)(row * delta + delta - 1);
  const unsigned c0 = (unsigned)(col * delta), c1 = (unsigned)(col * delta + delta - 1);
  double2 total = mk(0.0, 0.0);
  for (unsigned c = c0; c <= c1 && c < (unsigned)n; ++c) {
    double2 colsum = mk(0.0, 0.0);
    for (unsigned r = r0; r <= r1 && r < (unsigned)n; ++r)
      colsum = cadd(colsum, to_d(full[(long long)c * n + r]));
    total = cadd(total, colsum);
  }
  const double d2 = delta * delta;
  out[idx] = from_d<R>(mk(total.x / d2, total.y / d2));
}

cudaError_t launch_block_average(Precision p, const void *full, void *out, int n, int m,
                                 cudaStream_t s) {
  if (m <= 0 || m > n) return cudaErrorInvalidValue;
  const double delta = (double)n / (double)m;
  const long long total = (long long)m * m;
  const int T = 256;
  const int grid = (int)((total + T - 1) / T);
  if (p == kFP64)
    block_average_kernel<double><<<grid, T, 0, s>>>((const double2 *)full, (double2 *)out, n, m, delta);
  else
    block_average_kernel<float><<<grid, T, 0, s>>>((const float2 *)full, (float2 *)out, n, m, delta);
  return cudaGetLastError();
}

}  // namespace pxp
