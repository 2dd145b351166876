// post.cu -- device-side reductions for the post-processing modules.
//
// The reference's post:: modules (src/postProcessMod.cpp) turn the saved
// fields and the exit field into real arrays: |u| (post::Intensity, and the
// scale of IntensityUint8), arg u (post::Phase, ExitPhase), Re u
// (post::ExitField) and |u|^2 (post::ExitIntensity, computed as
// pow(abs(u), 2)).  These kernels compute them on the device from the
// resident fields, so a caller copies back 8 bytes per point instead of the
// complex field; max_abs_kernel gives the largest |u| over a set of saved
// fields (IntensityUint8's scale, src/postProcessMod.cpp:23).
#include "flux.cuh"
#include "pxp_complex.cuh"
#include "pxp_kernels.h"

namespace pxp {

template <typename R>
__global__ void post_kernel(const typename Cx<R>::T *__restrict__ in, double *__restrict__ out,
                            long long n, int quantity) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = to_d(in[i]);
    double r;
    switch (quantity) {
      case 0: r = hypot(v.x, v.y); break;  // std::abs(complex)
      case 1: r = atan2(v.y, v.x); break;  // std::arg
      case 2: r = v.x; break;
      default: {
        const double a = hypot(v.x, v.y);
        r = a * a;
      }
    }
    out[i] = r;
  }
}

// |u| >= 0, so the IEEE bit patterns order as the values: a 64-bit atomic
// max on the bits is a max on the values.
template <typename R>
__global__ void max_abs_kernel(const typename Cx<R>::T *__restrict__ in, long long n,
                               unsigned long long *__restrict__ result) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = to_d(in[i]);
    m = fmax(m, hypot(v.x, v.y));
  }
  for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, d));
  if ((threadIdx.x & 31) == 0) atomicMax(result, (unsigned long long)__double_as_longlong(m));
}

// The trapezoid sum of |u|^2 over [a, b] of the current field
// (Transmittivity's integral outside the step kernels, e.g. its intensity at
// zero), with the step kernels' summation.
template <typename R, int T>
__global__ void __launch_bounds__(T) flux_sum_kernel(const typename Cx<R>::T *__restrict__ u, int a,
                                                     int b, double *__restrict__ out) {
  __shared__ double red[flux_slots<T>()];
  double acc = 0.0;
  const int2 w = make_int2(a, b);
  for (int i = a + (int)threadIdx.x; i <= b; i += T) flux_add(acc, i, w, to_d(u[i]));
  flux_warp_total<T>(acc, red);
  __syncthreads();
  const FluxSpec f{nullptr, out, 0, 1};
  flux_store<T>(f, 0, red);
}

static int post_grid(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

cudaError_t launch_post(Precision p, const void *field, double *out, long long n, int quantity,
                        cudaStream_t s) {
  if (quantity < 0 || quantity > 3) return cudaErrorInvalidValue;
  if (p == kFP64)
    post_kernel<double><<<post_grid(n), 256, 0, s>>>((const double2 *)field, out, n, quantity);
  else
    post_kernel<float><<<post_grid(n), 256, 0, s>>>((const float2 *)field, out, n, quantity);
  return cudaGetLastError();
}

cudaError_t launch_max_abs(Precision p, const void *field, long long n, unsigned long long *result,
                           cudaStream_t s) {
  if (p == kFP64)
    max_abs_kernel<double><<<post_grid(n), 256, 0, s>>>((const double2 *)field, n, result);
  else
    max_abs_kernel<float><<<post_grid(n), 256, 0, s>>>((const float2 *)field, n, result);
  return cudaGetLastError();
}

cudaError_t launch_flux_sum(Precision p, const void *field, int a, int b, double *out,
                            cudaStream_t s) {
  if (p == kFP64)
    flux_sum_kernel<double, 256><<<1, 256, 0, s>>>((const double2 *)field, a, b, out);
  else
    flux_sum_kernel<float, 256><<<1, 256, 0, s>>>((const float2 *)field, a, b, out);
  return cudaGetLastError();
}

}  // namespace pxp
