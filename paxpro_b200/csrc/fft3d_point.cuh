// fft3d_point.cuh -- per-point arithmetic of the FFTSolver3D line passes:
// the material at a point (spheres or CSG), FFTSolver3D::refraction with its
// refraction integral (src/fftSolver3D.cpp:122-156, 253-273), the absorber
// bands (src/absorber.cpp:3-12), the spatial frequencies (:32-50) and the
// propagator product.  Shared by the line-pass kernels of fft3d.cu and
// fft3d_lines.cu so that both round every point identically.
#pragma once
#include "csg.cuh"
#include "fft_smem.cuh"
#include "pxp_kernels.h"
#include "pxp_sincos.h"

namespace pxp {

__device__ __forceinline__ void sph_eval(const Fft3dPass &q, double x, double y, double z,
                                         double &delta, double &beta) {
  if (q.csg.active) {
    csg_material(q.csg, x, y, z, delta, beta);
    return;
  }
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

// The index spatialFreq folds to: the propagator factor tables hold equal
// entries at idx and n - idx, and reading entries 0 .. n/2 only halves the
// part of a table a line pass keeps in L1.
__device__ __forceinline__ int kfold(int idx, int n) { return idx > n / 2 ? n - idx : idx; }

// spatialFreq: fold, then 2*PI*indx / (step*size)
__device__ __forceinline__ double kfreq(int idx, int n, double two_pi, double stepn) {
  if (idx > n / 2) idx = n - idx;
  return __ddiv_rn(__dmul_rn(two_pi, (double)idx), stepn);
}

// Propagator product of the x pass at column ix (kx2 = fl(kx*kx) there) of
// row iy (ky2 = fl(ky*ky)).  FP64: the product of the x and y factors of
// the propagator, exp(-i a kx^2) exp(-i a ky^2), from tables whose phases
// are reduced on the host in extended precision, rounded like one complex
// product with K; or, without tables (PXP_FFT3D_JOINT_PROP=1), the
// reference's argument fl(a * fl(kx2 + ky2)) and its sin/cos
// (src/fftSolver3D.cpp:24-30).  The two differ by the rounding of that
// argument (about 1e-13 rad at the largest frequencies, the same every
// step): 3.7e-13 relative L2 after 1000 steps of a field rich in high
// frequencies, against 30 FP64 operations a point saved.  FP32 multiplies
// by the split x and y factors.
__device__ __forceinline__ double2 prop3(const Fft3dPass &q, double2 u, double kx2, double ky2,
                                         int ix, int iy) {
  if (q.prop_x != nullptr) {
    const double2 *px = reinterpret_cast<const double2 *>(q.prop_x);
    const double2 *py = reinterpret_cast<const double2 *>(q.prop_y);
    return cx_mul_rn(u, cx_mul_rn(__ldg(px + kfold(ix, q.n)), __ldg(py + kfold(iy, q.n))));
  }
  const double phi = __dmul_rn(q.a, __dadd_rn(kx2, ky2));
  double sn, cs;
  sincos_cw(phi, &sn, &cs);
  return cx_mul_rn(u, mk(cs, -sn));
}
__device__ __forceinline__ float2 prop3(const Fft3dPass &q, float2 u, double, double, int ix,
                                        int iy) {
  const float4 *px = reinterpret_cast<const float4 *>(q.prop_x);
  const float4 *py = reinterpret_cast<const float4 *>(q.prop_y);
  return tw_mul(tw_mul(u, __ldg(px + kfold(ix, q.n))), __ldg(py + kfold(iy, q.n)));
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
                                                      int ix, int iy, double inv_norm) {
  const double x = __dadd_rn(q.xmin, __dmul_rn((double)ix, q.dx));
  const double y = __dadd_rn(q.ymin, __dmul_rn((double)iy, q.dy));
  double delta = 0.0, beta = 0.0;
  if (q.plane_delta) {
    const long long idx = (long long)ix * q.n + iy;
    delta = q.plane_delta[idx];
    beta = q.plane_beta[idx];
  } else if (q.nspheres > 0 || q.csg.active) {
    step_material(q, x, y, delta, beta);
  }
  if constexpr (sizeof(R) == 4) {
    // complex64 point with no material and no absorber band: the scaling by
    // 1/(n*n), a power of two, is exact in FP32
    if (delta == 0.0 && beta == 0.0 && inv_norm != 0.0 && q.thick_x == 0 && q.thick_y == 0) {
      const float sc = (float)inv_norm;
      return mk(uu.x * sc, uu.y * sc);
    }
  }
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
  // (u * t) / (n*n): when n*n is a power of two, multiplying by its exact
  // reciprocal rounds identically to the division; other sizes pass
  // inv_norm = 0 and divide
  u = inv_norm != 0.0 ? cx_scale_rn(u, inv_norm) : cx_div_real_rn(u, q.norm);
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

}  // namespace pxp

namespace pxp {

// Whether the y pass's refraction reduces to the scaling by 1/(n*n) at every
// point: no material sample in the step (no sphere meets the slab, no CSG
// or sampled plane), no absorber band, and n*n a power of two.
__device__ __forceinline__ bool refract3_is_scale(const Fft3dPass &q, double inv_norm) {
  return q.nspheres == 0 && !q.csg.active && q.plane_delta == nullptr && q.thick_x == 0 &&
         q.thick_y == 0 && inv_norm != 0.0;
}

// The register-resident line kernels unroll their points; refract3 inlined
// at every one of them (material lookups, refraction integral, exp and
// sin/cos, absorber) makes the y pass's code outgrow the instruction cache,
// and a call per point spills the caller's live registers.  So they apply
// the scaling-only case inline (refract3_is_scale: the same rounding as
// refract3, an exact power-of-two scale in either precision) and otherwise
// stage their points through shared memory and run refract3 in one
// non-unrolled loop over them.
template <typename C> __device__ __forceinline__ C scale_point(C u, double inv_norm);
template <> __device__ __forceinline__ double2 scale_point(double2 u, double inv_norm) {
  return cx_scale_rn(u, inv_norm);
}
template <> __device__ __forceinline__ float2 scale_point(float2 u, double inv_norm) {
  const float sc = (float)inv_norm;
  return mk(u.x * sc, u.y * sc);
}

}  // namespace pxp
