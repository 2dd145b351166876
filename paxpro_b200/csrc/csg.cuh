// csg.cuh -- constructive-solid-geometry material evaluated on the device.
//
// The reference's CSGMaterial::getXrayMatProp (src/materialFunction.cpp:3-13)
// over geom::Module / Part / Shape (src/geometry.cpp:91-108, 212-234,
// src/shape.cpp:59-70, 146-187), with every floating-point operation rounded
// as the reference's scalar code rounds it (no contraction):
//   * a shape transforms the point by its 4x4 matrix, each row summed left
//     to right (Armadillo's product of a 4x4 matrix and a 4-vector), the
//     fourth coordinate 1;
//   * sphere: sqrt((x*x + y*y) + z*z) < R; box: strict |x| < Lx/2 per axis;
//     cylinder: -h/2 < z < h/2 and sqrt(x*x + y*y) < (r2-r1)/h*(z + h/2) + r1;
//   * a part contains the point when its last shape (scanning backwards)
//     that contains it joined as a union; a module's last part (scanning
//     backwards) that contains the point decides: union -> its (delta,
//     beta), difference -> vacuum; the first module (in order) that decides
//     gives the material.
#pragma once
#include "pxp_kernels.h"

namespace pxp {

__device__ __forceinline__ double csg_row(const double *m, double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[0], x), __dmul_rn(m[1], y)), __dmul_rn(m[2], z)), m[3]);
}

__device__ __forceinline__ bool csg_shape_inside(const CsgShape &s, double x, double y, double z) {
  const double tx = csg_row(s.m, x, y, z), ty = csg_row(s.m + 4, x, y, z), tz = csg_row(s.m + 8, x, y, z);
  if (s.kind == 0) {  // sphere
    const double r = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)), __dmul_rn(tz, tz)));
    return r < s.size[0];
  }
  if (s.kind == 1) {  // box
    const double hx = s.size[0] / 2.0, hy = s.size[1] / 2.0, hz = s.size[2] / 2.0;
    return tx > -hx && tx < hx && ty > -hy && ty < hy && tz > -hz && tz < hz;
  }
  // cylinder
  const double h2 = s.size[0] / 2.0;
  if (!(tz < h2 && tz > -h2)) return false;
  const double slope = __ddiv_rn(__dsub_rn(s.size[2], s.size[1]), s.size[0]);
  const double radius = __dadd_rn(__dmul_rn(slope, __dadd_rn(tz, h2)), s.size[1]);
  const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(tx, tx), __dmul_rn(ty, ty)));
  return r < radius;
}

__device__ __forceinline__ bool csg_part_inside(const Csg &c, const CsgPart &p, double x, double y,
                                                double z) {
  for (int i = p.count - 1; i >= 0; --i) {
    const CsgShape &s = c.shapes[p.first + i];
    if (csg_shape_inside(s, x, y, z)) return s.op == 0;
  }
  return false;
}

__device__ __forceinline__ void csg_material(const Csg &c, double x, double y, double z,
                                             double &delta, double &beta) {
  delta = 0.0;
  beta = 0.0;
  for (int m = 0; m < c.nmodules; ++m) {
    if (!((c.active >> m) & 1ull)) continue;
    const CsgModule mod = c.modules[m];
    for (int i = mod.count - 1; i >= 0; --i) {
      const CsgPart &p = c.parts[mod.first + i];
      if (csg_part_inside(c, p, x, y, z)) {
        if (p.op == 0) {
          delta = p.delta;
          beta = p.beta;
        }
        return;
      }
    }
  }
}

}  // namespace pxp
