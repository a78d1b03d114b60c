// Scalar WENO5-JS / WENO7-Z reconstructions of the split characteristic
// fluxes at i+1/2.  Same formulas and evaluation order as the reference
// (reference src/WENO.cu:3059-3222); vp[] runs upwind-left to right, vm[]
// likewise, and the result is f+ + f-.
#pragma once

namespace cfk {

__device__ __forceinline__ double weno5_js(const double *vp, const double *vm, double eps) {
  constexpr double one6th{1.0 / 6}, t12{13.0 / 12};
  double v0 = one6th * (2 * vp[2] + 5 * vp[3] - vp[4]);
  double v1 = one6th * (-vp[1] + 5 * vp[2] + 2 * vp[3]);
  double v2 = one6th * (2 * vp[0] - 7 * vp[1] + 11 * vp[2]);
  double d0 = vp[2] + vp[4] - 2 * vp[3], e0 = 3 * vp[2] - 4 * vp[3] + vp[4];
  double d1 = vp[1] + vp[3] - 2 * vp[2], e1 = vp[1] - vp[3];
  double d2 = vp[0] + vp[2] - 2 * vp[1], e2 = vp[0] - 4 * vp[1] + 3 * vp[2];
  double beta0 = t12 * d0 * d0 + 0.25 * e0 * e0;
  double beta1 = t12 * d1 * d1 + 0.25 * e1 * e1;
  double beta2 = t12 * d2 * d2 + 0.25 * e2 * e2;
  double a0 = 0.3 / ((eps + beta0) * (eps + beta0));
  double a1 = 0.6 / ((eps + beta1) * (eps + beta1));
  double a2 = 0.1 / ((eps + beta2) * (eps + beta2));
  const double fPlus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);

  v0 = one6th * (11 * vm[2] - 7 * vm[3] + 2 * vm[4]);
  v1 = one6th * (2 * vm[1] + 5 * vm[2] - vm[3]);
  v2 = one6th * (-vm[0] + 5 * vm[1] + 2 * vm[2]);
  d0 = vm[2] + vm[4] - 2 * vm[3]; e0 = 3 * vm[2] - 4 * vm[3] + vm[4];
  d1 = vm[1] + vm[3] - 2 * vm[2]; e1 = vm[1] - vm[3];
  d2 = vm[0] + vm[2] - 2 * vm[1]; e2 = vm[0] - 4 * vm[1] + 3 * vm[2];
  beta0 = t12 * d0 * d0 + 0.25 * e0 * e0;
  beta1 = t12 * d1 * d1 + 0.25 * e1 * e1;
  beta2 = t12 * d2 * d2 + 0.25 * e2 * e2;
  a0 = 0.1 / ((eps + beta0) * (eps + beta0));
  a1 = 0.6 / ((eps + beta1) * (eps + beta1));
  a2 = 0.3 / ((eps + beta2) * (eps + beta2));
  const double fMinus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
  return fPlus + fMinus;
}

__device__ __forceinline__ double weno7_beta(double s1, double s2, double s3) {
  constexpr double d12{13.0 / 12.0}, d13{1043.0 / 960}, d14{1.0 / 12};
  return s1 * s1 + d12 * s2 * s2 + d13 * s3 * s3 + d14 * s1 * s3;
}

// One side of WENO7-Z: u[0..6] ordered from the far upwind point to the far
// downwind point of the stencil.
__device__ __forceinline__ double weno7_z_side(double u0, double u1, double u2, double u3, double u4, double u5,
                                               double u6, double eps) {
  constexpr double one6th{1.0 / 6};
  constexpr double c0{1.0 / 35}, c1{12.0 / 35}, c2{18.0 / 35}, c3{4.0 / 35};
  double s1 = one6th * (-2 * u0 + 9 * u1 - 18 * u2 + 11 * u3);
  double s2 = -u0 + 4 * u1 - 5 * u2 + 2 * u3;
  double s3 = -u0 + 3 * u1 - 3 * u2 + u3;
  const double beta0 = weno7_beta(s1, s2, s3);
  s1 = one6th * (u1 - 6 * u2 + 3 * u3 + 2 * u4);
  s2 = u2 - 2 * u3 + u4;
  s3 = -u1 + 3 * u2 - 3 * u3 + u4;
  const double beta1 = weno7_beta(s1, s2, s3);
  // stencil 2 shares the second difference of stencil 1 (reference src/WENO.cu:3137-3139)
  s1 = one6th * (-2 * u2 - 3 * u3 + 6 * u4 - u5);
  s3 = -u2 + 3 * u3 - 3 * u4 + u5;
  const double beta2 = weno7_beta(s1, s2, s3);
  s1 = one6th * (-11 * u3 + 18 * u4 - 9 * u5 + 2 * u6);
  s2 = 2 * u3 - 5 * u4 + 4 * u5 - u6;
  s3 = -u3 + 3 * u4 - 3 * u5 + u6;
  const double beta3 = weno7_beta(s1, s2, s3);
  double tau = beta0 + 3 * beta1 - 3 * beta2 - beta3;
  tau *= tau;
  const double a0 = c0 + c0 * tau / ((eps + beta0) * (eps + beta0));
  const double a1 = c1 + c1 * tau / ((eps + beta1) * (eps + beta1));
  const double a2 = c2 + c2 * tau / ((eps + beta2) * (eps + beta2));
  const double a3 = c3 + c3 * tau / ((eps + beta3) * (eps + beta3));
  const double v0 = -3 * u0 + 13 * u1 - 23 * u2 + 25 * u3;
  const double v1 = u1 - 5 * u2 + 13 * u3 + 3 * u4;
  const double v2 = -u2 + 7 * u3 + 7 * u4 - u5;
  const double v3 = 3 * u3 + 13 * u4 - 5 * u5 + u6;
  constexpr double one12th{1.0 / 12};
  return one12th * (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
}

__device__ __forceinline__ double weno7_z(const double *vp, const double *vm, double eps) {
  const double fPlus = weno7_z_side(vp[0], vp[1], vp[2], vp[3], vp[4], vp[5], vp[6], eps);
  const double fMinus = weno7_z_side(vm[6], vm[5], vm[4], vm[3], vm[2], vm[1], vm[0], eps);
  return fPlus + fMinus;
}

}  // namespace cfk
