// Scalar WENO5-JS / WENO7-Z reconstructions of the split characteristic
// fluxes at i+1/2 (reference src/WENO.cu:3059-3222): same substencils,
// smoothness indicators and weights; vp[] and vm[] run left to right and the
// result is f+ + f-.  The weight normalisation is rearranged so that a face
// costs one division per side pair instead of ten (WENO7) or six (WENO5).
#pragma once

namespace cfk {

// WENO5-JS, f+ + f-.  The weights a_k = d_k / (eps + beta_k)^2 enter only
// through sum(a_k v_k) / sum(a_k); both sums are multiplied through by the
// product of the three denominators, so one division per side remains.  The
// sides are not merged into one division: in flat regions the products are
// O(eps^4) and their cross product would underflow.  Same reconstruction as
// the reference; the rounding differs at the ulp level.
__device__ __forceinline__ void weno5_side(double u0, double u1, double u2, double u3, double u4, double eps,
                                           double d0, double d1, double d2, double &num, double &den) {
  constexpr double one6th{1.0 / 6}, t12{13.0 / 12};
  const double v0 = one6th * (2 * u2 + 5 * u3 - u4);
  const double v1 = one6th * (-u1 + 5 * u2 + 2 * u3);
  const double v2 = one6th * (2 * u0 - 7 * u1 + 11 * u2);
  const double g0 = u2 + u4 - 2 * u3, h0 = 3 * u2 - 4 * u3 + u4;
  const double g1 = u1 + u3 - 2 * u2, h1 = u1 - u3;
  const double g2 = u0 + u2 - 2 * u1, h2 = u0 - 4 * u1 + 3 * u2;
  const double b0 = eps + (t12 * g0 * g0 + 0.25 * h0 * h0);
  const double b1 = eps + (t12 * g1 * g1 + 0.25 * h1 * h1);
  const double b2 = eps + (t12 * g2 * g2 + 0.25 * h2 * h2);
  const double D0 = b0 * b0, D1 = b1 * b1, D2 = b2 * b2;
  const double a0 = d0 * (D1 * D2), a1 = d1 * (D0 * D2), a2 = d2 * (D0 * D1);
  num = a0 * v0 + a1 * v1 + a2 * v2;
  den = a0 + a1 + a2;
}

__device__ __forceinline__ double weno5_js(const double *vp, const double *vm, double eps) {
  double np, dp, nm, dm;
  weno5_side(vp[0], vp[1], vp[2], vp[3], vp[4], eps, 0.3, 0.6, 0.1, np, dp);
  // mirrored: minus-side substencil k is plus-side substencil 2-k, same linear weights
  weno5_side(vm[4], vm[3], vm[2], vm[1], vm[0], eps, 0.3, 0.6, 0.1, nm, dm);
  return np / dp + nm / dm;
}

__device__ __forceinline__ double weno7_beta(double s1, double s2, double s3) {
  constexpr double d12{13.0 / 12.0}, d13{1043.0 / 960}, d14{1.0 / 12};
  return s1 * s1 + d12 * s2 * s2 + d13 * s3 * s3 + d14 * s1 * s3;
}

// One side of WENO7-Z: u[0..6] ordered from the far upwind point to the far
// downwind point of the stencil.  Returns numerator and denominator of
// sum(a_k v_k) / sum(a_k) with a_k = c_k (1 + tau / (eps + beta_k)^2); the
// four reciprocals are formed from two divisions, 1/(D0 D1) and 1/(D2 D3).
__device__ __forceinline__ void weno7_z_side(double u0, double u1, double u2, double u3, double u4, double u5,
                                             double u6, double eps, double &num, double &den) {
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
  const double e0 = eps + beta0, e1 = eps + beta1, e2 = eps + beta2, e3 = eps + beta3;
  const double D0 = e0 * e0, D1 = e1 * e1, D2 = e2 * e2, D3 = e3 * e3;
  const double r01 = 1.0 / (D0 * D1), r23 = 1.0 / (D2 * D3);
  const double a0 = c0 + c0 * tau * (D1 * r01);
  const double a1 = c1 + c1 * tau * (D0 * r01);
  const double a2 = c2 + c2 * tau * (D3 * r23);
  const double a3 = c3 + c3 * tau * (D2 * r23);
  const double v0 = -3 * u0 + 13 * u1 - 23 * u2 + 25 * u3;
  const double v1 = u1 - 5 * u2 + 13 * u3 + 3 * u4;
  const double v2 = -u2 + 7 * u3 + 7 * u4 - u5;
  const double v3 = 3 * u3 + 13 * u4 - 5 * u5 + u6;
  num = a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3;
  den = a0 + a1 + a2 + a3;
}

// f+ + f-, one division shared by the two sides (each sum(a_k) >= 1/35, so
// the product of the two denominators cannot underflow).
__device__ __forceinline__ double weno7_z(const double *vp, const double *vm, double eps) {
  double np, dp, nm, dm;
  weno7_z_side(vp[0], vp[1], vp[2], vp[3], vp[4], vp[5], vp[6], eps, np, dp);
  weno7_z_side(vm[6], vm[5], vm[4], vm[3], vm[2], vm[1], vm[0], eps, nm, dm);
  constexpr double one12th{1.0 / 12};
  return one12th * ((np * dm + nm * dp) / (dp * dm));
}

// Linear branches of WENO5 / WENO7 used by the hybrid scheme away from
// shocks (reference src/WENO.cu:3100-3113 and 3204-3221): the substencil
// values combined with the optimal weights, which collapse to the 5- and
// 7-point upwind-biased stencils (UD5: (2, -13, 47, 27, -3) / 60;
// UD7: (-3, 25, -101, 319, 214, -38, 4) / 420).  The minus side is the plus
// side read right to left.
__device__ __forceinline__ double ud5_side(double u0, double u1, double u2, double u3, double u4) {
  constexpr double r60{1.0 / 60};
  return r60 * (2 * u0 - 13 * u1 + 47 * u2 + 27 * u3 - 3 * u4);
}

__device__ __forceinline__ double weno5_linear(const double *vp, const double *vm) {
  return ud5_side(vp[0], vp[1], vp[2], vp[3], vp[4]) + ud5_side(vm[4], vm[3], vm[2], vm[1], vm[0]);
}

__device__ __forceinline__ double ud7_side(double u0, double u1, double u2, double u3, double u4, double u5,
                                           double u6) {
  constexpr double r420{1.0 / 420};
  return r420 * (-3 * u0 + 25 * u1 - 101 * u2 + 319 * u3 + 214 * u4 - 38 * u5 + 4 * u6);
}

__device__ __forceinline__ double weno7_linear(const double *vp, const double *vm) {
  return ud7_side(vp[0], vp[1], vp[2], vp[3], vp[4], vp[5], vp[6]) +
         ud7_side(vm[6], vm[5], vm[4], vm[3], vm[2], vm[1], vm[0]);
}

// Hybrid switch of the WENO sweeps (reference src/WENO.cu:839-849, 1580-1590
// and the z sweep): the face between node idf and idf + sd takes the
// nonlinear weights when the sensor of any node idf + ii*sd, ii in
// [-g+1, g], exceeds the threshold.  sensor == nullptr: WENO everywhere.
__device__ __forceinline__ bool face_shocked(const double *sensor, int64_t idf, int64_t sd, int g,
                                             double threshold) {
  if (sensor == nullptr) return true;
  for (int ii = -g + 1; ii <= g; ++ii)
    if (__ldg(sensor + idf + ii * sd) > threshold) return true;
  return false;
}

}  // namespace cfk
