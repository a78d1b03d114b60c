// Primitive-variable approximate Riemann solvers for a thermally perfect
// mixture of NS species (NASA-7 thermo), one face at a time, in the
// reference's arithmetic order (reference src/InviscidScheme.cu):
//   side energies and gamma of the reconstructed states (:184-213),
//   AUSM+ (:397-469), HLLC with the Roe-averaged mixture sound speed
//   (:471-599), Roe with the species terms of the eigen-decomposition and the
//   half sum of the left/right fluxes (:601-765).
// The reference has no Lax-Friedrichs flux for mixtures (:767-770).
// States: rho, u, v, w, p, Y_1..Y_NS, then E per volume (slot NV) and gamma
// (slot NV + 1), NV = 5 + NS.
#pragma once

#include "chem_fast.cuh"
#include "cfk_common.cuh"
#include "thermo.cuh"

namespace cfk {

// E and gamma of a reconstructed state, from its T = p / (rho R_u sum Y/W).
template <int NS>
__device__ __forceinline__ void add_energy_mix(const Thermo *th, double *s) {
  constexpr int NV = 5 + NS;
  double e = 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]);
  double mw_inv = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) mw_inv += s[5 + l] * th->imw[l];
  const double t = s[4] / (s[0] * kRu * mw_inv);
  double h[NS], cp_i[NS];
  enthalpy_cp_ns<NS>(th, t, h, cp_i);
  double cp = 0, cv = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    cp += cp_i[l] * s[l + 5];
    cv += s[l + 5] * (cp_i[l] - th->gas_const[l]);
    e += h[l] * s[l + 5];
  }
  s[NV] = s[0] * e - s[4];
  s[NV + 1] = cp / cv;
}

template <int NS>
__device__ __forceinline__ void ausm_plus_mix(const double *pl, const double *pr, const double m[2][3],
                                              const double jac[2], double *fc) {
  constexpr int NV = 5 + NS;
  const double k1 = 0.5 * (jac[0] * m[0][0] + jac[1] * m[1][0]);
  const double k2 = 0.5 * (jac[0] * m[0][1] + jac[1] * m[1][1]);
  const double k3 = 0.5 * (jac[0] * m[0][2] + jac[1] * m[1][2]);
  const double grad_k_div_jac = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / grad_k_div_jac;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / grad_k_div_jac;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double c = 0.5 * (sqrt(pl[NV + 1] * p_l / rho_l) + sqrt(pr[NV + 1] * p_r / rho_r));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  constexpr double alpha = 3 / 16.0;
  if (fabs(mach_l) > 1) {
    mlp = 0.5 * (mach_l + fabs(mach_l));
    plp = mlp / mach_l;
  } else {
    const double a = (mach_l + 1) * (mach_l + 1) * 0.25;
    const double b = (mach_l * mach_l - 1) * (mach_l * mach_l - 1);
    mlp = a + 0.125 * b;
    plp = a * (2 - mach_l) + alpha * mach_l * b;
  }
  if (fabs(mach_r) > 1) {
    mrn = 0.5 * (mach_r - fabs(mach_r));
    prn = mrn / mach_r;
  } else {
    const double a = (mach_r - 1) * (mach_r - 1) * 0.25;
    const double b = (mach_r * mach_r - 1) * (mach_r * mach_r - 1);
    mrn = -a - 0.125 * b;
    prn = a * (2 + mach_r) - alpha * mach_r * b;
  }
  const double p_coeff = plp * p_l + prn * p_r;
  const double m_half = mlp + mrn;
  const double mach_pos = 0.5 * (m_half + fabs(m_half));
  const double mach_neg = 0.5 * (m_half - fabs(m_half));
  const double mass_flux_half = c * (rho_l * mach_pos + rho_r * mach_neg);
  const double coeff = mass_flux_half * grad_k_div_jac;
  const double *pv = mass_flux_half >= 0 ? pl : pr;
  fc[0] = coeff;
  fc[1] = coeff * pv[1] + p_coeff * k1;
  fc[2] = coeff * pv[2] + p_coeff * k2;
  fc[3] = coeff * pv[3] + p_coeff * k3;
  fc[4] = coeff * (pv[NV] + pv[4]) / pv[0];
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] = coeff * pv[l];
}

template <int NS>
__device__ __forceinline__ void hllc_mix(const Thermo *th, const double *pl, const double *pr, const double m[2][3],
                                         const double jac[2], double *fc) {
  constexpr int NV = 5 + NS;
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double u_tilde = pl[1] * rl_c + pr[1] * rr_c;
  const double v_tilde = pl[2] * rl_c + pr[2] * rr_c;
  const double w_tilde = pl[3] * rl_c + pr[3] * rr_c;
  double c_tilde;
  {
    double mw_inv = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) mw_inv += (rl_c * pl[l + 5] + rr_c * pr[l + 5]) * th->imw[l];
    const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
    const double t = (rl_c * tl + rr_c * tr) / (kRu * mw_inv);
    double cp_i[NS], h_i[NS];
    enthalpy_cp_ns<NS>(th, t, h_i, cp_i);
    double cv = 0, cp = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double svm = rl_c * pl[l + 5] + rr_c * pr[l + 5];
      cp += cp_i[l] * svm;
      cv += svm * (cp_i[l] - th->gas_const[l]);
    }
    const double gamma = cp / cv;
    c_tilde = sqrt(gamma * kRu * mw_inv * t);
  }
  const double kx = 0.5 * (m[0][0] + m[1][0]);
  const double ky = 0.5 * (m[0][1] + m[1][1]);
  const double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double U_tilde_bar = (kx * u_tilde + ky * v_tilde + kz * w_tilde) / gradK;
  const double jac_ave = 0.5 * (jac[0] + jac[1]);
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(pl[NV + 1] * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, U_tilde_bar - c_tilde);
  if (sl >= 0) {
    const double rhoUk = pl[0] * Ul;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pl[1] + pl[4] * kx);
    fc[2] = jac_ave * (rhoUk * pl[2] + pl[4] * ky);
    fc[3] = jac_ave * (rhoUk * pl[3] + pl[4] * kz);
    fc[4] = jac_ave * ((pl[NV] + pl[4]) * Ul);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] = jac_ave * rhoUk * pl[l];
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(pr[NV + 1] * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, U_tilde_bar + c_tilde);
  if (sr < 0) {
    const double rhoUk = pr[0] * Ur;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pr[1] + pr[4] * kx);
    fc[2] = jac_ave * (rhoUk * pr[2] + pr[4] * ky);
    fc[3] = jac_ave * (rhoUk * pr[3] + pr[4] * kz);
    fc[4] = jac_ave * ((pr[NV] + pr[4]) * Ur);
#pragma unroll
    for (int l = 5; l < NV; ++l) fc[l] = jac_ave * rhoUk * pr[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  const bool left = sm >= 0;
  const double *ps = left ? pl : pr;
  const double ss = left ? sl : sr, Us = left ? Ul : Ur;
  const double pCoeff = 1.0 / (ss - sm);
  const double QCoeff = jac_ave * pCoeff * sm * (ss * gradK - Us) * ps[0];
  fc[0] = QCoeff;
  const double dP = (ss * pm - sm * ps[4]) * pCoeff * jac_ave;
  fc[1] = QCoeff * ps[1] + dP * kx;
  fc[2] = QCoeff * ps[2] + dP * ky;
  fc[3] = QCoeff * ps[3] + dP * kz;
  fc[4] = QCoeff * ps[NV] / ps[0] + pCoeff * jac_ave * (ss * pm * sm * gradK - sm * ps[4] * Us);
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] = QCoeff * ps[l];
}

// Entropy-fix width at a node; the acoustic speed comes from the property array.
__device__ __forceinline__ double entropy_fix_delta_mix(double u, double v, double w, double acoustic_speed,
                                                        const double *mt, int dim, double factor) {
  const double U = fabs(u * mt[0] + v * mt[1] + w * mt[2]);
  const double V = fabs(u * mt[3] + v * mt[4] + w * mt[5]);
  const double W = fabs(u * mt[6] + v * mt[7] + w * mt[8]);
  const double kx = sqrt(mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2]);
  const double ky = sqrt(mt[3] * mt[3] + mt[4] * mt[4] + mt[5] * mt[5]);
  const double kz = sqrt(mt[6] * mt[6] + mt[7] * mt[7] + mt[8] * mt[8]);
  if (dim == 2) return factor * (U + V + acoustic_speed * 0.5 * (kx + ky));
  return factor * (U + V + W + acoustic_speed * (kx + ky + kz) / 3.0);
}

template <int NS>
__device__ __forceinline__ void roe_mix(const Thermo *th, const double *pl, const double *pr, const double m[2][3],
                                        const double jac[2], const double delta[2], double *fc) {
  constexpr int NV = 5 + NS;
  double JacKx = jac[0] * m[0][0], JacKy = jac[0] * m[0][1], JacKz = jac[0] * m[0][2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[NV]);
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] = 0.5 * coeff * pl[l];
  JacKx = jac[1] * m[1][0];
  JacKy = jac[1] * m[1][1];
  JacKz = jac[1] * m[1][2];
  Uk = pr[1] * JacKx + pr[2] * JacKy + pr[3] * JacKz;
  coeff = Uk * pr[0];
  fc[0] += 0.5 * coeff;
  fc[1] += 0.5 * (coeff * pr[1] + pr[4] * JacKx);
  fc[2] += 0.5 * (coeff * pr[2] + pr[4] * JacKy);
  fc[3] += 0.5 * (coeff * pr[3] + pr[4] * JacKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[NV]);
#pragma unroll
  for (int l = 5; l < NV; ++l) fc[l] += 0.5 * coeff * pr[l];

  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv_denominator = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_denominator;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_denominator;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_denominator;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[NV] + pl[4]) / pl[0];
  const double hr = (pr[NV] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_denominator;
  double svm[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_denominator;
  double h_i[NS], mw_inv = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) mw_inv += svm[l] * th->imw[l];
  const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
  const double t = (dl * tl + dr * tr) * inv_denominator / (kRu * mw_inv);
  double gamma;
  {
    double cp_i[NS];
    enthalpy_cp_ns<NS>(th, t, h_i, cp_i);
    double cv = 0, cp = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      cp += cp_i[l] * svm[l];
      cv += svm[l] * (cp_i[l] - th->gas_const[l]);
    }
    gamma = cp / cv;
  }
  const double c = sqrt(gamma * kRu * mw_inv * t);
  const double mw = 1.0 / mw_inv;

  double kx = 0.5 * (m[0][0] + m[1][0]);
  double ky = 0.5 * (m[0][1] + m[1][1]);
  double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  double Ukk = kx * u + ky * v + kz * w;
  double ch[3] = {Ukk - gradK * c, Ukk, Ukk + gradK * c};
  const double entropy_fix_delta_ave = 0.5 * (delta[0] + delta[1]);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double cc = fabs(ch[q]);
    if (cc < entropy_fix_delta_ave) cc = 0.5 * (cc * cc / entropy_fix_delta_ave + entropy_fix_delta_ave);
    ch[q] = cc;
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Ukk /= gradK;

  const double jac_ave = 0.5 * (jac[0] + jac[1]);
  double dq[NV];
  dq[0] = jac_ave * (pr[0] - pl[0]);
#pragma unroll
  for (int l = 1; l < NV; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[NV] - pl[NV]);

  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Ukk * dq[0]) / c;
#pragma unroll
  for (int l = 0; l < NS; ++l) c1 += (mw * th->imw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double LDq[NV];
  LDq[0] = 0.5 * (c1 - c2);
  LDq[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  LDq[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  LDq[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  LDq[4] = 0.5 * (c1 + c2);
#pragma unroll
  for (int l = 0; l < NS; ++l) LDq[l + 5] = dq[l + 5] - svm[l] * dq[0];

  double b[NV];
  b[0] = -ch[0] * LDq[0];
#pragma unroll
  for (int l = 1; l < NV; ++l) b[l] = -ch[1] * LDq[l];
  b[4] = -ch[2] * LDq[4];

  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) c3 += (h_i[l] - mw * th->imw[l] * c * c / (gamma - 1)) * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Ukk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
#pragma unroll
  for (int l = 0; l < NS; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

}  // namespace cfk
