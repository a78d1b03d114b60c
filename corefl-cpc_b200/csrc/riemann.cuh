// Primitive-variable reconstruction and approximate Riemann solvers for
// calorically perfect air, one face at a time, in the reference's arithmetic
// order:
//   first order / MUSCL (kappa = 1/3) / NND2 with minmod
//       (reference src/Reconstruction.cu:5-45, src/Limiter.cuh:14-41; both
//        limiter codes select the same minmod body),
//   energy of the reconstructed states (src/InviscidScheme.cu:212-217),
//   AUSM+ (:397-469), HLLC (:471-599), Lax-Friedrichs (:767-805), Roe with
//   the Harten entropy fix and the half sum of the left/right fluxes
//   (:601-765), entropy-fix width at a node (:269-304).
// State vectors: rho, u, v, w, p and the total energy per volume in slot 5.
// m[q][l]: this direction's metric row at the face's left (q = 0) and right
// (q = 1) nodes; jac[q] the Jacobians there.
#pragma once

#include "cfk_common.cuh"

namespace cfk {

__device__ __forceinline__ double minmod_ref(double a, double b) {
  // gxl::sgn returns +1 for zero
  const int sa = a < 0 ? -1 : 1, sb = b < 0 ? -1 : 1;
  return 0.5 * (sa + sb) * fmin(fabs(a), fabs(b));
}

// v0..v3: one primitive variable at nodes i-1, i, i+1, i+2 -> states at i+1/2
template <int RECON>
__device__ __forceinline__ void reconstruct_var(double v0, double v1, double v2, double v3, double &l, double &r) {
  if (RECON == 2) {
    constexpr double kappa = 1.0 / 3.0;
    const double delta_i = v1 - v0, delta_i1 = v2 - v1, delta_i2 = v3 - v2;
    const double delta_neg_l = minmod_ref(delta_i, delta_i1);
    const double delta_pos_l = minmod_ref(delta_i1, delta_i);
    const double delta_neg_r = minmod_ref(delta_i1, delta_i2);
    const double delta_pos_r = minmod_ref(delta_i2, delta_i1);
    l = v1 + 0.25 * ((1 - kappa) * delta_neg_l + (1 + kappa) * delta_pos_l);
    r = v2 - 0.25 * ((1 - kappa) * delta_pos_r + (1 + kappa) * delta_neg_r);
  } else if (RECON == 3) {
    const double delta_i = v1 - v0, delta_i1 = v2 - v1, delta_i2 = v3 - v2;
    l = v1 + 0.5 * minmod_ref(delta_i, delta_i1);
    r = v2 - 0.5 * minmod_ref(delta_i1, delta_i2);
  } else {
    l = v1;
    r = v2;
  }
}

__device__ __forceinline__ void add_energy_air(double *s) {
  const double e = 0.5 * (s[1] * s[1] + s[2] * s[2] + s[3] * s[3]);
  s[5] = e * s[0] + s[4] / (kGammaAir - 1);
}

__device__ __forceinline__ void ausm_plus_air(const double *pl, const double *pr, const double m[2][3],
                                              const double jac[2], double *fc) {
  const double k1 = 0.5 * (jac[0] * m[0][0] + jac[1] * m[1][0]);
  const double k2 = 0.5 * (jac[0] * m[0][1] + jac[1] * m[1][1]);
  const double k3 = 0.5 * (jac[0] * m[0][2] + jac[1] * m[1][2]);
  const double grad_k_div_jac = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / grad_k_div_jac;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / grad_k_div_jac;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double c = 0.5 * (sqrt(kGammaAir * p_l / rho_l) + sqrt(kGammaAir * p_r / rho_r));
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
  fc[4] = coeff * (pv[5] + pv[4]) / pv[0];
}

__device__ __forceinline__ void hllc_air(const double *pl, const double *pr, const double m[2][3], const double jac[2],
                                         double *fc) {
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double u_tilde = pl[1] * rl_c + pr[1] * rr_c;
  const double v_tilde = pl[2] * rl_c + pr[2] * rr_c;
  const double w_tilde = pl[3] * rl_c + pr[3] * rr_c;
  constexpr double gamma = kGammaAir;
  const double hl = (pl[5] + pl[4]) / pl[0];
  const double hr = (pr[5] + pr[4]) / pr[0];
  const double h_tilde = hl * rl_c + hr * rr_c;
  const double ek_tilde = 0.5 * (u_tilde * u_tilde + v_tilde * v_tilde + w_tilde * w_tilde);
  const double c_tilde = sqrt((gamma - 1) * (h_tilde - ek_tilde));
  const double kx = 0.5 * (m[0][0] + m[1][0]);
  const double ky = 0.5 * (m[0][1] + m[1][1]);
  const double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double U_tilde_bar = (kx * u_tilde + ky * v_tilde + kz * w_tilde) / gradK;
  const double jac_ave = 0.5 * (jac[0] + jac[1]);
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(kGammaAir * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, U_tilde_bar - c_tilde);
  if (sl >= 0) {
    const double rhoUk = pl[0] * Ul;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pl[1] + pl[4] * kx);
    fc[2] = jac_ave * (rhoUk * pl[2] + pl[4] * ky);
    fc[3] = jac_ave * (rhoUk * pl[3] + pl[4] * kz);
    fc[4] = jac_ave * ((pl[5] + pl[4]) * Ul);
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(kGammaAir * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, U_tilde_bar + c_tilde);
  if (sr < 0) {
    const double rhoUk = pr[0] * Ur;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pr[1] + pr[4] * kx);
    fc[2] = jac_ave * (rhoUk * pr[2] + pr[4] * ky);
    fc[3] = jac_ave * (rhoUk * pr[3] + pr[4] * kz);
    fc[4] = jac_ave * ((pr[5] + pr[4]) * Ur);
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
  fc[4] = QCoeff * ps[5] / ps[0] + pCoeff * jac_ave * (ss * pm * sm * gradK - sm * ps[4] * Us);
}

__device__ __forceinline__ void lax_friedrichs_air(const double *pl, const double *pr, const double m[2][3],
                                                   const double jac[2], double *fc) {
  const double kx = 0.5 * (m[0][0] + m[1][0]);
  const double ky = 0.5 * (m[0][1] + m[1][1]);
  const double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const double Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = sqrt(kGammaAir * pl[4] / pl[0]);
  const double cr = sqrt(kGammaAir * pr[4] / pr[0]);
  const double spectral_radius = fmax(fabs(Ukl) + cl * gradK, fabs(Ukr) + cr * gradK);
  const double half_jac_ave = 0.5 * 0.5 * (jac[0] + jac[1]);
  const double rhoUl = pl[0] * Ukl;
  const double rhoUr = pr[0] * Ukr;
  fc[0] = (rhoUl + rhoUr - spectral_radius * (pr[0] - pl[0])) * half_jac_ave;
  fc[1] = (rhoUl * pl[1] + rhoUr * pr[1] + kx * (pl[4] + pr[4]) - spectral_radius * (pr[1] * pr[0] - pl[1] * pl[0])) *
          half_jac_ave;
  fc[2] = (rhoUl * pl[2] + rhoUr * pr[2] + ky * (pl[4] + pr[4]) - spectral_radius * (pr[2] * pr[0] - pl[2] * pl[0])) *
          half_jac_ave;
  fc[3] = (rhoUl * pl[3] + rhoUr * pr[3] + kz * (pl[4] + pr[4]) - spectral_radius * (pr[3] * pr[0] - pl[3] * pl[0])) *
          half_jac_ave;
  fc[4] = ((pl[5] + pl[4]) * Ukl + (pr[5] + pr[4]) * Ukr - spectral_radius * (pr[5] - pl[5])) * half_jac_ave;
}

// Entropy-fix width at a node from its state and all nine metric terms.
__device__ __forceinline__ double entropy_fix_delta_air(double rho, double u, double v, double w, double p,
                                                        const double *mt, int dim, double factor) {
  const double U = fabs(u * mt[0] + v * mt[1] + w * mt[2]);
  const double V = fabs(u * mt[3] + v * mt[4] + w * mt[5]);
  const double W = fabs(u * mt[6] + v * mt[7] + w * mt[8]);
  const double kx = sqrt(mt[0] * mt[0] + mt[1] * mt[1] + mt[2] * mt[2]);
  const double ky = sqrt(mt[3] * mt[3] + mt[4] * mt[4] + mt[5] * mt[5]);
  const double kz = sqrt(mt[6] * mt[6] + mt[7] * mt[7] + mt[8] * mt[8]);
  const double acoustic_speed = sqrt(kGammaAir * p / rho);
  if (dim == 2) return factor * (U + V + acoustic_speed * 0.5 * (kx + ky));
  return factor * (U + V + W + acoustic_speed * (kx + ky + kz) / 3.0);
}

__device__ __forceinline__ void roe_air(const double *pl, const double *pr, const double m[2][3], const double jac[2],
                                        const double delta[2], double *fc) {
  double JacKx = jac[0] * m[0][0], JacKy = jac[0] * m[0][1], JacKz = jac[0] * m[0][2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[5]);
  JacKx = jac[1] * m[1][0];
  JacKy = jac[1] * m[1][1];
  JacKz = jac[1] * m[1][2];
  Uk = pr[1] * JacKx + pr[2] * JacKy + pr[3] * JacKz;
  coeff = Uk * pr[0];
  fc[0] += 0.5 * coeff;
  fc[1] += 0.5 * (coeff * pr[1] + pr[4] * JacKx);
  fc[2] += 0.5 * (coeff * pr[2] + pr[4] * JacKy);
  fc[3] += 0.5 * (coeff * pr[3] + pr[4] * JacKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[5]);

  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv_denominator = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_denominator;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_denominator;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_denominator;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[5] + pl[4]) / pl[0];
  const double hr = (pr[5] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_denominator;
  constexpr double gamma = kGammaAir;
  const double c = sqrt((gamma - 1) * (h - ek));

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
  double dq[5];
  dq[0] = jac_ave * (pr[0] - pl[0]);
#pragma unroll
  for (int l = 1; l < 4; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[5] - pl[5]);

  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Ukk * dq[0]) / c;
  double c3 = dq[0] - c1;
  double LDq[5];
  LDq[0] = 0.5 * (c1 - c2);
  LDq[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  LDq[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  LDq[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  LDq[4] = 0.5 * (c1 + c2);

  double b[5];
  b[0] = -ch[0] * LDq[0];
  b[1] = -ch[1] * LDq[1];
  b[2] = -ch[1] * LDq[2];
  b[3] = -ch[1] * LDq[3];
  b[4] = -ch[2] * LDq[4];

  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Ukk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
}

}  // namespace cfk
