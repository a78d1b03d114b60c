/*
 * CPU oracle: primitive-variable reconstruction (first order, MUSCL, NND2
 * with the minmod limiter) and the Lax-Friedrichs, Roe (Harten entropy fix),
 * AUSM+ and HLLC Riemann solvers, for calorically perfect air and for
 * thermally perfect mixtures (species mass fractions reconstructed with the
 * flow variables, side energies and gamma from NASA-7 thermo; the reference
 * has no Lax-Friedrichs flux for mixtures).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates, in the reference's arithmetic order:
 *   compute_inviscid_flux dispatch       src/InviscidScheme.cu:12-26
 *   compute_convective_term_pv(_1D)      src/InviscidScheme.cu:28-169
 *   reconstruction                       src/InviscidScheme.cu:171-219
 *   Roe_compute_inviscid_flux(_1D)       src/InviscidScheme.cu:221-267, 306-395
 *   compute_entropy_fix_delta            src/InviscidScheme.cu:269-304
 *   riemannSolver_ausmPlus               src/InviscidScheme.cu:397-469
 *   riemannSolver_hllc                   src/InviscidScheme.cu:471-599
 *   compute_half_sum_left_right_flux     src/InviscidScheme.cu:601-633
 *   riemannSolver_Roe                    src/InviscidScheme.cu:635-765
 *   riemannSolver_laxFriedrich (air)     src/InviscidScheme.cu:767-805
 *   first_order / MUSCL / NND2           src/Reconstruction.cu:5-45
 *   minmod limiter                       src/Limiter.cuh:14-41 (both limiter
 *                                        codes select the same minmod body)
 * Face fluxes go to fFlux/gFlux/hFlux at the index of the face's left node
 * (faces -1 .. m-1), then dq(i) -= F(i) - F(i-1); the k sweep runs only when
 * mz > 1, as in the reference.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define GAMMA_AIR 1.4
#define R_U 8314.462618
/* reconstructed state: rho, u, v, w, p, Y_1..Y_ns, then E (slot nv) and gamma (slot nv + 1) */
#define NRMAX (ORC_MAX_SPEC + 7)

static inline long psz(const orc_zone *z, int g) {
  return (long)(z->mx + 2 * g) * (z->my + 2 * g) * (z->mz + 2 * g);
}
static inline long pidx(const orc_zone *z, int g, int i, int j, int k) {
  return ((long)(k + g) * (z->my + 2 * g) + (j + g)) * (z->mx + 2 * g) + (i + g);
}
static inline long pstride(const orc_zone *z, int g, int dir) {
  if (dir == 0) return 1;
  if (dir == 1) return z->mx + 2 * g;
  return (long)(z->mx + 2 * g) * (z->my + 2 * g);
}

/* gxl::sgn (src/gxl_lib/Math.hpp:10-12): -1 for negative, +1 otherwise */
static inline int sgn(double a) { return a < 0 ? -1 : 1; }
static inline double minmod(double a, double b) { return 0.5 * (sgn(a) + sgn(b)) * fmin(fabs(a), fabs(b)); }

/* pv[4][*]: the nv primitive variables at nodes i-1, i, i+1, i+2; out: left
 * and right states at i+1/2 with the total energy per volume in slot nv and,
 * for mixtures, gamma in slot nv + 1 (src/InviscidScheme.cu:171-219). */
static void reconstruct(const double pv[4][NRMAX], int nv, int recon, const orc_mech *mech, double *pl,
                        double *pr) {
  for (int l = 0; l < nv; ++l) {
    if (recon == 2) {
      const double kappa = 1.0 / 3.0;
      const double delta_i = pv[1][l] - pv[0][l];
      const double delta_i1 = pv[2][l] - pv[1][l];
      const double delta_i2 = pv[3][l] - pv[2][l];
      const double delta_neg_l = minmod(delta_i, delta_i1);
      const double delta_pos_l = minmod(delta_i1, delta_i);
      const double delta_neg_r = minmod(delta_i1, delta_i2);
      const double delta_pos_r = minmod(delta_i2, delta_i1);
      pl[l] = pv[1][l] + 0.25 * ((1 - kappa) * delta_neg_l + (1 + kappa) * delta_pos_l);
      pr[l] = pv[2][l] - 0.25 * ((1 - kappa) * delta_pos_r + (1 + kappa) * delta_neg_r);
    } else if (recon == 3) {
      const double delta_i = pv[1][l] - pv[0][l];
      const double delta_i1 = pv[2][l] - pv[1][l];
      const double delta_i2 = pv[3][l] - pv[2][l];
      pl[l] = pv[1][l] + 0.5 * minmod(delta_i, delta_i1);
      pr[l] = pv[2][l] - 0.5 * minmod(delta_i1, delta_i2);
    } else {
      pl[l] = pv[1][l];
      pr[l] = pv[2][l];
    }
  }
  if (mech) {
    const int ns = mech->n_spec;
    double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    double mw_inv_l = 0, mw_inv_r = 0;
    for (int l = 0; l < ns; ++l) {
      mw_inv_l += pl[5 + l] * mech->imw[l];
      mw_inv_r += pr[5 + l] * mech->imw[l];
    }
    const double t_l = pl[4] / (pl[0] * R_U * mw_inv_l);
    const double t_r = pr[4] / (pr[0] * R_U * mw_inv_r);
    double hl[ORC_MAX_SPEC], hr[ORC_MAX_SPEC], cpl_i[ORC_MAX_SPEC], cpr_i[ORC_MAX_SPEC];
    orc_enthalpy_and_cp(mech, t_l, hl, cpl_i);
    orc_enthalpy_and_cp(mech, t_r, hr, cpr_i);
    double cpl = 0, cpr = 0, cvl = 0, cvr = 0;
    for (int l = 0; l < ns; ++l) {
      cpl += cpl_i[l] * pl[l + 5];
      cpr += cpr_i[l] * pr[l + 5];
      cvl += pl[l + 5] * (cpl_i[l] - mech->gas_const[l]);
      cvr += pr[l + 5] * (cpr_i[l] - mech->gas_const[l]);
      el += hl[l] * pl[l + 5];
      er += hr[l] * pr[l + 5];
    }
    pl[nv] = pl[0] * el - pl[4];
    pr[nv] = pr[0] * er - pr[4];
    pl[nv + 1] = cpl / cvl;
    pr[nv + 1] = cpr / cvr;
  } else {
    const double el = 0.5 * (pl[1] * pl[1] + pl[2] * pl[2] + pl[3] * pl[3]);
    const double er = 0.5 * (pr[1] * pr[1] + pr[2] * pr[2] + pr[3] * pr[3]);
    pl[nv] = el * pl[0] + pl[4] / (GAMMA_AIR - 1);
    pr[nv] = er * pr[0] + pr[4] / (GAMMA_AIR - 1);
  }
}

/* m[2][3]: this direction's metric row at nodes i, i+1; jac[2]. */
static void ausm_plus(const double *pl, const double *pr, int nv, const orc_mech *mech, const double m[2][3],
                      const double jac[2], double *fc) {
  const double k1 = 0.5 * (jac[0] * m[0][0] + jac[1] * m[1][0]);
  const double k2 = 0.5 * (jac[0] * m[0][1] + jac[1] * m[1][1]);
  const double k3 = 0.5 * (jac[0] * m[0][2] + jac[1] * m[1][2]);
  const double grad_k_div_jac = sqrt(k1 * k1 + k2 * k2 + k3 * k3);
  const double ul = (k1 * pl[1] + k2 * pl[2] + k3 * pl[3]) / grad_k_div_jac;
  const double ur = (k1 * pr[1] + k2 * pr[2] + k3 * pr[3]) / grad_k_div_jac;
  const double p_l = pl[4], p_r = pr[4], rho_l = pl[0], rho_r = pr[0];
  const double gam_l = mech ? pl[nv + 1] : GAMMA_AIR, gam_r = mech ? pr[nv + 1] : GAMMA_AIR;
  const double c = 0.5 * (sqrt(gam_l * p_l / rho_l) + sqrt(gam_r * p_r / rho_r));
  const double mach_l = ul / c, mach_r = ur / c;
  double mlp, mrn, plp, prn;
  const double alpha = 3 / 16.0;
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
  fc[4] = coeff * (pv[nv] + pv[4]) / pv[0];
  for (int l = 5; l < nv; ++l) fc[l] = coeff * pv[l];
}

static void hllc(const double *pl, const double *pr, int nv, const orc_mech *mech, const double m[2][3],
                 const double jac[2], double *fc) {
  const double rl_c = sqrt(pl[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double rr_c = sqrt(pr[0]) / (sqrt(pl[0]) + sqrt(pr[0]));
  const double u_tilde = pl[1] * rl_c + pr[1] * rr_c;
  const double v_tilde = pl[2] * rl_c + pr[2] * rr_c;
  const double w_tilde = pl[3] * rl_c + pr[3] * rr_c;
  double gamma = GAMMA_AIR, c_tilde;
  if (!mech) {
    const double hl = (pl[nv] + pl[4]) / pl[0];
    const double hr = (pr[nv] + pr[4]) / pr[0];
    const double h_tilde = hl * rl_c + hr * rr_c;
    const double ek_tilde = 0.5 * (u_tilde * u_tilde + v_tilde * v_tilde + w_tilde * w_tilde);
    c_tilde = sqrt((gamma - 1) * (h_tilde - ek_tilde));
  } else {
    const int ns = mech->n_spec;
    double svm[ORC_MAX_SPEC];
    for (int l = 0; l < nv - 5; ++l) svm[l] = rl_c * pl[l + 5] + rr_c * pr[l + 5];
    double mw_inv = 0;
    for (int l = 0; l < ns; ++l) mw_inv += svm[l] * mech->imw[l];
    const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
    const double t = (rl_c * tl + rr_c * tr) / (R_U * mw_inv);
    double cp_i[ORC_MAX_SPEC], h_i[ORC_MAX_SPEC];
    orc_enthalpy_and_cp(mech, t, h_i, cp_i);
    double cv = 0, cp = 0;
    for (int l = 0; l < ns; ++l) {
      cp += cp_i[l] * svm[l];
      cv += svm[l] * (cp_i[l] - mech->gas_const[l]);
    }
    gamma = cp / cv;
    c_tilde = sqrt(gamma * R_U * mw_inv * t);
  }
  const double kx = 0.5 * (m[0][0] + m[1][0]);
  const double ky = 0.5 * (m[0][1] + m[1][1]);
  const double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double U_tilde_bar = (kx * u_tilde + ky * v_tilde + kz * w_tilde) / gradK;
  const double jac_ave = 0.5 * (jac[0] + jac[1]);
  const double gamma_l = mech ? pl[nv + 1] : GAMMA_AIR, gamma_r = mech ? pr[nv + 1] : GAMMA_AIR;
  const double Ul = kx * pl[1] + ky * pl[2] + kz * pl[3];
  const double cl = sqrt(gamma_l * pl[4] / pl[0]);
  const double sl = fmin(Ul / gradK - cl, U_tilde_bar - c_tilde);
  if (sl >= 0) {
    const double rhoUk = pl[0] * Ul;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pl[1] + pl[4] * kx);
    fc[2] = jac_ave * (rhoUk * pl[2] + pl[4] * ky);
    fc[3] = jac_ave * (rhoUk * pl[3] + pl[4] * kz);
    fc[4] = jac_ave * ((pl[nv] + pl[4]) * Ul);
    for (int l = 5; l < nv; ++l) fc[l] = jac_ave * rhoUk * pl[l];
    return;
  }
  const double Ur = kx * pr[1] + ky * pr[2] + kz * pr[3];
  const double cr = sqrt(gamma_r * pr[4] / pr[0]);
  const double sr = fmax(Ur / gradK + cr, U_tilde_bar + c_tilde);
  if (sr < 0) {
    const double rhoUk = pr[0] * Ur;
    fc[0] = jac_ave * rhoUk;
    fc[1] = jac_ave * (rhoUk * pr[1] + pr[4] * kx);
    fc[2] = jac_ave * (rhoUk * pr[2] + pr[4] * ky);
    fc[3] = jac_ave * (rhoUk * pr[3] + pr[4] * kz);
    fc[4] = jac_ave * ((pr[nv] + pr[4]) * Ur);
    for (int l = 5; l < nv; ++l) fc[l] = jac_ave * rhoUk * pr[l];
    return;
  }
  const double sm = ((pr[0] * Ur * (sr - Ur / gradK) - pl[0] * Ul * (sl - Ul / gradK)) / gradK + pl[4] - pr[4]) /
                    (pr[0] * (sr - Ur / gradK) - pl[0] * (sl - Ul / gradK));
  const double pm = pl[0] * (sl - Ul / gradK) * (sm - Ul / gradK) + pl[4];
  if (sm >= 0) {
    const double pCoeff = 1.0 / (sl - sm);
    const double QlCoeff = jac_ave * pCoeff * sm * (sl * gradK - Ul) * pl[0];
    fc[0] = QlCoeff;
    const double dP = (sl * pm - sm * pl[4]) * pCoeff * jac_ave;
    fc[1] = QlCoeff * pl[1] + dP * kx;
    fc[2] = QlCoeff * pl[2] + dP * ky;
    fc[3] = QlCoeff * pl[3] + dP * kz;
    fc[4] = QlCoeff * pl[nv] / pl[0] + pCoeff * jac_ave * (sl * pm * sm * gradK - sm * pl[4] * Ul);
    for (int l = 5; l < nv; ++l) fc[l] = QlCoeff * pl[l];
  } else {
    const double pCoeff = 1.0 / (sr - sm);
    const double QrCoeff = jac_ave * pCoeff * sm * (sr * gradK - Ur) * pr[0];
    fc[0] = QrCoeff;
    const double dP = (sr * pm - sm * pr[4]) * pCoeff * jac_ave;
    fc[1] = QrCoeff * pr[1] + dP * kx;
    fc[2] = QrCoeff * pr[2] + dP * ky;
    fc[3] = QrCoeff * pr[3] + dP * kz;
    fc[4] = QrCoeff * pr[nv] / pr[0] + pCoeff * jac_ave * (sr * pm * sm * gradK - sm * pr[4] * Ur);
    for (int l = 5; l < nv; ++l) fc[l] = QrCoeff * pr[l];
  }
}

/* air only: the reference prints a message and leaves the flux zero for mixtures */
static void lax_friedrichs(const double *pl, const double *pr, const double m[2][3], const double jac[2],
                           double *fc) {
  const double kx = 0.5 * (m[0][0] + m[1][0]);
  const double ky = 0.5 * (m[0][1] + m[1][1]);
  const double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  const double Ukl = pl[1] * kx + pl[2] * ky + pl[3] * kz;
  const double Ukr = pr[1] * kx + pr[2] * ky + pr[3] * kz;
  const double cl = sqrt(GAMMA_AIR * pl[4] / pl[0]);
  const double cr = sqrt(GAMMA_AIR * pr[4] / pr[0]);
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

/* Entropy-fix width at one node (compute_entropy_fix_delta); mixtures take
 * the node's acoustic speed from the property array. */
static double entropy_fix_delta(const orc_zone *z, const orc_param *p, long id) {
  const long sz = psz(z, z->ngg);
  const double *bv = z->bv, *mt = z->metric;
  const double u = bv[id + sz], v = bv[id + 2 * sz], w = bv[id + 3 * sz];
  const double U = fabs(u * mt[id] + v * mt[id + sz] + w * mt[id + 2 * sz]);
  const double V = fabs(u * mt[id + 3 * sz] + v * mt[id + 4 * sz] + w * mt[id + 5 * sz]);
  const double W = fabs(u * mt[id + 6 * sz] + v * mt[id + 7 * sz] + w * mt[id + 8 * sz]);
  const double kx = sqrt(mt[id] * mt[id] + mt[id + sz] * mt[id + sz] + mt[id + 2 * sz] * mt[id + 2 * sz]);
  const double ky = sqrt(mt[id + 3 * sz] * mt[id + 3 * sz] + mt[id + 4 * sz] * mt[id + 4 * sz] +
                         mt[id + 5 * sz] * mt[id + 5 * sz]);
  const double kz = sqrt(mt[id + 6 * sz] * mt[id + 6 * sz] + mt[id + 7 * sz] * mt[id + 7 * sz] +
                         mt[id + 8 * sz] * mt[id + 8 * sz]);
  const double acoustic_speed = p->mech ? z->acoustic_speed[id] : sqrt(GAMMA_AIR * bv[id + 4 * sz] / bv[id]);
  if (p->dim == 2) return p->entropy_fix_factor * (U + V + acoustic_speed * 0.5 * (kx + ky));
  return p->entropy_fix_factor * (U + V + W + acoustic_speed * (kx + ky + kz) / 3.0);
}

static void roe(const double *pl, const double *pr, int nv, const orc_mech *mech, const double m[2][3],
                const double jac[2], const double delta[2], double *fc) {
  /* half sum of the left and right fluxes with the node metrics */
  double JacKx = jac[0] * m[0][0], JacKy = jac[0] * m[0][1], JacKz = jac[0] * m[0][2];
  double Uk = pl[1] * JacKx + pl[2] * JacKy + pl[3] * JacKz;
  double coeff = Uk * pl[0];
  fc[0] = 0.5 * coeff;
  fc[1] = 0.5 * (coeff * pl[1] + pl[4] * JacKx);
  fc[2] = 0.5 * (coeff * pl[2] + pl[4] * JacKy);
  fc[3] = 0.5 * (coeff * pl[3] + pl[4] * JacKz);
  fc[4] = 0.5 * Uk * (pl[4] + pl[nv]);
  for (int l = 5; l < nv; ++l) fc[l] = 0.5 * coeff * pl[l];
  JacKx = jac[1] * m[1][0];
  JacKy = jac[1] * m[1][1];
  JacKz = jac[1] * m[1][2];
  Uk = pr[1] * JacKx + pr[2] * JacKy + pr[3] * JacKz;
  coeff = Uk * pr[0];
  fc[0] += 0.5 * coeff;
  fc[1] += 0.5 * (coeff * pr[1] + pr[4] * JacKx);
  fc[2] += 0.5 * (coeff * pr[2] + pr[4] * JacKy);
  fc[3] += 0.5 * (coeff * pr[3] + pr[4] * JacKz);
  fc[4] += 0.5 * Uk * (pr[4] + pr[nv]);
  for (int l = 5; l < nv; ++l) fc[l] += 0.5 * coeff * pr[l];

  /* Roe averages */
  const double dl = sqrt(pl[0]), dr = sqrt(pr[0]);
  const double inv_denominator = 1.0 / (dl + dr);
  const double u = (dl * pl[1] + dr * pr[1]) * inv_denominator;
  const double v = (dl * pl[2] + dr * pr[2]) * inv_denominator;
  const double w = (dl * pl[3] + dr * pr[3]) * inv_denominator;
  const double ek = 0.5 * (u * u + v * v + w * w);
  const double hl = (pl[nv] + pl[4]) / pl[0];
  const double hr = (pr[nv] + pr[4]) / pr[0];
  const double h = (dl * hl + dr * hr) * inv_denominator;
  double gamma = GAMMA_AIR;
  double c = sqrt((gamma - 1) * (h - ek));
  double mw = 28.9647;
  double svm[ORC_MAX_SPEC] = {0};
  for (int l = 0; l < nv - 5; ++l) svm[l] = (dl * pl[l + 5] + dr * pr[l + 5]) * inv_denominator;
  double h_i[ORC_MAX_SPEC] = {0};
  const int ns = mech ? mech->n_spec : 0;
  if (mech) {
    double mw_inv = 0;
    for (int l = 0; l < ns; ++l) mw_inv += svm[l] * mech->imw[l];
    const double tl = pl[4] / pl[0], tr = pr[4] / pr[0];
    const double t = (dl * tl + dr * tr) * inv_denominator / (R_U * mw_inv);
    double cp_i[ORC_MAX_SPEC];
    orc_enthalpy_and_cp(mech, t, h_i, cp_i);
    double cv = 0, cp = 0;
    for (int l = 0; l < ns; ++l) {
      cp += cp_i[l] * svm[l];
      cv += svm[l] * (cp_i[l] - mech->gas_const[l]);
    }
    gamma = cp / cv;
    c = sqrt(gamma * R_U * mw_inv * t);
    mw = 1.0 / mw_inv;
  }

  double kx = 0.5 * (m[0][0] + m[1][0]);
  double ky = 0.5 * (m[0][1] + m[1][1]);
  double kz = 0.5 * (m[0][2] + m[1][2]);
  const double gradK = sqrt(kx * kx + ky * ky + kz * kz);
  double Ukk = kx * u + ky * v + kz * w;
  double characteristic[3] = {Ukk - gradK * c, Ukk, Ukk + gradK * c};
  const double entropy_fix_delta_ave = 0.5 * (delta[0] + delta[1]);
  for (int q = 0; q < 3; ++q) {
    double cc = fabs(characteristic[q]);
    if (cc < entropy_fix_delta_ave) cc = 0.5 * (cc * cc / entropy_fix_delta_ave + entropy_fix_delta_ave);
    characteristic[q] = cc;
  }
  kx /= gradK;
  ky /= gradK;
  kz /= gradK;
  Ukk /= gradK;

  const double jac_ave = 0.5 * (jac[0] + jac[1]);
  double dq[NRMAX];
  dq[0] = jac_ave * (pr[0] - pl[0]);
  for (int l = 1; l < nv; ++l) dq[l] = jac_ave * (pr[0] * pr[l] - pl[0] * pl[l]);
  dq[4] = jac_ave * (pr[nv] - pl[nv]);

  double c1 = (gamma - 1) * (ek * dq[0] - u * dq[1] - v * dq[2] - w * dq[3] + dq[4]) / (c * c);
  double c2 = (kx * dq[1] + ky * dq[2] + kz * dq[3] - Ukk * dq[0]) / c;
  for (int l = 0; l < ns; ++l) c1 += (mw * mech->imw[l] - h_i[l] * (gamma - 1) / (c * c)) * dq[l + 5];
  double c3 = dq[0] - c1;
  double LDq[NRMAX];
  LDq[0] = 0.5 * (c1 - c2);
  LDq[1] = kx * c3 - ((kz * v - ky * w) * dq[0] - kz * dq[2] + ky * dq[3]) / c;
  LDq[2] = ky * c3 - ((kx * w - kz * u) * dq[0] - kx * dq[3] + kz * dq[1]) / c;
  LDq[3] = kz * c3 - ((ky * u - kx * v) * dq[0] - ky * dq[1] + kx * dq[2]) / c;
  LDq[4] = 0.5 * (c1 + c2);
  for (int l = 0; l < nv - 5; ++l) LDq[l + 5] = dq[l + 5] - svm[l] * dq[0];

  double b[NRMAX];
  b[0] = -characteristic[0] * LDq[0];
  for (int l = 1; l < nv; ++l) b[l] = -characteristic[1] * LDq[l];
  b[4] = -characteristic[2] * LDq[4];

  const double c0 = kx * b[1] + ky * b[2] + kz * b[3];
  c1 = c0 + b[0] + b[4];
  c2 = c * (b[4] - b[0]);
  c3 = 0;
  for (int l = 0; l < ns; ++l) c3 += (h_i[l] - mw * mech->imw[l] * c * c / (gamma - 1)) * b[l + 5];
  fc[0] += 0.5 * c1;
  fc[1] += 0.5 * (u * c1 + kx * c2 - c * (kz * b[2] - ky * b[3]));
  fc[2] += 0.5 * (v * c1 + ky * c2 - c * (kx * b[3] - kz * b[1]));
  fc[3] += 0.5 * (w * c1 + kz * c2 - c * (ky * b[1] - kx * b[2]));
  fc[4] += 0.5 * (h * c1 + Ukk * c2 - c * c * c0 / (gamma - 1) +
                  c * ((kz * v - ky * w) * b[1] + (kx * w - kz * u) * b[2] + (ky * u - kx * v) * b[3]) + c3);
  for (int l = 0; l < nv - 5; ++l) fc[5 + l] += 0.5 * (b[l + 5] + svm[l] * c1);
}

static void pv_direction(orc_zone *z, const orc_param *p, int dir) {
  const int ngg = z->ngg, mx = z->mx, my = z->my, mz = z->mz, nv = p->n_var;
  const long sz = psz(z, ngg), s = pstride(z, ngg, dir);
  double *flux = dir == 0 ? z->fFlux : (dir == 1 ? z->gFlux : z->hFlux);
  const int mm = 3 * dir;
  const int i0 = dir == 0 ? -1 : 0, j0 = dir == 1 ? -1 : 0, k0 = dir == 2 ? -1 : 0;
  const int sch = p->inviscid_scheme;
  const orc_mech *mech = p->mech;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < mz; ++k) {
    for (int j = j0; j < my; ++j) {
      for (int i = i0; i < mx; ++i) {
        const long id = pidx(z, ngg, i, j, k);
        double pv[4][NRMAX], m[2][3], jac[2], pl[NRMAX], pr[NRMAX], fc[NRMAX];
        for (int q = 0; q < 4; ++q) {
          for (int l = 0; l < 5; ++l) pv[q][l] = z->bv[id + (q - 1) * s + l * sz];
          for (int l = 5; l < nv; ++l) pv[q][l] = z->sv[id + (q - 1) * s + (l - 5) * sz];
        }
        for (int q = 0; q < 2; ++q) {
          for (int l = 0; l < 3; ++l) m[q][l] = z->metric[id + q * s + (mm + l) * sz];
          jac[q] = z->jac[id + q * s];
        }
        reconstruct(pv, nv, p->reconstruction, mech, pl, pr);
        if (sch == 2) {
          const double delta[2] = {entropy_fix_delta(z, p, id), entropy_fix_delta(z, p, id + s)};
          roe(pl, pr, nv, mech, m, jac, delta, fc);
        } else if (sch == 1) {
          lax_friedrichs(pl, pr, m, jac, fc);
        } else if (sch == 4) {
          hllc(pl, pr, nv, mech, m, jac, fc);
        } else {
          ausm_plus(pl, pr, nv, mech, m, jac, fc);
        }
        for (int l = 0; l < nv; ++l) flux[id + l * sz] = fc[l];
      }
    }
  }
  const long szq = psz(z, 0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k) {
    for (int j = 0; j < my; ++j) {
      for (int i = 0; i < mx; ++i) {
        const long iq = pidx(z, 0, i, j, k);
        const long ic = pidx(z, ngg, i, j, k), im = ic - s;
        for (int l = 0; l < nv; ++l) z->dq[iq + l * szq] -= flux[ic + l * sz] - flux[im + l * sz];
      }
    }
  }
}

void orc_roe_like_inviscid(orc_zone *z, const orc_param *p) {
  if (p->mech && p->inviscid_scheme == 1) {
    fprintf(stderr, "oracle: the reference has no Lax-Friedrichs flux for mixtures\n");
    abort();
  }
  pv_direction(z, p, 0);
  pv_direction(z, p, 1);
  if (z->mz > 1) pv_direction(z, p, 2);
}
