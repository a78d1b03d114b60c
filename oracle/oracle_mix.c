/*
 * CPU oracle, mixture model: NASA-7 thermo, temperature Newton iteration,
 * mixture-averaged transport, the characteristic WENO projection with
 * species, species diffusion in the viscous flux, finite-rate kinetics with
 * the point-implicit substep of Wu's splitting.  TEST INFRASTRUCTURE ONLY
 * (see oracle.h).  Each routine names the reference file:line it restates.
 */
#include "oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define R_U 8314.462618
#define P_ATM 101325.0
#define PI 3.141592653589793

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

/* ------------------------------------------------------------------------ */
/* NASA-7 two-range thermo with linear extrapolation (src/Thermo.cu:385-633) */
/* ------------------------------------------------------------------------ */
void orc_enthalpy_and_cp(const orc_mech *m, double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < m->n_spec; ++i) {
    if (t < m->t_low[i] || t > m->t_high[i]) {
      const int lo = t < m->t_low[i];
      const double tt = lo ? m->t_low[i] : m->t_high[i];
      const double *c = lo ? m->low_coeff[i] : m->high_coeff[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = t < m->t_mid[i] ? m->low_coeff[i] : m->high_coeff[i];
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    h[i] *= m->gas_const[i];
    cp[i] *= m->gas_const[i];
  }
}

void orc_enthalpy(const orc_mech *m, double t, double *h) {
  double cp[ORC_MAX_SPEC];
  orc_enthalpy_and_cp(m, t, h, cp);
}

void orc_cp(const orc_mech *m, double t, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < m->n_spec; ++i) {
    if (t < m->t_low[i]) {
      const double tt = m->t_low[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = m->low_coeff[i];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else if (t > m->t_high[i]) {
      const double tt = m->t_high[i], tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      const double *c = m->high_coeff[i];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    } else {
      const double *c = t < m->t_mid[i] ? m->low_coeff[i] : m->high_coeff[i];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    cp[i] *= m->gas_const[i];
  }
}

/* compute_gibbs_div_rt, NASA-7 branch (src/Thermo.cu:576-606) */
void orc_gibbs_div_rt(const orc_mech *m, double t, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t_inv = 1 / t, log_t = log(t);
  for (int i = 0; i < m->n_spec; ++i) {
    if (t < m->t_low[i] || t > m->t_high[i]) {
      const int lo = t < m->t_low[i];
      const double tt = lo ? m->t_low[i] : m->t_high[i];
      const double *c = lo ? m->low_coeff[i] : m->high_coeff[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt_inv = 1 / tt, log_tt = log(tt);
      g[i] = c[0] * (1.0 - log_tt) - 0.5 * c[1] * tt - c[2] * tt2 / 6.0 - c[3] * tt3 / 12.0 - c[4] * tt4 * 0.05 +
             c[5] * tt_inv - c[6];
    } else {
      const double *c = t < m->t_mid[i] ? m->low_coeff[i] : m->high_coeff[i];
      g[i] = c[0] * (1.0 - log_t) - 0.5 * c[1] * t - c[2] * t2 / 6.0 - c[3] * t3 / 12.0 - c[4] * t4 * 0.05 +
             c[5] * t_inv - c[6];
    }
  }
}

/* compute_temperature_and_pressure (src/FieldOperation.cu:4-45) on a node */
void orc_temperature_and_pressure(orc_zone *z, const orc_param *p, long id, double total_energy) {
  const orc_mech *m = p->mech;
  const int ns = m->n_spec;
  const long sz = psz(z, z->ngg);
  double gas_const = 0;
  for (int l = 0; l < ns; ++l) gas_const += z->sv[id + l * sz] * m->gas_const[l];
  const double u = z->bv[id + sz], v = z->bv[id + 2 * sz], w = z->bv[id + 3 * sz];
  const double e = total_energy / z->bv[id] - 0.5 * (u * u + v * v + w * w);
  double err = 1, t = z->bv[id + 5 * sz];
  int iter = 0;
  double h_i[ORC_MAX_SPEC], cp_i[ORC_MAX_SPEC];
  while (err > 1e-5 && iter++ < 1000) {
    orc_enthalpy_and_cp(m, t, h_i, cp_i);
    double cp_tot = 0, h = 0;
    for (int l = 0; l < ns; ++l) {
      cp_tot += cp_i[l] * z->sv[id + l * sz];
      h += h_i[l] * z->sv[id + l * sz];
    }
    const double e_t = h - gas_const * t;
    const double cv = cp_tot - gas_const;
    const double t1 = t - (e_t - e) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  z->bv[id + 5 * sz] = t;
  z->bv[id + 4 * sz] = z->bv[id] * t * gas_const;
}

/* compute_total_energy, mixture branch (src/FieldOperation.cuh:16-37) */
void orc_total_energy_mixture(orc_zone *z, const orc_param *p, long id) {
  const orc_mech *m = p->mech;
  const long sz = psz(z, z->ngg);
  const double *bv = z->bv;
  const double V2 = bv[id + sz] * bv[id + sz] + bv[id + 2 * sz] * bv[id + 2 * sz] + bv[id + 3 * sz] * bv[id + 3 * sz];
  double total_energy = 0.5 * V2;
  double h[ORC_MAX_SPEC];
  orc_enthalpy(m, bv[id + 5 * sz], h);
  for (int l = 0; l < m->n_spec; ++l) total_energy += h[l] * z->sv[id + l * sz];
  total_energy *= bv[id];
  total_energy -= bv[id + 4 * sz];
  z->cv[id + 4 * sz] = total_energy;
}

/* ------------------------------------------------------------------------ */
/* update_physical_properties, mixture branch (src/FieldOperation.cuh:95-114)*/
/* with compute_transport_property (src/Transport.cu:43-165, 182-184).        */
/* ------------------------------------------------------------------------ */
static double omega_d(double t_red) { return 1.0548 * pow(t_red, -0.15504) + pow(t_red + 0.55909, -2.1705); }

void orc_update_physical_properties_mixture_point(orc_zone *z, const orc_param *p, long id) {
  const orc_mech *m = p->mech;
  const int ns = m->n_spec;
  const long sz = psz(z, z->ngg);
  const double temperature = z->bv[id + 5 * sz];
  const double uu = z->bv[id + sz], vv = z->bv[id + 2 * sz], ww = z->bv[id + 3 * sz];
  const double V = sqrt(uu * uu + vv * vv + ww * ww);
  double imw = 0, temp = 0, cp[ORC_MAX_SPEC];
  orc_cp(m, temperature, cp);
  for (int l = 0; l < ns; ++l) {
    const double y = z->sv[id + l * sz];
    imw = fma(y, m->imw[l], imw);
    temp = fma(y, cp[l], temp);
  }
  const double R = R_U * imw;
  temp = temp / (temp - R);
  z->gamma[id] = temp;
  temp = sqrt(temp * R * temperature);
  z->acoustic_speed[id] = temp;
  z->mach[id] = V / temp;

  /* transport */
  const double mw_total = 1 / imw;
  double X[ORC_MAX_SPEC], vis_denom[ORC_MAX_SPEC];
  temp = sqrt(temperature);
  for (int l = 0; l < ns; ++l) {
    X[l] = z->sv[id + l * sz] * mw_total / m->mw[l];
    const double t_dl = temperature * m->LJ_potent_inv[l];
    vis_denom[l] = m->vis_coeff[l] * temp / (1.147 * pow(t_dl, -0.145) + pow(t_dl + 0.5, -2));
  }
  const double t_3over2_over_p = temperature * temp;
  double viscosity = 0, conductivity = 0;
  for (int mm = 0; mm < ns; ++mm) {
    double Rm = m->gas_const[mm];
    double lambda = 15 * 0.25 * vis_denom[mm] * Rm;
    const int geom = (int)m->geometry[mm];
    if (geom == 1 || geom == 2) {
      const double t_red = temperature * m->kb_over_eps_jk[mm][mm];
      const double tRedInv = 1 / t_red;
      temp = sqrt(tRedInv * PI) * PI;
      const double FT = 1 + 0.5 * temp + (2 + 0.25 * PI * PI) * tRedInv + temp * tRedInv;
      const double rhoD = m->binary_diffusivity_coeff[mm][mm] * t_3over2_over_p / (omega_d(t_red) * Rm * temperature);
      if (geom == 1) {
        const double ADivPiB = (2.5 * vis_denom[mm] - rhoD) /
                               ((PI * m->ZRotF298[mm] / FT * vis_denom[mm] + 10.0 / 3 * vis_denom[mm] + 2.0 * rhoD));
        lambda += -5 * ADivPiB * vis_denom[mm] * Rm + rhoD * cp[mm] + rhoD * (2 * ADivPiB - 2.5) * Rm;
      } else {
        const double ADivPiB = (2.5 * vis_denom[mm] - rhoD) /
                               ((PI * m->ZRotF298[mm] / FT * vis_denom[mm] + 5 * vis_denom[mm] + 2.0 * rhoD));
        lambda += -7.5 * ADivPiB * vis_denom[mm] * Rm + rhoD * cp[mm] + rhoD * (3 * ADivPiB - 2.5) * Rm;
      }
    }
    temp = 0;
    Rm = sqrt(vis_denom[mm]);
    for (int n = 0; n < ns; ++n) {
      double partition_func = 1.0;
      if (mm != n) {
        const double numerator = 1.0 + (1.0 / sqrt(vis_denom[n])) * (Rm * m->WjDivWi_to_One4th[mm][n]);
        partition_func = numerator * numerator * m->sqrt_WiDivWjPl1Mul8[mm][n];
      }
      temp += partition_func * X[n];
    }
    viscosity += vis_denom[mm] * X[mm] / temp;
    conductivity += lambda * X[mm] / (1.065 * temp - 0.065 * X[mm]);
  }
  z->mul[id] = viscosity;
  z->thermal_conductivity[id] = conductivity;
  const double eps = 1e-12;
  double sum = 0;
  for (int l = 0; l < ns; ++l) {
    temp = (X[l] + eps) * m->mw[l];
    cp[l] = temp;
    sum += temp;
    vis_denom[l] = 0;
  }
  for (int l = 0; l < ns; ++l) cp[l] = sum - cp[l];
  for (int l = 0; l < ns; ++l)
    for (int n = l + 1; n < ns; ++n) {
      temp = omega_d(temperature * m->kb_over_eps_jk[l][n]) / (m->binary_diffusivity_coeff[l][n] * t_3over2_over_p);
      vis_denom[l] += (X[n] + eps) * temp;
      vis_denom[n] += (X[l] + eps) * temp;
    }
  temp = 1.0 / (temperature * R_U);
  for (int l = 0; l < ns; ++l) z->rho_D[id + l * sz] = cp[l] * temp / vis_denom[l];
}

/* viscous spectral velocity of the mixture (src/TimeAdvanceFunc.cuh:72-85) */
double orc_mixture_max_diffuse_vel(const orc_zone *z, const orc_param *p, long id) {
  const orc_mech *m = p->mech;
  const long sz = psz(z, z->ngg);
  const double iRho = 1.0 / z->bv[id];
  double cpl[ORC_MAX_SPEC];
  orc_cp(m, z->bv[id + 5 * sz], cpl);
  double cp = 0, max_rhoD = 0;
  for (int l = 0; l < m->n_spec; ++l) {
    cp += cpl[l] * z->sv[id + l * sz];
    max_rhoD = max_rhoD > z->rho_D[id + l * sz] ? max_rhoD : z->rho_D[id + l * sz];
  }
  double mdv = z->mul[id] * iRho;
  const double a = z->thermal_conductivity[id] * iRho * z->gamma[id] / cp;
  mdv = mdv > a ? mdv : a;
  const double b = max_rhoD * iRho;
  return mdv > b ? mdv : b;
}

/* ------------------------------------------------------------------------ */
/* Characteristic WENO face flux with species (src/WENO.cu:1096-1469)        */
/* ------------------------------------------------------------------------ */
void orc_weno_face_mixture(const orc_zone *z, const orc_param *p, int dir, long idx, double kx, double ky,
                           double kz, double eps_ref, int if_shock, double *fc) {
  const orc_mech *mech = p->mech;
  const int ngg = z->ngg, ns = mech->n_spec, nv = p->n_var;
  const long sz = psz(z, ngg), s = pstride(z, ngg, dir);
  const int mm = 3 * dir;
  const int order7 = p->inviscid_scheme == 72;
  const int lo = order7 ? -3 : -2, np = order7 ? 8 : 6;
  double Q[ORC_MAX_SPEC + 5][8], F[7][8];
  for (int m = 0; m < np; ++m) {
    const long id = idx + (long)(lo + m) * s;
    const double q0 = z->cv[id], q1 = z->cv[id + sz], q2 = z->cv[id + 2 * sz], q3 = z->cv[id + 3 * sz],
                 q4 = z->cv[id + 4 * sz];
    Q[0][m] = q0; Q[1][m] = q1; Q[2][m] = q2; Q[3][m] = q3; Q[4][m] = q4;
    const double m0 = z->metric[id + mm * sz], m1 = z->metric[id + (mm + 1) * sz], m2 = z->metric[id + (mm + 2) * sz];
    const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
    const double pk = z->bv[id + 4 * sz];
    F[0][m] = Uk;
    F[1][m] = fma(q1, Uk, pk * m0);
    F[2][m] = fma(q2, Uk, pk * m1);
    F[3][m] = fma(q3, Uk, pk * m2);
    F[4][m] = pk;
    for (int l = 5; l < nv; ++l) Q[l][m] = z->cv[id + l * sz];
    F[5][m] = sqrt(m0 * m0 + m1 * m1 + m2 * m2) * z->acoustic_speed[id];
    F[6][m] = z->jac[id];
  }
  const int c = -lo;
  const double rho_l = Q[0][c], rho_r = Q[0][c + 1];
  double temp1 = sqrt(rho_l * rho_r);
  const double rlc = 1 / (rho_l + temp1);
  const double rrc = 1 / (temp1 + rho_r);
  const double um = rlc * Q[1][c] + rrc * Q[1][c + 1];
  const double vm = rlc * Q[2][c] + rrc * Q[2][c + 1];
  const double wm = rlc * Q[3][c] + rrc * Q[3][c + 1];
  double svm[ORC_MAX_SPEC];
  for (int l = 0; l < nv - 5; ++l) svm[l] = rlc * Q[l + 5][c] + rrc * Q[l + 5][c + 1];
  temp1 = 0;
  for (int l = 0; l < ns; ++l) temp1 += svm[l] * mech->gas_const[l];
  double temp3 = (rlc * F[4][c] + rrc * F[4][c + 1]) / temp1;
  double fChar[5 + ORC_MAX_SPEC], hI_alpI[ORC_MAX_SPEC];
  orc_enthalpy_and_cp(mech, temp3, hI_alpI, fChar);
  double temp2 = 0;
  for (int l = 0; l < ns; ++l) temp2 += svm[l] * fChar[l];
  const double gamma = temp2 / (temp2 - temp1);
  const double cm = sqrt(gamma * temp1 * temp3);
  const double gm1 = gamma - 1;
  temp1 = 1.0 / sqrt(kx * kx + ky * ky + kz * kz);
  kx *= temp1; ky *= temp1; kz *= temp1;
  const double Uk_bar = kx * um + ky * vm + kz * wm;
  double nx = 0, ny = 0, nz = 0, qx, qy, qz;
  if (fabs(kx) > 0.8) { nx = -kz; nz = kx; }
  else { ny = kz; nz = -ky; }
  temp1 = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= temp1; ny *= temp1; nz *= temp1;
  qx = ky * nz - kz * ny; qy = kz * nx - kx * nz; qz = kx * ny - ky * nx;
  temp1 = 1.0 / sqrt(qx * qx + qy * qy + qz * qz);
  qx *= temp1; qy *= temp1; qz *= temp1;
  const double Un = nx * um + ny * vm + nz * wm;
  const double Uq = qx * um + qy * vm + qz * wm;
  temp2 = 1.0 / (cm * cm);
  for (int l = 0; l < ns; ++l) {
    hI_alpI[l] = gamma * mech->gas_const[l] * temp3 - gm1 * hI_alpI[l];
    hI_alpI[l] *= temp2;
  }
  temp3 = 0.5 * gm1 * (um * um + vm * vm + wm * wm);
  double max_lambda = 0;
  for (int m = 0; m < np; ++m) {
    const double lam = fabs(F[0][m]) + F[5][m];
    if (lam > max_lambda) max_lambda = lam;
  }
  double sumBetaQ[8], sumBetaF[8];
  for (int m = 0; m < np; ++m) {
    double sp = 0, sm = 0;
    for (int n = 0; n < ns; ++n) {
      sp = fma(hI_alpI[n], Q[5 + n][m], sp);
      sm = fma(hI_alpI[n], Q[5 + n][m] * F[0][m], sm);
    }
    sumBetaQ[m] = sp;
    sumBetaF[m] = sm;
  }
  for (int l = 0; l < 5; ++l) {
    double L[5];
    temp1 = 0.5;
    switch (l) {
      case 0:
        L[0] = (temp3 + Uk_bar * cm) * temp2 * 0.5;
        L[1] = -(gm1 * um + kx * cm) * temp2 * 0.5;
        L[2] = -(gm1 * vm + ky * cm) * temp2 * 0.5;
        L[3] = -(gm1 * wm + kz * cm) * temp2 * 0.5;
        L[4] = gm1 * temp2 * 0.5;
        break;
      case 1:
        temp1 = 0; L[0] = -Un; L[1] = nx; L[2] = ny; L[3] = nz; L[4] = 0;
        break;
      case 2:
        temp1 = 0; L[0] = -Uq; L[1] = qx; L[2] = qy; L[3] = qz; L[4] = 0;
        break;
      case 3:
        temp1 = -1;
        L[0] = 1 - temp3 * temp2;
        L[1] = gm1 * um * temp2;
        L[2] = gm1 * vm * temp2;
        L[3] = gm1 * wm * temp2;
        L[4] = -gm1 * temp2;
        break;
      default:
        L[0] = (temp3 - Uk_bar * cm) * temp2 * 0.5;
        L[1] = -(gm1 * um - kx * cm) * temp2 * 0.5;
        L[2] = -(gm1 * vm - ky * cm) * temp2 * 0.5;
        L[3] = -(gm1 * wm - kz * cm) * temp2 * 0.5;
        L[4] = gm1 * temp2 * 0.5;
        break;
    }
    double vPlus[8], vMinus[8];
    for (int m = 0; m < np; ++m) {
      const double LFm = L[0] * (Q[0][m] * F[0][m]) + L[1] * F[1][m] + L[2] * F[2][m] + L[3] * F[3][m] +
                         L[4] * ((Q[4][m] + F[4][m]) * F[0][m]) + temp1 * sumBetaF[m];
      const double LQm = L[0] * Q[0][m] + L[1] * Q[1][m] + L[2] * Q[2][m] + L[3] * Q[3][m] + L[4] * Q[4][m] +
                         temp1 * sumBetaQ[m];
      if (m < np - 1) vPlus[m] = 0.5 * F[6][m] * (LFm + max_lambda * LQm);
      if (m > 0) vMinus[m - 1] = 0.5 * F[6][m] * (LFm - max_lambda * LQm);
    }
    fChar[l] = order7 ? orc_weno7(vPlus, vMinus, eps_ref, if_shock) : orc_weno5(vPlus, vMinus, eps_ref, if_shock);
  }
  for (int l = 0; l < ns; ++l) {
    double vPlus[8], vMinus[8];
    for (int m = 0; m < np; ++m) {
      const double LFm = F[0][m] * (Q[5 + l][m] - svm[l] * Q[0][m]);
      const double LQm = Q[5 + l][m] - svm[l] * Q[0][m];
      if (m < np - 1) vPlus[m] = 0.5 * F[6][m] * (LFm + max_lambda * LQm);
      if (m > 0) vMinus[m - 1] = 0.5 * F[6][m] * (LFm - max_lambda * LQm);
    }
    fChar[5 + l] = order7 ? orc_weno7(vPlus, vMinus, eps_ref, if_shock) : orc_weno5(vPlus, vMinus, eps_ref, if_shock);
  }
  temp1 = fChar[0] + fChar[3] + fChar[4];
  temp3 = fChar[0] - fChar[4];
  fc[0] = temp1;
  fc[1] = um * temp1 - kx * cm * temp3 + nx * fChar[1] + qx * fChar[2];
  fc[2] = vm * temp1 - ky * cm * temp3 + ny * fChar[1] + qy * fChar[2];
  fc[3] = wm * temp1 - kz * cm * temp3 + nz * fChar[1] + qz * fChar[2];
  temp2 = rlc * (Q[4][c] + F[4][c]) + rrc * (Q[4][c + 1] + F[4][c + 1]);
  fc[4] = temp2 * temp1 - Uk_bar * cm * temp3 + Un * fChar[1] + Uq * fChar[2] - cm * cm / gm1 * fChar[3];
  temp2 = 0;
  for (int l = 0; l < ns; ++l) {
    fc[5 + l] = svm[l] * temp1 + fChar[l + 5];
    temp2 += hI_alpI[l] * fChar[l + 5];
  }
  fc[4] -= temp2 * cm * cm / gm1;
}

/* Positive-preserving limiter of the species face fluxes, characteristic
 * branch of the x sweep (src/WENO.cu:1471-1540).  For each species whose
 * one-sided updates alpha/2 J rhoY -/+ dt f would go negative, the face flux
 * is blended towards a first-order flux f1 with theta in [0, 1].  dt is the
 * step's dt (DParameter::dt); when that is not positive the reference reads
 * dt_local(i, j, k), which for the i = -1 face lies outside the array — here
 * that face takes node 0's value. */
void orc_positive_preserving_face(const orc_zone *z, const orc_param *p, int dir, int i, int j, int k, double *fc) {
  const int ngg = z->ngg, ns = p->n_var - 5;
  const long sz = psz(z, ngg), s = pstride(z, ngg, dir);
  const long il = pidx(z, ngg, i, j, k), ir = il + s;
  double dt = z->dt_step;
  if (!(dt > 0)) dt = z->dt_local[pidx(z, 0, i < 0 ? 0 : i, j, k)];
  const double alpha = p->dim == 3 ? 1.0 / 3.0 : 0.5;
  const double jac_l = z->jac[il], jac_r = z->jac[ir];
  const double alphaL = 0.5 * alpha * jac_l, alphaR = 0.5 * alpha * jac_r;
  int start_l = -1;
  for (int l = 0; l < ns; ++l) {
    const double up = alphaL * z->cv[il + (5 + l) * sz] - dt * fc[5 + l];
    const double um = alphaR * z->cv[ir + (5 + l) * sz] + dt * fc[5 + l];
    if (up < 0 || um < 0) { start_l = l; break; }
  }
  if (start_l < 0) return;
  /* Uk and c|grad k| of the two nodes (the staged F[0], F[5], F[6] of
   * src/WENO.cu:1112-1137) */
  double Uk[2], cg[2], J[2];
  const long nd[2] = {il, ir};
  const int mo = 3 * dir;
  for (int n = 0; n < 2; ++n) {
    const long id = nd[n];
    const double q0 = z->cv[id], q1 = z->cv[id + sz], q2 = z->cv[id + 2 * sz], q3 = z->cv[id + 3 * sz];
    const double m0 = z->metric[id + mo * sz], m1 = z->metric[id + (mo + 1) * sz], m2 = z->metric[id + (mo + 2) * sz];
    Uk[n] = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
    cg[n] = sqrt(m0 * m0 + m1 * m1 + m2 * m2) * z->acoustic_speed[id];
    J[n] = z->jac[id];
  }
  const double U1 = Uk[0] * jac_l, U2 = Uk[1] * jac_r;
  for (int l = start_l; l < ns; ++l) {
    double f1 = 0;
    int f1_computed = 0;
    double theta_p = 1.0, theta_m = 1.0;
    const double rhoYL = z->cv[il + (5 + l) * sz], rhoYR = z->cv[ir + (5 + l) * sz];
    const double fp = 0.5 * J[0] * (Uk[0] + cg[0]) * rhoYL;
    const double fm = 0.5 * J[1] * (Uk[1] - cg[1]) * rhoYR;
    const double up = alphaL * rhoYL - dt * fc[5 + l];
    if (up < 0) {
      f1 = 0.5 * (fp + U1 * rhoYL) + 0.5 * (fm - U2 * rhoYR);
      f1_computed = 1;
      const double up_lf = alphaL * rhoYL - dt * f1;
      if (fabs(up - up_lf) > 1e-20 * p->rho_ref) {
        theta_p = (0 - up_lf) / (up - up_lf);
        if (theta_p > 1) theta_p = 1.0;
        else if (theta_p < 0) theta_p = 0;
      }
    }
    const double um = alphaR * rhoYR + dt * fc[5 + l];
    if (um < 0) {
      if (!f1_computed) f1 = 0.5 * (fp + U1 * rhoYL) + 0.5 * (fm - U2 * rhoYR);
      const double um_lf = alphaR * rhoYR + dt * f1;
      if (fabs(um - um_lf) > 1e-20 * p->rho_ref) {
        theta_m = (0 - um_lf) / (um - um_lf);
        if (theta_m > 1) theta_m = 1.0;
        else if (theta_m < 0) theta_m = 0;
      }
    }
    fc[5 + l] = fmin(theta_p, theta_m) * (fc[5 + l] - f1) + f1;
  }
}

/* ------------------------------------------------------------------------ */
/* Species diffusion part of the viscous face flux (src/ViscousScheme.cu:    */
/* 700-790 and the g/h analogues), with the grad-p term of                   */
/* gradPInDiffusionFlux (:742-766, 931-955, 1115-1139) when it is set.       */
/* ------------------------------------------------------------------------ */
void orc_viscous_species_face(const orc_zone *z, const orc_param *p, int dir, int i, int j, int k,
                              const double gm[9], const double gk[3], double *fv) {
  const orc_mech *m = p->mech;
  const int ns = m->n_spec, ngg = z->ngg;
  const long sz = psz(z, ngg);
  const long id = pidx(z, ngg, i, j, k), sd = pstride(z, ngg, dir), idn = id + sd;
  const int da = (dir + 1) % 3, db = (dir + 2) % 3;
  const long sa = pstride(z, ngg, da), sb = pstride(z, ngg, db);
  const double *y = z->sv;
  double diffusivity[ORC_MAX_SPEC], yk[ORC_MAX_SPEC], ddf[ORC_MAX_SPEC];
  double sum_GradXi_cdot_GradY_over_wl = 0, sum_rhoDkYk = 0, CorrectionVelocityTerm = 0, mw_tot = 0;
  for (int l = 0; l < ns; ++l) {
    const double *yl = y + l * sz;
    yk[l] = 0.5 * (yl[id] + yl[idn]);
    diffusivity[l] = 0.5 * (z->rho_D[id + l * sz] + z->rho_D[idn + l * sz]);
    double d3[3];
    d3[dir] = yl[idn] - yl[id];
    d3[da] = 0.25 * (yl[id + sa] - yl[id - sa] + yl[idn + sa] - yl[idn - sa]);
    d3[db] = 0.25 * (yl[id + sb] - yl[id - sb] + yl[idn + sb] - yl[idn - sb]);
    const double y_x = d3[0] * gm[0] + d3[1] * gm[3] + d3[2] * gm[6];
    const double y_y = d3[0] * gm[1] + d3[1] * gm[4] + d3[2] * gm[7];
    const double y_z = d3[0] * gm[2] + d3[1] * gm[5] + d3[2] * gm[8];
    const double GradXi_cdot_GradY = gk[0] * y_x + gk[1] * y_y + gk[2] * y_z;
    ddf[l] = GradXi_cdot_GradY;
    CorrectionVelocityTerm += diffusivity[l] * GradXi_cdot_GradY;
    sum_GradXi_cdot_GradY_over_wl += GradXi_cdot_GradY * m->imw[l];
    mw_tot += yk[l] * m->imw[l];
    sum_rhoDkYk += diffusivity[l] * yk[l];
  }
  mw_tot = 1.0 / mw_tot;
  CorrectionVelocityTerm -= mw_tot * sum_rhoDkYk * sum_GradXi_cdot_GradY_over_wl;
  if (p->gradPInDiffusionFlux) {
    const double *pv = z->bv + 4 * sz;
    double d3[3];
    d3[dir] = pv[idn] - pv[id];
    d3[da] = 0.25 * (pv[id + sa] - pv[id - sa] + pv[idn + sa] - pv[idn - sa]);
    d3[db] = 0.25 * (pv[id + sb] - pv[id - sb] + pv[idn + sb] - pv[idn - sb]);
    const double p_x = d3[0] * gm[0] + d3[1] * gm[3] + d3[2] * gm[6];
    const double p_y = d3[0] * gm[1] + d3[1] * gm[4] + d3[2] * gm[7];
    const double p_z = d3[0] * gm[2] + d3[1] * gm[5] + d3[2] * gm[8];
    const double gradXi_cdot_gradP_over_p = (gk[0] * p_x + gk[1] * p_y + gk[2] * p_z) / (0.5 * (pv[idn] + pv[id]));
    for (int l = 0; l < ns; ++l) {
      ddf[l] += (mw_tot * m->imw[l] - 1) * yk[l] * gradXi_cdot_gradP_over_p;
      CorrectionVelocityTerm += (mw_tot * m->imw[l] - 1) * yk[l] * gradXi_cdot_gradP_over_p * diffusivity[l];
    }
  }
  double h[ORC_MAX_SPEC];
  const double tm = 0.5 * (z->bv[id + 5 * sz] + z->bv[idn + 5 * sz]);
  orc_enthalpy(m, tm, h);
  for (int l = 0; l < ns; ++l) {
    const double diffusion_flux =
        diffusivity[l] * (ddf[l] - mw_tot * yk[l] * sum_GradXi_cdot_GradY_over_wl) - yk[l] * CorrectionVelocityTerm;
    fv[4 + l] = diffusion_flux;
    fv[3] += h[l] * diffusion_flux;
  }
}

/* MUSCL + Roe/AUSM+/HLLC paths are restated in oracle_riemann.c */
void orc_roe_like_inviscid(orc_zone *z, const orc_param *p);

/* ------------------------------------------------------------------------ */
/* Finite-rate kinetics (generic mechanism, src/FiniteRateChem.cu:1466-1605) */
/* ------------------------------------------------------------------------ */
static double arrhenius(double t, double A, double b, double Ea) { return A * pow(t, b) * exp(-Ea / t); }

void orc_forward_rate(const orc_mech *m, double t, const double *c, double *kf) {
  for (int i = 0; i < m->n_reac; ++i) {
    kf[i] = arrhenius(t, m->A[i], m->b[i], m->Ea[i]);
    const int type = m->reac_type[i];
    if (type == 3) {
      kf[i] += arrhenius(t, m->A2[i], m->b2[i], m->Ea2[i]);
    } else if (type > 3) {
      double cc = 0;
      for (int l = 0; l < m->n_spec; ++l) cc += c[l] * m->third_body_coeff[i][l];
      if (type == 4) {
        kf[i] *= cc;
      } else {
        const double kf_low = arrhenius(t, m->A2[i], m->b2[i], m->Ea2[i]);
        const double kf_high = kf[i];
        if (kf_high < 1e-25 && kf_low < 1e-25) {
          kf[i] = 0;
          continue;
        }
        const double reduced_pressure = kf_low * cc / kf_high;
        double F = 1.0;
        if (type > 5) {
          double f_cent = (1 - m->troe_alpha[i]) * exp(-t / m->troe_t3[i]) + m->troe_alpha[i] * exp(-t / m->troe_t1[i]);
          if (type == 7) f_cent += exp(-m->troe_t2[i] / t);
          const double logFc = log10(f_cent);
          const double cq = -0.4 - 0.67 * logFc;
          const double n = 0.75 - 1.27 * logFc;
          const double logPr = log10(reduced_pressure);
          const double tempo = (logPr + cq) / (n - 0.14 * (logPr + cq));
          const double pp = logFc / (1.0 + tempo * tempo);
          F = pow(10, pp);
        }
        kf[i] = kf_high * reduced_pressure / (1.0 + reduced_pressure) * F;
      }
    }
  }
}

void orc_backward_rate(const orc_mech *m, double t, const double *kf, const double *c, double *kb) {
  int n_gibbs = m->n_reac;
  for (int i = 0; i < m->n_reac; ++i) {
    if (m->reac_type[i] == 0) {
      kb[i] = 0;
      --n_gibbs;
    } else if (m->rev_type[i] == 1) {
      kb[i] = arrhenius(t, m->A2[i], m->b2[i], m->Ea2[i]);
      if (m->reac_type[i] == 4) {
        double cc = 0;
        for (int l = 0; l < m->n_spec; ++l) cc += c[l] * m->third_body_coeff[i][l];
        kb[i] *= cc;
      }
      --n_gibbs;
    }
  }
  if (n_gibbs < 1) return;
  double g[ORC_MAX_SPEC];
  orc_gibbs_div_rt(m, t, g);
  const double temp_p = P_ATM / R_U * 1e-3;
  const double temp_t = temp_p / t;
  /* as in the reference, every reversible reaction (also REV ones) ends with
   * kb = kf / Kc (src/FiniteRateChem.cu:1549-1559) */
  for (int i = 0; i < m->n_reac; ++i) {
    if (m->reac_type[i] != 2 && m->reac_type[i] != 0) {
      double d_gibbs = 0;
      for (int l = 0; l < m->n_spec; ++l) d_gibbs += g[l] * (m->stoi_b[i][l] - m->stoi_f[i][l]);
      const double kc = pow(temp_t, m->reac_order[i]) * exp(-d_gibbs);
      kb[i] = kf[i] / kc;
    }
  }
}

void orc_rate_of_progress(const orc_mech *m, const double *kf, const double *kb, const double *c, double *q1,
                          double *q2) {
  for (int i = 0; i < m->n_reac; ++i) {
    q1[i] = 1.0;
    q2[i] = m->reac_type[i] != 0 ? 1.0 : 0.0;
    for (int j = 0; j < m->n_spec; ++j) {
      q1[i] *= pow(c[j], m->stoi_f[i][j]);
      if (m->reac_type[i] != 0) q2[i] *= pow(c[j], m->stoi_b[i][j]);
    }
    q1[i] *= kf[i];
    if (m->reac_type[i] != 0) q2[i] *= kb[i];
  }
}

void orc_chemical_source(const orc_mech *m, const double *q1, const double *q2, double *omega_d, double *omega) {
  for (int i = 0; i < m->n_spec; ++i) {
    double creation = 0;
    omega_d[i] = 0;
    for (int j = 0; j < m->n_reac; ++j) {
      creation += q2[j] * m->stoi_f[j][i] + q1[j] * m->stoi_b[j][i];
      omega_d[i] += q1[j] * m->stoi_f[j][i] + q2[j] * m->stoi_b[j][i];
    }
    creation *= 1e+3 / m->imw[i];
    omega_d[i] *= 1e+3 / m->imw[i];
    omega[i] = creation - omega_d[i];
  }
}

/* solve_chem_system: column-pivoted Crout-type LU (src/FiniteRateChem.cu:1769-1822) */
void orc_solve_chem_system(double *lhs, double *rhs, int dim) {
  int ipiv[ORC_MAX_SPEC] = {0};
  for (int n = 0; n < dim; ++n) {
    int ik = n;
    for (int m = n; m < dim; ++m) {
      for (int t = 0; t < n; ++t) lhs[m * dim + n] -= lhs[m * dim + t] * lhs[t * dim + n];
      if (fabs(lhs[m * dim + n]) > fabs(lhs[ik * dim + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n)
      for (int t = 0; t < dim; ++t) {
        const double mid = lhs[ik * dim + t];
        lhs[ik * dim + t] = lhs[n * dim + t];
        lhs[n * dim + t] = mid;
      }
    for (int pp = n + 1; pp < dim; ++pp)
      for (int t = 0; t < n; ++t) lhs[n * dim + pp] -= lhs[n * dim + t] * lhs[t * dim + pp];
    for (int m = n + 1; m < dim; ++m) lhs[m * dim + n] /= lhs[n * dim + n];
  }
  for (int m = 0; m < dim; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      const double mid = rhs[t];
      rhs[t] = rhs[m];
      rhs[m] = mid;
    }
  }
  for (int m = 1; m < dim; ++m)
    for (int t = 0; t < m; ++t) rhs[m] -= lhs[m * dim + t] * rhs[t];
  rhs[dim - 1] /= lhs[dim * dim - 1];
  for (int m = dim - 2; m >= 0; --m) {
    for (int t = m + 1; t < dim; ++t) rhs[m] -= lhs[m * dim + t] * rhs[t];
    rhs[m] /= lhs[m * dim + m];
  }
}

/* ------------------------------------------------------------------------ */
/* One point-implicit (method 1) or explicit (method 0) 0-D substep of Wu's  */
/* splitting at a node: wu_zeroDReaction (src/StrangSplitting.cu:43-224).    */
/* ------------------------------------------------------------------------ */
static void wu_zero_d(orc_zone *z, const orc_param *p, double dt, long id, long iq, const double *cn,
                      const double *cnY, double *timeScale) {
  const orc_mech *m = p->mech;
  const int ns = m->n_spec, nr = m->n_reac;
  const long sz = psz(z, z->ngg);
  double *cv = z->cv, *bv = z->bv;
  double c[ORC_MAX_SPEC], kf[ORC_MAX_REAC], kb[ORC_MAX_REAC] = {0}, q1[ORC_MAX_REAC], q2[ORC_MAX_REAC];
  double omega[ORC_MAX_SPEC], omega_d[ORC_MAX_SPEC];
  for (int l = 0; l < ns; ++l) c[l] = cv[id + (l + 5) * sz] * m->imw[l] * 1e-3;
  const double t = bv[id + 5 * sz];
  const double iJac = 1.0 / z->jac[id];
  (void)iq;
  orc_forward_rate(m, t, c, kf);
  orc_backward_rate(m, t, kf, c, kb);
  orc_rate_of_progress(m, kf, kb, c, q1, q2);
  orc_chemical_source(m, q1, q2, omega_d, omega);
  for (int l = 0; l < ns; ++l) c[l] *= 1e+3 / m->imw[l];
  if (p->chem_advance_method == 1) {
    double jac[ORC_MAX_SPEC * ORC_MAX_SPEC];
    for (int a = 0; a < ns; ++a)
      for (int n = 0; n < ns; ++n) {
        double zz = 0;
        const double rhoY = c[n];
        if (rhoY > 1e-25) {
          for (int r = 0; r < nr; ++r)
            zz += (m->stoi_b[r][a] - m->stoi_f[r][a]) * (m->stoi_f[r][n] * q1[r] - m->stoi_b[r][n] * q2[r]);
          zz /= rhoY;
        }
        jac[a * ns + n] = zz * 1e+3 / m->imw[a];
      }
    for (int a = 0; a < ns; ++a)
      for (int n = 0; n < ns; ++n) jac[a * ns + n] = (a == n ? 1 : 0) - dt * jac[a * ns + n];
    orc_solve_chem_system(jac, omega, ns);
  }
  for (int l = 0; l < 5; ++l) cv[id + l * sz] += cn[l] * dt * iJac;
  double time_scale = 1e6;
  for (int l = 0; l < ns; ++l) {
    const double rY = cv[id + (5 + l) * sz];
    if (rY > 1e-25 && fabs(omega_d[l]) > 1e-25) {
      const double ts = fabs(rY / omega_d[l]);
      time_scale = ts < time_scale ? ts : time_scale;
    }
    cv[id + (5 + l) * sz] += (omega[l] + cnY[l] * iJac) * dt;
  }
  *timeScale = time_scale;
  bv[id] = cv[id];
  const double density_inv = 1.0 / cv[id];
  bv[id + sz] = cv[id + sz] * density_inv;
  bv[id + 2 * sz] = cv[id + 2 * sz] * density_inv;
  bv[id + 3 * sz] = cv[id + 3 * sz] * density_inv;
  double sum_part_den = 0;
  for (int l = 0; l < ns; ++l) {
    if (cv[id + (5 + l) * sz] < 0) cv[id + (5 + l) * sz] = 0;
    else sum_part_den += cv[id + (l + 5) * sz];
  }
  sum_part_den = 1.0 / sum_part_den;
  const double den_ratio = cv[id] * sum_part_den;
  for (int l = 0; l < ns; ++l) {
    z->sv[id + l * sz] = cv[id + (5 + l) * sz] * sum_part_den;
    cv[id + (5 + l) * sz] *= den_ratio;
  }
  for (int l = ns; l < p->n_scalar; ++l) z->sv[id + l * sz] = cv[id + (5 + l) * sz] * density_inv;
  orc_temperature_and_pressure(z, p, id, cv[id + 4 * sz]);
}

/* wu_reaction_step (src/StrangSplitting.cu:373-421): n_sub = int(dt/tau)
 * substeps of dt/(n_sub+1) and a last one of dt - n_sub*dt/(n_sub+1).
 * Returns the number of substeps taken at each node in nsub_out (optional). */
void orc_wu_reaction_step(orc_zone *z, const orc_param *p, double dt, int *nsub_out) {
  const int ns = p->mech->n_spec, g = z->ngg;
  const long szq = psz(z, 0);
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = 0; k < z->mz; ++k)
    for (int j = 0; j < z->my; ++j)
      for (int i = 0; i < z->mx; ++i) {
        const long id = pidx(z, g, i, j, k), iq = pidx(z, 0, i, j, k);
        double Cn[5], CnY[ORC_MAX_SPEC];
        for (int l = 0; l < 5; ++l) Cn[l] = z->Cn[iq + l * szq];
        for (int l = 0; l < ns; ++l) CnY[l] = z->Cn[iq + (l + 5) * szq];
        double reaction_timescale = z->reaction_timeScale[id];
        if (reaction_timescale < 1e-15) reaction_timescale = 0.2 * dt;
        const int n_sub = (int)(dt / reaction_timescale);
        double dt_reaction = dt / (n_sub + 1);
        double *timeScale = &z->reaction_timeScale[id];
        for (int n = 0; n < n_sub; ++n) wu_zero_d(z, p, dt_reaction, id, iq, Cn, CnY, timeScale);
        dt_reaction = dt - dt_reaction * n_sub;
        int taken = n_sub;
        if (fabs(dt_reaction) > 1e-12) {
          wu_zero_d(z, p, dt_reaction, id, iq, Cn, CnY, timeScale);
          ++taken;
        }
        if (nsub_out) nsub_out[iq] = taken;
      }
}

/* finite_rate_chemistry, explicit source into dq (src/FiniteRateChem.cu:1388-1464) */
void orc_finite_rate_chemistry(orc_zone *z, const orc_param *p) {
  const orc_mech *m = p->mech;
  const int ns = m->n_spec, g = z->ngg;
  const long sz = psz(z, g), szq = psz(z, 0);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z->mz; ++k)
    for (int j = 0; j < z->my; ++j)
      for (int i = 0; i < z->mx; ++i) {
        const long id = pidx(z, g, i, j, k), iq = pidx(z, 0, i, j, k);
        double c[ORC_MAX_SPEC], kf[ORC_MAX_REAC], kb[ORC_MAX_REAC] = {0}, q1[ORC_MAX_REAC], q2[ORC_MAX_REAC];
        double omega[ORC_MAX_SPEC], omega_d[ORC_MAX_SPEC];
        const double density = z->bv[id];
        for (int l = 0; l < ns; ++l) c[l] = density * z->sv[id + l * sz] * m->imw[l] * 1e-3;
        const double t = z->bv[id + 5 * sz];
        orc_forward_rate(m, t, c, kf);
        orc_backward_rate(m, t, kf, c, kb);
        orc_rate_of_progress(m, kf, kb, c, q1, q2);
        orc_chemical_source(m, q1, q2, omega_d, omega);
        double time_scale = 1e6;
        for (int l = 0; l < ns; ++l) {
          z->dq[iq + (l + 5) * szq] += z->jac[id] * omega[l];
          const double y = z->sv[id + l * sz];
          if (y > 1e-25 && fabs(omega_d[l]) > 1e-25) {
            const double ts = fabs(density * y / omega_d[l]);
            time_scale = ts < time_scale ? ts : time_scale;
          }
        }
        z->reaction_timeScale[id] = time_scale;
      }
}
