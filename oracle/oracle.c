/*
 * CPU oracle: plain-C restatement of the reference solver's per-stage
 * right-hand side and SSP-RK3 update (air model; the mixture model and the
 * chemistry live in oracle_mix.c).  TEST INFRASTRUCTURE ONLY: it is the
 * checker for the CUDA path and the timed CPU baseline, never the product.
 *
 * Every routine names the reference file:line it restates.  The arithmetic
 * order follows the reference; where the reference calls a CUDA intrinsic
 * (rnorm3d, norm3d) the oracle uses the textbook formula, which agrees to a
 * few ulp.
 */
#include "oracle.h"
#include <stdint.h>

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* physical constants, reference src/Constants.h */
#define R_U 8314.462618
#define MW_AIR 28.9647
#define GAMMA_AIR 1.4
#define R_AIR (R_U / MW_AIR)
#define EPS_WENO 1e-40 /* src/WENO.cu:8 */

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static inline long psz(const orc_zone *z, int g) {
  return (long)(z->mx + 2 * g) * (z->my + 2 * g) * (z->mz + 2 * g);
}
/* ggxl::VectorField3D column-major index (src/gxl_lib/Array.cuh:246-322) */
static inline long pidx(const orc_zone *z, int g, int i, int j, int k) {
  return ((long)(k + g) * (z->my + 2 * g) + (j + g)) * (z->mx + 2 * g) + (i + g);
}
static inline long pstride(const orc_zone *z, int g, int dir) {
  if (dir == 0) return 1;
  if (dir == 1) return z->mx + 2 * g;
  return (long)(z->mx + 2 * g) * (z->my + 2 * g);
}

int orc_zone_alloc(orc_zone *z, int mx, int my, int mz, int ngg, int n_var, int n_spec, int n_scalar) {
  memset(z, 0, sizeof(*z));
  z->mx = mx; z->my = my; z->mz = mz; z->ngg = ngg;
  const long P = psz(z, ngg), N = psz(z, 0), P1 = psz(z, 1);
  int ns = n_spec > 0 ? n_spec : 1, nsc = n_scalar > 0 ? n_scalar : 1;
#define AL(ptr, n) do { ptr = (double *)calloc((size_t)(n), sizeof(double)); if (!ptr) return -1; } while (0)
  AL(z->cv, P * n_var); AL(z->bv, P * 6); AL(z->sv, P * nsc); AL(z->qn, P * n_var);
  AL(z->metric, P * 9); AL(z->jac, P); AL(z->mul, P); AL(z->mach, P);
  AL(z->fFlux, P * n_var); AL(z->gFlux, P * n_var); AL(z->hFlux, P * n_var);
  AL(z->acoustic_speed, P); AL(z->gamma, P); AL(z->thermal_conductivity, P);
  AL(z->rho_D, P * ns); AL(z->reaction_timeScale, P);
  AL(z->dq, N * n_var); AL(z->dt_local, N); AL(z->Cn, N * n_var);
  AL(z->vis_flux, P1 * (n_var - 1));
#undef AL
  return 0;
}

void orc_zone_free(orc_zone *z) {
  double *ptrs[] = {z->cv, z->bv, z->sv, z->qn, z->metric, z->jac, z->mul, z->mach, z->fFlux, z->gFlux, z->hFlux,
                    z->acoustic_speed, z->gamma, z->thermal_conductivity, z->rho_D, z->reaction_timeScale,
                    z->dq, z->dt_local, z->Cn, z->vis_flux};
  for (size_t n = 0; n < sizeof(ptrs) / sizeof(ptrs[0]); ++n) free(ptrs[n]);
  memset(z, 0, sizeof(*z));
}

double orc_sutherland(double t) {
  /* src/Transport.cu:6-9 */
  return 1.7894e-5 * pow(t / 288.16, 1.5) * (288.16 + 110) / (t + 110);
}

/* ------------------------------------------------------------------------ */
/* WENO5-JS and WENO7-Z scalar reconstructions, src/WENO.cu:3059-3222        */
/* ------------------------------------------------------------------------ */
double orc_weno5(const double *vp, const double *vm, double eps, int if_shock) {
  const double one6th = 1.0 / 6;
  if (if_shock) {
    double v0 = one6th * (2 * vp[2] + 5 * vp[3] - vp[4]);
    double v1 = one6th * (-vp[1] + 5 * vp[2] + 2 * vp[3]);
    double v2 = one6th * (2 * vp[0] - 7 * vp[1] + 11 * vp[2]);
    const double t12 = 13.0 / 12;
    double beta0 = t12 * (vp[2] + vp[4] - 2 * vp[3]) * (vp[2] + vp[4] - 2 * vp[3]) +
                   0.25 * (3 * vp[2] - 4 * vp[3] + vp[4]) * (3 * vp[2] - 4 * vp[3] + vp[4]);
    double beta1 = t12 * (vp[1] + vp[3] - 2 * vp[2]) * (vp[1] + vp[3] - 2 * vp[2]) +
                   0.25 * (vp[1] - vp[3]) * (vp[1] - vp[3]);
    double beta2 = t12 * (vp[0] + vp[2] - 2 * vp[1]) * (vp[0] + vp[2] - 2 * vp[1]) +
                   0.25 * (vp[0] - 4 * vp[1] + 3 * vp[2]) * (vp[0] - 4 * vp[1] + 3 * vp[2]);
    double a0 = 0.3 / ((eps + beta0) * (eps + beta0));
    double a1 = 0.6 / ((eps + beta1) * (eps + beta1));
    double a2 = 0.1 / ((eps + beta2) * (eps + beta2));
    const double fPlus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);

    v0 = one6th * (11 * vm[2] - 7 * vm[3] + 2 * vm[4]);
    v1 = one6th * (2 * vm[1] + 5 * vm[2] - vm[3]);
    v2 = one6th * (-vm[0] + 5 * vm[1] + 2 * vm[2]);
    beta0 = t12 * (vm[2] + vm[4] - 2 * vm[3]) * (vm[2] + vm[4] - 2 * vm[3]) +
            0.25 * (3 * vm[2] - 4 * vm[3] + vm[4]) * (3 * vm[2] - 4 * vm[3] + vm[4]);
    beta1 = t12 * (vm[1] + vm[3] - 2 * vm[2]) * (vm[1] + vm[3] - 2 * vm[2]) +
            0.25 * (vm[1] - vm[3]) * (vm[1] - vm[3]);
    beta2 = t12 * (vm[0] + vm[2] - 2 * vm[1]) * (vm[0] + vm[2] - 2 * vm[1]) +
            0.25 * (vm[0] - 4 * vm[1] + 3 * vm[2]) * (vm[0] - 4 * vm[1] + 3 * vm[2]);
    a0 = 0.1 / ((eps + beta0) * (eps + beta0));
    a1 = 0.6 / ((eps + beta1) * (eps + beta1));
    a2 = 0.3 / ((eps + beta2) * (eps + beta2));
    const double fMinus = (a0 * v0 + a1 * v1 + a2 * v2) / (a0 + a1 + a2);
    return fPlus + fMinus;
  }
  double v0 = one6th * (2 * vp[2] + 5 * vp[3] - vp[4]);
  double v1 = one6th * (-vp[1] + 5 * vp[2] + 2 * vp[3]);
  double v2 = one6th * (2 * vp[0] - 7 * vp[1] + 11 * vp[2]);
  const double fPlus = 0.3 * v0 + 0.6 * v1 + 0.1 * v2;
  v0 = one6th * (11 * vm[2] - 7 * vm[3] + 2 * vm[4]);
  v1 = one6th * (2 * vm[1] + 5 * vm[2] - vm[3]);
  v2 = one6th * (-vm[0] + 5 * vm[1] + 2 * vm[2]);
  const double fMinus = 0.1 * v0 + 0.6 * v1 + 0.3 * v2;
  return fPlus + fMinus;
}

static inline double weno7_beta(double s1, double s2, double s3) {
  const double d12 = 13.0 / 12.0, d13 = 1043.0 / 960, d14 = 1.0 / 12;
  return s1 * s1 + d12 * s2 * s2 + d13 * s3 * s3 + d14 * s1 * s3;
}

double orc_weno7(const double *vp, const double *vm, double eps, int if_shock) {
  const double one6th = 1.0 / 6, one12th = 1.0 / 12;
  const double c0 = 1.0 / 35, c1 = 12.0 / 35, c2 = 18.0 / 35, c3 = 4.0 / 35;
  if (if_shock) {
    double s1 = one6th * (-2 * vp[0] + 9 * vp[1] - 18 * vp[2] + 11 * vp[3]);
    double s2 = -vp[0] + 4 * vp[1] - 5 * vp[2] + 2 * vp[3];
    double s3 = -vp[0] + 3 * vp[1] - 3 * vp[2] + vp[3];
    double beta0 = weno7_beta(s1, s2, s3);
    s1 = one6th * (vp[1] - 6 * vp[2] + 3 * vp[3] + 2 * vp[4]);
    s2 = vp[2] - 2 * vp[3] + vp[4];
    s3 = -vp[1] + 3 * vp[2] - 3 * vp[3] + vp[4];
    double beta1 = weno7_beta(s1, s2, s3);
    /* the reference reuses s2 of stencil 1 for stencil 2 (src/WENO.cu:3137-3139) */
    s1 = one6th * (-2 * vp[2] - 3 * vp[3] + 6 * vp[4] - vp[5]);
    s3 = -vp[2] + 3 * vp[3] - 3 * vp[4] + vp[5];
    double beta2 = weno7_beta(s1, s2, s3);
    s1 = one6th * (-11 * vp[3] + 18 * vp[4] - 9 * vp[5] + 2 * vp[6]);
    s2 = 2 * vp[3] - 5 * vp[4] + 4 * vp[5] - vp[6];
    s3 = -vp[3] + 3 * vp[4] - 3 * vp[5] + vp[6];
    double beta3 = weno7_beta(s1, s2, s3);
    double tau = beta0 + 3 * beta1 - 3 * beta2 - beta3;
    tau *= tau;
    double a0 = c0 + c0 * tau / ((eps + beta0) * (eps + beta0));
    double a1 = c1 + c1 * tau / ((eps + beta1) * (eps + beta1));
    double a2 = c2 + c2 * tau / ((eps + beta2) * (eps + beta2));
    double a3 = c3 + c3 * tau / ((eps + beta3) * (eps + beta3));
    double v0 = -3 * vp[0] + 13 * vp[1] - 23 * vp[2] + 25 * vp[3];
    double v1 = vp[1] - 5 * vp[2] + 13 * vp[3] + 3 * vp[4];
    double v2 = -vp[2] + 7 * vp[3] + 7 * vp[4] - vp[5];
    double v3 = 3 * vp[3] + 13 * vp[4] - 5 * vp[5] + vp[6];
    const double fPlus = one12th * (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);

    s1 = one6th * (-2 * vm[6] + 9 * vm[5] - 18 * vm[4] + 11 * vm[3]);
    s2 = -vm[6] + 4 * vm[5] - 5 * vm[4] + 2 * vm[3];
    s3 = -vm[6] + 3 * vm[5] - 3 * vm[4] + vm[3];
    beta0 = weno7_beta(s1, s2, s3);
    s1 = one6th * (vm[5] - 6 * vm[4] + 3 * vm[3] + 2 * vm[2]);
    s2 = vm[4] - 2 * vm[3] + vm[2];
    s3 = -vm[5] + 3 * vm[4] - 3 * vm[3] + vm[2];
    beta1 = weno7_beta(s1, s2, s3);
    s1 = one6th * (-2 * vm[4] - 3 * vm[3] + 6 * vm[2] - vm[1]);
    s3 = -vm[4] + 3 * vm[3] - 3 * vm[2] + vm[1];
    beta2 = weno7_beta(s1, s2, s3);
    s1 = one6th * (-11 * vm[3] + 18 * vm[2] - 9 * vm[1] + 2 * vm[0]);
    s2 = 2 * vm[3] - 5 * vm[2] + 4 * vm[1] - vm[0];
    s3 = -vm[3] + 3 * vm[2] - 3 * vm[1] + vm[0];
    beta3 = weno7_beta(s1, s2, s3);
    tau = beta0 + 3 * beta1 - 3 * beta2 - beta3;
    tau *= tau;
    a0 = c0 + c0 * tau / ((eps + beta0) * (eps + beta0));
    a1 = c1 + c1 * tau / ((eps + beta1) * (eps + beta1));
    a2 = c2 + c2 * tau / ((eps + beta2) * (eps + beta2));
    a3 = c3 + c3 * tau / ((eps + beta3) * (eps + beta3));
    v0 = -3 * vm[6] + 13 * vm[5] - 23 * vm[4] + 25 * vm[3];
    v1 = vm[5] - 5 * vm[4] + 13 * vm[3] + 3 * vm[2];
    v2 = -vm[4] + 7 * vm[3] + 7 * vm[2] - vm[1];
    v3 = 3 * vm[3] + 13 * vm[2] - 5 * vm[1] + vm[0];
    const double fMinus = one12th * (a0 * v0 + a1 * v1 + a2 * v2 + a3 * v3) / (a0 + a1 + a2 + a3);
    return fPlus + fMinus;
  }
  double v3 = 3 * vp[3] + 13 * vp[4] - 5 * vp[5] + vp[6];
  double v2 = -vp[2] + 7 * vp[3] + 7 * vp[4] - vp[5];
  double v1 = vp[1] - 5 * vp[2] + 13 * vp[3] + 3 * vp[4];
  double v0 = -3 * vp[0] + 13 * vp[1] - 23 * vp[2] + 25 * vp[3];
  const double fPlus = one12th * (c0 * v0 + c1 * v1 + c2 * v2 + c3 * v3);
  v0 = -3 * vm[6] + 13 * vm[5] - 23 * vm[4] + 25 * vm[3];
  v1 = vm[5] - 5 * vm[4] + 13 * vm[3] + 3 * vm[2];
  v2 = -vm[4] + 7 * vm[3] + 7 * vm[2] - vm[1];
  v3 = 3 * vm[3] + 13 * vm[2] - 5 * vm[1] + vm[0];
  const double fMinus = one12th * (c0 * v0 + c1 * v1 + c2 * v2 + c3 * v3);
  return fPlus + fMinus;
}

/* ------------------------------------------------------------------------ */
/* Inviscid WENO flux at face (node idx, node idx+s) in direction dir.        */
/* Component-wise LLF (51/71): src/WENO.cu:890-1089.                         */
/* Characteristic (52/72), air: src/WENO.cu:1090-1138 + weno_ch_air_x/_yz    */
/* (src/WENO.cu:10-244, 414-654).  Mixture branch lives in oracle_mix.c.      */
/* ------------------------------------------------------------------------ */
void orc_weno_face_mixture(const orc_zone *z, const orc_param *p, int dir, long idx, double kx, double ky,
                           double kz, double eps_ref, int if_shock, double *fc);

static void weno_face_air_or_cp(const orc_zone *z, const orc_param *p, int dir, long idx, double kx, double ky,
                                double kz, double eps_ref, int if_shock, double *fc) {
  const int ngg = z->ngg, nv = p->n_var, sch = p->inviscid_scheme;
  const long sz = psz(z, ngg), s = pstride(z, ngg, dir);
  const int mm = 3 * dir;
  const int order7 = (sch == 71 || sch == 72);
  const int lo = order7 ? -3 : -2, hi = order7 ? 4 : 3; /* stencil point offsets */
  const int np = hi - lo + 1;

  if (sch == 51 || sch == 71) {
    double fp[ORC_MAX_SPEC + 5][8], fm[ORC_MAX_SPEC + 5][8];
    for (int m = 0; m < np; ++m) {
      const long id = idx + (long)(lo + m) * s;
      const double q0 = z->cv[id], q1 = z->cv[id + sz], q2 = z->cv[id + 2 * sz], q3 = z->cv[id + 3 * sz],
                   q4 = z->cv[id + 4 * sz];
      double pk = z->bv[id + 4 * sz];
      const double m0 = z->metric[id + mm * sz], m1 = z->metric[id + (mm + 1) * sz], m2 = z->metric[id + (mm + 2) * sz];
      const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
      double cGradK = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
      if (p->mech) cGradK *= z->acoustic_speed[id];
      else cGradK *= sqrt(GAMMA_AIR * R_AIR * z->bv[id + 5 * sz]);
      const double lambda0 = fabs(Uk) + cGradK;
      const double jac = z->jac[id];
      const double sPlus = 0.5 * jac * (Uk + lambda0);
      const double sMinus = 0.5 * jac * (Uk - lambda0);
      pk *= 0.5 * jac;
      fp[0][m] = sPlus * q0;
      fp[1][m] = fma(sPlus, q1, pk * m0);
      fp[2][m] = fma(sPlus, q2, pk * m1);
      fp[3][m] = fma(sPlus, q3, pk * m2);
      fp[4][m] = fma(sPlus, q4, pk * Uk);
      fm[0][m] = sMinus * q0;
      fm[1][m] = fma(sMinus, q1, pk * m0);
      fm[2][m] = fma(sMinus, q2, pk * m1);
      fm[3][m] = fma(sMinus, q3, pk * m2);
      fm[4][m] = fma(sMinus, q4, pk * Uk);
      for (int l = 5; l < nv; ++l) {
        const double ql = z->cv[id + l * sz];
        fp[l][m] = sPlus * ql;
        fm[l][m] = sMinus * ql;
      }
    }
    double eps_scaled[3];
    eps_scaled[0] = eps_ref;
    eps_scaled[1] = eps_ref * p->v_ref * p->v_ref;
    eps_scaled[2] = eps_scaled[1] * p->v_ref * p->v_ref;
    for (int l = 0; l < nv; ++l) {
      double eps_here = eps_scaled[0];
      if (l == 1 || l == 2 || l == 3) eps_here = eps_scaled[1];
      else if (l == 4) eps_here = eps_scaled[2];
      if (order7) {
        /* vp = fp[i-3..i+3], vm = fm[i-2..i+4]; point m corresponds to offset m-3 */
        fc[l] = orc_weno7(&fp[l][0], &fm[l][1], eps_here, if_shock);
      } else {
        fc[l] = orc_weno5(&fp[l][0], &fm[l][1], eps_here, if_shock);
      }
    }
    return;
  }

  if (p->mech) {
    orc_weno_face_mixture(z, p, dir, idx, kx, ky, kz, eps_ref, if_shock, fc);
    return;
  }

  /* characteristic, air */
  double Q[5][8], F[7][8];
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
    F[5][m] = sqrt(m0 * m0 + m1 * m1 + m2 * m2) * sqrt(GAMMA_AIR * R_AIR * z->bv[id + 5 * sz]);
    F[6][m] = z->jac[id];
  }
  const int c = -lo; /* local index of node i */
  const double rho_l = Q[0][c], rho_r = Q[0][c + 1];
  double temp1 = sqrt(rho_l * rho_r);
  const double rlc = 1 / (rho_l + temp1);
  const double rrc = 1 / (temp1 + rho_r);
  const double um = rlc * Q[1][c] + rrc * Q[1][c + 1];
  const double vm = rlc * Q[2][c] + rrc * Q[2][c + 1];
  const double wm = rlc * Q[3][c] + rrc * Q[3][c + 1];
  double temp3 = (rlc * F[4][c] + rrc * F[4][c + 1]) / R_AIR;
  const double cm = sqrt(GAMMA_AIR * R_AIR * temp3);
  const double gm1 = GAMMA_AIR - 1;

  temp1 = 1.0 / sqrt(kx * kx + ky * ky + kz * kz);
  kx *= temp1; ky *= temp1; kz *= temp1;
  const double Uk_bar = kx * um + ky * vm + kz * wm;
  double nx = 0, ny = 0, nz = 0, qx, qy, qz;
  if (fabs(kx) > 0.8) { nx = -kz; nz = kx; }
  else { ny = kz; nz = -ky; }
  temp1 = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= temp1; ny *= temp1; nz *= temp1;
  qx = ky * nz - kz * ny;
  qy = kz * nx - kx * nz;
  qz = kx * ny - ky * nx;
  temp1 = 1.0 / sqrt(qx * qx + qy * qy + qz * qz);
  qx *= temp1; qy *= temp1; qz *= temp1;
  const double Un = nx * um + ny * vm + nz * wm;
  const double Uq = qx * um + qy * vm + qz * wm;
  double temp2 = 1.0 / (cm * cm);
  temp3 = 0.5 * gm1 * (um * um + vm * vm + wm * wm);

  double max_lambda = 0;
  for (int m = 0; m < np; ++m) {
    const double lam = fabs(F[0][m]) + F[5][m];
    if (lam > max_lambda) max_lambda = lam;
  }
  double fChar[5];
  for (int l = 0; l < 5; ++l) {
    double L[5];
    switch (l) {
      case 0:
        L[0] = (temp3 + Uk_bar * cm) * temp2 * 0.5;
        L[1] = -(gm1 * um + kx * cm) * temp2 * 0.5;
        L[2] = -(gm1 * vm + ky * cm) * temp2 * 0.5;
        L[3] = -(gm1 * wm + kz * cm) * temp2 * 0.5;
        L[4] = gm1 * temp2 * 0.5;
        break;
      case 1:
        L[0] = -Un; L[1] = nx; L[2] = ny; L[3] = nz; L[4] = 0;
        break;
      case 2:
        L[0] = -Uq; L[1] = qx; L[2] = qy; L[3] = qz; L[4] = 0;
        break;
      case 3:
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
                         L[4] * ((Q[4][m] + F[4][m]) * F[0][m]);
      const double LQm = L[0] * Q[0][m] + L[1] * Q[1][m] + L[2] * Q[2][m] + L[3] * Q[3][m] + L[4] * Q[4][m];
      if (m < np - 1) vPlus[m] = 0.5 * F[6][m] * (LFm + max_lambda * LQm);
      if (m > 0) vMinus[m - 1] = 0.5 * F[6][m] * (LFm - max_lambda * LQm);
    }
    fChar[l] = order7 ? orc_weno7(vPlus, vMinus, eps_ref, if_shock) : orc_weno5(vPlus, vMinus, eps_ref, if_shock);
  }
  temp1 = fChar[0] + fChar[3] + fChar[4];
  temp3 = fChar[0] - fChar[4];
  fc[0] = temp1;
  fc[1] = um * temp1 - kx * cm * temp3 + nx * fChar[1] + qx * fChar[2];
  fc[2] = vm * temp1 - ky * cm * temp3 + ny * fChar[1] + qy * fChar[2];
  fc[3] = wm * temp1 - kz * cm * temp3 + nz * fChar[1] + qz * fChar[2];
  temp2 = rlc * (Q[4][c] + F[4][c]) + rrc * (Q[4][c + 1] + F[4][c + 1]);
  fc[4] = temp2 * temp1 - Uk_bar * cm * temp3 + Un * fChar[1] + Uq * fChar[2] - cm * cm / gm1 * fChar[3];
}

void orc_positive_preserving_face(const orc_zone *z, const orc_param *p, int dir, int i, int j, int k, double *fc);

/* compute_convective_term_weno (src/WENO.cu:2914-2946): x, y, z face fluxes then
 * compute_derivative_{x,y,z} (src/WENO.cu:1544, 2219, 2885). */
static void weno_direction(orc_zone *z, const orc_param *p, int dir) {
  const int ngg = z->ngg, nv = p->n_var, mx = z->mx, my = z->my, mz = z->mz;
  const long sz = psz(z, ngg), s = pstride(z, ngg, dir);
  const double eps_ref = EPS_WENO * p->weno_eps_scale;
  double *flux = dir == 0 ? z->fFlux : (dir == 1 ? z->gFlux : z->hFlux);
  const int mm = 3 * dir;
  const int i0 = dir == 0 ? -1 : 0, j0 = dir == 1 ? -1 : 0, k0 = dir == 2 ? -1 : 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < mz; ++k) {
    for (int j = j0; j < my; ++j) {
      for (int i = i0; i < mx; ++i) {
        const long id = pidx(z, ngg, i, j, k);
        /* face normal: x averages with i+1; y and z also average with (i+1,j,k)
         * exactly as the reference does (src/WENO.cu:1627-1629, 2303-2305). */
        const long idn = id + 1;
        const double kx = 0.5 * (z->metric[id + mm * sz] + z->metric[idn + mm * sz]);
        const double ky = 0.5 * (z->metric[id + (mm + 1) * sz] + z->metric[idn + (mm + 1) * sz]);
        const double kz = 0.5 * (z->metric[id + (mm + 2) * sz] + z->metric[idn + (mm + 2) * sz]);
        /* hybrid scheme: linear weights unless a node of the stencil is
         * shocked (src/WENO.cu:839-849, 1580-1590 and the z analogue) */
        int if_shock = 1;
        if (p->sensor_threshold > 1e-10) {
          if_shock = 0;
          for (int ii = -ngg + 1; ii <= ngg; ++ii)
            if (z->shock_sensor[id + ii * s] > p->sensor_threshold) { if_shock = 1; break; }
        }
        double fc[ORC_MAX_SPEC + 5];
        weno_face_air_or_cp(z, p, dir, id, kx, ky, kz, eps_ref, if_shock, fc);
        /* characteristic WENO: the limiter exists in the x sweep only
         * (src/WENO.cu:1471-1540; the y and z sweeps have none) */
        if (p->positive_preserving && nv > 5 && dir == 0) orc_positive_preserving_face(z, p, dir, i, j, k, fc);
        for (int l = 0; l < nv; ++l) flux[id + l * sz] = fc[l];
      }
    }
  }
  /* derivative: dq -= F(i) - F(i-1) */
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

void orc_roe_like_inviscid(orc_zone *z, const orc_param *p);

void orc_compute_inviscid_flux(orc_zone *z, const orc_param *p) {
  const int sch = p->inviscid_scheme;
  if (sch == 51 || sch == 52 || sch == 71 || sch == 72) {
    weno_direction(z, p, 0);
    weno_direction(z, p, 1);
    if (z->mz > 1) weno_direction(z, p, 2);
  } else {
    orc_roe_like_inviscid(z, p);
  }
}

/* ------------------------------------------------------------------------ */
/* Second-order viscous flux, air branch and mixture hook:                   */
/* compute_fv/gv/hv_2nd_order + compute_dFv_dx/dGv_dy/dHv_dz                 */
/* (src/ViscousScheme.cu:75-127, 614-1173).                                  */
/* ------------------------------------------------------------------------ */
void orc_viscous_species_face(const orc_zone *z, const orc_param *p, int dir, int i, int j, int k,
                              const double gm[9], const double gradk_div_jac[3], double *fv_out);

static void viscous_direction(orc_zone *z, const orc_param *p, int dir) {
  const int ngg = z->ngg, nv = p->n_var, mx = z->mx, my = z->my, mz = z->mz;
  const long sz = psz(z, ngg), szv = psz(z, 1);
  const long sd = pstride(z, ngg, dir);
  const int i0 = dir == 0 ? -1 : 0, j0 = dir == 1 ? -1 : 0, k0 = dir == 2 ? -1 : 0;
  const int da = (dir + 1) % 3, db = (dir + 2) % 3; /* the two cross directions */
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = k0; k < mz; ++k) {
    for (int j = j0; j < my; ++j) {
      for (int i = i0; i < mx; ++i) {
        const long id = pidx(z, ngg, i, j, k), idn = id + sd;
        double gm[9];
        for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (z->metric[id + l * sz] + z->metric[idn + l * sz]);
        const double *pv = z->bv;
        /* derivative of variable at slot v with respect to xi, eta, zeta at the face */
        double d[4][3]; /* u, v, w, T */
        const int slots[4] = {1, 2, 3, 5};
        for (int a = 0; a < 4; ++a) {
          const double *f = pv + slots[a] * sz;
          double dd[3];
          dd[dir] = f[idn] - f[id];
          const int cr[2] = {da, db};
          for (int c = 0; c < 2; ++c) {
            const long sc = pstride(z, ngg, cr[c]);
            /* the reference orders the terms as (n,+)-(n,-)+(n+1,+)-(n+1,-) */
            dd[cr[c]] = 0.25 * (f[id + sc] - f[id - sc] + f[idn + sc] - f[idn - sc]);
          }
          d[a][0] = dd[0]; d[a][1] = dd[1]; d[a][2] = dd[2];
        }
        const double xi_x = gm[0], xi_y = gm[1], xi_z = gm[2], eta_x = gm[3], eta_y = gm[4], eta_z = gm[5],
                     zeta_x = gm[6], zeta_y = gm[7], zeta_z = gm[8];
        const double u_x = d[0][0] * xi_x + d[0][1] * eta_x + d[0][2] * zeta_x;
        const double u_y = d[0][0] * xi_y + d[0][1] * eta_y + d[0][2] * zeta_y;
        const double u_z = d[0][0] * xi_z + d[0][1] * eta_z + d[0][2] * zeta_z;
        const double v_x = d[1][0] * xi_x + d[1][1] * eta_x + d[1][2] * zeta_x;
        const double v_y = d[1][0] * xi_y + d[1][1] * eta_y + d[1][2] * zeta_y;
        const double v_z = d[1][0] * xi_z + d[1][1] * eta_z + d[1][2] * zeta_z;
        const double w_x = d[2][0] * xi_x + d[2][1] * eta_x + d[2][2] * zeta_x;
        const double w_y = d[2][0] * xi_y + d[2][1] * eta_y + d[2][2] * zeta_y;
        const double w_z = d[2][0] * xi_z + d[2][1] * eta_z + d[2][2] * zeta_z;
        const double mul = 0.5 * (z->mul[id] + z->mul[idn]);
        const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
        const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
        const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
        const double tau_xy = mul * (u_y + v_x);
        const double tau_xz = mul * (u_z + w_x);
        const double tau_yz = mul * (v_z + w_y);
        const int mm = 3 * dir;
        double gk[3];
        for (int c = 0; c < 3; ++c)
          gk[c] = 0.5 * (z->metric[id + (mm + c) * sz] * z->jac[id] + z->metric[idn + (mm + c) * sz] * z->jac[idn]);
        const long iv = pidx(z, 1, i, j, k);
        double fv[ORC_MAX_SPEC + 4];
        fv[0] = gk[0] * tau_xx + gk[1] * tau_xy + gk[2] * tau_xz;
        fv[1] = gk[0] * tau_xy + gk[1] * tau_yy + gk[2] * tau_yz;
        fv[2] = gk[0] * tau_xz + gk[1] * tau_yz + gk[2] * tau_zz;
        const double umv = 0.5 * (pv[id + sz] + pv[idn + sz]);
        const double vmv = 0.5 * (pv[id + 2 * sz] + pv[idn + 2 * sz]);
        const double wmv = 0.5 * (pv[id + 3 * sz] + pv[idn + 3 * sz]);
        const double t_x = d[3][0] * xi_x + d[3][1] * eta_x + d[3][2] * zeta_x;
        const double t_y = d[3][0] * xi_y + d[3][1] * eta_y + d[3][2] * zeta_y;
        const double t_z = d[3][0] * xi_z + d[3][1] * eta_z + d[3][2] * zeta_z;
        double conductivity;
        if (p->mech) {
          conductivity = 0.5 * (z->thermal_conductivity[id] + z->thermal_conductivity[idn]);
        } else {
          const double cp = GAMMA_AIR * R_AIR / (GAMMA_AIR - 1);
          conductivity = mul / p->Pr * cp;
        }
        fv[3] = umv * fv[0] + vmv * fv[1] + wmv * fv[2] + conductivity * (gk[0] * t_x + gk[1] * t_y + gk[2] * t_z);
        if (p->mech) orc_viscous_species_face(z, p, dir, i, j, k, gm, gk, fv);
        for (int l = 0; l < nv - 1; ++l) z->vis_flux[iv + l * szv] = fv[l];
      }
    }
  }
  const long szq = psz(z, 0), sv1 = pstride(z, 1, dir);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k) {
    for (int j = 0; j < my; ++j) {
      for (int i = 0; i < mx; ++i) {
        const long iq = pidx(z, 0, i, j, k), ic = pidx(z, 1, i, j, k), im = ic - sv1;
        for (int l = 1; l < nv; ++l) z->dq[iq + l * szq] += z->vis_flux[ic + (l - 1) * szv] - z->vis_flux[im + (l - 1) * szv];
      }
    }
  }
}

void orc_viscous_flux_8th(orc_zone *z, const orc_param *p);

void orc_compute_viscous_flux(orc_zone *z, const orc_param *p) {
  if (p->viscous_order == 8 || p->viscous_order == 4) {
    orc_viscous_flux_8th(z, p);
    return;
  }
  if (p->viscous_order != 2) return;
  viscous_direction(z, p, 0);
  viscous_direction(z, p, 1);
  if (z->mz > 1) viscous_direction(z, p, 2);
}

/* ------------------------------------------------------------------------ */
/* Stage update (src/RK.cuh:11-15, 224-281).                                 */
/* ------------------------------------------------------------------------ */
static const double RK_A[3] = {1.0, 0.75, 1.0 / 3.0};
static const double RK_B[3] = {0.0, 0.25, 2.0 / 3.0};
static const double RK_C[3] = {1.0, 0.25, 2.0 / 3.0};

void orc_temperature_and_pressure(orc_zone *z, const orc_param *p, long id, double total_energy);

static void update_cv_and_bv(orc_zone *z, const orc_param *p, double dt, int rk, int minus_cn);

void orc_update_cv_and_bv_rk(orc_zone *z, const orc_param *p, double dt, int rk) { update_cv_and_bv(z, p, dt, rk, 0); }

/* update_cv_and_bv_rk_wu (src/StrangSplitting.cu:504-562): the same update
 * with dq - Cn, the transport part frozen at the start of the step. */
void orc_update_cv_and_bv_rk_wu(orc_zone *z, const orc_param *p, double dt, int rk) {
  update_cv_and_bv(z, p, dt, rk, 1);
}

static void update_cv_and_bv(orc_zone *z, const orc_param *p, double dt, int rk, int minus_cn) {
  const int ngg = z->ngg, nv = p->n_var, mx = z->mx, my = z->my, mz = z->mz;
  const long sz = psz(z, ngg), szq = psz(z, 0);
  const int ns = p->n_spec;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k) {
    for (int j = 0; j < my; ++j) {
      for (int i = 0; i < mx; ++i) {
        const long id = pidx(z, ngg, i, j, k), iq = pidx(z, 0, i, j, k);
        double *cv = z->cv, *bv = z->bv, *sv = z->sv;
        const double dt_div_jac = dt / z->jac[id];
        for (int l = 0; l < nv; ++l) {
          const double r = minus_cn ? z->dq[iq + l * szq] - z->Cn[iq + l * szq] : z->dq[iq + l * szq];
          cv[id + l * sz] = RK_A[rk] * z->qn[id + l * sz] + RK_B[rk] * cv[id + l * sz] + RK_C[rk] * dt_div_jac * r;
        }
        if (mz == 1) cv[id + 3 * sz] = 0;
        bv[id] = cv[id];
        const double density_inv = 1.0 / cv[id];
        bv[id + sz] = cv[id + sz] * density_inv;
        bv[id + 2 * sz] = cv[id + 2 * sz] * density_inv;
        bv[id + 3 * sz] = cv[id + 3 * sz] * density_inv;
        const double V2 = bv[id + sz] * bv[id + sz] + bv[id + 2 * sz] * bv[id + 2 * sz] + bv[id + 3 * sz] * bv[id + 3 * sz];
        double sum_part_den = 0;
        for (int l = 0; l < ns; ++l) {
          if (cv[id + (5 + l) * sz] < 0) cv[id + (5 + l) * sz] = 0;
          else sum_part_den += cv[id + (l + 5) * sz];
        }
        sum_part_den = 1.0 / sum_part_den;
        const double denComDivDenReal = cv[id] * sum_part_den;
        for (int l = 0; l < ns; ++l) {
          sv[id + l * sz] = cv[id + (5 + l) * sz] * sum_part_den;
          cv[id + (5 + l) * sz] *= denComDivDenReal;
        }
        for (int l = ns; l < p->n_scalar; ++l) sv[id + l * sz] = cv[id + (5 + l) * sz] * density_inv;
        if (p->mech) {
          orc_temperature_and_pressure(z, p, id, cv[id + 4 * sz]);
        } else {
          bv[id + 4 * sz] = (GAMMA_AIR - 1) * (cv[id + 4 * sz] - 0.5 * bv[id] * V2);
          bv[id + 5 * sz] = bv[id + 4 * sz] * MW_AIR * density_inv / R_U;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* cv from bv over the padded domain (src/FieldOperation.cuh:16-64)           */
/* ------------------------------------------------------------------------ */
void orc_total_energy_mixture(orc_zone *z, const orc_param *p, long id);

static void cv_from_bv_point(orc_zone *z, const orc_param *p, long id) {
  const long sz = psz(z, z->ngg);
  double *cv = z->cv, *bv = z->bv;
  const double rho = bv[id];
  cv[id] = rho;
  cv[id + sz] = rho * bv[id + sz];
  cv[id + 2 * sz] = rho * bv[id + 2 * sz];
  cv[id + 3 * sz] = rho * bv[id + 3 * sz];
  for (int l = 0; l < p->n_scalar; ++l) cv[id + (5 + l) * sz] = rho * z->sv[id + l * sz];
  if (p->mech) {
    orc_total_energy_mixture(z, p, id);
  } else {
    const double V2 = bv[id + sz] * bv[id + sz] + bv[id + 2 * sz] * bv[id + 2 * sz] + bv[id + 3 * sz] * bv[id + 3 * sz];
    double total_energy = 0.5 * V2;
    total_energy *= bv[id];
    total_energy += bv[id + 4 * sz] / (GAMMA_AIR - 1);
    cv[id + 4 * sz] = total_energy;
  }
}

void orc_compute_cv_from_bv(orc_zone *z, const orc_param *p) {
  const int g = z->ngg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -g; k < z->mz + g; ++k)
    for (int j = -g; j < z->my + g; ++j)
      for (int i = -g; i < z->mx + g; ++i) cv_from_bv_point(z, p, pidx(z, g, i, j, k));
}

/* ------------------------------------------------------------------------ */
/* update_physical_properties, air branch (src/FieldOperation.cuh:86-120)    */
/* ------------------------------------------------------------------------ */
void orc_update_physical_properties_mixture_point(orc_zone *z, const orc_param *p, long id);

void orc_update_physical_properties(orc_zone *z, const orc_param *p) {
  const int g = z->ngg;
  const long sz = psz(z, g);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = -g; k < z->mz + g; ++k)
    for (int j = -g; j < z->my + g; ++j)
      for (int i = -g; i < z->mx + g; ++i) {
        const long id = pidx(z, g, i, j, k);
        if (p->mech) {
          orc_update_physical_properties_mixture_point(z, p, id);
          continue;
        }
        const double t = z->bv[id + 5 * sz];
        const double u = z->bv[id + sz], v = z->bv[id + 2 * sz], w = z->bv[id + 3 * sz];
        const double V = sqrt(u * u + v * v + w * w);
        const double c_temp = GAMMA_AIR * R_U / MW_AIR;
        z->mul[id] = orc_sutherland(t);
        z->mach[id] = V / sqrt(c_temp * t);
      }
}

/* ------------------------------------------------------------------------ */
/* local and global time step (src/TimeAdvanceFunc.cuh:28-115,               */
/* src/TimeAdvanceFunc.cu:102-152)                                           */
/* ------------------------------------------------------------------------ */
double orc_mixture_max_diffuse_vel(const orc_zone *z, const orc_param *p, long id);

static void local_time_step(orc_zone *z, const orc_param *p, int with_reaction);

void orc_local_time_step(orc_zone *z, const orc_param *p) { local_time_step(z, p, 1); }

/* local_time_step_without_reaction (src/TimeAdvanceFunc.cu:21-100) */
void orc_local_time_step_without_reaction(orc_zone *z, const orc_param *p) { local_time_step(z, p, 0); }

static void local_time_step(orc_zone *z, const orc_param *p, int with_reaction) {
  const int g = z->ngg, mx = z->mx, my = z->my, mz = z->mz;
  const long sz = psz(z, g);
  const int dim = mz == 1 ? 2 : 3;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k)
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        const long id = pidx(z, g, i, j, k);
        const double *mt = z->metric;
        const double grad_xi = sqrt(mt[id] * mt[id] + mt[id + sz] * mt[id + sz] + mt[id + 2 * sz] * mt[id + 2 * sz]);
        const double grad_eta = sqrt(mt[id + 3 * sz] * mt[id + 3 * sz] + mt[id + 4 * sz] * mt[id + 4 * sz] +
                                     mt[id + 5 * sz] * mt[id + 5 * sz]);
        const double grad_zeta = sqrt(mt[id + 6 * sz] * mt[id + 6 * sz] + mt[id + 7 * sz] * mt[id + 7 * sz] +
                                      mt[id + 8 * sz] * mt[id + 8 * sz]);
        const double u = z->bv[id + sz], v = z->bv[id + 2 * sz], w = z->bv[id + 3 * sz];
        const double U = u * mt[id] + v * mt[id + sz] + w * mt[id + 2 * sz];
        const double V = u * mt[id + 3 * sz] + v * mt[id + 4 * sz] + w * mt[id + 5 * sz];
        const double W = u * mt[id + 6 * sz] + v * mt[id + 7 * sz] + w * mt[id + 8 * sz];
        double a;
        if (p->mech) a = z->acoustic_speed[id];
        else a = sqrt(GAMMA_AIR * R_AIR * z->bv[id + 5 * sz]);
        const double r0 = fabs(U) + a * grad_xi;
        const double r1 = fabs(V) + a * grad_eta;
        double max_sr = r0 > r1 ? r0 : r1;
        if (dim == 3) {
          const double r2 = fabs(W) + a * grad_zeta;
          max_sr = max_sr > r2 ? max_sr : r2;
        }
        if (p->viscous_order > 0) {
          double max_length = grad_xi;
          max_length = max_length > grad_eta ? max_length : grad_eta;
          if (dim == 3) max_length = max_length > grad_zeta ? max_length : grad_zeta;
          double mdv;
          const double iRho = 1.0 / z->bv[id];
          if (p->mech) {
            mdv = orc_mixture_max_diffuse_vel(z, p, id);
          } else {
            mdv = (GAMMA_AIR > 4.0 / 3.0 ? GAMMA_AIR : 4.0 / 3.0) * iRho;
            mdv *= z->mul[id] / p->Pr;
          }
          const double vr = max_length * max_length * mdv;
          max_sr = max_sr > vr ? max_sr : vr;
        }
        double dt = p->cfl / max_sr;
        if (with_reaction && p->mech && p->n_reac > 0) {
          const double reaction_dt = p->cfl * z->reaction_timeScale[id];
          if (reaction_dt > 1e-20 && reaction_dt < 1e-5) dt = dt < reaction_dt ? dt : reaction_dt;
        }
        z->dt_local[pidx(z, 0, i, j, k)] = dt;
      }
}

/* ------------------------------------------------------------------------ */
/* Shock sensors (src/FieldOperation.cu:74-179)                               */
/* ------------------------------------------------------------------------ */
static double ducros_sensor(const orc_zone *z, double eps, long id) {
  const long sz = psz(z, z->ngg);
  const long si = 1, sj = pstride(z, z->ngg, 1), sk = pstride(z, z->ngg, 2);
  const double *mt = z->metric, *bv = z->bv;
  const double xi_x = mt[id], xi_y = mt[id + sz], xi_z = mt[id + 2 * sz];
  const double eta_x = mt[id + 3 * sz], eta_y = mt[id + 4 * sz], eta_z = mt[id + 5 * sz];
  const double zeta_x = mt[id + 6 * sz], zeta_y = mt[id + 7 * sz], zeta_z = mt[id + 8 * sz];
  const double oneD12 = 1.0 / 12.0, twoD3 = 2.0 / 3.0;
  double d[3][3];
  for (int v = 0; v < 3; ++v) {
    const double *f = bv + (v + 1) * sz;
    const long st[3] = {si, sj, sk};
    for (int a = 0; a < 3; ++a)
      d[v][a] = oneD12 * f[id - 2 * st[a]] - twoD3 * f[id - st[a]] + twoD3 * f[id + st[a]] - oneD12 * f[id + 2 * st[a]];
  }
  const double duDx = d[0][0] * xi_x + d[0][1] * eta_x + d[0][2] * zeta_x;
  const double dvDy = d[1][0] * xi_y + d[1][1] * eta_y + d[1][2] * zeta_y;
  const double dwDz = d[2][0] * xi_z + d[2][1] * eta_z + d[2][2] * zeta_z;
  double divV2 = duDx + dvDy + dwDz;
  if (divV2 > 0) return 0;
  const double duDy = d[0][0] * xi_y + d[0][1] * eta_y + d[0][2] * zeta_y;
  const double duDz = d[0][0] * xi_z + d[0][1] * eta_z + d[0][2] * zeta_z;
  const double dvDx = d[1][0] * xi_x + d[1][1] * eta_x + d[1][2] * zeta_x;
  const double dvDz = d[1][0] * xi_z + d[1][1] * eta_z + d[1][2] * zeta_z;
  const double dwDx = d[2][0] * xi_x + d[2][1] * eta_x + d[2][2] * zeta_x;
  const double dwDy = d[2][0] * xi_y + d[2][1] * eta_y + d[2][2] * zeta_y;
  divV2 *= divV2;
  const double curl2 = (dwDy - dvDz) * (dwDy - dvDz) + (duDz - dwDx) * (duDz - dwDx) + (dvDx - duDy) * (dvDx - duDy);
  return divV2 / (divV2 + curl2 + eps);
}

static double jameson_sensor(const orc_zone *z, long id) {
  const long sz = psz(z, z->ngg), sj = pstride(z, z->ngg, 1), sk = pstride(z, z->ngg, 2);
  const double *p = z->bv + 4 * sz;
  const double twoP = p[id] * 2;
  const double pI = p[id + 1] + p[id - 1], pJ = p[id + sj] + p[id - sj], pK = p[id + sk] + p[id - sk];
  return fabs(pI - twoP) / (pI + twoP) + fabs(pJ - twoP) / (pJ + twoP) + fabs(pK - twoP) / (pK + twoP);
}

static double jump_sensor(const orc_zone *z, long id) {
  const long sz = psz(z, z->ngg), sj = pstride(z, z->ngg, 1), sk = pstride(z, z->ngg, 2);
  const double *bv = z->bv;
  const double rho = bv[id], rhoI = 1.0 / rho, p = bv[id + 4 * sz], pI = 1.0 / p;
  double s = 0;
  s = fmax(s, fabs(bv[id + 1] - rho) * rhoI);
  s = fmax(s, fabs(bv[id + sj] - rho) * rhoI);
  s = fmax(s, fabs(bv[id + sk] - rho) * rhoI);
  s = fmax(s, fabs(bv[id + 1 + 4 * sz] - p) * pI);
  s = fmax(s, fabs(bv[id + sj + 4 * sz] - p) * pI);
  s = fmax(s, fabs(bv[id + sk + 4 * sz] - p) * pI);
  return s;
}

void orc_compute_shock_sensor(orc_zone *z, const orc_param *p) {
  const int g = z->ngg;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < z->mz; ++k)
    for (int j = 0; j < z->my; ++j)
      for (int i = 0; i < z->mx; ++i) {
        const long id = pidx(z, g, i, j, k);
        double sensor;
        if (p->shock_sensor == 1) sensor = jameson_sensor(z, id);
        else if (p->shock_sensor == 2) sensor = jump_sensor(z, id);
        else sensor = ducros_sensor(z, p->sensor_eps, id);
        z->shock_sensor[id] = sensor;
      }
}

double orc_global_time_step(const orc_zone *z) {
  const long n = psz(z, 0);
  double dt = 1e6;
  for (long i = 0; i < n; ++i) dt = z->dt_local[i] < dt ? z->dt_local[i] : dt;
  return dt;
}

/* ------------------------------------------------------------------------ */
/* Boundary conditions: outflow (src/BoundCond.cu:2065-2171, plain branch),  */
/* periodic (src/BoundCond.cu:3033-3080), symmetry (src/BoundCond.cu:2002),  */
/* no-slip wall (src/BoundCond.cu:2761-3031), inflow (src/BoundCond.cu:2190) */
/* applied per label in the reference's priority order                       */
/* (src/BoundCond.cu:3489-3619): outflow, inflow, symmetry, wall, periodic.  */
/* Each face covers its tangential range, widened by ngg ghosts only when    */
/* viscous_order == 2 (src/Mesh.cpp:14-31, 637: need_extend_boundary); for  */
/* a 2-D block the k range is then [-ngg, ngg], else [0, 0].                 */
/* ------------------------------------------------------------------------ */
static void face_range(const orc_zone *z, const orc_param *p, const orc_face *f, int lo[3], int hi[3]) {
  const int g = p->viscous_order == 2 ? z->ngg : 0;
  const int m[3] = {z->mx, z->my, z->mz};
  for (int d = 0; d < 3; ++d) {
    if (d == f->face) {
      lo[d] = hi[d] = f->direction < 0 ? 0 : m[d] - 1;
    } else {
      lo[d] = -g;
      hi[d] = m[d] - 1 + g;
    }
  }
  if (z->mz == 1) { lo[2] = -g; hi[2] = g; }
}

static void apply_outflow_face(orc_zone *z, const orc_param *p, const orc_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  int lo[3], hi[3];
  face_range(z, p, f, lo, hi);
  const long s = pstride(z, g, f->face) * f->direction;
  const int ns = p->mech ? p->n_spec : 0;
  double *bv = z->bv, *sv = z->sv;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const long id = pidx(z, g, i, j, k);
        if (!p->outflow_back_pressure_on) {
          for (int gg = 1; gg <= g; ++gg) {
            const long gi = id + gg * s;
            for (int l = 0; l < 6; ++l) bv[gi + l * sz] = bv[id + l * sz];
            for (int l = 0; l < p->n_scalar; ++l) sv[gi + l * sz] = sv[id + l * sz];
            cv_from_bv_point(z, p, gi);
          }
          continue;
        }
        /* back-pressure branch (src/BoundCond.cu:2082-2171) */
        const int mf = 3 * f->face;
        const double *mt = z->metric;
        double nx = mt[id + mf * sz], ny = mt[id + (mf + 1) * sz], nz = mt[id + (mf + 2) * sz];
        const double grad_n_inv = f->direction / sqrt(nx * nx + ny * ny + nz * nz);
        nx *= grad_n_inv; ny *= grad_n_inv; nz *= grad_n_inv;
        double u_b = bv[id + sz], v_b = bv[id + 2 * sz], w_b = bv[id + 3 * sz];
        const double u_face = nx * u_b + ny * v_b + nz * w_b;
        double p_b = bv[id + 4 * sz], rho_b = bv[id];
        double gamma = GAMMA_AIR, yk_b[ORC_MAX_SPEC], cpk[ORC_MAX_SPEC];
        if (ns > 0) {
          orc_cp(p->mech, bv[id + 5 * sz], cpk);
          double cp = 0, R = 0;
          for (int l = 0; l < ns; ++l) {
            yk_b[l] = sv[id + l * sz];
            cp += sv[id + l * sz] * cpk[l];
            R += sv[id + l * sz] * p->mech->gas_const[l];
          }
          gamma = cp / (cp - R);
        }
        const double a_b = sqrt(gamma * p_b / rho_b);
        const double mach_b = fabs(u_face / a_b);
        if (mach_b < 1) {
          p_b = p->outflow_back_pressure;
          const long i1 = id - s;
          const double d1 = bv[i1], u1 = bv[i1 + sz], v1 = bv[i1 + 2 * sz], w1 = bv[i1 + 3 * sz], p1 = bv[i1 + 4 * sz];
          gamma = GAMMA_AIR;
          if (ns > 0) {
            orc_cp(p->mech, bv[i1 + 5 * sz], cpk);
            double cp = 0, R = 0;
            for (int l = 0; l < ns; ++l) {
              cp += sv[i1 + l * sz] * cpk[l];
              R += sv[i1 + l * sz] * p->mech->gas_const[l];
            }
            gamma = cp / (cp - R);
          }
          const double c1 = sqrt(gamma * p1 / d1);
          const double temp = (p_b - p1) / c1;
          rho_b = d1 + temp / c1;
          u_b = u1 - nx * temp / d1;
          v_b = v1 - ny * temp / d1;
          w_b = w1 - nz * temp / d1;
          for (int gg = 1; gg <= g; ++gg) {
            const long gi = id + gg * s, ii = id - gg * s;
            const double p_g = 2 * p_b - bv[ii + 4 * sz], rho_g = 2 * rho_b - bv[ii];
            bv[gi] = rho_g;
            bv[gi + sz] = 2 * u_b - bv[ii + sz];
            bv[gi + 2 * sz] = 2 * v_b - bv[ii + 2 * sz];
            bv[gi + 3 * sz] = 2 * w_b - bv[ii + 3 * sz];
            bv[gi + 4 * sz] = p_g;
            double R = R_AIR;
            if (ns > 0) {
              R = 0;
              for (int l = 0; l < ns; ++l) {
                sv[gi + l * sz] = 2 * yk_b[l] - sv[ii + l * sz];
                R += sv[gi + l * sz] * p->mech->gas_const[l];
              }
            }
            bv[gi + 5 * sz] = p_g / (rho_g * R);
            cv_from_bv_point(z, p, gi);
          }
        } else {
          for (int gg = 1; gg <= g; ++gg) {
            const long gi = id + gg * s;
            bv[gi] = rho_b; bv[gi + sz] = u_b; bv[gi + 2 * sz] = v_b; bv[gi + 3 * sz] = w_b;
            bv[gi + 4 * sz] = p_b; bv[gi + 5 * sz] = bv[id + 5 * sz];
            for (int l = 0; l < p->n_scalar; ++l) sv[gi + l * sz] = sv[id + l * sz];
            cv_from_bv_point(z, p, gi);
          }
        }
      }
}

static void apply_symmetry_face(orc_zone *z, const orc_param *p, const orc_face *f);

static void apply_periodic_face(orc_zone *z, const orc_param *p, const orc_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  int lo[3], hi[3];
  face_range(z, p, f, lo, hi);
  const int m[3] = {z->mx, z->my, z->mz};
  const long sd = pstride(z, g, f->face);
  const long s = sd * f->direction;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const long id = pidx(z, g, i, j, k);
        /* partner node on the opposite face */
        const long io = id + (long)(f->direction < 0 ? (m[f->face] - 1) : -(m[f->face] - 1)) * sd;
        for (int l = 0; l < 6; ++l) {
          const double ave = 0.5 * (z->bv[id + l * sz] + z->bv[io + l * sz]);
          z->bv[id + l * sz] = ave;
          z->bv[io + l * sz] = ave;
        }
        for (int l = 0; l < p->n_scalar; ++l) {
          const double ave = 0.5 * (z->sv[id + l * sz] + z->sv[io + l * sz]);
          z->sv[id + l * sz] = ave;
          z->sv[io + l * sz] = ave;
        }
        cv_from_bv_point(z, p, id);
        for (int gg = 1; gg <= g; ++gg) {
          const long gi = id + gg * s, ii = io + gg * s;
          for (int l = 0; l < 6; ++l) z->bv[gi + l * sz] = z->bv[ii + l * sz];
          for (int l = 0; l < p->n_scalar; ++l) z->sv[gi + l * sz] = z->sv[ii + l * sz];
          cv_from_bv_point(z, p, gi);
        }
      }
}

/* apply_wall (src/BoundCond.cu:2761-3031) without its jet, shock-blowing and
 * wall-fluctuation branches (so v_blow = 0).  The boundary node takes zero
 * velocity, its inner neighbour's pressure, the wall temperature (isothermal)
 * or the inner neighbour's temperature (adiabatic), the mass fractions of the
 * inner neighbour (non-catalytic) or of the wall (catalytic), and
 * rho = p / (R T).  Ghost layer g mirrors inner node g: velocity reversed,
 * pressure copied, temperature copied (adiabatic) or reflected about the wall
 * temperature, T_g = 2 T_w - T_i, replaced by T_w when at or below 0.1 T_w
 * (isothermal).  As in the reference the catalytic ghosts' gas constant is
 * summed from the boundary node's (just written) mass fractions. */
static void apply_wall_face(orc_zone *z, const orc_param *p, const orc_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  int lo[3], hi[3];
  face_range(z, p, f, lo, hi);
  const long s = pstride(z, g, f->face) * f->direction;
  const int ns = p->mech ? p->n_spec : 0;
  const int catalytic = ns > 0 && p->wall_catalytic_type == 1;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const long id = pidx(z, g, i, j, k), in = id - s;
        double *bv = z->bv, *sv = z->sv;
        const double t_wall = p->wall_thermal_type == 0 ? p->wall_temperature : bv[in + 5 * sz];
        const double pw = bv[in + 4 * sz];
        double R = R_AIR;
        if (ns > 0) {
          R = 0;
          for (int l = 0; l < ns; ++l) {
            sv[id + l * sz] = catalytic ? p->wall_yk[l] : sv[in + l * sz];
            R += sv[id + l * sz] * p->mech->gas_const[l];
          }
        }
        bv[id] = pw / (t_wall * R);
        bv[id + sz] = 0;
        bv[id + 2 * sz] = 0;
        bv[id + 3 * sz] = 0;
        bv[id + 4 * sz] = pw;
        bv[id + 5 * sz] = t_wall;
        cv_from_bv_point(z, p, id);
        const double v_blow = 0;
        for (int gg = 1; gg <= g; ++gg) {
          const long ii = id - gg * s, gi = id + gg * s;
          const double p_i = bv[ii + 4 * sz], t_i = bv[ii + 5 * sz];
          double t_g = t_i;
          if (p->wall_thermal_type == 0) {
            t_g = 2 * t_wall - t_i;
            if (t_g <= 0.1 * t_wall) t_g = t_wall;
          }
          if (ns > 0) {
            R = 0;
            for (int l = 0; l < ns; ++l) {
              if (catalytic) {
                sv[gi + l * sz] = p->wall_yk[l];
                R += sv[id + l * sz] * p->mech->gas_const[l];
              } else {
                sv[gi + l * sz] = sv[ii + l * sz];
                R += sv[ii + l * sz] * p->mech->gas_const[l];
              }
            }
          }
          bv[gi] = p_i / (t_g * R);
          bv[gi + sz] = -bv[ii + sz];
          bv[gi + 2 * sz] = v_blow * 2 - bv[ii + 2 * sz];
          bv[gi + 3 * sz] = -bv[ii + 3 * sz];
          bv[gi + 4 * sz] = p_i;
          bv[gi + 5 * sz] = t_g;
          cv_from_bv_point(z, p, gi);
        }
      }
}

/* Seeded white noise of the fluctuating inflow (test infrastructure: the
 * same integer steps as the library's counter-based stream): the SplitMix64
 * output function (Steele, Lea and Flood, OOPSLA 2014) on a key of seed,
 * application count and face node gives uniforms in (0, 1]; Box-Muller gives
 * the normal deviates. */
static uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

double orc_noise_uniform(unsigned long long seed, unsigned long long call, unsigned long long node,
                         unsigned long long n) {
  const uint64_t key = splitmix64(seed ^ splitmix64((call << 24) ^ node));
  const uint64_t r = splitmix64(key + n * 0x9E3779B97F4A7C15ull);
  return (double)((r >> 11) + 1) * 0x1.0p-53;
}

static void noise_normal_pair(uint64_t seed, uint64_t call, uint64_t node, uint64_t m, double *n0, double *n1) {
  const double u1 = orc_noise_uniform(seed, call, node, 2 * m), u2 = orc_noise_uniform(seed, call, node, 2 * m + 1);
  const double r = sqrt(-2.0 * log(u1));
  const double a = 2.0 * 3.141592653589793 * u2;
  *n0 = r * cos(a);
  *n1 = r * sin(a);
}

/* index of a face node in its padded face plane (src/BoundCond.cu:2485-2496) */
static uint64_t inflow_noise_node(const orc_zone *z, int face, int i, int j, int k) {
  const int g = z->ngg;
  if (face == 1) return (uint64_t)(k + g) * (uint64_t)(z->mx + 2 * g) + (uint64_t)(i + g);
  if (face == 2) return (uint64_t)(j + g) * (uint64_t)(z->mx + 2 * g) + (uint64_t)(i + g);
  return (uint64_t)(k + g) * (uint64_t)(z->my + 2 * g) + (uint64_t)(j + g);
}

/* apply_inflow (src/BoundCond.cu:2190-2705): the constant inflow
 * (inflow_type 0, with inflow_sub and with the white noise on u of
 * :2573-2596) and the mixing-layer inflow (inflow_type 2, :2455-2506, with
 * the white noise on u, v, w).  Profile inflows and the other fluctuation
 * forms are not restated. */
static void apply_inflow_face(orc_zone *z, const orc_param *p, const orc_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  int lo[3], hi[3];
  face_range(z, p, f, lo, hi);
  const long s = pstride(z, g, f->face) * f->direction;
  const int mix = p->mech != NULL;
  double *bv = z->bv, *sv = z->sv;
  const uint64_t call = z->inflow_draws;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const long id = pidx(z, g, i, j, k);
        double density = p->inflow_density, u = p->inflow_u, v = p->inflow_v, w = p->inflow_w;
        double pr = p->inflow_pressure, T = p->inflow_temperature;
        const double *svb = p->inflow_sv;
        if (p->inflow_type == 2) {
          const double y = z->y[id];
          u = 0.5 * (p->inflow_u + p->inflow_u_lower) +
              0.5 * (p->inflow_u - p->inflow_u_lower) * tanh(2 * y / p->inflow_delta_omega);
          if (!(y >= 0)) {
            density = p->inflow_density_lower;
            v = p->inflow_v_lower;
            w = p->inflow_w_lower;
            pr = p->inflow_p_lower;
            T = p->inflow_t_lower;
            svb = p->inflow_sv_lower;
          }
          if (p->inflow_fluctuation_type == 1) {
            const uint64_t node = inflow_noise_node(z, f->face, i, j, k);
            const double rms = p->inflow_fluctuation_intensity * u * exp(-y * y);
            double n0, n1, n2, n3;
            noise_normal_pair(p->inflow_seed, call, node, 0, &n0, &n1);
            noise_normal_pair(p->inflow_seed, call, node, 1, &n2, &n3);
            u += n0 * rms;
            v += n1 * rms;
            w += n2 * rms;
          }
        } else if (p->inflow_subsonic) {
          const double *mt = z->metric;
          const int mf = 3 * f->face;
          double nx = mt[id + mf * sz], ny = mt[id + (mf + 1) * sz], nz = mt[id + (mf + 2) * sz];
          const double grad_n_inv = f->direction / sqrt(nx * nx + ny * ny + nz * nz);
          nx *= grad_n_inv;
          ny *= grad_n_inv;
          nz *= grad_n_inv;
          const double c0 = mix ? z->acoustic_speed[id] : sqrt(GAMMA_AIR * R_AIR * bv[id + 5 * sz]);
          const double Mn = (bv[id + sz] * nx + bv[id + 2 * sz] * ny + bv[id + 3 * sz] * nz) / c0;
          if (!(Mn < -1.0)) {
            const long i1 = id - s;
            const double c1 = mix ? z->acoustic_speed[i1] : sqrt(GAMMA_AIR * R_AIR * bv[i1 + 5 * sz]);
            const double rho1 = bv[i1], p1 = bv[i1 + 4 * sz];
            pr = 0.5 * (p1 + p->inflow_pressure -
                        rho1 * c1 * ((p->inflow_u - bv[i1 + sz]) * nx + (p->inflow_v - bv[i1 + 2 * sz]) * ny +
                                     (p->inflow_w - bv[i1 + 3 * sz]) * nz));
            density = p->inflow_density + (pr - p->inflow_pressure) / (c1 * c1);
            u = p->inflow_u - (pr - p->inflow_pressure) / (rho1 * c1) * nx;
            v = p->inflow_v - (pr - p->inflow_pressure) / (rho1 * c1) * ny;
            w = p->inflow_w - (pr - p->inflow_pressure) / (rho1 * c1) * nz;
            T = mix ? pr * p->inflow_mw / (density * R_U) : pr / (density * R_AIR);
          }
        } else if (p->inflow_fluctuation_type == 1) {
          const uint64_t node = inflow_noise_node(z, f->face, i, j, k);
          double n0, n1;
          noise_normal_pair(p->inflow_seed, call, node, 0, &n0, &n1);
          u += n0 * p->inflow_fluctuation_intensity *
               sqrt(p->inflow_u * p->inflow_u + p->inflow_v * p->inflow_v + p->inflow_w * p->inflow_w);
        }
        bv[id] = density; bv[id + sz] = u; bv[id + 2 * sz] = v; bv[id + 3 * sz] = w;
        bv[id + 4 * sz] = pr; bv[id + 5 * sz] = T;
        for (int l = 0; l < p->n_scalar; ++l) sv[id + l * sz] = svb[l];
        cv_from_bv_point(z, p, id);
        for (int gg = 1; gg <= g; ++gg) {
          const long gi = id + gg * s;
          for (int l = 0; l < p->n_scalar; ++l) sv[gi + l * sz] = svb[l];
          if (p->inflow_subsonic) {
            const long ii = id - gg * s;
            double rho2 = 2 * density - bv[ii], p2 = 2 * pr - bv[ii + 4 * sz];
            if (p2 <= 0.1 * pr) p2 = 0.1 * pr;
            if (rho2 <= 0.1 * density) rho2 = 0.1 * density;
            bv[gi] = rho2;
            bv[gi + sz] = 2 * u - bv[ii + sz];
            bv[gi + 2 * sz] = 2 * v - bv[ii + 2 * sz];
            bv[gi + 3 * sz] = 2 * w - bv[ii + 3 * sz];
            bv[gi + 4 * sz] = p2;
            bv[gi + 5 * sz] = mix ? p2 * p->inflow_mw / (rho2 * R_U) : p2 / (rho2 * R_AIR);
          } else {
            bv[gi] = density; bv[gi + sz] = u; bv[gi + 2 * sz] = v; bv[gi + 3 * sz] = w;
            bv[gi + 4 * sz] = pr; bv[gi + 5 * sz] = T;
          }
          cv_from_bv_point(z, p, gi);
        }
      }
  if (p->inflow_fluctuation_type == 1) z->inflow_draws += 1;
}

void orc_apply_boundary_conditions(orc_zone *z, const orc_param *p) {
  static const int order[] = {6, 5, 3, 2, 8};
  for (int o = 0; o < 5; ++o)
    for (int n = 0; n < p->n_face; ++n) {
      const orc_face *f = &p->faces[n];
      if (f->label != order[o]) continue;
      if (f->label == 6) apply_outflow_face(z, p, f);
      else if (f->label == 5) apply_inflow_face(z, p, f);
      else if (f->label == 3) apply_symmetry_face(z, p, f);
      else if (f->label == 2) apply_wall_face(z, p, f);
      else if (f->label == 8) apply_periodic_face(z, p, f);
    }
}

/* apply_symmetry (src/BoundCond.cu:2002-2063).  The boundary node takes the
 * tangential velocity and rho, p, T, scalars of its inner neighbour; as in the
 * reference its cv is not recomputed, only the ghosts' cv are. */
static void apply_symmetry_face(orc_zone *z, const orc_param *p, const orc_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  int lo[3], hi[3];
  face_range(z, p, f, lo, hi);
  const long s = pstride(z, g, f->face) * f->direction;
  const int mf = 3 * f->face;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const long id = pidx(z, g, i, j, k), in = id - s;
        const double *mt = z->metric;
        double k_x = mt[id + mf * sz], k_y = mt[id + (mf + 1) * sz], k_z = mt[id + (mf + 2) * sz];
        const double k_magnitude = sqrt(k_x * k_x + k_y * k_y + k_z * k_z);
        k_x /= k_magnitude; k_y /= k_magnitude; k_z /= k_magnitude;
        const double u1 = z->bv[in + sz], v1 = z->bv[in + 2 * sz], w1 = z->bv[in + 3 * sz];
        double u_k = k_x * u1 + k_y * v1 + k_z * w1;
        const double u_t = u1 - k_x * u_k, v_t = v1 - k_y * u_k, w_t = w1 - k_z * u_k;
        z->bv[id + sz] = u_t;
        z->bv[id + 2 * sz] = v_t;
        z->bv[id + 3 * sz] = w_t;
        z->bv[id] = z->bv[in];
        z->bv[id + 4 * sz] = z->bv[in + 4 * sz];
        z->bv[id + 5 * sz] = z->bv[in + 5 * sz];
        for (int l = 0; l < p->n_scalar; ++l) z->sv[id + l * sz] = z->sv[in + l * sz];
        for (int gg = 1; gg <= g; ++gg) {
          const long gi = id + gg * s, ii = id - gg * s;
          z->bv[gi] = z->bv[ii];
          const double u = z->bv[ii + sz], v = z->bv[ii + 2 * sz], w = z->bv[ii + 3 * sz];
          u_k = k_x * u + k_y * v + k_z * w;
          z->bv[gi + sz] = u - 2 * u_k * k_x;
          z->bv[gi + 2 * sz] = v - 2 * u_k * k_y;
          z->bv[gi + 3 * sz] = w - 2 * u_k * k_z;
          z->bv[gi + 4 * sz] = z->bv[ii + 4 * sz];
          z->bv[gi + 5 * sz] = z->bv[ii + 5 * sz];
          for (int l = 0; l < p->n_scalar; ++l) z->sv[gi + l * sz] = z->sv[ii + l * sz];
          cv_from_bv_point(z, p, gi);
        }
      }
}

/* ------------------------------------------------------------------------ */
/* Multi-block meshes: InnerFace::register_boundary (src/Mesh.cpp:39-172)    */
/* and inner_communication (src/DataCommunication.cu:36-102).                */
/* ------------------------------------------------------------------------ */
static int isgn(int a) { return a > 0 ? 1 : (a < 0 ? -1 : 0); }

int orc_register_inner_face(int dim, int ngg, const int src[6], const int tar[6], int target_block,
                            orc_inner_face *o) {
  int rs[3], re[3], ts[3], te[3], st[3] = {0, 0, 0};
  int face = -1, dir = 1, tface = -1, tdir = 1;
  for (int i = 0; i < 3; ++i) {
    rs[i] = src[2 * i]; re[i] = src[2 * i + 1];
    ts[i] = tar[2 * i]; te[i] = tar[2 * i + 1];
  }
  for (int i = 0; i < dim && face < 0; ++i)
    if (rs[i] == re[i]) {
      face = i;
      if (rs[i] == 1) dir = -1;
      rs[i] -= 1; re[i] -= 1;
    }
  for (int i = 0; i < dim && tface < 0; ++i)
    if (ts[i] == te[i]) {
      tface = i;
      if (ts[i] == 1) tdir = -1;
      ts[i] -= 1; te[i] -= 1;
    }
  if (face < 0 || tface < 0) return -1;
  st[tface] = -(dir * tdir) * (face + 1);
  if (dim == 2) {
    const int nf = 1 - face, tnf = 1 - tface;
    rs[nf] = abs(rs[nf]) - 1; re[nf] = abs(re[nf]) - 1;
    ts[tnf] = abs(ts[tnf]) - 1; te[tnf] = abs(te[tnf]) - 1;
    st[tnf] = isgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1);
    st[2] = 3;
    rs[2] = re[2] = ts[2] = te[2] = 0;
  } else {
    int nf = -1, tnf = -1;
    for (int i = 0; i < dim && nf < 0; ++i)
      if (rs[i] < 0) { nf = i; rs[i] = -rs[i] - 1; re[i] = -re[i] - 1; }
    for (int i = 0; i < dim && tnf < 0; ++i)
      if (ts[i] < 0) { tnf = i; ts[i] = -ts[i] - 1; te[i] = -te[i] - 1; }
    if (nf < 0 || tnf < 0) return -1;
    st[tnf] = isgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1);
    nf = 3 - face - nf;
    tnf = 3 - tface - tnf;
    rs[nf] -= 1; re[nf] -= 1;
    ts[tnf] -= 1; te[tnf] -= 1;
    st[tnf] = isgn((te[tnf] - ts[tnf]) * (re[nf] - rs[nf])) * (nf + 1);
  }
  rs[face] = dir < 0 ? -ngg : re[face];
  re[face] = dir < 0 ? 0 : re[face] + ngg;
  const int sg = isgn(st[tface]);
  if (tdir > 0) ts[tface] = sg > 0 ? te[tface] - ngg : te[tface];
  else ts[tface] = sg > 0 ? 0 : ngg;
  for (int i = 0; i < 3; ++i) {
    o->range_start[i] = rs[i]; o->range_end[i] = re[i];
    o->target_start[i] = ts[i]; o->target_end[i] = te[i];
    o->loop_dir[i] = rs[i] <= re[i] ? 1 : -1;
    o->target_loop_dir[i] = isgn(st[i]);
    o->src_tar[i] = abs(st[i]) - 1;
    o->n_point[i] = abs(rs[i] - re[i]) + 1;
  }
  o->face = face; o->direction = dir;
  o->target_face = tface; o->target_direction = tdir;
  o->target_block = target_block - 1;
  return 0;
}

/* The speed test uses sqrt(u^2 + v^2 + w^2) where the reference calls norm3d;
 * the two can differ in the last bit, which matters only for speeds within
 * an ulp of the 1e-15 threshold. */
void orc_inner_communication(orc_zone *z, orc_zone *tz, const orc_param *p, const orc_inner_face *f) {
  const int g = z->ngg;
  const long sz = psz(z, g), tsz = psz(tz, g);
  const int face_node = f->direction > 0 ? f->range_start[f->face] : f->range_end[f->face];
  for (int n2 = 0; n2 < f->n_point[2]; ++n2)
    for (int n1 = 0; n1 < f->n_point[1]; ++n1)
      for (int n0 = 0; n0 < f->n_point[0]; ++n0) {
        const int n[3] = {n0, n1, n2};
        int idx[3], d_idx[3], idt[3];
        for (int a = 0; a < 3; ++a) {
          d_idx[a] = f->loop_dir[a] * n[a];
          idx[a] = f->range_start[a] + d_idx[a];
        }
        for (int a = 0; a < 3; ++a) idt[a] = f->target_start[a] + f->target_loop_dir[a] * d_idx[f->src_tar[a]];
        const long id = pidx(z, g, idx[0], idx[1], idx[2]), it = pidx(tz, g, idt[0], idt[1], idt[2]);
        double *bv = z->bv, *tbv = tz->bv, *sv = z->sv, *tsv = tz->sv;
        if (idx[f->face] == face_node) {
          const double u_this = sqrt(bv[id + sz] * bv[id + sz] + bv[id + 2 * sz] * bv[id + 2 * sz] +
                                     bv[id + 3 * sz] * bv[id + 3 * sz]);
          if (fabs(u_this) > 1e-15) {
            const double u_that = sqrt(tbv[it + tsz] * tbv[it + tsz] + tbv[it + 2 * tsz] * tbv[it + 2 * tsz] +
                                       tbv[it + 3 * tsz] * tbv[it + 3 * tsz]);
            if (fabs(u_that) < 1e-15) {
              for (int l = 0; l < 6; ++l) bv[id + l * sz] = tbv[it + l * tsz];
              for (int l = 0; l < p->n_scalar; ++l) sv[id + l * sz] = tsv[it + l * tsz];
            } else {
              for (int l = 0; l < 6; ++l) {
                const double ave = 0.5 * (tbv[it + l * tsz] + bv[id + l * sz]);
                bv[id + l * sz] = ave;
                tbv[it + l * tsz] = ave;
              }
              for (int l = 0; l < p->n_scalar; ++l) {
                const double ave = 0.5 * (tsv[it + l * tsz] + sv[id + l * sz]);
                sv[id + l * sz] = ave;
                tsv[it + l * tsz] = ave;
              }
            }
          }
        } else {
          for (int l = 0; l < 6; ++l) bv[id + l * sz] = tbv[it + l * tsz];
          for (int l = 0; l < p->n_scalar; ++l) sv[id + l * sz] = tsv[it + l * tsz];
        }
        cv_from_bv_point(z, p, id);
      }
}

static int unphysical(const double *v, const double *ll, const double *ul) {
  for (int l = 0; l < 5; ++l)
    if (isnan(v[l]) || v[l] < ll[l] || v[l] > ul[l]) return 1;
  return 0;
}

int orc_limit_flow(orc_zone *z, const orc_param *p, const double ll[5], const double ul[5]) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  const long nn = (long)z->mx * z->my * z->mz;
  double *snap = (double *)malloc(sizeof(double) * 5 * nn);
  if (!snap) return -1;
#define SNAP(i, j, k) (snap + 5 * (((long)(k) * z->my + (j)) * z->mx + (i)))
  for (int k = 0; k < z->mz; ++k)
    for (int j = 0; j < z->my; ++j)
      for (int i = 0; i < z->mx; ++i)
        for (int l = 0; l < 5; ++l) SNAP(i, j, k)[l] = z->bv[pidx(z, g, i, j, k) + l * sz];
  int repaired = 0;
  for (int k = 0; k < z->mz; ++k)
    for (int j = 0; j < z->my; ++j)
      for (int i = 0; i < z->mx; ++i) {
        const double *var = SNAP(i, j, k);
        if (!unphysical(var, ll, ul)) continue;
        double upd[5] = {0, 0, 0, 0, 0};
        int kn = 0;
        for (int ka = -1; ka < 2; ++ka) {
          const int k1 = k + ka;
          if (k1 < 0 || k1 >= z->mz) continue;
          for (int ja = -1; ja < 2; ++ja) {
            const int j1 = j + ja;
            if (j1 < 0 || j1 >= z->my) continue;
            for (int ia = -1; ia < 2; ++ia) {
              const int i1 = i + ia;
              if (i1 < 0 || i1 >= z->mx) continue;
              const double *nb = SNAP(i1, j1, k1);
              if (unphysical(nb, ll, ul)) continue;
              for (int l = 0; l < 5; ++l) upd[l] += nb[l];
              ++kn;
            }
          }
        }
        if (kn > 0) {
          const double kn_inv = 1.0 / kn;
          for (int l = 0; l < 5; ++l) upd[l] *= kn_inv;
        } else {
          for (int l = 0; l < 5; ++l) {
            upd[l] = var[l] > ll[l] ? var[l] : ll[l];
            upd[l] = upd[l] < ul[l] ? upd[l] : ul[l];
          }
        }
        const long id = pidx(z, g, i, j, k);
        for (int l = 0; l < 5; ++l) z->bv[id + l * sz] = upd[l];
        if (p->mech) {
          double R = 0;
          for (int l = 0; l < p->n_spec; ++l) R += z->sv[id + l * sz] * p->mech->gas_const[l];
          z->bv[id + 5 * sz] = upd[4] / (upd[0] * R);
        } else {
          z->bv[id + 5 * sz] = upd[4] * MW_AIR / (upd[0] * R_U);
        }
        cv_from_bv_point(z, p, id);
        ++repaired;
      }
#undef SNAP
  free(snap);
  return repaired;
}

/* eliminate_k_gradient (src/FieldOperation.cu:47-72) */
void orc_eliminate_k_gradient(orc_zone *z, const orc_param *p) {
  const int g = z->ngg;
  const long sz = psz(z, g);
  for (int j = -g; j < z->my + g; ++j)
    for (int i = -g; i < z->mx + g; ++i) {
      const long i0 = pidx(z, g, i, j, 0);
      for (int k = 1; k <= g; ++k) {
        const long ip = pidx(z, g, i, j, k), im = pidx(z, g, i, j, -k);
        for (int l = 0; l < 6; ++l) { z->bv[ip + l * sz] = z->bv[i0 + l * sz]; z->bv[im + l * sz] = z->bv[i0 + l * sz]; }
        for (int l = 0; l < p->n_scalar; ++l) { z->sv[ip + l * sz] = z->sv[i0 + l * sz]; z->sv[im + l * sz] = z->sv[i0 + l * sz]; }
        for (int l = 0; l < p->n_var; ++l) { z->cv[ip + l * sz] = z->cv[i0 + l * sz]; z->cv[im + l * sz] = z->cv[i0 + l * sz]; }
      }
    }
}

/* ------------------------------------------------------------------------ */
/* One SSP-RK3 step: src/RK.cuh:84-212 (single block, no MPI).               */
/* ------------------------------------------------------------------------ */
/* One step of Wu's splitting, the loop body of wu_splitting
 * (src/StrangSplitting.cu:683-861): dt without the reaction limit;
 * compute_cn (:15-41): Cn = viscous + inviscid right-hand side;
 * wu_reaction_subStep (:475-502): the reaction step over dt with the frozen
 * Cn, BCs, 2-D k-ghost copy, properties; wu_RK_subStep (:564-634): SSP-RK3
 * over dt/2 on dq - Cn with BCs (no property update inside). */
double orc_wu_splitting_step(orc_zone *z, const orc_param *p, double dt_fixed) {
  const long sz = psz(z, z->ngg), szq = psz(z, 0);
  double dt = dt_fixed;
  if (!p->fixed_dt) {
    orc_local_time_step_without_reaction(z, p);
    dt = orc_global_time_step(z);
  }
  z->dt_step = dt;
  if (p->sensor_threshold > 1e-10) orc_compute_shock_sensor(z, p); /* src/StrangSplitting.cu:19-24 */
  memset(z->dq, 0, sizeof(double) * szq * p->n_var);
  orc_compute_viscous_flux(z, p);
  orc_compute_inviscid_flux(z, p);
  memcpy(z->Cn, z->dq, sizeof(double) * szq * p->n_var);
  orc_wu_reaction_step(z, p, dt, NULL);
  orc_apply_boundary_conditions(z, p);
  if (z->mz == 1) orc_eliminate_k_gradient(z, p);
  orc_update_physical_properties(z, p);
  memcpy(z->qn, z->cv, sizeof(double) * sz * p->n_var);
  for (int rk = 0; rk < 3; ++rk) {
    memset(z->dq, 0, sizeof(double) * szq * p->n_var);
    orc_compute_viscous_flux(z, p);
    orc_compute_inviscid_flux(z, p);
    orc_update_cv_and_bv_rk_wu(z, p, 0.5 * dt, rk);
    if (p->limit_flow) orc_limit_flow(z, p, p->limit_ll, p->limit_ul);
    orc_apply_boundary_conditions(z, p);
    if (z->mz == 1) orc_eliminate_k_gradient(z, p);
  }
  return dt;
}

double orc_rk3_step(orc_zone *z, const orc_param *p, double dt_fixed) {
  const long sz = psz(z, z->ngg), szq = psz(z, 0);
  memcpy(z->qn, z->cv, sizeof(double) * sz * p->n_var);
  if (p->sensor_threshold > 1e-10) orc_compute_shock_sensor(z, p); /* src/RK.cuh:112-116 */
  double dt = dt_fixed;
  if (!p->fixed_dt) {
    orc_local_time_step(z, p);
    dt = orc_global_time_step(z);
  }
  z->dt_step = dt;
  for (int rk = 0; rk < 3; ++rk) {
    memset(z->dq, 0, sizeof(double) * szq * p->n_var);
    orc_compute_viscous_flux(z, p);
    /* explicit chemical source of a reacting mixture (src/RK.cuh:147-149) */
    if (p->mech && p->n_reac > 0) orc_finite_rate_chemistry(z, p);
    orc_compute_inviscid_flux(z, p);
    orc_update_cv_and_bv_rk(z, p, dt, rk);
    if (p->limit_flow) orc_limit_flow(z, p, p->limit_ll, p->limit_ul);
    orc_apply_boundary_conditions(z, p);
    if (z->mz == 1) orc_eliminate_k_gradient(z, p);
    orc_update_physical_properties(z, p);
  }
  return dt;
}

/* Halo of a block face shared with another rank's block: setup_data_to_be_sent
 * and assign_data_received (src/DataCommunication.cu:210-307) over a whole
 * block face (face 0/1/2, direction -1/+1), tangential nodes of the block
 * only.  Buffer per face node t (first tangential axis fastest), layer q =
 * 0..ngg (q-th node inwards), 6 basic variables then n_scalar scalars. */
static void halo_geom(const orc_zone *z, int face, int direction, int *a, int *b, int *na, int *nb, int *f0) {
  const int m[3] = {z->mx, z->my, z->mz};
  *a = face == 0 ? 1 : 0;
  *b = face == 2 ? 1 : 2;
  *na = m[*a];
  *nb = m[*b];
  *f0 = direction < 0 ? 0 : m[face] - 1;
}

long orc_halo_size(const orc_zone *z, const orc_param *p, int face) {
  int a, b, na, nb, f0;
  halo_geom(z, face, -1, &a, &b, &na, &nb, &f0);
  return (long)na * nb * (z->ngg + 1) * (6 + p->n_scalar);
}

void orc_halo_pack(const orc_zone *z, const orc_param *p, int face, int direction, double *buf) {
  int a, b, na, nb, f0;
  halo_geom(z, face, direction, &a, &b, &na, &nb, &f0);
  const int g = z->ngg, nt = 6 + p->n_scalar;
  const long sz = psz(z, g);
  for (int t = 0; t < na * nb; ++t)
    for (int q = 0; q <= g; ++q) {
      int idx[3];
      idx[a] = t % na;
      idx[b] = t / na;
      idx[face] = f0 - q * direction;
      const long id = pidx(z, g, idx[0], idx[1], idx[2]);
      double *o = buf + ((long)t * (g + 1) + q) * nt;
      for (int l = 0; l < 6; ++l) o[l] = z->bv[id + l * sz];
      for (int l = 0; l < p->n_scalar; ++l) o[6 + l] = z->sv[id + l * sz];
    }
}

void orc_halo_assign(orc_zone *z, const orc_param *p, int face, int direction, const double *buf) {
  int a, b, na, nb, f0;
  halo_geom(z, face, direction, &a, &b, &na, &nb, &f0);
  const int g = z->ngg, nt = 6 + p->n_scalar;
  const long sz = psz(z, g);
  for (int t = 0; t < na * nb; ++t) {
    const double *in = buf + (long)t * (g + 1) * nt;
    int idx[3];
    idx[a] = t % na;
    idx[b] = t / na;
    idx[face] = f0;
    long id = pidx(z, g, idx[0], idx[1], idx[2]);
    const double *bv = z->bv;
    const double u_this = sqrt(bv[id + sz] * bv[id + sz] + bv[id + 2 * sz] * bv[id + 2 * sz] +
                               bv[id + 3 * sz] * bv[id + 3 * sz]);
    if (fabs(u_this) > 1e-15) {
      if (sqrt(in[1] * in[1] + in[2] * in[2] + in[3] * in[3]) < 1e-15) {
        for (int l = 0; l < 6; ++l) z->bv[id + l * sz] = in[l];
        for (int l = 0; l < p->n_scalar; ++l) z->sv[id + l * sz] = in[6 + l];
      } else {
        for (int l = 0; l < 6; ++l) z->bv[id + l * sz] = 0.5 * (z->bv[id + l * sz] + in[l]);
        for (int l = 0; l < p->n_scalar; ++l) z->sv[id + l * sz] = 0.5 * (z->sv[id + l * sz] + in[6 + l]);
      }
      cv_from_bv_point(z, p, id);
    }
    for (int q = 1; q <= g; ++q) {
      idx[face] = f0 + q * direction;
      id = pidx(z, g, idx[0], idx[1], idx[2]);
      const double *v = in + q * nt;
      for (int l = 0; l < 6; ++l) z->bv[id + l * sz] = v[l];
      for (int l = 0; l < p->n_scalar; ++l) z->sv[id + l * sz] = v[6 + l];
      cv_from_bv_point(z, p, id);
    }
  }
}
