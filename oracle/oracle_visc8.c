/*
 * CPU oracle: the collocated viscous schemes, 8th order (viscous_order = 8,
 * the reference's) and 4th order (viscous_order = 4: the same scheme with the
 * reference's 4th-order central operator of its n = 2 boundary row used in
 * the interior, and its n = 0 / n = 1 one-sided rows at physical faces; the
 * reference has no 4th-order viscous scheme, so this one is checked by its
 * own exactness and convergence, not against a reference build).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * Restates, in the reference's arithmetic order:
 *   compute_viscous_flux, order-8 branch      src/ViscousScheme.cu:41-70
 *   d_dXi / d_dEta / d_dZeta<8>               src/ViscousScheme.cu:129-308
 *     (8th-order central differences; at a physical boundary face the
 *      reference switches to 4th/6th-order one-sided and reduced stencils
 *      on the four nodes next to it; periodic faces count as inner)
 *   compute_viscous_flux_collocated<8>        src/ViscousScheme.cu:309-412
 *   compute_viscous_flux_collocated_scalar<8> src/ViscousScheme.cu:414-560
 *   exchange_value(task 1), periodic faces    src/DataCommunication.cu:436-456, 628-672
 *   compute_viscous_flux_derivative<8>        src/ViscousScheme.cu:562-612
 * The node fluxes go to fFlux/gFlux/hFlux (slots 1..nv-1) on the interior
 * nodes; the periodic exchange averages the two coincident face nodes and
 * fills ngg ghost layers from the other side, face by face in the boundary
 * list's order.  In 2-D (mz = 1) the zeta derivative of hFlux only reads
 * ghost planes that nothing writes and that the reference allocates zeroed,
 * so it is zero and is left out.
 */
#include "oracle.h"

#include <math.h>
#include <string.h>

#define R_U 8314.462618
#define GAMMA_AIR 1.4
#define R_AIR (R_U / 28.9647)

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

/* d f / d(xi_dir) at node index n (0..nn-1) of a line through f[id], stride s */
static int g_order = 8; /* set by the entry point before the kernels run */

static double d8(const double *f, long id, long s, int n, int nn, int left, int right) {
  double df = 0;
  int computed = 0;
#define F(o) f[id + (long)(o) * s]
  if (g_order == 4) {
    if (left && n == 0) return -25.0 / 12 * F(0) + 4.0 * F(1) - 3 * F(2) + 4.0 / 3 * F(3) - 0.25 * F(4);
    if (left && n == 1) return -0.25 * F(-1) - 5.0 / 6 * F(0) + 1.5 * F(1) - 0.5 * F(2) + 1.0 / 12 * F(3);
    if (right && n == nn - 1) return 25.0 / 12 * F(0) - 4.0 * F(-1) + 3 * F(-2) - 4.0 / 3 * F(-3) + 0.25 * F(-4);
    if (right && n == nn - 2) return 0.25 * F(1) + 5.0 / 6 * F(0) - 1.5 * F(-1) + 0.5 * F(-2) - 1.0 / 12 * F(-3);
    return -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
  }
  if (left) {
    if (n == 0) {
      df = -25.0 / 12 * F(0) + 4.0 * F(1) - 3 * F(2) + 4.0 / 3 * F(3) - 0.25 * F(4);
      computed = 1;
    } else if (n == 1) {
      df = -0.25 * F(-1) - 5.0 / 6 * F(0) + 1.5 * F(1) - 0.5 * F(2) + 1.0 / 12 * F(3);
      computed = 1;
    } else if (n == 2) {
      df = -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
      computed = 1;
    } else if (n == 3) {
      df = 0.75 * (F(1) - F(-1)) - 0.15 * (F(2) - F(-2)) + 1.0 / 60 * (F(3) - F(-3));
      computed = 1;
    }
  }
  if (right) {
    if (n == nn - 1) {
      df = 25.0 / 12 * F(0) - 4.0 * F(-1) + 3 * F(-2) - 4.0 / 3 * F(-3) + 0.25 * F(-4);
      computed = 1;
    } else if (n == nn - 2) {
      df = 0.25 * F(1) + 5.0 / 6 * F(0) - 1.5 * F(-1) + 0.5 * F(-2) - 1.0 / 12 * F(-3);
      computed = 1;
    } else if (n == nn - 3) {
      df = -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
      computed = 1;
    } else if (n == nn - 4) {
      df = 0.75 * (F(1) - F(-1)) - 0.15 * (F(2) - F(-2)) + 1.0 / 60 * (F(3) - F(-3));
      computed = 1;
    }
  }
  if (!computed) {
    const double a1 = 0.8, a2 = -0.2, a3 = 4.0 / 105, a4 = -1.0 / 280;
    df = a1 * (F(1) - F(-1)) + a2 * (F(2) - F(-2)) + a3 * (F(3) - F(-3)) + a4 * (F(4) - F(-4));
  }
#undef F
  return df;
}

/* physical (non-periodic) boundary on each side of each direction */
static void boundary_types(const orc_param *p, int bt[3][2]) {
  memset(bt, 0, sizeof(int) * 6);
  for (int n = 0; n < p->n_face; ++n) {
    const orc_face *f = &p->faces[n];
    if (f->label != 8) bt[f->face][f->direction < 0 ? 0 : 1] = 1;
  }
}

void orc_enthalpy(const orc_mech *m, double t, double *h);

static void collocated(orc_zone *z, const orc_param *p, const int bt[3][2]) {
  const int g = z->ngg, mx = z->mx, my = z->my, mz = z->mz, nv = p->n_var;
  const long sz = psz(z, g), sj = pstride(z, g, 1), sk = pstride(z, g, 2);
  const orc_mech *m = p->mech;
  const int ns = m ? m->n_spec : 0;
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k)
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        const long id = pidx(z, g, i, j, k);
        const double *bv = z->bv;
        double dv[4][3];
        const int slots[4] = {1, 2, 3, 5};
        for (int q = 0; q < 4; ++q) {
          const double *f = bv + slots[q] * sz;
          dv[q][0] = d8(f, id, 1, i, mx, bt[0][0], bt[0][1]);
          dv[q][1] = d8(f, id, sj, j, my, bt[1][0], bt[1][1]);
          dv[q][2] = d8(f, id, sk, k, mz, bt[2][0], bt[2][1]);
        }
        const double *mt = z->metric;
        const double xi_x = mt[id], xi_y = mt[id + sz], xi_z = mt[id + 2 * sz];
        const double eta_x = mt[id + 3 * sz], eta_y = mt[id + 4 * sz], eta_z = mt[id + 5 * sz];
        const double zeta_x = mt[id + 6 * sz], zeta_y = mt[id + 7 * sz], zeta_z = mt[id + 8 * sz];
        const double u_x = dv[0][0] * xi_x + dv[0][1] * eta_x + dv[0][2] * zeta_x;
        const double u_y = dv[0][0] * xi_y + dv[0][1] * eta_y + dv[0][2] * zeta_y;
        const double u_z = dv[0][0] * xi_z + dv[0][1] * eta_z + dv[0][2] * zeta_z;
        const double v_x = dv[1][0] * xi_x + dv[1][1] * eta_x + dv[1][2] * zeta_x;
        const double v_y = dv[1][0] * xi_y + dv[1][1] * eta_y + dv[1][2] * zeta_y;
        const double v_z = dv[1][0] * xi_z + dv[1][1] * eta_z + dv[1][2] * zeta_z;
        const double w_x = dv[2][0] * xi_x + dv[2][1] * eta_x + dv[2][2] * zeta_x;
        const double w_y = dv[2][0] * xi_y + dv[2][1] * eta_y + dv[2][2] * zeta_y;
        const double w_z = dv[2][0] * xi_z + dv[2][1] * eta_z + dv[2][2] * zeta_z;
        const double mul = z->mul[id];
        const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
        const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
        const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
        const double tau_xy = mul * (u_y + v_x);
        const double tau_xz = mul * (u_z + w_x);
        const double tau_yz = mul * (v_z + w_y);
        double *fv = z->fFlux, *gv = z->gFlux, *hv = z->hFlux;
        fv[id + 1 * sz] = xi_x * tau_xx + xi_y * tau_xy + xi_z * tau_xz;
        fv[id + 2 * sz] = xi_x * tau_xy + xi_y * tau_yy + xi_z * tau_yz;
        fv[id + 3 * sz] = xi_x * tau_xz + xi_y * tau_yz + xi_z * tau_zz;
        gv[id + 1 * sz] = eta_x * tau_xx + eta_y * tau_xy + eta_z * tau_xz;
        gv[id + 2 * sz] = eta_x * tau_xy + eta_y * tau_yy + eta_z * tau_yz;
        gv[id + 3 * sz] = eta_x * tau_xz + eta_y * tau_yz + eta_z * tau_zz;
        hv[id + 1 * sz] = zeta_x * tau_xx + zeta_y * tau_xy + zeta_z * tau_xz;
        hv[id + 2 * sz] = zeta_x * tau_xy + zeta_y * tau_yy + zeta_z * tau_yz;
        hv[id + 3 * sz] = zeta_x * tau_xz + zeta_y * tau_yz + zeta_z * tau_zz;
        const double t_x = dv[3][0] * xi_x + dv[3][1] * eta_x + dv[3][2] * zeta_x;
        const double t_y = dv[3][0] * xi_y + dv[3][1] * eta_y + dv[3][2] * zeta_y;
        const double t_z = dv[3][0] * xi_z + dv[3][1] * eta_z + dv[3][2] * zeta_z;
        const double cp_air = GAMMA_AIR * R_AIR / (GAMMA_AIR - 1);
        const double conductivity = m ? z->thermal_conductivity[id] : mul / p->Pr * cp_air;
        const double u = bv[id + sz], v = bv[id + 2 * sz], w = bv[id + 3 * sz];
        const double Ex = u * tau_xx + v * tau_xy + w * tau_xz + conductivity * t_x;
        const double Ey = u * tau_xy + v * tau_yy + w * tau_yz + conductivity * t_y;
        const double Ez = u * tau_xz + v * tau_yz + w * tau_zz + conductivity * t_z;
        fv[id + 4 * sz] = xi_x * Ex + xi_y * Ey + xi_z * Ez;
        gv[id + 4 * sz] = eta_x * Ex + eta_y * Ey + eta_z * Ez;
        hv[id + 4 * sz] = zeta_x * Ex + zeta_y * Ey + zeta_z * Ez;
        if (!m) continue;
        /* species diffusion (collocated_scalar), with the grad-p term of
         * gradPInDiffusionFlux when it is set (src/ViscousScheme.cu:495-520) */
        double diffusivity[ORC_MAX_SPEC], yk[ORC_MAX_SPEC], dfx[ORC_MAX_SPEC], dfy[ORC_MAX_SPEC], dfz[ORC_MAX_SPEC];
        double sx = 0, sy = 0, szz = 0, sum_rhoDkYk = 0, cv0 = 0, cv1 = 0, cv2 = 0, mw_tot = 0;
        for (int l = 0; l < ns; ++l) {
          const double *y = z->sv + l * sz;
          yk[l] = y[id];
          diffusivity[l] = z->rho_D[id + l * sz];
          const double y_xi = d8(y, id, 1, i, mx, bt[0][0], bt[0][1]);
          const double y_eta = d8(y, id, sj, j, my, bt[1][0], bt[1][1]);
          const double y_zeta = d8(y, id, sk, k, mz, bt[2][0], bt[2][1]);
          const double y_x = y_xi * xi_x + y_eta * eta_x + y_zeta * zeta_x;
          const double y_y = y_xi * xi_y + y_eta * eta_y + y_zeta * zeta_y;
          const double y_z = y_xi * xi_z + y_eta * eta_z + y_zeta * zeta_z;
          const double gx = xi_x * y_x + xi_y * y_y + xi_z * y_z;
          const double gy = eta_x * y_x + eta_y * y_y + eta_z * y_z;
          const double gz = zeta_x * y_x + zeta_y * y_y + zeta_z * y_z;
          dfx[l] = gx;
          dfy[l] = gy;
          dfz[l] = gz;
          cv0 += diffusivity[l] * gx;
          cv1 += diffusivity[l] * gy;
          cv2 += diffusivity[l] * gz;
          sx += gx * m->imw[l];
          sy += gy * m->imw[l];
          szz += gz * m->imw[l];
          mw_tot += yk[l] * m->imw[l];
          sum_rhoDkYk += diffusivity[l] * yk[l];
        }
        mw_tot = 1.0 / mw_tot;
        cv0 -= mw_tot * sum_rhoDkYk * sx;
        cv1 -= mw_tot * sum_rhoDkYk * sy;
        cv2 -= mw_tot * sum_rhoDkYk * szz;
        if (p->gradPInDiffusionFlux) {
          const double *pp = bv + 4 * sz;
          const double p_xi = d8(pp, id, 1, i, mx, bt[0][0], bt[0][1]);
          const double p_eta = d8(pp, id, sj, j, my, bt[1][0], bt[1][1]);
          const double p_zeta = d8(pp, id, sk, k, mz, bt[2][0], bt[2][1]);
          const double p_x = p_xi * xi_x + p_eta * eta_x + p_zeta * zeta_x;
          const double p_y = p_xi * xi_y + p_eta * eta_y + p_zeta * zeta_y;
          const double p_z = p_xi * xi_z + p_eta * eta_z + p_zeta * zeta_z;
          const double gxp = (xi_x * p_x + xi_y * p_y + xi_z * p_z) / pp[id];
          const double gyp = (eta_x * p_x + eta_y * p_y + eta_z * p_z) / pp[id];
          const double gzp = (zeta_x * p_x + zeta_y * p_y + zeta_z * p_z) / pp[id];
          for (int l = 0; l < ns; ++l) {
            const double coefficient = (mw_tot * m->imw[l] - 1) * yk[l];
            dfx[l] += coefficient * gxp;
            dfy[l] += coefficient * gyp;
            dfz[l] += coefficient * gzp;
            cv0 += coefficient * gxp * diffusivity[l];
            cv1 += coefficient * gyp * diffusivity[l];
            cv2 += coefficient * gzp * diffusivity[l];
          }
        }
        double h[ORC_MAX_SPEC];
        orc_enthalpy(m, bv[id + 5 * sz], h);
        for (int l = 0; l < ns; ++l) {
          double df = diffusivity[l] * (dfx[l] - mw_tot * yk[l] * sx) - yk[l] * cv0;
          fv[id + (5 + l) * sz] = df;
          fv[id + 4 * sz] += h[l] * df;
          df = diffusivity[l] * (dfy[l] - mw_tot * yk[l] * sy) - yk[l] * cv1;
          gv[id + (5 + l) * sz] = df;
          gv[id + 4 * sz] += h[l] * df;
          df = diffusivity[l] * (dfz[l] - mw_tot * yk[l] * szz) - yk[l] * cv2;
          hv[id + (5 + l) * sz] = df;
          hv[id + 4 * sz] += h[l] * df;
        }
        (void)nv;
      }
}

/* exchange_value(task 1) on the periodic faces, in the face list's order */
static void periodic_exchange(orc_zone *z, const orc_param *p) {
  const int g = z->ngg, nv = p->n_var;
  const long sz = psz(z, g);
  double *arr[3] = {z->fFlux, z->gFlux, z->hFlux};
  const int ext[3] = {z->mx, z->my, z->mz};
  for (int n = 0; n < p->n_face; ++n) {
    const orc_face *f = &p->faces[n];
    if (f->label != 8) continue;
    const int d = f->face, a = (d + 1) % 3, b = (d + 2) % 3;
    const int here = f->direction < 0 ? 0 : ext[d] - 1, other = f->direction < 0 ? ext[d] - 1 : 0;
    const long s = pstride(z, g, d);
    for (int ib = 0; ib < ext[b]; ++ib)
      for (int ia = 0; ia < ext[a]; ++ia) {
        int c[3];
        c[d] = here;
        c[a] = ia;
        c[b] = ib;
        const long idh = pidx(z, g, c[0], c[1], c[2]);
        c[d] = other;
        const long ido = pidx(z, g, c[0], c[1], c[2]);
        for (int l = 0; l < nv; ++l)
          for (int q = 0; q < 3; ++q) {
            const double ave = 0.5 * (arr[q][idh + l * sz] + arr[q][ido + l * sz]);
            arr[q][idh + l * sz] = ave;
            arr[q][ido + l * sz] = ave;
          }
        for (int gg = 1; gg <= g; ++gg) {
          const long gh = idh + (long)gg * f->direction * s, go = ido + (long)gg * f->direction * s;
          for (int l = 0; l < nv; ++l)
            for (int q = 0; q < 3; ++q) arr[q][gh + l * sz] = arr[q][go + l * sz];
        }
      }
  }
}

static void derivative(orc_zone *z, const orc_param *p, const int bt[3][2]) {
  const int g = z->ngg, mx = z->mx, my = z->my, mz = z->mz, nv = p->n_var;
  const long sz = psz(z, g), szq = psz(z, 0), sj = pstride(z, g, 1), sk = pstride(z, g, 2);
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < mz; ++k)
    for (int j = 0; j < my; ++j)
      for (int i = 0; i < mx; ++i) {
        const long id = pidx(z, g, i, j, k), iq = pidx(z, 0, i, j, k);
        const double jac = z->jac[id];
        for (int l = 1; l < nv; ++l) {
          double s = d8(z->fFlux + l * sz, id, 1, i, mx, bt[0][0], bt[0][1]) +
                     d8(z->gFlux + l * sz, id, sj, j, my, bt[1][0], bt[1][1]);
          if (mz > 1) s += d8(z->hFlux + l * sz, id, sk, k, mz, bt[2][0], bt[2][1]);
          z->dq[iq + l * szq] += s * jac;
        }
      }
}

void orc_viscous_flux_8th(orc_zone *z, const orc_param *p) {
  g_order = p->viscous_order == 4 ? 4 : 8;
  int bt[3][2];
  boundary_types(p, bt);
  collocated(z, p, bt);
  periodic_exchange(z, p);
  derivative(z, p, bt);
}
