// Mixture thermodynamics and transport on the device.
//
// NASA-7 two-range polynomials with linear extrapolation outside
// [t_low, t_high] (the Combustion2Part branch, reference
// src/Thermo.cu:385-633), the temperature Newton iteration of
// compute_temperature_and_pressure (reference src/FieldOperation.cu:4-45) and
// the mixture-averaged viscosity / conductivity / diffusivity of
// compute_transport_property (reference src/Transport.cu:43-165).  The
// tables live in one device-resident Thermo block read through the uniform
// (warp-broadcast) cache.
#pragma once

#include "cfk_common.cuh"

namespace cfk {

struct Thermo {
  int n_spec;
  double imw[kMaxSpec], gas_const[kMaxSpec], mw[kMaxSpec];
  double t_low[kMaxSpec], t_mid[kMaxSpec], t_high[kMaxSpec];
  double low[kMaxSpec][7], high[kMaxSpec][7];
  // transport
  int geometry[kMaxSpec];
  double LJ_potent_inv[kMaxSpec], vis_coeff[kMaxSpec], ZRotF298[kMaxSpec];
  double WjDivWi_to_One4th[kMaxSpec][kMaxSpec];
  double sqrt_WiDivWjPl1Mul8[kMaxSpec][kMaxSpec];
  double binary_diffusivity_coeff[kMaxSpec][kMaxSpec];
  double kb_over_eps_jk[kMaxSpec][kMaxSpec];
};

__host__ __device__ inline double sutherland(double t) {
  // reference src/Transport.cu:6-9; (T/288.16)^1.5 as x sqrt(x) (correctly
  // rounded sqrt and one product) instead of the general power function
  const double x = t / 288.16;
  return 1.7894e-5 * (x * sqrt(x)) * (288.16 + 110) / (t + 110);
}

__device__ __forceinline__ void compute_enthalpy_and_cp(const Thermo *th, double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < th->n_spec; ++i) {
    if (t < th->t_low[i] || t > th->t_high[i]) {
      const bool lo = t < th->t_low[i];
      const double tt = lo ? th->t_low[i] : th->t_high[i];
      const double *c = lo ? th->low[i] : th->high[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cp[i] * (t - tt);
    } else {
      const double *c = t < th->t_mid[i] ? th->low[i] : th->high[i];
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
      cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    }
    h[i] *= th->gas_const[i];
    cp[i] *= th->gas_const[i];
  }
}

__device__ __forceinline__ void compute_enthalpy(const Thermo *th, double t, double *h) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  for (int i = 0; i < th->n_spec; ++i) {
    if (t < th->t_low[i] || t > th->t_high[i]) {
      const bool lo = t < th->t_low[i];
      const double tt = lo ? th->t_low[i] : th->t_high[i];
      const double *c = lo ? th->low[i] : th->high[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt, tt5 = tt4 * tt;
      h[i] = c[0] * tt + 0.5 * c[1] * tt2 + c[2] * tt3 / 3 + 0.25 * c[3] * tt4 + 0.2 * c[4] * tt5 + c[5];
      const double cpl = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
      h[i] += cpl * (t - tt);
    } else {
      const double *c = t < th->t_mid[i] ? th->low[i] : th->high[i];
      h[i] = c[0] * t + 0.5 * c[1] * t2 + c[2] * t3 / 3 + 0.25 * c[3] * t4 + 0.2 * c[4] * t5 + c[5];
    }
    h[i] *= th->gas_const[i];
  }
}

__device__ __forceinline__ void compute_cp(const Thermo *th, double t, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < th->n_spec; ++i) {
    double tt = t;
    const double *c;
    if (t < th->t_low[i]) { tt = th->t_low[i]; c = th->low[i]; }
    else if (t > th->t_high[i]) { tt = th->t_high[i]; c = th->high[i]; }
    else c = t < th->t_mid[i] ? th->low[i] : th->high[i];
    if (tt == t) cp[i] = c[0] + c[1] * t + c[2] * t2 + c[3] * t3 + c[4] * t4;
    else {
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      cp[i] = c[0] + c[1] * tt + c[2] * tt2 + c[3] * tt3 + c[4] * tt4;
    }
    cp[i] *= th->gas_const[i];
  }
}

// T from the internal energy by Newton's method, eps = 1e-5, at most 1000
// iterations, starting from the previous T (reference src/FieldOperation.cu:4-45).
// Returns false if the iteration cap was reached (the reference then keeps
// the last iterate; so does this routine).
__device__ __forceinline__ bool temperature_newton(const Thermo *th, int ns, const double *yk, double total_energy,
                                                   double rho, double V2, double &t, double &p) {
  double gas_const = 0;
  for (int l = 0; l < ns; ++l) gas_const += yk[l] * th->gas_const[l];
  const double e = total_energy / rho - 0.5 * V2;
  double err = 1;
  int iter = 0;
  double h_i[kMaxSpec], cp_i[kMaxSpec];
  while (err > 1e-5 && iter++ < 1000) {
    compute_enthalpy_and_cp(th, t, h_i, cp_i);
    double cp_tot = 0, h = 0;
    for (int l = 0; l < ns; ++l) {
      cp_tot += cp_i[l] * yk[l];
      h += h_i[l] * yk[l];
    }
    const double e_t = h - gas_const * t;
    const double cv = cp_tot - gas_const;
    const double t1 = t - (e_t - e) / cv;
    err = abs(1 - t1 / t);
    t = t1;
  }
  p = rho * t * gas_const;
  return err <= 1e-5;
}

__device__ __forceinline__ double omega_d(double t_red) {
  // reference src/Transport.cu:182-184
  return 1.0548 * pow(t_red, -0.15504) + pow(t_red + 0.55909, -2.1705);
}

// gamma, acoustic speed, Mach, mu, kappa, rho*D_k at one node
// (reference src/FieldOperation.cuh:95-114, src/Transport.cu:43-165).
__device__ __forceinline__ void mixture_properties_point(const Zone &z, const Param &p, const Thermo *th, int64_t id,
                                                         double temperature, double V) {
  const int64_t sz = z.d.plane(z.d.ngg);
  const int ns = p.n_spec;
  double imw = 0, cpm = 0;
  double cp[kMaxSpec], yk[kMaxSpec];
  compute_cp(th, temperature, cp);
  for (int l = 0; l < ns; ++l) {
    yk[l] = z.sv[id + l * sz];
    imw = fma(yk[l], th->imw[l], imw);
    cpm = fma(yk[l], cp[l], cpm);
  }
  const double R = kRu * imw;
  double gam = cpm / (cpm - R);
  z.gamma[id] = gam;
  const double a = sqrt(gam * R * temperature);
  z.acoustic_speed[id] = a;
  if (z.mach) z.mach[id] = V / a;

  const double mw_total = 1 / imw;
  double X[kMaxSpec], vis_denom[kMaxSpec];
  double temp = sqrt(temperature);
  for (int l = 0; l < ns; ++l) {
    X[l] = yk[l] * mw_total / th->mw[l];
    const double t_dl = temperature * th->LJ_potent_inv[l];
    const double t5 = t_dl + 0.5;  // (t_dl + 0.5)^-2 as a reciprocal square, not the general power
    vis_denom[l] = th->vis_coeff[l] * temp / (1.147 * pow(t_dl, -0.145) + 1.0 / (t5 * t5));
  }
  const double t_3over2_over_p = temperature * temp;
  double viscosity = 0, conductivity = 0;
  constexpr double pi = 3.141592653589793;
  for (int m = 0; m < ns; ++m) {
    double Rm = th->gas_const[m];
    double lambda = 15 * 0.25 * vis_denom[m] * Rm;
    const int geom = th->geometry[m];
    if (geom == 1 || geom == 2) {
      const double t_red = temperature * th->kb_over_eps_jk[m][m];
      const double tRedInv = 1 / t_red;
      temp = sqrt(tRedInv * pi) * pi;
      const double FT = 1 + 0.5 * temp + (2 + 0.25 * pi * pi) * tRedInv + temp * tRedInv;
      const double rhoD = th->binary_diffusivity_coeff[m][m] * t_3over2_over_p / (omega_d(t_red) * Rm * temperature);
      if (geom == 1) {
        const double ADivPiB = (2.5 * vis_denom[m] - rhoD) /
                               ((pi * th->ZRotF298[m] / FT * vis_denom[m] + 10.0 / 3 * vis_denom[m] + 2.0 * rhoD));
        lambda += -5 * ADivPiB * vis_denom[m] * Rm + rhoD * cp[m] + rhoD * (2 * ADivPiB - 2.5) * Rm;
      } else {
        const double ADivPiB = (2.5 * vis_denom[m] - rhoD) /
                               ((pi * th->ZRotF298[m] / FT * vis_denom[m] + 5 * vis_denom[m] + 2.0 * rhoD));
        lambda += -7.5 * ADivPiB * vis_denom[m] * Rm + rhoD * cp[m] + rhoD * (3 * ADivPiB - 2.5) * Rm;
      }
    }
    temp = 0;
    const double sq = sqrt(vis_denom[m]);
    for (int n = 0; n < ns; ++n) {
      double partition_func = 1.0;
      if (m != n) {
        const double numerator = 1.0 + rsqrt(vis_denom[n]) * (sq * th->WjDivWi_to_One4th[m][n]);
        partition_func = numerator * numerator * th->sqrt_WiDivWjPl1Mul8[m][n];
      }
      temp += partition_func * X[n];
    }
    viscosity += vis_denom[m] * X[m] / temp;
    conductivity += lambda * X[m] / (1.065 * temp - 0.065 * X[m]);
  }
  z.mul[id] = viscosity;
  z.thermal_conductivity[id] = conductivity;
  constexpr double eps = 1e-12;
  double sum = 0;
  for (int l = 0; l < ns; ++l) {
    temp = (X[l] + eps) * th->mw[l];
    cp[l] = temp;
    sum += temp;
    vis_denom[l] = 0;
  }
  for (int l = 0; l < ns; ++l) cp[l] = sum - cp[l];
  for (int l = 0; l < ns; ++l) {
    for (int n = l + 1; n < ns; ++n) {
      temp = omega_d(temperature * th->kb_over_eps_jk[l][n]) / (th->binary_diffusivity_coeff[l][n] * t_3over2_over_p);
      vis_denom[l] += (X[n] + eps) * temp;
      vis_denom[n] += (X[l] + eps) * temp;
    }
  }
  temp = 1.0 / (temperature * kRu);
  for (int l = 0; l < ns; ++l) z.rho_D[id + l * sz] = cp[l] * temp / vis_denom[l];
}

// Viscous spectral-radius velocity of the mixture (reference
// src/TimeAdvanceFunc.cuh:72-85).
__device__ __forceinline__ double mixture_max_diffuse_vel(const Zone &z, const Param &p, const Thermo *th, int64_t id,
                                                          double iRho) {
  const int64_t sz = z.d.plane(z.d.ngg);
  double cpl[kMaxSpec];
  compute_cp(th, z.bv[id + 5 * sz], cpl);
  double cp = 0, max_rhoD = 0;
  for (int l = 0; l < p.n_spec; ++l) {
    cp += cpl[l] * z.sv[id + l * sz];
    max_rhoD = max(max_rhoD, z.rho_D[id + l * sz]);
  }
  double mdv = z.mul[id] * iRho;
  mdv = max(mdv, z.thermal_conductivity[id] * iRho * z.gamma[id] / cp);
  mdv = max(mdv, max_rhoD * iRho);
  return mdv;
}

}  // namespace cfk
