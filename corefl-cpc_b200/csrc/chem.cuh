// Finite-rate kinetics on the device: forward/backward rates, rates of
// progress, species sources, the analytic source Jacobian and the pivoted LU
// solve of the point-implicit system (reference src/FiniteRateChem.cu:1466-1822).
//
// Differences in form, not in the model: A T^b exp(-Ea/T) is evaluated as
// A exp(b ln T - Ea/T) with ln T and 1/T formed once per call; the
// equilibrium constant's (p_atm / R_u T)^order is an integer power; the
// sums over reactions run over per-reaction species lists prepared on the
// host, in the reference's reaction order, so only zero terms are skipped.
#pragma once

#include "cfk_common.cuh"
#include "thermo.cuh"

namespace cfk {

constexpr int kMaxReac = 24;
constexpr int kMaxInvolved = 6;  // distinct species appearing in one reaction

struct Kinetics {
  int n_reac;
  int type[kMaxReac], rev[kMaxReac], order[kMaxReac];
  double A[kMaxReac], b[kMaxReac], Ea[kMaxReac], A2[kMaxReac], b2[kMaxReac], Ea2[kMaxReac];
  double troe_alpha[kMaxReac], troe_t3[kMaxReac], troe_t1[kMaxReac], troe_t2[kMaxReac];
  double tb[kMaxReac][kMaxSpec];  // third-body efficiencies
  // species of reaction r: index, forward and backward stoichiometry
  int n_inv[kMaxReac];
  int inv_sp[kMaxReac][kMaxInvolved];
  int inv_f[kMaxReac][kMaxInvolved], inv_b[kMaxReac][kMaxInvolved];
  // the same stoichiometry dense per species, with bit masks of the species
  // involved (inv_mask) and of those with a non-zero net coefficient
  // (net_mask), for loops whose species index is a compile-time constant
  signed char stf[kMaxReac][kMaxSpec], stb[kMaxReac][kMaxSpec];
  unsigned int inv_mask[kMaxReac], net_mask[kMaxReac];
};

// Mixture and mechanism tables in one device block.
struct Mech {
  Thermo th;
  Kinetics kn;
};

__device__ __forceinline__ double ipow(double c, int n) {
  double r = 1.0;
  for (int k = 0; k < n; ++k) r *= c;
  return r;
}

// G_k / (R T), NASA-7 branch of compute_gibbs_div_rt (reference src/Thermo.cu:576-606)
__device__ __forceinline__ void gibbs_div_rt(const Thermo *th, double t, double lnT, double iT, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
  for (int i = 0; i < th->n_spec; ++i) {
    if (t < th->t_low[i] || t > th->t_high[i]) {
      const bool lo = t < th->t_low[i];
      const double tt = lo ? th->t_low[i] : th->t_high[i];
      const double *c = lo ? th->low[i] : th->high[i];
      const double tt2 = tt * tt, tt3 = tt2 * tt, tt4 = tt3 * tt;
      g[i] = c[0] * (1.0 - log(tt)) - 0.5 * c[1] * tt - c[2] * tt2 / 6.0 - c[3] * tt3 / 12.0 - c[4] * tt4 * 0.05 +
             c[5] / tt - c[6];
    } else {
      const double *c = t < th->t_mid[i] ? th->low[i] : th->high[i];
      g[i] = c[0] * (1.0 - lnT) - 0.5 * c[1] * t - c[2] * t2 / 6.0 - c[3] * t3 / 12.0 - c[4] * t4 * 0.05 + c[5] * iT -
             c[6];
    }
  }
}

// Rates of progress q1 (forward) and q2 (backward) in mol/(cm^3 s) from the
// concentrations c in mol/cm^3 (forward_reaction_rate, backward_reaction_rate,
// rate_of_progress: reference src/FiniteRateChem.cu:1466-1587).
__device__ __forceinline__ void rates_of_progress(const Mech *mc, double t, const double *c, double *q1,
                                                  double *q2) {
  const Kinetics &kn = mc->kn;
  const int ns = mc->th.n_spec;
  const double lnT = log(t), iT = 1.0 / t;
  double g[kMaxSpec];
  gibbs_div_rt(&mc->th, t, lnT, iT, g);
  constexpr double temp_p = 101325.0 / kRu * 1e-3;  // mol K / cm^3
  const double temp_t = temp_p * iT;
  for (int r = 0; r < kn.n_reac; ++r) {
    const int type = kn.type[r];
    double kf = kn.A[r] * exp(kn.b[r] * lnT - kn.Ea[r] * iT);
    double cc = 0;
    if (type > 3)
      for (int l = 0; l < ns; ++l) cc += c[l] * kn.tb[r][l];
    if (type == 3) {
      kf += kn.A2[r] * exp(kn.b2[r] * lnT - kn.Ea2[r] * iT);
    } else if (type == 4) {
      kf *= cc;
    } else if (type > 4) {
      const double kf_low = kn.A2[r] * exp(kn.b2[r] * lnT - kn.Ea2[r] * iT);
      const double kf_high = kf;
      if (kf_high < 1e-25 && kf_low < 1e-25) {
        kf = 0;
      } else {
        const double pr = kf_low * cc / kf_high;
        double F = 1.0;
        if (type > 5) {
          double f_cent = (1 - kn.troe_alpha[r]) * exp(-t / kn.troe_t3[r]) + kn.troe_alpha[r] * exp(-t / kn.troe_t1[r]);
          if (type == 7) f_cent += exp(-kn.troe_t2[r] * iT);
          const double logFc = log10(f_cent);
          const double cq = -0.4 - 0.67 * logFc;
          const double n = 0.75 - 1.27 * logFc;
          const double logPr = log10(pr);
          const double tempo = (logPr + cq) / (n - 0.14 * (logPr + cq));
          F = exp10(logFc / (1.0 + tempo * tempo));
        }
        kf = kf_high * pr / (1.0 + pr) * F;
      }
    }
    double kb = 0;
    if (type != 0) {
      // kb = kf / Kc for every reversible reaction, including REV ones, as the
      // reference's second loop does (reference src/FiniteRateChem.cu:1549-1559)
      double d_gibbs = 0;
      for (int q = 0; q < kn.n_inv[r]; ++q)
        d_gibbs += g[kn.inv_sp[r][q]] * (kn.inv_b[r][q] - kn.inv_f[r][q]);
      const int o = kn.order[r];
      double pw = 1.0;
      for (int k = 0; k < (o < 0 ? -o : o); ++k) pw *= temp_t;
      const double kc = (o < 0 ? 1.0 / pw : pw) * exp(-d_gibbs);
      kb = kf / kc;
    }
    double a = kf, bb = kb;
    for (int q = 0; q < kn.n_inv[r]; ++q) {
      const double cs = c[kn.inv_sp[r][q]];
      a *= ipow(cs, kn.inv_f[r][q]);
      bb *= ipow(cs, kn.inv_b[r][q]);
    }
    q1[r] = a;
    q2[r] = type != 0 ? bb : 0.0;
  }
}

// Species sources omega and destruction rates omega_d in kg/(m^3 s)
// (chemical_source, reference src/FiniteRateChem.cu:1589-1605).
__device__ __forceinline__ void species_sources(const Mech *mc, const double *q1, const double *q2, double *omega,
                                                double *omega_d) {
  const Kinetics &kn = mc->kn;
  const int ns = mc->th.n_spec;
  double creation[kMaxSpec];
  for (int l = 0; l < ns; ++l) { creation[l] = 0; omega_d[l] = 0; }
  for (int r = 0; r < kn.n_reac; ++r)
    for (int q = 0; q < kn.n_inv[r]; ++q) {
      const int l = kn.inv_sp[r][q];
      const double f = kn.inv_f[r][q], bq = kn.inv_b[r][q];
      creation[l] += q2[r] * f + q1[r] * bq;
      omega_d[l] += q1[r] * f + q2[r] * bq;
    }
  for (int l = 0; l < ns; ++l) {
    const double w = 1e+3 / mc->th.imw[l];
    creation[l] *= w;
    omega_d[l] *= w;
    omega[l] = creation[l] - omega_d[l];
  }
}

// In-place column-pivoted LU solve of lhs x = rhs, the reference's
// Crout-type elimination order (reference src/FiniteRateChem.cu:1769-1822).
__device__ __forceinline__ void solve_chem_system(double *lhs, double *rhs, int dim) {
  int ipiv[kMaxSpec];
  for (int n = 0; n < dim; ++n) {
    int ik = n;
    for (int m = n; m < dim; ++m) {
      for (int t = 0; t < n; ++t) lhs[m * dim + n] -= lhs[m * dim + t] * lhs[t * dim + n];
      if (abs(lhs[m * dim + n]) > abs(lhs[ik * dim + n])) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n)
      for (int t = 0; t < dim; ++t) {
        const double mid = lhs[ik * dim + t];
        lhs[ik * dim + t] = lhs[n * dim + t];
        lhs[n * dim + t] = mid;
      }
    for (int p = n + 1; p < dim; ++p)
      for (int t = 0; t < n; ++t) lhs[n * dim + p] -= lhs[n * dim + t] * lhs[t * dim + p];
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

}  // namespace cfk
