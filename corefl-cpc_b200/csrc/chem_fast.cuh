// Point-implicit reaction substep with the species count fixed at compile
// time.  Same model and, term by term, the same arithmetic order as the
// runtime-count path in chem.cu/chem.cuh (reference
// src/FiniteRateChem.cu:1466-1822, src/StrangSplitting.cu:43-224), laid out
// for the GPU:
//  * every per-species quantity is a register array indexed by compile-time
//    constants; a reaction's species are selected with the uniform bit masks
//    of the dense stoichiometry tables (all lanes process the same reaction,
//    so these branches never diverge);
//  * rates of progress are consumed as soon as they are formed: sources,
//    destruction rates and the Jacobian are accumulated reaction by reaction
//    (each accumulator still sums the reactions in mechanism order);
//  * the NS x NS system matrix and right-hand side live in shared memory,
//    entry e of lane t at base[e * stride + t], so the Jacobian's sparse
//    accumulation and the pivoted LU's runtime row indices address shared
//    memory rather than local memory;
//  * the mechanism tables are a __grid_constant__ kernel parameter: uniform
//    reads through the constant cache;
//  * divisions by the same value are one reciprocal and products, so results
//    match the runtime-count path to rounding, not bit for bit.
#pragma once

#include "chem.cuh"
#include "thermo.cuh"

namespace cfk {

template <int NS>
__device__ __forceinline__ void enthalpy_cp_ns(const Thermo *th, double t, double *h, double *cp) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
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

template <int NS>
__device__ __forceinline__ bool temperature_newton_ns(const Thermo *th, const double *yk, double total_energy,
                                                      double rho, double V2, double &t, double &p) {
  double gas_const = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) gas_const += yk[l] * th->gas_const[l];
  const double e = total_energy / rho - 0.5 * V2;
  double err = 1;
  int iter = 0;
  while (err > 1e-5 && iter++ < 1000) {
    double h_i[NS], cp_i[NS];
    enthalpy_cp_ns<NS>(th, t, h_i, cp_i);
    double cp_tot = 0, h = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
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

template <int NS>
__device__ __forceinline__ void gibbs_ns(const Thermo *th, double t, double lnT, double iT, double *g) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
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

// A per-lane slot in shared memory: entry e at p[e * stride].
struct LaneSlot {
  double *p;
  int stride;
  __device__ __forceinline__ double &operator()(int e) const { return p[e * stride]; }
};

// Column-pivoted LU solve of L x = R in the elimination order of
// solve_chem_system (divisions by a pivot as one reciprocal each); L and R
// are overwritten, x returned in registers.
template <int NS>
__device__ __forceinline__ void lu_solve_ns(const LaneSlot &L, const LaneSlot &R, double *x) {
  int ipiv[NS];
  double rdiag[NS];
#pragma unroll
  for (int n = 0; n < NS; ++n) {
    int ik = n;
#pragma unroll
    for (int m = n; m < NS; ++m) {
      double v = L(m * NS + n);
#pragma unroll
      for (int t = 0; t < n; ++t) v -= L(m * NS + t) * L(t * NS + n);
      L(m * NS + n) = v;
      if (abs(v) > abs(L(ik * NS + n))) ik = m;
    }
    ipiv[n] = ik;
    if (ik != n) {
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        const double mid = L(ik * NS + t);
        L(ik * NS + t) = L(n * NS + t);
        L(n * NS + t) = mid;
      }
    }
#pragma unroll
    for (int p = n + 1; p < NS; ++p) {
      double v = L(n * NS + p);
#pragma unroll
      for (int t = 0; t < n; ++t) v -= L(n * NS + t) * L(t * NS + p);
      L(n * NS + p) = v;
    }
    rdiag[n] = 1.0 / L(n * NS + n);
#pragma unroll
    for (int m = n + 1; m < NS; ++m) L(m * NS + n) *= rdiag[n];
  }
#pragma unroll
  for (int m = 0; m < NS; ++m) {
    const int t = ipiv[m];
    if (t != m) {
      const double mid = R(t);
      R(t) = R(m);
      R(m) = mid;
    }
  }
#pragma unroll
  for (int m = 0; m < NS; ++m) x[m] = R(m);
#pragma unroll
  for (int m = 1; m < NS; ++m)
#pragma unroll
    for (int t = 0; t < m; ++t) x[m] -= L(m * NS + t) * x[t];
  x[NS - 1] *= rdiag[NS - 1];
#pragma unroll
  for (int m = NS - 2; m >= 0; --m) {
#pragma unroll
    for (int t = m + 1; t < NS; ++t) x[m] -= L(m * NS + t) * x[t];
    x[m] *= rdiag[m];
  }
}

template <int NS>
struct NodeStateN {
  double q[5];
  double rY[NS];
  double T;
  double cn[5], cnY[NS];
  double iJac;
  double ts;  // reaction time scale
};

template <int NS>
__device__ __forceinline__ void load_node_ns(const Zone &z, int64_t id, int64_t iq, NodeStateN<NS> &s, double *yk,
                                             double &pres) {
  const int64_t sz = z.d.plane(z.d.ngg), szq = z.d.plane(0);
#pragma unroll
  for (int l = 0; l < 5; ++l) s.q[l] = z.cv[id + l * sz];
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    s.rY[l] = z.cv[id + (5 + l) * sz];
    yk[l] = z.sv[id + l * sz];
  }
  s.T = z.bv[id + 5 * sz];
  pres = z.bv[id + 4 * sz];
  if (z.Cn) {
#pragma unroll
    for (int l = 0; l < 5; ++l) s.cn[l] = z.Cn[iq + l * szq];
#pragma unroll
    for (int l = 0; l < NS; ++l) s.cnY[l] = z.Cn[iq + (5 + l) * szq];
  } else {
#pragma unroll
    for (int l = 0; l < 5; ++l) s.cn[l] = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) s.cnY[l] = 0;
  }
  s.iJac = 1.0 / z.jac[id];
  s.ts = z.reaction_timeScale[id];
}

template <int NS>
__device__ __forceinline__ void store_node_ns(const Zone &z, int n_scalar, int64_t id, const NodeStateN<NS> &s,
                                              const double *yk, double pres) {
  const int64_t sz = z.d.plane(z.d.ngg);
#pragma unroll
  for (int l = 0; l < 5; ++l) z.cv[id + l * sz] = s.q[l];
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    z.cv[id + (5 + l) * sz] = s.rY[l];
    z.sv[id + l * sz] = yk[l];
  }
  const double rho_inv = 1.0 / s.q[0];
  for (int l = NS; l < n_scalar; ++l) z.sv[id + l * sz] = z.cv[id + (5 + l) * sz] * rho_inv;
  z.bv[id] = s.q[0];
  z.bv[id + sz] = s.q[1] * rho_inv;
  z.bv[id + 2 * sz] = s.q[2] * rho_inv;
  z.bv[id + 3 * sz] = s.q[3] * rho_inv;
  z.bv[id + 4 * sz] = pres;
  z.bv[id + 5 * sz] = s.T;
  z.reaction_timeScale[id] = s.ts;
}

// One substep of wu_zeroDReaction (methods 0 and 1).
template <int NS>
__device__ __forceinline__ bool zero_d_substep_ns(const Mech *mc, int method, double dt, NodeStateN<NS> &s,
                                                  double *yk, double &pres, const LaneSlot &L, const LaneSlot &R) {
  const Thermo *th = &mc->th;
  const Kinetics &kn = mc->kn;
  double c[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) c[l] = s.rY[l] * th->imw[l] * 1e-3;
  const double t = s.T, lnT = log(t), iT = 1.0 / t;
  double g[NS];
  gibbs_ns<NS>(th, t, lnT, iT, g);
  constexpr double temp_p = 101325.0 / kRu * 1e-3;  // mol K / cm^3
  const double temp_t = temp_p * iT;
  double creation[NS], omega_d[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) { creation[l] = 0; omega_d[l] = 0; }
  if (method == 1) {
#pragma unroll
    for (int e = 0; e < NS * NS; ++e) L(e) = 0;
  }
  for (int r = 0; r < kn.n_reac; ++r) {
    const int type = kn.type[r];
    const unsigned inv = kn.inv_mask[r];
    double kf = kn.A[r] * exp(kn.b[r] * lnT - kn.Ea[r] * iT);
    double cc = 0;
    if (type > 3) {
#pragma unroll
      for (int l = 0; l < NS; ++l) cc += c[l] * kn.tb[r][l];
    }
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
      double d_gibbs = 0;
#pragma unroll
      for (int l = 0; l < NS; ++l)
        if (inv >> l & 1u) d_gibbs += g[l] * (kn.stb[r][l] - kn.stf[r][l]);
      const int o = kn.order[r];
      double pw = 1.0;
      for (int k = 0; k < (o < 0 ? -o : o); ++k) pw *= temp_t;
      const double kc = (o < 0 ? 1.0 / pw : pw) * exp(-d_gibbs);
      kb = kf / kc;
    }
    double a = kf, bb = kb;
#pragma unroll
    for (int l = 0; l < NS; ++l)
      if (inv >> l & 1u) {
        a *= ipow(c[l], kn.stf[r][l]);
        bb *= ipow(c[l], kn.stb[r][l]);
      }
    const double q1 = a, q2 = type != 0 ? bb : 0.0;
#pragma unroll
    for (int l = 0; l < NS; ++l)
      if (inv >> l & 1u) {
        const double f = kn.stf[r][l], bq = kn.stb[r][l];
        creation[l] += q2 * f + q1 * bq;
        omega_d[l] += q1 * f + q2 * bq;
      }
    if (method == 1) {
      // the matrix is in shared memory: its runtime row/column indices are free
      const int ni = kn.n_inv[r];
      for (int qa = 0; qa < ni; ++qa) {
        const double net = kn.inv_b[r][qa] - kn.inv_f[r][qa];
        if (net == 0) continue;
        const int m = kn.inv_sp[r][qa];
        for (int qb = 0; qb < ni; ++qb)
          L(m * NS + kn.inv_sp[r][qb]) += net * (kn.inv_f[r][qb] * q1 - kn.inv_b[r][qb] * q2);
      }
    }
  }
  double omega[NS];
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    const double w = 1e+3 / th->imw[l];
    creation[l] *= w;
    omega_d[l] *= w;
    omega[l] = creation[l] - omega_d[l];
  }
#pragma unroll
  for (int l = 0; l < NS; ++l) c[l] *= 1e+3 / th->imw[l];
  if (method == 1) {
    // (I - dt J): J_mn / rhoY_n * 1e3 / imw_m, with the 2 NS divisions hoisted
    double rc[NS], wm[NS];
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      rc[n] = c[n] > 1e-25 ? 1.0 / c[n] : 0.0;
      wm[n] = 1e+3 / th->imw[n];
    }
#pragma unroll
    for (int m = 0; m < NS; ++m)
#pragma unroll
      for (int n = 0; n < NS; ++n) L(m * NS + n) = (m == n ? 1 : 0) - dt * (L(m * NS + n) * rc[n] * wm[m]);
#pragma unroll
    for (int l = 0; l < NS; ++l) R(l) = omega[l];
    lu_solve_ns<NS>(L, R, omega);
  }
#pragma unroll
  for (int l = 0; l < 5; ++l) s.q[l] += s.cn[l] * dt * s.iJac;
  double time_scale = 1e6;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    if (s.rY[l] > 1e-25 && abs(omega_d[l]) > 1e-25) time_scale = min(time_scale, abs(s.rY[l] / omega_d[l]));
    s.rY[l] += (omega[l] + s.cnY[l] * s.iJac) * dt;
  }
  s.ts = time_scale;
  const double rho = s.q[0];
  const double rho_inv = 1.0 / rho;
  const double u = s.q[1] * rho_inv, v = s.q[2] * rho_inv, w = s.q[3] * rho_inv;
  double sum = 0;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    if (s.rY[l] < 0) s.rY[l] = 0;
    else sum += s.rY[l];
  }
  sum = 1.0 / sum;
  const double ratio = rho * sum;
#pragma unroll
  for (int l = 0; l < NS; ++l) {
    yk[l] = s.rY[l] * sum;
    s.rY[l] *= ratio;
  }
  return temperature_newton_ns<NS>(th, yk, s.q[4], rho, u * u + v * v + w * w, s.T, pres);
}

}  // namespace cfk
