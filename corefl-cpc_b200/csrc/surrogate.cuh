// MLP chemistry surrogate: parameter layout, feature transform and the
// element-conservation projection shared by the surrogate kernels.
//
// The network maps one cell's state before a reaction step of length dt to
// its change over that step:
//   inputs  (12): T, ln p, bc(Y_0..Y_8), ln dt
//   outputs (11): bc(Y_k,new) - bc(Y_k,old) for k = 0..8, T_new - T_old,
//                 ln(reaction time scale after the step)
// with bc the Box-Cox transform bc(Y) = ((Y + 1e-20)^0.1 - 1) / 0.1, which
// resolves trace radicals on a log-like scale.  Inputs are standardised with
// the training set's mean and standard deviation, outputs de-standardised.
//
// Network: 16 -> 128 -> 128 -> 128 -> 16 (three tanh hidden layers, linear
// output), BF16 operands with FP32 accumulation on the tensor cores.  Biases
// are folded into the GEMMs: input column 15 is the constant 1 (its weight
// column is the first layer's bias) and every hidden activation tile carries
// a constant-1 column 128 (the next layer's bias), padded to 144 columns.
// Weight blocks (rows = outputs, cols = inputs incl. bias/pad):
//   W0 128x16, W1 128x144, W2 128x144, W3 16x144.
// The FP32 master copy is row-major per block, concatenated in that order;
// the BF16 copy uses the same element count per block in the tensor-core
// core-matrix layout (rows grouped by 8, 8 columns = 16 bytes per row).
#pragma once

#include <cstdint>

#include "cfk_common.cuh"
#include "chem.cuh"
#include "thermo.cuh"

namespace cfk {

constexpr int kSgIn = 12, kSgOut = 11, kSgK0 = 16, kSgH = 128, kSgKH = 144, kSgNO = 16;
constexpr int kSgW0 = 0;
constexpr int kSgW1 = kSgW0 + 128 * 16;
constexpr int kSgW2 = kSgW1 + 128 * 144;
constexpr int kSgW3 = kSgW2 + 128 * 144;
constexpr int kSgNParam = kSgW3 + 16 * 144;  // 41216
constexpr int kSgWBytes = 2 * kSgNParam;     // 82432 bytes of BF16 weights
constexpr double kSgLambda = 0.1, kSgEps = 1e-20;

// Standardisation of inputs / outputs and the training range of the
// standardised inputs (out-of-distribution gate).  Output j is learnt as
// z_j = asinh(g_j / out_scale[j]) (g_j itself where out_scale[j] == 0),
// standardised with out_mean / out_std: increments far below the scale are
// resolved linearly, large ones (ignition) logarithmically.
struct SgNorm {
  float in_mean[kSgIn], in_rstd[kSgIn];
  float out_mean[kSgOut], out_std[kSgOut];
  float in_lo[kSgIn], in_hi[kSgIn];
  float out_scale[kSgOut];
};
static_assert(sizeof(SgNorm) == 81 * 4, "SgNorm is exchanged as 81 floats");

// raw target -> learnt variable, and back
__host__ __device__ inline double sg_target_fwd(double g, float scale) { return scale > 0 ? asinh(g / scale) : g; }
__host__ __device__ inline double sg_target_inv(double z, float scale) { return scale > 0 ? scale * sinh(z) : z; }

struct SgGate {
  double ood_margin;      // allowed excursion beyond the training range, standardised units
  double dT_max;          // |T change| per step above which the plain integrator runs (K)
  double dT_consistency;  // |network dT - energy-consistent dT| above which it runs (K)
  double judge_tol_T;     // judged cell: |T_surrogate - T_plain| tolerance (K)
  double judge_tol_bc;    // judged cell: max_k |bc(Y_surrogate) - bc(Y_plain)| tolerance
  double min_substeps;    // cells the plain integrator would finish in fewer substeps stay on it
  int judge_stride;       // every judge_stride-th cell (rotating) is judged; 0 = none
  int judge_salt;         // rotation of the judged subset (the step index)
  int revert_steps;       // steps a cell that failed the judge stays on the plain integrator
};

// Element mass fractions Z_e = sum_k mu[e][k] Y_k, mu = a_ek W_e / W_k.
struct SgProj {
  int n_elem;
  double mu[4][kMaxSpec];
};

struct SgJudge {
  unsigned int cell;
  float T;
  float Y[kMaxSpec];
};

enum SgCount {
  SG_CELLS = 0, SG_SURROGATE, SG_OOD, SG_IGNITION, SG_CONSISTENCY, SG_REVERT, SG_JUDGED, SG_JUDGE_FAILED,
  SG_NEWTON_FAILED, SG_CHEAP, SG_NCOUNT
};
struct SgCounters {
  unsigned long long n[SG_NCOUNT];
  unsigned long long judge_max_dT_bits, judge_max_dbc_bits;  // non-negative doubles as ordered bits
  double judge_sum_dT;
};

__host__ __device__ inline double sg_boxcox(double y) {
  return (pow((y > 0 ? y : 0.0) + kSgEps, kSgLambda) - 1.0) / kSgLambda;
}

// Inverse of sg_boxcox for lambda = 0.1: (1 + 0.1 b)^10 - eps, clipped at 0.
__host__ __device__ inline double sg_boxcox_inv(double b) {
  const double x = 1.0 + kSgLambda * b;
  if (x <= 0) return 0.0;
  const double x2 = x * x, x4 = x2 * x2, x5 = x4 * x;
  const double y = x5 * x5 - kSgEps;
  return y > 0 ? y : 0.0;
}

__host__ __device__ inline void sg_raw_features(double T, double p, const double *Y, int ns, double dt, double *f) {
  f[0] = T;
  f[1] = log(p);
  for (int k = 0; k < kMaxSpec; ++k) f[2 + k] = k < ns ? sg_boxcox(Y[k]) : 0.0;
  f[11] = log(dt);
}

// The state a node reaches when the frozen transport term of Wu's splitting
// acts alone for the fraction f of the reaction step: conserved variables
// q = q0 + f cq (cq = Cn dt / J over the whole step), partial densities
// rY0 + f crY clipped at 0 and scaled to the new density, Y = rY / rho, and T,
// p from the energy by the Newton iteration (T_guess to start).  Returns
// false when no partial density is left or the iteration fails.  Inside a
// flow the surrogate reads its features at f = 1/2 (the mid-step state the
// frozen transport passes through) and applies its predicted change to the
// f = 1 state; with Cn = 0 both are the node's own state.
__device__ inline bool sg_transported(const Thermo *th, int ns, const double *q0, const double *rY0, const double *cq,
                                      const double *crY, double f, double T_guess, double *q, double *Y, double &T,
                                      double &p) {
#pragma unroll
  for (int l = 0; l < 5; ++l) q[l] = q0[l] + f * cq[l];
  double sum = 0;
  for (int l = 0; l < ns; ++l) {
    Y[l] = fmax(rY0[l] + f * crY[l], 0.0);
    sum += Y[l];
  }
  if (!(sum > 0) || !(q[0] > 0)) return false;
  for (int l = 0; l < ns; ++l) Y[l] /= sum;
  for (int l = ns; l < kMaxSpec; ++l) Y[l] = 0.0;
  const double rinv = 1.0 / q[0];
  const double u = q[1] * rinv, v = q[2] * rinv, w = q[3] * rinv;
  T = T_guess;
  return temperature_newton(th, ns, Y, q[4], q[0], u * u + v * v + w * w, T, p);
}

// Both transported states of a node in one out-of-line call: the mid-step
// state (f = 1/2, Newton from T0) the features are read at, and the end state
// (f = 1, Newton from the mid-step T) the predicted change applies to.  With
// two inlined sg_transported calls in one kernel, nvcc 12.9 for sm_100a
// returned a wrong end state (a composition unrelated to q0 + cq and a
// spurious negative temperature root) while the mid-step state was right;
// the out-of-line form computes both correctly.
static __device__ __noinline__ bool sg_transported_pair(const Thermo *th, int ns, const double *q0, const double *rY0,
                                                        const double *cq, const double *crY, double T0, double *qm,
                                                        double *Ym, double &Tm, double &pm, double *qe, double *Ye,
                                                        double &Te, double &pe) {
  if (!sg_transported(th, ns, q0, rY0, cq, crY, 0.5, T0, qm, Ym, Tm, pm)) return false;
  return sg_transported(th, ns, q0, rY0, cq, crY, 1.0, Tm, qe, Ye, Te, pe);
}

// Weighted least-squares projection of Y onto {mu Y = Z0, Y >= 0}: the
// correction of species k is proportional to (Y_k + 1e-12), so trace species
// move least; species driven negative are clipped to 0 and frozen, and the
// projection is repeated over the rest (at most ns passes).  Returns false
// if the element residual max_e |mu Y - Z0| stays above 1e-10 (the caller
// then leaves the node to the plain integrator).  Y sums to 1 on success.
__device__ inline bool sg_project(const SgProj &pj, int ns, const double *Z0, double *Y) {
  const int ne = pj.n_elem;
  unsigned active = (1u << ns) - 1u;
  for (int pass = 0; pass < ns; ++pass) {
    double w[kMaxSpec], A[4][5];
    for (int k = 0; k < ns; ++k) w[k] = (active >> k & 1u) ? Y[k] + 1e-12 : 0.0;
    for (int e = 0; e < ne; ++e) {
      double r = Z0[e];
      for (int k = 0; k < ns; ++k) r -= pj.mu[e][k] * Y[k];
      A[e][ne] = r;
      for (int f = 0; f < ne; ++f) {
        double acc = 0;
        for (int k = 0; k < ns; ++k) acc += pj.mu[e][k] * w[k] * pj.mu[f][k];
        A[e][f] = acc;
      }
    }
    // Gaussian elimination with partial pivoting on the ne x ne system
    for (int c = 0; c < ne; ++c) {
      int piv = c;
      for (int r = c + 1; r < ne; ++r)
        if (fabs(A[r][c]) > fabs(A[piv][c])) piv = r;
      if (piv != c)
        for (int q = 0; q <= ne; ++q) { const double t = A[c][q]; A[c][q] = A[piv][q]; A[piv][q] = t; }
      if (!(fabs(A[c][c]) > 1e-300)) return false;
      const double inv = 1.0 / A[c][c];
      for (int r = c + 1; r < ne; ++r) {
        const double f = A[r][c] * inv;
        for (int q = c; q <= ne; ++q) A[r][q] -= f * A[c][q];
      }
    }
    double lam[4];
    for (int c = ne - 1; c >= 0; --c) {
      double acc = A[c][ne];
      for (int q = c + 1; q < ne; ++q) acc -= A[c][q] * lam[q];
      lam[c] = acc / A[c][c];
    }
    bool clipped = false;
    for (int k = 0; k < ns; ++k) {
      if (!(active >> k & 1u)) continue;
      double d = 0;
      for (int e = 0; e < ne; ++e) d += pj.mu[e][k] * lam[e];
      Y[k] += w[k] * d;
      if (Y[k] < 0) {
        Y[k] = 0;
        active &= ~(1u << k);
        clipped = true;
      }
    }
    if (!clipped) break;
  }
  double res = 0, sum = 0;
  for (int e = 0; e < ne; ++e) {
    double r = Z0[e];
    for (int k = 0; k < ns; ++k) r -= pj.mu[e][k] * Y[k];
    res = fmax(res, fabs(r));
  }
  for (int k = 0; k < ns; ++k) sum += Y[k];
  if (!(res <= 1e-10) || !(sum > 0)) return false;
  const double inv = 1.0 / sum;
  for (int k = 0; k < ns; ++k) Y[k] *= inv;
  return true;
}

}  // namespace cfk
