// Fused characteristic WENO flux + flux difference for a reacting mixture
// (NS species, thermally perfect, NASA-7 thermo).
//
// Restates compute_convective_term_weno_{x,y,z} with the mixture branch of
// the characteristic reconstruction (reference src/WENO.cu:1096-1469) and
// compute_derivative_{x,y,z} (:1544, 2219, 2885) in the stage / faces / diff
// structure of weno_air.cu:
//   stage — Q[5], the species densities rho*Y_k, the face-normal flux
//           G = (rho U, rho u U + p k_x, ..., (rho E + p) U), U, p, J and the
//           spectral radius |U| + c|grad k| (c from the acoustic-speed array)
//           of every stencil point, in shared memory;
//   faces — Roe average of u, v, w, Y_k and T, mixture gamma and c from the
//           NASA-7 cp at the averaged temperature, the five characteristic
//           fields with the species coupling terms (beta_k = (gamma R_k T -
//           (gamma-1) h_k) / c^2), NS species fields (rho Y_k - Y~_k rho),
//           LLF split, WENO5-JS / WENO7-Z, back projection;
//   diff  — dq -= F(n+1/2) - F(n-1/2) for all 5 + NS variables.
// The mixture tables are a __grid_constant__ parameter (constant bank).
#include "cfk_common.cuh"
#include "chem_fast.cuh"
#include "thermo.cuh"
#include "weno.cuh"

namespace cfk {

namespace {

// staged values per point: Q0..4, G0..4, U, p, J, lambda, rhoY[NS]
template <int NS>
struct MixVals {
  static constexpr int U = 10, P = 11, J = 12, LAM = 13, Y0 = 14, N = 14 + NS;
};

// Tile shapes of a sweep (nodes per column TN x columns C); VAR is chosen per
// direction by the tile autotuner.
template <int DIR, int VAR>
struct MixShape {
  static constexpr int TN = DIR == 0 ? (VAR == 0 ? 63 : VAR == 1 ? 127 : 31) : (VAR == 0 ? 15 : VAR == 1 ? 31 : 63);
  static constexpr int C = DIR == 0 ? (VAR == 0 ? 4 : VAR == 1 ? 2 : 8) : (VAR == 0 ? 16 : VAR == 1 ? 8 : 4);
};

template <int DIR, int ORD, int NS, int VAR = 0>
struct MixTile {
  static constexpr int R = ORD == 7 ? 3 : 2;
  static constexpr int NPF = 2 * R + 2;
  static constexpr int TN = MixShape<DIR, VAR>::TN;
  static constexpr int C = MixShape<DIR, VAR>::C;
  static constexpr int NF = TN + 1;
  static constexpr int NPT = TN + 2 * R + 2;
  static constexpr int NT = 256;
  static constexpr int NQ = MixVals<NS>::N;
  static constexpr int NV = 5 + NS;
  __device__ static int spt(int q, int c, int t) {
    return DIR == 0 ? (q * C + c) * NPT + t : (q * NPT + t) * C + c;
  }
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(NQ * C * NPT + NV * C * NF); }
};

// Positive-preserving limiter of the species face fluxes (reference
// src/WENO.cu:1471-1540; the characteristic scheme has it in the x sweep
// only).  For each species whose one-sided updates alpha/2 J rhoY -/+ dt f
// would go negative, the face flux is blended towards the first-order flux
// f1 = 1/2 (fp + U_L J_L rhoY_L) + 1/2 (fm - U_R J_R rhoY_R) with
// fp/m = 1/2 J (U +/- c|grad k|) rhoY, theta in [0, 1].  Out of line: the
// branch is rare and must not add registers to the face loop.  s/sf point at
// the staged values and face fluxes of this tile; the species face fluxes
// are updated in shared memory.
template <int ORD, int NS, int VAR>
__device__ __noinline__ void pp_limit_x(const double *s, double *sf, int c, int t, const Zone &z, int64_t idl,
                                        double dt, double alpha_dim, double rho_ref) {
  using T = MixTile<0, ORD, NS, VAR>;
  using V = MixVals<NS>;
  const int pc = t + T::R;
  const double jac_l = s[T::spt(V::J, c, pc)], jac_r = s[T::spt(V::J, c, pc + 1)];
  const double alphaL = 0.5 * alpha_dim * jac_l, alphaR = 0.5 * alpha_dim * jac_r;
  int start_l = -1;
  for (int l = 0; l < NS; ++l) {
    const double fl = sf[T::sfl(5 + l, c, t)];
    const double up = alphaL * s[T::spt(V::Y0 + l, c, pc)] - dt * fl;
    const double um = alphaR * s[T::spt(V::Y0 + l, c, pc + 1)] + dt * fl;
    if (up < 0 || um < 0) { start_l = l; break; }
  }
  if (start_l < 0) return;
  // c|grad k| of the two nodes, as staged by the reference (F[5])
  const int64_t sz = z.d.plane(z.d.ngg);
  double cg[2];
  for (int n = 0; n < 2; ++n) {
    const int64_t id = idl + n;
    const double m0 = z.metric[id], m1 = z.metric[id + sz], m2 = z.metric[id + 2 * sz];
    cg[n] = sqrt(m0 * m0 + m1 * m1 + m2 * m2) * z.acoustic_speed[id];
  }
  const double UkL = s[T::spt(V::U, c, pc)], UkR = s[T::spt(V::U, c, pc + 1)];
  const double U1 = UkL * jac_l, U2 = UkR * jac_r;
  for (int l = start_l; l < NS; ++l) {
    const double fc = sf[T::sfl(5 + l, c, t)];
    double f1 = 0, theta_p = 1.0, theta_m = 1.0;
    bool f1_computed = false;
    const double rhoYL = s[T::spt(V::Y0 + l, c, pc)], rhoYR = s[T::spt(V::Y0 + l, c, pc + 1)];
    const double fp = 0.5 * jac_l * (UkL + cg[0]) * rhoYL;
    const double fm = 0.5 * jac_r * (UkR - cg[1]) * rhoYR;
    const double up = alphaL * rhoYL - dt * fc;
    if (up < 0) {
      f1 = 0.5 * (fp + U1 * rhoYL) + 0.5 * (fm - U2 * rhoYR);
      f1_computed = true;
      const double up_lf = alphaL * rhoYL - dt * f1;
      if (abs(up - up_lf) > 1e-20 * rho_ref) theta_p = min(max((0 - up_lf) / (up - up_lf), 0.0), 1.0);
    }
    const double um = alphaR * rhoYR + dt * fc;
    if (um < 0) {
      if (!f1_computed) f1 = 0.5 * (fp + U1 * rhoYL) + 0.5 * (fm - U2 * rhoYR);
      const double um_lf = alphaR * rhoYR + dt * f1;
      if (abs(um - um_lf) > 1e-20 * rho_ref) theta_m = min(max((0 - um_lf) / (um - um_lf), 0.0), 1.0);
    }
    sf[T::sfl(5 + l, c, t)] = min(theta_p, theta_m) * (fc - f1) + f1;
  }
}

// Settings of the positive-preserving limiter: off unless `on`; the step's
// dt from the device (CFL runs) or the host (fixed dt); dt <= 0 selects the
// node's dt_local as the reference does.
struct PPArgs {
  int on;
  const double *dt_dev;
  double dt_host, alpha_dim, rho_ref;
};

}  // namespace

// HYB: hybrid UD/WENO scheme, the face switches on the shock sensor.
// VAR: tile shape (MixShape).
template <int DIR, int ORD, int NS, bool HYB, int VAR>
__global__ void __launch_bounds__(256) weno_mix_flux_diff(Zone z, double eps_ref, const __grid_constant__ Thermo thermo,
                                                          const double *sensor, double threshold, PPArgs pp) {
  using T = MixTile<DIR, ORD, NS, VAR>;
  using V = MixVals<NS>;
  constexpr int R = T::R, NPF = T::NPF, TN = T::TN, C = T::C, NF = T::NF, NPT = T::NPT;
  const Thermo *th = &thermo;
  extern __shared__ double sm[];
  double *spts = sm;
  double *sflx = sm + T::NQ * C * NPT;

  const Dims d = z.d;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int m = d.ext(DIR);
  int n0, cbase, cfix;
  if (DIR == 0) { n0 = blockIdx.x * TN; cbase = blockIdx.y * C; cfix = blockIdx.z; }
  else { n0 = blockIdx.y * TN; cbase = blockIdx.x * C; cfix = blockIdx.z; }
  const int ncol_max = DIR == 0 ? d.my : d.mx;
  auto node_idx = [&](int g_, int c, int a) -> int64_t {
    const int cc = cbase + c;
    if (DIR == 0) return d.idx(g_, a, cc, cfix);
    if (DIR == 1) return d.idx(g_, cc, a, cfix);
    return d.idx(g_, cc, cfix, a);
  };
  auto split = [&](int item, int n_t, int &c, int &t) {
    if (DIR == 0) { c = item / n_t; t = item - c * n_t; }
    else { t = item / C; c = item - t * C; }
  };
  const int mmo = 3 * DIR;
  double dt_pp = 0;
  if (DIR == 0 && pp.on) dt_pp = pp.dt_dev ? *pp.dt_dev : pp.dt_host;

  // ---- stage ------------------------------------------------------------
  for (int item = threadIdx.x; item < NPT * C; item += T::NT) {
    int c, t;
    split(item, NPT, c, t);
    const int a = n0 - 1 - R + t;
    if (cbase + c >= ncol_max || a > m + R) continue;
    const int64_t id = node_idx(g, c, a);
    const double q0 = z.cv[id], q1 = z.cv[id + sz], q2 = z.cv[id + 2 * sz], q3 = z.cv[id + 3 * sz],
                 q4 = z.cv[id + 4 * sz];
    const double m0 = z.metric[id + mmo * sz], m1 = z.metric[id + (mmo + 1) * sz], m2 = z.metric[id + (mmo + 2) * sz];
    const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
    const double pk = z.bv[id + 4 * sz];
    double *s = spts;
    s[T::spt(0, c, t)] = q0;
    s[T::spt(1, c, t)] = q1;
    s[T::spt(2, c, t)] = q2;
    s[T::spt(3, c, t)] = q3;
    s[T::spt(4, c, t)] = q4;
    s[T::spt(5, c, t)] = q0 * Uk;
    s[T::spt(6, c, t)] = fma(q1, Uk, pk * m0);
    s[T::spt(7, c, t)] = fma(q2, Uk, pk * m1);
    s[T::spt(8, c, t)] = fma(q3, Uk, pk * m2);
    s[T::spt(9, c, t)] = (q4 + pk) * Uk;
    s[T::spt(V::U, c, t)] = Uk;
    s[T::spt(V::P, c, t)] = pk;
    s[T::spt(V::J, c, t)] = z.jac[id];
    s[T::spt(V::LAM, c, t)] = abs(Uk) + sqrt(m0 * m0 + m1 * m1 + m2 * m2) * z.acoustic_speed[id];
#pragma unroll
    for (int l = 0; l < NS; ++l) s[T::spt(V::Y0 + l, c, t)] = z.cv[id + (5 + l) * sz];
  }
  __syncthreads();

  // ---- face fluxes ------------------------------------------------------
  for (int item = threadIdx.x; item < NF * C; item += T::NT) {
    int c, t;
    split(item, NF, c, t);
    const int f = n0 - 1 + t;
    if (cbase + c >= ncol_max || f > m - 1) continue;
    const double *s = spts;
    const int pc = t + R;
    // face normal averaged with the (i+1) node, as the reference does
    const int64_t idf = node_idx(g, c, f);
    double kx = 0.5 * (z.metric[idf + mmo * sz] + z.metric[idf + 1 + mmo * sz]);
    double ky = 0.5 * (z.metric[idf + (mmo + 1) * sz] + z.metric[idf + 1 + (mmo + 1) * sz]);
    double kz = 0.5 * (z.metric[idf + (mmo + 2) * sz] + z.metric[idf + 1 + (mmo + 2) * sz]);

    const double rho_l = s[T::spt(0, c, pc)], rho_r = s[T::spt(0, c, pc + 1)];
    double temp1 = sqrt(rho_l * rho_r);
    const double rlc = 1 / (rho_l + temp1);
    const double rrc = 1 / (temp1 + rho_r);
    const double um = rlc * s[T::spt(1, c, pc)] + rrc * s[T::spt(1, c, pc + 1)];
    const double vm = rlc * s[T::spt(2, c, pc)] + rrc * s[T::spt(2, c, pc + 1)];
    const double wm = rlc * s[T::spt(3, c, pc)] + rrc * s[T::spt(3, c, pc + 1)];
    double svm[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l)
      svm[l] = rlc * s[T::spt(V::Y0 + l, c, pc)] + rrc * s[T::spt(V::Y0 + l, c, pc + 1)];
    temp1 = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) temp1 += svm[l] * th->gas_const[l];
    double temp3 = (rlc * s[T::spt(V::P, c, pc)] + rrc * s[T::spt(V::P, c, pc + 1)]) / temp1;
    double hb[NS], cpb[NS];
    enthalpy_cp_ns<NS>(th, temp3, hb, cpb);  // compute_enthalpy_and_cp at the averaged T
    double temp2 = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) temp2 += svm[l] * cpb[l];
    const double gamma = temp2 / (temp2 - temp1);
    const double cm = sqrt(gamma * temp1 * temp3);
    const double gm1 = gamma - 1;
    temp1 = 1.0 / sqrt(kx * kx + ky * ky + kz * kz);
    kx *= temp1; ky *= temp1; kz *= temp1;
    const double Uk_bar = kx * um + ky * vm + kz * wm;
    double nx = 0, ny = 0, nz = 0;
    if (abs(kx) > 0.8) { nx = -kz; nz = kx; }
    else { ny = kz; nz = -ky; }
    temp1 = 1.0 / sqrt(nx * nx + ny * ny + nz * nz);
    nx *= temp1; ny *= temp1; nz *= temp1;
    double qx = ky * nz - kz * ny, qy = kz * nx - kx * nz, qz = kx * ny - ky * nx;
    temp1 = 1.0 / sqrt(qx * qx + qy * qy + qz * qz);
    qx *= temp1; qy *= temp1; qz *= temp1;
    const double Un = nx * um + ny * vm + nz * wm;
    const double Uq = qx * um + qy * vm + qz * wm;
    temp2 = 1.0 / (cm * cm);
    double beta[NS];
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      beta[l] = gamma * th->gas_const[l] * temp3 - gm1 * hb[l];
      beta[l] *= temp2;
    }
    const double alpha = 0.5 * gm1 * (um * um + vm * vm + wm * wm);
    double lam = 0;
#pragma unroll
    for (int q = 0; q < NPF; ++q) lam = max(lam, s[T::spt(V::LAM, c, t + q)]);
    const bool shock = !HYB || face_shocked(sensor, idf, d.stride(g, DIR), g, threshold);
    double sbq[NPF], sbf[NPF];
#pragma unroll
    for (int q = 0; q < NPF; ++q) {
      const int tq = t + q;
      const double uq = s[T::spt(V::U, c, tq)];
      double sp = 0, sn = 0;
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        const double ry = s[T::spt(V::Y0 + n, c, tq)];
        sp = fma(beta[n], ry, sp);
        sn = fma(beta[n], ry * uq, sn);
      }
      sbq[q] = sp;
      sbf[q] = sn;
    }

    double fChar[5 + NS];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      asm volatile("" ::: "memory");
      double L0, L1, L2, L3, L4, tb = 0.5;
      if (l == 0) {
        L0 = (alpha + Uk_bar * cm) * temp2 * 0.5;
        L1 = -(gm1 * um + kx * cm) * temp2 * 0.5;
        L2 = -(gm1 * vm + ky * cm) * temp2 * 0.5;
        L3 = -(gm1 * wm + kz * cm) * temp2 * 0.5;
        L4 = gm1 * temp2 * 0.5;
      } else if (l == 1) {
        tb = 0; L0 = -Un; L1 = nx; L2 = ny; L3 = nz; L4 = 0;
      } else if (l == 2) {
        tb = 0; L0 = -Uq; L1 = qx; L2 = qy; L3 = qz; L4 = 0;
      } else if (l == 3) {
        tb = -1;
        L0 = 1 - alpha * temp2;
        L1 = gm1 * um * temp2;
        L2 = gm1 * vm * temp2;
        L3 = gm1 * wm * temp2;
        L4 = -gm1 * temp2;
      } else {
        L0 = (alpha - Uk_bar * cm) * temp2 * 0.5;
        L1 = -(gm1 * um - kx * cm) * temp2 * 0.5;
        L2 = -(gm1 * vm - ky * cm) * temp2 * 0.5;
        L3 = -(gm1 * wm - kz * cm) * temp2 * 0.5;
        L4 = gm1 * temp2 * 0.5;
      }
      double vp[NPF - 1], vmn[NPF - 1];
#pragma unroll
      for (int q = 0; q < NPF; ++q) {
        const int tq = t + q;
        double LF = L0 * s[T::spt(5, c, tq)] + L1 * s[T::spt(6, c, tq)] + L2 * s[T::spt(7, c, tq)] +
                    L3 * s[T::spt(8, c, tq)];
        double LQ = L0 * s[T::spt(0, c, tq)] + L1 * s[T::spt(1, c, tq)] + L2 * s[T::spt(2, c, tq)] +
                    L3 * s[T::spt(3, c, tq)];
        if (l != 1 && l != 2) {  // the rows of fields 1 and 2 have no energy or species term
          LF = LF + L4 * s[T::spt(9, c, tq)] + tb * sbf[q];
          LQ = LQ + L4 * s[T::spt(4, c, tq)] + tb * sbq[q];
        }
        const double jq = s[T::spt(V::J, c, tq)];
        if (q < NPF - 1) vp[q] = 0.5 * jq * (LF + lam * LQ);
        if (q > 0) vmn[q - 1] = 0.5 * jq * (LF - lam * LQ);
      }
      if constexpr (ORD == 7) fChar[l] = shock ? weno7_z(vp, vmn, eps_ref) : weno7_linear(vp, vmn);
      else fChar[l] = shock ? weno5_js(vp, vmn, eps_ref) : weno5_linear(vp, vmn);
    }
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      asm volatile("" ::: "memory");
      double vp[NPF - 1], vmn[NPF - 1];
#pragma unroll
      for (int q = 0; q < NPF; ++q) {
        const int tq = t + q;
        const double LQ = s[T::spt(V::Y0 + l, c, tq)] - svm[l] * s[T::spt(0, c, tq)];
        const double LF = s[T::spt(V::U, c, tq)] * LQ;
        const double jq = s[T::spt(V::J, c, tq)];
        if (q < NPF - 1) vp[q] = 0.5 * jq * (LF + lam * LQ);
        if (q > 0) vmn[q - 1] = 0.5 * jq * (LF - lam * LQ);
      }
      if constexpr (ORD == 7) fChar[5 + l] = shock ? weno7_z(vp, vmn, eps_ref) : weno7_linear(vp, vmn);
      else fChar[5 + l] = shock ? weno5_js(vp, vmn, eps_ref) : weno5_linear(vp, vmn);
    }
    const double f034 = fChar[0] + fChar[3] + fChar[4];
    const double f04 = fChar[0] - fChar[4];
    const double H = rlc * (s[T::spt(4, c, pc)] + s[T::spt(V::P, c, pc)]) +
                     rrc * (s[T::spt(4, c, pc + 1)] + s[T::spt(V::P, c, pc + 1)]);
    sflx[T::sfl(0, c, t)] = f034;
    sflx[T::sfl(1, c, t)] = um * f034 - kx * cm * f04 + nx * fChar[1] + qx * fChar[2];
    sflx[T::sfl(2, c, t)] = vm * f034 - ky * cm * f04 + ny * fChar[1] + qy * fChar[2];
    sflx[T::sfl(3, c, t)] = wm * f034 - kz * cm * f04 + nz * fChar[1] + qz * fChar[2];
    double f4 = H * f034 - Uk_bar * cm * f04 + Un * fChar[1] + Uq * fChar[2] - cm * cm / gm1 * fChar[3];
    double bsum = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      sflx[T::sfl(5 + l, c, t)] = svm[l] * f034 + fChar[5 + l];
      bsum += beta[l] * fChar[5 + l];
    }
    f4 -= bsum * cm * cm / gm1;
    sflx[T::sfl(4, c, t)] = f4;
    if constexpr (DIR == 0) {
      if (pp.on) {
        const double dt = dt_pp > 0 ? dt_pp : z.dt_local[node_idx(0, c, f < 0 ? 0 : f)];
        pp_limit_x<ORD, NS, VAR>(s, sflx, c, t, z, idf, dt, pp.alpha_dim, pp.rho_ref);
      }
    }
  }
  __syncthreads();

  // ---- flux difference into dq -----------------------------------------
  for (int item = threadIdx.x; item < TN * C; item += T::NT) {
    int c, t;
    split(item, TN, c, t);
    const int a = n0 + t;
    if (cbase + c >= ncol_max || a > m - 1) continue;
    const int64_t iq = node_idx(0, c, a);
#pragma unroll
    for (int v = 0; v < T::NV; ++v) z.dq[iq + v * szq] -= sflx[T::sfl(v, c, t + 1)] - sflx[T::sfl(v, c, t)];
  }
}

namespace {

template <int DIR, int ORD, int VAR>
cudaError_t launch_mix_var(const Zone &z, double eps_ref, const Thermo &th, const double *sensor, double threshold,
                           const PPArgs &pp, cudaStream_t st) {
  using T = MixTile<DIR, ORD, kMaxSpec, VAR>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  if (sensor)
    weno_mix_flux_diff<DIR, ORD, kMaxSpec, true, VAR>
        <<<grid, T::NT, T::smem_bytes(), st>>>(z, eps_ref, th, sensor, threshold, pp);
  else
    weno_mix_flux_diff<DIR, ORD, kMaxSpec, false, VAR>
        <<<grid, T::NT, T::smem_bytes(), st>>>(z, eps_ref, th, nullptr, threshold, pp);
  return cudaGetLastError();
}

template <int DIR, int ORD>
cudaError_t launch_mix_dir(const Zone &z, double eps_ref, const Thermo &th, const double *sensor, double threshold,
                           const PPArgs &pp, int var, cudaStream_t st) {
  if (var == 1) return launch_mix_var<DIR, ORD, 1>(z, eps_ref, th, sensor, threshold, pp, st);
  if (var == 2) return launch_mix_var<DIR, ORD, 2>(z, eps_ref, th, sensor, threshold, pp, st);
  return launch_mix_var<DIR, ORD, 0>(z, eps_ref, th, sensor, threshold, pp, st);
}

template <int DIR, int ORD, int VAR>
cudaError_t set_mix_attr() {
  const int b = (int)MixTile<DIR, ORD, kMaxSpec, VAR>::smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(weno_mix_flux_diff<DIR, ORD, kMaxSpec, false, VAR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(weno_mix_flux_diff<DIR, ORD, kMaxSpec, true, VAR>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

template <int DIR, int ORD>
cudaError_t set_mix_attrs() {
  cudaError_t e;
  if ((e = set_mix_attr<DIR, ORD, 0>()) != cudaSuccess) return e;
  if ((e = set_mix_attr<DIR, ORD, 1>()) != cudaSuccess) return e;
  return set_mix_attr<DIR, ORD, 2>();
}

}  // namespace

cudaError_t weno_mix_init_attributes() {
  cudaError_t e;
  if ((e = set_mix_attrs<0, 5>()) != cudaSuccess) return e;
  if ((e = set_mix_attrs<1, 5>()) != cudaSuccess) return e;
  if ((e = set_mix_attrs<2, 5>()) != cudaSuccess) return e;
  if ((e = set_mix_attrs<0, 7>()) != cudaSuccess) return e;
  if ((e = set_mix_attrs<1, 7>()) != cudaSuccess) return e;
  return set_mix_attrs<2, 7>();
}

// One sweep (dir 0/1/2) with tile variant var; the species count is fixed at
// 9 (kMaxSpec).  dt_dev / dt_host: the step's dt for the positive-preserving
// limiter (x sweep only, as in the reference).
cudaError_t launch_weno_mix_dir(const Zone &z, const Param &p, const Thermo &th, const double *dt_dev,
                                double dt_host, int dir, int var, cudaStream_t st) {
  const double eps_ref = kEpsWeno * p.weno_eps_scale;
  const double tr = p.sensor_threshold;
  const double *sn = tr > 1e-10 ? z.shock_sensor : nullptr;  // hybrid UD + WENO
  const PPArgs pp{p.positive_preserving && dir == 0 ? 1 : 0, dt_dev, dt_host, p.dim == 3 ? 1.0 / 3.0 : 0.5,
                  p.rho_ref};
  const bool w7 = p.inviscid_scheme == 72;
  if (dir == 0)
    return w7 ? launch_mix_dir<0, 7>(z, eps_ref, th, sn, tr, pp, var, st)
              : launch_mix_dir<0, 5>(z, eps_ref, th, sn, tr, pp, var, st);
  if (dir == 1)
    return w7 ? launch_mix_dir<1, 7>(z, eps_ref, th, sn, tr, pp, var, st)
              : launch_mix_dir<1, 5>(z, eps_ref, th, sn, tr, pp, var, st);
  return w7 ? launch_mix_dir<2, 7>(z, eps_ref, th, sn, tr, pp, var, st)
            : launch_mix_dir<2, 5>(z, eps_ref, th, sn, tr, pp, var, st);
}

// x, y and (3-D) z sweeps; var[d] is the tile variant of sweep d.
cudaError_t launch_weno_mix(const Zone &z, const Param &p, const Thermo &th, const double *dt_dev, double dt_host,
                            const int *var, cudaStream_t st, int *n_launch) {
  const int nd = z.d.mz > 1 ? 3 : 2;
  for (int dir = 0; dir < nd; ++dir) {
    cudaError_t e = launch_weno_mix_dir(z, p, th, dt_dev, dt_host, dir, var[dir], st);
    if (e != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
