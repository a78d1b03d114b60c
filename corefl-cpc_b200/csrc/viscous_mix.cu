// Fused second-order viscous flux + flux difference for a mixture.
//
// Restates compute_{f,g,h}v_2nd_order, mixture branch (reference
// src/ViscousScheme.cu:614-1173: stress, heat flux with the mixture
// conductivity, mixture-averaged species diffusion rho D_k (grad Y_k -
// Y_k grad W / W) with the correction velocity, and the enthalpy flux
// sum h_k J_k at the face temperature), and compute_dFv_dx / dGv_dy / dHv_dz
// (:75-127).  Same face tiling as viscous_air.cu; the face fluxes of all
// 4 + NS viscous components stay in shared memory.  With gradp set the
// diffusion driving force also carries the pressure-gradient term
// (W/W_k - 1) Y_k grad(xi).grad(p) / p of gradPInDiffusionFlux (reference
// src/ViscousScheme.cu:742-766, 931-955, 1115-1139), p taken at the face.
#include "cfk_common.cuh"
#include "chem_fast.cuh"
#include "thermo.cuh"

namespace cfk {

namespace {
template <int DIR, int NS>
struct VisMixTile {
  static constexpr int TN = DIR == 0 ? 63 : 15;
  static constexpr int C = DIR == 0 ? 4 : 16;
  static constexpr int NF = TN + 1;
  static constexpr int NT = 256;
  static constexpr int NVF = 4 + NS;
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(NVF * C * NF); }
};
}  // namespace

template <int DIR, int NS>
__global__ void __launch_bounds__(256) viscous_mix_flux_diff(Zone z, const __grid_constant__ Thermo thermo,
                                                             int gradp) {
  using T = VisMixTile<DIR, NS>;
  constexpr int TN = T::TN, C = T::C, NF = T::NF;
  const Thermo *th = &thermo;
  extern __shared__ double sflx[];
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
  const int64_t sd = d.stride(g, DIR);
  constexpr int DA = (DIR + 1) % 3, DB = (DIR + 2) % 3;
  const int64_t sa = d.stride(g, DA), sb = d.stride(g, DB);

  for (int item = threadIdx.x; item < NF * C; item += T::NT) {
    int c, t;
    split(item, NF, c, t);
    const int f = n0 - 1 + t;
    if (cbase + c >= ncol_max || f > m - 1) continue;
    const int64_t id = node_idx(g, c, f), idn = id + sd;
    const double *mt = z.metric;
    double gm[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (mt[id + l * sz] + mt[idn + l * sz]);
    const double *pv = z.bv;
    double dd[4][3];
    const int slots[4] = {1, 2, 3, 5};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const double *fa = pv + slots[a] * sz;
      dd[a][DIR] = fa[idn] - fa[id];
      dd[a][DA] = 0.25 * (fa[id + sa] - fa[id - sa] + fa[idn + sa] - fa[idn - sa]);
      dd[a][DB] = 0.25 * (fa[id + sb] - fa[id - sb] + fa[idn + sb] - fa[idn - sb]);
    }
    const double u_x = dd[0][0] * gm[0] + dd[0][1] * gm[3] + dd[0][2] * gm[6];
    const double u_y = dd[0][0] * gm[1] + dd[0][1] * gm[4] + dd[0][2] * gm[7];
    const double u_z = dd[0][0] * gm[2] + dd[0][1] * gm[5] + dd[0][2] * gm[8];
    const double v_x = dd[1][0] * gm[0] + dd[1][1] * gm[3] + dd[1][2] * gm[6];
    const double v_y = dd[1][0] * gm[1] + dd[1][1] * gm[4] + dd[1][2] * gm[7];
    const double v_z = dd[1][0] * gm[2] + dd[1][1] * gm[5] + dd[1][2] * gm[8];
    const double w_x = dd[2][0] * gm[0] + dd[2][1] * gm[3] + dd[2][2] * gm[6];
    const double w_y = dd[2][0] * gm[1] + dd[2][1] * gm[4] + dd[2][2] * gm[7];
    const double w_z = dd[2][0] * gm[2] + dd[2][1] * gm[5] + dd[2][2] * gm[8];
    const double mul = 0.5 * (z.mul[id] + z.mul[idn]);
    const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
    const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
    const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
    const double tau_xy = mul * (u_y + v_x);
    const double tau_xz = mul * (u_z + w_x);
    const double tau_yz = mul * (v_z + w_y);
    const int mo = 3 * DIR;
    const double ja = z.jac[id], jb = z.jac[idn];
    const double gk0 = 0.5 * (mt[id + mo * sz] * ja + mt[idn + mo * sz] * jb);
    const double gk1 = 0.5 * (mt[id + (mo + 1) * sz] * ja + mt[idn + (mo + 1) * sz] * jb);
    const double gk2 = 0.5 * (mt[id + (mo + 2) * sz] * ja + mt[idn + (mo + 2) * sz] * jb);
    const double f0 = gk0 * tau_xx + gk1 * tau_xy + gk2 * tau_xz;
    const double f1 = gk0 * tau_xy + gk1 * tau_yy + gk2 * tau_yz;
    const double f2 = gk0 * tau_xz + gk1 * tau_yz + gk2 * tau_zz;
    const double um = 0.5 * (pv[id + sz] + pv[idn + sz]);
    const double vm = 0.5 * (pv[id + 2 * sz] + pv[idn + 2 * sz]);
    const double wm = 0.5 * (pv[id + 3 * sz] + pv[idn + 3 * sz]);
    const double t_x = dd[3][0] * gm[0] + dd[3][1] * gm[3] + dd[3][2] * gm[6];
    const double t_y = dd[3][0] * gm[1] + dd[3][1] * gm[4] + dd[3][2] * gm[7];
    const double t_z = dd[3][0] * gm[2] + dd[3][1] * gm[5] + dd[3][2] * gm[8];
    const double conductivity = 0.5 * (z.thermal_conductivity[id] + z.thermal_conductivity[idn]);
    double f3 = um * f0 + vm * f1 + wm * f2 + conductivity * (gk0 * t_x + gk1 * t_y + gk2 * t_z);

    // species diffusion with the correction velocity (mixture-averaged)
    const double *y = z.sv;
    double yk[NS], diffusivity[NS], ddf[NS];
    double sum_grad_over_w = 0, sum_rhoDkYk = 0, correction = 0, mw_tot = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double *yl = y + l * sz;
      yk[l] = 0.5 * (yl[id] + yl[idn]);
      diffusivity[l] = 0.5 * (z.rho_D[id + l * sz] + z.rho_D[idn + l * sz]);
      double d3[3];
      d3[DIR] = yl[idn] - yl[id];
      d3[DA] = 0.25 * (yl[id + sa] - yl[id - sa] + yl[idn + sa] - yl[idn - sa]);
      d3[DB] = 0.25 * (yl[id + sb] - yl[id - sb] + yl[idn + sb] - yl[idn - sb]);
      const double y_x = d3[0] * gm[0] + d3[1] * gm[3] + d3[2] * gm[6];
      const double y_y = d3[0] * gm[1] + d3[1] * gm[4] + d3[2] * gm[7];
      const double y_z = d3[0] * gm[2] + d3[1] * gm[5] + d3[2] * gm[8];
      const double gy = gk0 * y_x + gk1 * y_y + gk2 * y_z;
      ddf[l] = gy;
      correction += diffusivity[l] * gy;
      sum_grad_over_w += gy * th->imw[l];
      mw_tot += yk[l] * th->imw[l];
      sum_rhoDkYk += diffusivity[l] * yk[l];
    }
    mw_tot = 1.0 / mw_tot;
    correction -= mw_tot * sum_rhoDkYk * sum_grad_over_w;
    if (gradp) {
      const double *pp = pv + 4 * sz;
      double d3[3];
      d3[DIR] = pp[idn] - pp[id];
      d3[DA] = 0.25 * (pp[id + sa] - pp[id - sa] + pp[idn + sa] - pp[idn - sa]);
      d3[DB] = 0.25 * (pp[id + sb] - pp[id - sb] + pp[idn + sb] - pp[idn - sb]);
      const double p_x = d3[0] * gm[0] + d3[1] * gm[3] + d3[2] * gm[6];
      const double p_y = d3[0] * gm[1] + d3[1] * gm[4] + d3[2] * gm[7];
      const double p_z = d3[0] * gm[2] + d3[1] * gm[5] + d3[2] * gm[8];
      const double gp = (gk0 * p_x + gk1 * p_y + gk2 * p_z) / (0.5 * (pp[idn] + pp[id]));
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        ddf[l] += (mw_tot * th->imw[l] - 1) * yk[l] * gp;
        correction += (mw_tot * th->imw[l] - 1) * yk[l] * gp * diffusivity[l];
      }
    }
    double h[NS], cp_unused[NS];
    enthalpy_cp_ns<NS>(th, 0.5 * (pv[id + 5 * sz] + pv[idn + 5 * sz]), h, cp_unused);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double flux = diffusivity[l] * (ddf[l] - mw_tot * yk[l] * sum_grad_over_w) - yk[l] * correction;
      sflx[T::sfl(4 + l, c, t)] = flux;
      f3 += h[l] * flux;
    }
    sflx[T::sfl(0, c, t)] = f0;
    sflx[T::sfl(1, c, t)] = f1;
    sflx[T::sfl(2, c, t)] = f2;
    sflx[T::sfl(3, c, t)] = f3;
  }
  __syncthreads();
  for (int item = threadIdx.x; item < TN * C; item += T::NT) {
    int c, t;
    split(item, TN, c, t);
    const int a = n0 + t;
    if (cbase + c >= ncol_max || a > m - 1) continue;
    const int64_t iq = node_idx(0, c, a);
#pragma unroll
    for (int v = 0; v < T::NVF; ++v) z.dq[iq + (v + 1) * szq] += sflx[T::sfl(v, c, t + 1)] - sflx[T::sfl(v, c, t)];
  }
}

namespace {

template <int DIR>
cudaError_t launch_vis_mix_dir(const Zone &z, const Thermo &th, int gradp, cudaStream_t st) {
  using T = VisMixTile<DIR, kMaxSpec>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  viscous_mix_flux_diff<DIR, kMaxSpec><<<grid, T::NT, T::smem_bytes(), st>>>(z, th, gradp);
  return cudaGetLastError();
}

template <int DIR>
cudaError_t set_vis_mix_attr() {
  return cudaFuncSetAttribute(viscous_mix_flux_diff<DIR, kMaxSpec>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)VisMixTile<DIR, kMaxSpec>::smem_bytes());
}

}  // namespace

cudaError_t viscous_mix_init_attributes() {
  cudaError_t e;
  if ((e = set_vis_mix_attr<0>()) != cudaSuccess) return e;
  if ((e = set_vis_mix_attr<1>()) != cudaSuccess) return e;
  return set_vis_mix_attr<2>();
}

cudaError_t launch_viscous_mix(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st, int *n_launch) {
  const int gradp = p.gradPInDiffusionFlux;
  cudaError_t e = launch_vis_mix_dir<0>(z, th, gradp, st);
  if (e != cudaSuccess) return e;
  e = launch_vis_mix_dir<1>(z, th, gradp, st);
  if (e != cudaSuccess) return e;
  *n_launch += 2;
  if (z.d.mz > 1) {
    e = launch_vis_mix_dir<2>(z, th, gradp, st);
    if (e != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
