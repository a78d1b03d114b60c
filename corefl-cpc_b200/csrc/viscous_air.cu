// Fused second-order viscous flux + flux difference, calorically perfect air.
//
// Restates compute_{f,g,h}v_2nd_order (air branch, reference
// src/ViscousScheme.cu:614-1173) and compute_dFv_dx / dGv_dy / dHv_dz
// (reference src/ViscousScheme.cu:75-127).  The staggered face flux is
// computed into shared memory and differenced in the same kernel, so the
// vis_flux array of the reference never reaches HBM.
#include "cfk_common.cuh"

namespace cfk {

namespace {
template <int DIR>
struct VisTile {
  static constexpr int TN = DIR == 0 ? 63 : 15;
  static constexpr int C = DIR == 0 ? 4 : 32;
  static constexpr int NF = TN + 1;
  static constexpr int NT = 256;
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
};
}  // namespace

template <int DIR>
__global__ void __launch_bounds__(256) viscous_air_flux_diff(Zone z, double Pr) {
  using T = VisTile<DIR>;
  constexpr int TN = T::TN, C = T::C, NF = T::NF;
  __shared__ double sflx[4 * C * NF];
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
    // d/d(xi_dir) across the face and the averaged central cross derivatives
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
    constexpr double cp = kGammaAir * kRAir / (kGammaAir - 1);
    const double conductivity = mul / Pr * cp;
    sflx[T::sfl(0, c, t)] = f0;
    sflx[T::sfl(1, c, t)] = f1;
    sflx[T::sfl(2, c, t)] = f2;
    sflx[T::sfl(3, c, t)] = um * f0 + vm * f1 + wm * f2 + conductivity * (gk0 * t_x + gk1 * t_y + gk2 * t_z);
  }
  __syncthreads();
  for (int item = threadIdx.x; item < TN * C; item += T::NT) {
    int c, t;
    split(item, TN, c, t);
    const int a = n0 + t;
    if (cbase + c >= ncol_max || a > m - 1) continue;
    const int64_t iq = node_idx(0, c, a);
#pragma unroll
    for (int v = 0; v < 4; ++v) z.dq[iq + (v + 1) * szq] += sflx[T::sfl(v, c, t + 1)] - sflx[T::sfl(v, c, t)];
  }
}

template <int DIR>
static cudaError_t launch_vis_dir(const Zone &z, double Pr, cudaStream_t st) {
  using T = VisTile<DIR>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  viscous_air_flux_diff<DIR><<<grid, T::NT, 0, st>>>(z, Pr);
  return cudaGetLastError();
}

cudaError_t launch_viscous_air(const Zone &z, const Param &p, cudaStream_t st, int *n_launch) {
  cudaError_t e = launch_vis_dir<0>(z, p.Pr, st);
  if (e != cudaSuccess) return e;
  e = launch_vis_dir<1>(z, p.Pr, st);
  if (e != cudaSuccess) return e;
  *n_launch += 2;
  if (z.d.mz > 1) {
    e = launch_vis_dir<2>(z, p.Pr, st);
    if (e != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
