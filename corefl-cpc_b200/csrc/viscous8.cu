// Collocated viscous schemes, air and 9-species mixtures: the reference's
// 8th-order scheme (viscous_order = 8) and a 4th-order variant
// (viscous_order = 4, not in the reference) built from the same pieces: the
// reference's 4th-order central operator (its row for the third node from a
// wall) in the interior and its two one-sided rows at physical faces.
//
// Restates the order-8 branch of compute_viscous_flux (reference
// src/ViscousScheme.cu:41-70) as three steps:
//   collocated — one thread per interior node (i on the lanes): 8th-order
//                central derivatives of u, v, w, T (and Y_k) along xi, eta,
//                zeta (one-sided 4th/6th-order forms on the four nodes next
//                to a physical boundary face, reference :129-308), the
//                stress, heat flux (and mixture-averaged species diffusion
//                with the correction velocity and enthalpy flux, :414-560)
//                contracted with the three metric rows into the node fluxes
//                Fv, Gv, Hv (reference :309-412);
//   exchange   — per periodic face in the boundary list's order: average the
//                two coincident face nodes and fill the ghost layers from the
//                other side (exchange_value task 1, reference
//                src/DataCommunication.cu:628-672);
//   derivative — dq(l) += (dFv/dxi + dGv/deta + dHv/dzeta)(l) * J with the
//                same difference operators (reference :562-612).
// The node fluxes live in a context-owned array of 3 x (nv - 1) planes with
// ngg ghosts; the k-derivative is skipped in 2-D, where it only reads ghost
// planes that nothing writes (zero in the reference's zero-initialised
// arrays).
#include "cfk_common.cuh"
#include "chem_fast.cuh"
#include "thermo.cuh"

namespace cfk {

namespace {

// derivative along one direction at node n of nn; f points at the node, s
// is the stride; left/right: the line ends at a physical boundary face.
template <int ORDER>
__device__ __forceinline__ double d8(const double *__restrict__ f, int64_t s, int n, int nn, bool left, bool right) {
  auto F = [&](int o) { return f[o * s]; };
  if constexpr (ORDER == 4) {
    if (left && n == 0) return -25.0 / 12 * F(0) + 4.0 * F(1) - 3 * F(2) + 4.0 / 3 * F(3) - 0.25 * F(4);
    if (left && n == 1) return -0.25 * F(-1) - 5.0 / 6 * F(0) + 1.5 * F(1) - 0.5 * F(2) + 1.0 / 12 * F(3);
    if (right && n == nn - 1) return 25.0 / 12 * F(0) - 4.0 * F(-1) + 3 * F(-2) - 4.0 / 3 * F(-3) + 0.25 * F(-4);
    if (right && n == nn - 2) return 0.25 * F(1) + 5.0 / 6 * F(0) - 1.5 * F(-1) + 0.5 * F(-2) - 1.0 / 12 * F(-3);
    return -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
  }
  double df = 0;
  bool computed = false;
  if (left) {
    if (n == 0) {
      df = -25.0 / 12 * F(0) + 4.0 * F(1) - 3 * F(2) + 4.0 / 3 * F(3) - 0.25 * F(4);
      computed = true;
    } else if (n == 1) {
      df = -0.25 * F(-1) - 5.0 / 6 * F(0) + 1.5 * F(1) - 0.5 * F(2) + 1.0 / 12 * F(3);
      computed = true;
    } else if (n == 2) {
      df = -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
      computed = true;
    } else if (n == 3) {
      df = 0.75 * (F(1) - F(-1)) - 0.15 * (F(2) - F(-2)) + 1.0 / 60 * (F(3) - F(-3));
      computed = true;
    }
  }
  if (right) {
    if (n == nn - 1) {
      df = 25.0 / 12 * F(0) - 4.0 * F(-1) + 3 * F(-2) - 4.0 / 3 * F(-3) + 0.25 * F(-4);
      computed = true;
    } else if (n == nn - 2) {
      df = 0.25 * F(1) + 5.0 / 6 * F(0) - 1.5 * F(-1) + 0.5 * F(-2) - 1.0 / 12 * F(-3);
      computed = true;
    } else if (n == nn - 3) {
      df = -1.0 / 12 * (F(2) - F(-2)) + 2.0 / 3 * (F(1) - F(-1));
      computed = true;
    } else if (n == nn - 4) {
      df = 0.75 * (F(1) - F(-1)) - 0.15 * (F(2) - F(-2)) + 1.0 / 60 * (F(3) - F(-3));
      computed = true;
    }
  }
  if (!computed) {
    constexpr double a1{0.8}, a2{-0.2}, a3{4.0 / 105}, a4{-1.0 / 280};
    df = a1 * (F(1) - F(-1)) + a2 * (F(2) - F(-2)) + a3 * (F(3) - F(-3)) + a4 * (F(4) - F(-4));
  }
  return df;
}

struct Bnd {
  bool l[3], r[3];  // physical (non-periodic) boundary face on the min / max side of each direction
};

template <int ORDER>
__device__ __forceinline__ void grad3(const double *f, int64_t sj, int64_t sk, int i, int j, int k, const Dims &d,
                                      const Bnd &b, double &dx, double &dy, double &dz) {
  dx = d8<ORDER>(f, 1, i, d.mx, b.l[0], b.r[0]);
  dy = d8<ORDER>(f, sj, j, d.my, b.l[1], b.r[1]);
  dz = d8<ORDER>(f, sk, k, d.mz, b.l[2], b.r[2]);
}

// NS = 0: calorically perfect air
template <int NS, int ORDER>
__global__ void __launch_bounds__(128) visc8_collocated(Zone z, double *fvis, Bnd b, double Pr,
                                                        const __grid_constant__ Thermo thermo, int gradp) {
  constexpr int NV = 5 + NS;
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= d.mx) return;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), sj = d.stride(g, 1), sk = d.stride(g, 2);
  const int64_t id = d.idx(g, i, j, k);
  double u_xi, u_eta, u_zeta, v_xi, v_eta, v_zeta, w_xi, w_eta, w_zeta, t_xi, t_eta, t_zeta;
  grad3<ORDER>(z.bv + sz + id, sj, sk, i, j, k, d, b, u_xi, u_eta, u_zeta);
  grad3<ORDER>(z.bv + 2 * sz + id, sj, sk, i, j, k, d, b, v_xi, v_eta, v_zeta);
  grad3<ORDER>(z.bv + 3 * sz + id, sj, sk, i, j, k, d, b, w_xi, w_eta, w_zeta);
  grad3<ORDER>(z.bv + 5 * sz + id, sj, sk, i, j, k, d, b, t_xi, t_eta, t_zeta);
  const double *mt = z.metric + id;
  const double xi_x = mt[0], xi_y = mt[sz], xi_z = mt[2 * sz];
  const double eta_x = mt[3 * sz], eta_y = mt[4 * sz], eta_z = mt[5 * sz];
  const double zeta_x = mt[6 * sz], zeta_y = mt[7 * sz], zeta_z = mt[8 * sz];
  const double u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
  const double u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
  const double u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
  const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
  const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
  const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
  const double w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
  const double w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
  const double w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
  const double mul = z.mul[id];
  const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double tau_xy = mul * (u_y + v_x);
  const double tau_xz = mul * (u_z + w_x);
  const double tau_yz = mul * (v_z + w_y);
  // slot l (1..NV-1) of direction q at fvis[(q * (NV - 1) + l - 1) * sz]
  double *fv = fvis + id - sz, *gv = fv + (NV - 1) * sz, *hv = gv + (NV - 1) * sz;
  fv[1 * sz] = xi_x * tau_xx + xi_y * tau_xy + xi_z * tau_xz;
  fv[2 * sz] = xi_x * tau_xy + xi_y * tau_yy + xi_z * tau_yz;
  fv[3 * sz] = xi_x * tau_xz + xi_y * tau_yz + xi_z * tau_zz;
  gv[1 * sz] = eta_x * tau_xx + eta_y * tau_xy + eta_z * tau_xz;
  gv[2 * sz] = eta_x * tau_xy + eta_y * tau_yy + eta_z * tau_yz;
  gv[3 * sz] = eta_x * tau_xz + eta_y * tau_yz + eta_z * tau_zz;
  hv[1 * sz] = zeta_x * tau_xx + zeta_y * tau_xy + zeta_z * tau_xz;
  hv[2 * sz] = zeta_x * tau_xy + zeta_y * tau_yy + zeta_z * tau_yz;
  hv[3 * sz] = zeta_x * tau_xz + zeta_y * tau_yz + zeta_z * tau_zz;
  const double t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
  const double t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
  const double t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
  double conductivity;
  if constexpr (NS > 0) {
    conductivity = z.thermal_conductivity[id];
  } else {
    constexpr double cp{kGammaAir * kRAir / (kGammaAir - 1)};
    conductivity = mul / Pr * cp;
  }
  const double u = z.bv[id + sz], v = z.bv[id + 2 * sz], w = z.bv[id + 3 * sz];
  const double Ex = u * tau_xx + v * tau_xy + w * tau_xz + conductivity * t_x;
  const double Ey = u * tau_xy + v * tau_yy + w * tau_yz + conductivity * t_y;
  const double Ez = u * tau_xz + v * tau_yz + w * tau_zz + conductivity * t_z;
  double f4 = xi_x * Ex + xi_y * Ey + xi_z * Ez;
  double g4 = eta_x * Ex + eta_y * Ey + eta_z * Ez;
  double h4 = zeta_x * Ex + zeta_y * Ey + zeta_z * Ez;
  if constexpr (NS > 0) {
    const Thermo *th = &thermo;
    double diffusivity[NS], yk[NS], dfx[NS], dfy[NS], dfz[NS];
    double sx = 0, sy = 0, szt = 0, sum_rhoDkYk = 0, c0 = 0, c1 = 0, c2 = 0, mw_tot = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double *y = z.sv + l * sz + id;
      yk[l] = y[0];
      diffusivity[l] = z.rho_D[id + l * sz];
      double y_xi, y_eta, y_zeta;
      grad3<ORDER>(y, sj, sk, i, j, k, d, b, y_xi, y_eta, y_zeta);
      const double y_x = y_xi * xi_x + y_eta * eta_x + y_zeta * zeta_x;
      const double y_y = y_xi * xi_y + y_eta * eta_y + y_zeta * zeta_y;
      const double y_z = y_xi * xi_z + y_eta * eta_z + y_zeta * zeta_z;
      const double gx = xi_x * y_x + xi_y * y_y + xi_z * y_z;
      const double gy = eta_x * y_x + eta_y * y_y + eta_z * y_z;
      const double gz = zeta_x * y_x + zeta_y * y_y + zeta_z * y_z;
      dfx[l] = gx;
      dfy[l] = gy;
      dfz[l] = gz;
      c0 += diffusivity[l] * gx;
      c1 += diffusivity[l] * gy;
      c2 += diffusivity[l] * gz;
      sx += gx * th->imw[l];
      sy += gy * th->imw[l];
      szt += gz * th->imw[l];
      mw_tot += yk[l] * th->imw[l];
      sum_rhoDkYk += diffusivity[l] * yk[l];
    }
    mw_tot = 1.0 / mw_tot;
    c0 -= mw_tot * sum_rhoDkYk * sx;
    c1 -= mw_tot * sum_rhoDkYk * sy;
    c2 -= mw_tot * sum_rhoDkYk * szt;
    if (gradp) {  // pressure-gradient term of the driving force (reference src/ViscousScheme.cu:495-520)
      double p_xi, p_eta, p_zeta;
      grad3<ORDER>(z.bv + 4 * sz + id, sj, sk, i, j, k, d, b, p_xi, p_eta, p_zeta);
      const double p_x = p_xi * xi_x + p_eta * eta_x + p_zeta * zeta_x;
      const double p_y = p_xi * xi_y + p_eta * eta_y + p_zeta * zeta_y;
      const double p_z = p_xi * xi_z + p_eta * eta_z + p_zeta * zeta_z;
      const double pn = z.bv[id + 4 * sz];
      const double gxp = (xi_x * p_x + xi_y * p_y + xi_z * p_z) / pn;
      const double gyp = (eta_x * p_x + eta_y * p_y + eta_z * p_z) / pn;
      const double gzp = (zeta_x * p_x + zeta_y * p_y + zeta_z * p_z) / pn;
#pragma unroll
      for (int l = 0; l < NS; ++l) {
        const double coefficient = (mw_tot * th->imw[l] - 1) * yk[l];
        dfx[l] += coefficient * gxp;
        dfy[l] += coefficient * gyp;
        dfz[l] += coefficient * gzp;
        c0 += coefficient * gxp * diffusivity[l];
        c1 += coefficient * gyp * diffusivity[l];
        c2 += coefficient * gzp * diffusivity[l];
      }
    }
    double h[NS], cp_unused[NS];
    enthalpy_cp_ns<NS>(th, z.bv[id + 5 * sz], h, cp_unused);
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      double df = diffusivity[l] * (dfx[l] - mw_tot * yk[l] * sx) - yk[l] * c0;
      fv[(5 + l) * sz] = df;
      f4 += h[l] * df;
      df = diffusivity[l] * (dfy[l] - mw_tot * yk[l] * sy) - yk[l] * c1;
      gv[(5 + l) * sz] = df;
      g4 += h[l] * df;
      df = diffusivity[l] * (dfz[l] - mw_tot * yk[l] * szt) - yk[l] * c2;
      hv[(5 + l) * sz] = df;
      h4 += h[l] * df;
    }
  }
  fv[4 * sz] = f4;
  gv[4 * sz] = g4;
  hv[4 * sz] = h4;
}

// One periodic face: thread per face node (a, b tangential).
__global__ void visc8_periodic_exchange(Zone z, double *fvis, int nplanes, int dir, int direction) {
  const Dims d = z.d;
  const int a_dir = (dir + 1) % 3, b_dir = (dir + 2) % 3;
  const int ia = blockIdx.x * blockDim.x + threadIdx.x, ib = blockIdx.y;
  if (ia >= d.ext(a_dir)) return;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), s = d.stride(g, dir);
  int c[3];
  c[a_dir] = ia;
  c[b_dir] = ib;
  c[dir] = direction < 0 ? 0 : d.ext(dir) - 1;
  const int64_t idh = d.idx(g, c[0], c[1], c[2]);
  c[dir] = direction < 0 ? d.ext(dir) - 1 : 0;
  const int64_t ido = d.idx(g, c[0], c[1], c[2]);
  for (int l = 0; l < nplanes; ++l) {
    const double ave = 0.5 * (fvis[idh + l * sz] + fvis[ido + l * sz]);
    fvis[idh + l * sz] = ave;
    fvis[ido + l * sz] = ave;
  }
  for (int gg = 1; gg <= g; ++gg) {
    const int64_t gh = idh + (int64_t)gg * direction * s, go = ido + (int64_t)gg * direction * s;
    for (int l = 0; l < nplanes; ++l) fvis[gh + l * sz] = fvis[go + l * sz];
  }
}

template <int NV, int ORDER>
__global__ void __launch_bounds__(128) visc8_derivative(Zone z, const double *fvis, Bnd b) {
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= d.mx) return;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0), sj = d.stride(g, 1), sk = d.stride(g, 2);
  const int64_t id = d.idx(g, i, j, k), iq = d.idx(0, i, j, k);
  const double jac = z.jac[id];
  const bool three_d = d.mz > 1;
#pragma unroll
  for (int l = 1; l < NV; ++l) {
    const double *fv = fvis + (l - 1) * sz + id, *gv = fvis + (NV - 1 + l - 1) * sz + id,
                 *hv = fvis + (2 * (NV - 1) + l - 1) * sz + id;
    double s = d8<ORDER>(fv, 1, i, d.mx, b.l[0], b.r[0]) + d8<ORDER>(gv, sj, j, d.my, b.l[1], b.r[1]);
    if (three_d) s += d8<ORDER>(hv, sk, k, d.mz, b.l[2], b.r[2]);
    z.dq[iq + l * szq] += s * jac;
  }
}

Bnd boundary_flags(const cfk_face *faces, int n_face) {
  Bnd b{};
  for (int n = 0; n < n_face; ++n)
    if (faces[n].label != 8) (faces[n].direction < 0 ? b.l : b.r)[faces[n].face] = true;
  return b;
}

}  // namespace

// Node fluxes, periodic exchange (face list order), derivative into dq.
// fvis: 3 x (nv - 1) planes with ngg ghosts; th: nullptr for air.
cudaError_t launch_viscous8(const Zone &z, const Param &p, const Thermo *th, const cfk_face *faces, int n_face,
                            double *fvis, cudaStream_t st, int *n_launch) {
  const Dims &d = z.d;
  const Bnd b = boundary_flags(faces, n_face);
  const dim3 grid((d.mx + 127) / 128, d.my, d.mz);
  static const Thermo no_thermo{};
  const bool o4 = p.viscous_order == 4;
  const int gradp = p.gradPInDiffusionFlux;
  if (th && o4) visc8_collocated<kMaxSpec, 4><<<grid, 128, 0, st>>>(z, fvis, b, p.Pr, *th, gradp);
  else if (th) visc8_collocated<kMaxSpec, 8><<<grid, 128, 0, st>>>(z, fvis, b, p.Pr, *th, gradp);
  else if (o4) visc8_collocated<0, 4><<<grid, 128, 0, st>>>(z, fvis, b, p.Pr, no_thermo, 0);
  else visc8_collocated<0, 8><<<grid, 128, 0, st>>>(z, fvis, b, p.Pr, no_thermo, 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  *n_launch += 1;
  const int nplanes = 3 * (p.n_var - 1);
  for (int n = 0; n < n_face; ++n) {
    if (faces[n].label != 8) continue;
    const int dir = faces[n].face, a_dir = (dir + 1) % 3, b_dir = (dir + 2) % 3;
    const dim3 g2((d.ext(a_dir) + 127) / 128, d.ext(b_dir));
    visc8_periodic_exchange<<<g2, 128, 0, st>>>(z, fvis, nplanes, dir, faces[n].direction);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    *n_launch += 1;
  }
  if (th && o4) visc8_derivative<5 + kMaxSpec, 4><<<grid, 128, 0, st>>>(z, fvis, b);
  else if (th) visc8_derivative<5 + kMaxSpec, 8><<<grid, 128, 0, st>>>(z, fvis, b);
  else if (o4) visc8_derivative<5, 4><<<grid, 128, 0, st>>>(z, fvis, b);
  else visc8_derivative<5, 8><<<grid, 128, 0, st>>>(z, fvis, b);
  *n_launch += 1;
  return cudaGetLastError();
}

}  // namespace cfk
