// Shock sensor of the hybrid UD/WENO schemes (reference
// src/FieldOperation.cu:74-179, compute_shock_sensor): one value per interior
// node, written into the context's ghost-padded sensor array whose ghost
// layers stay zero.  Sensor 0 is the modified Ducros sensor (4th-order
// central velocity derivatives, div^2 / (div^2 + |curl|^2 + eps), zero in
// expansions), 1 the modified Jameson pressure sensor, 2 the density/pressure
// jump sensor.  One thread per node, consecutive i on consecutive lanes; the
// +-2 neighbours along j and k are re-read from L1/L2.
#include "cfk_common.cuh"

namespace cfk {

namespace {

__device__ __forceinline__ double d4(const double *f, int64_t id, int64_t s) {
  constexpr double oneD12{1.0 / 12.0}, twoD3{2.0 / 3.0};
  return oneD12 * f[id - 2 * s] - twoD3 * f[id - s] + twoD3 * f[id + s] - oneD12 * f[id + 2 * s];
}

__device__ double ducros(const Zone &z, int64_t id, int64_t sz, int64_t sj, int64_t sk, double eps) {
  const double *u = z.bv + sz, *v = z.bv + 2 * sz, *w = z.bv + 3 * sz;
  const double *mt = z.metric;
  const double xi_x = mt[id], xi_y = mt[id + sz], xi_z = mt[id + 2 * sz];
  const double eta_x = mt[id + 3 * sz], eta_y = mt[id + 4 * sz], eta_z = mt[id + 5 * sz];
  const double zeta_x = mt[id + 6 * sz], zeta_y = mt[id + 7 * sz], zeta_z = mt[id + 8 * sz];
  const double du1 = d4(u, id, 1), du2 = d4(u, id, sj), du3 = d4(u, id, sk);
  const double dv1 = d4(v, id, 1), dv2 = d4(v, id, sj), dv3 = d4(v, id, sk);
  const double dw1 = d4(w, id, 1), dw2 = d4(w, id, sj), dw3 = d4(w, id, sk);
  double div = (du1 * xi_x + du2 * eta_x + du3 * zeta_x) + (dv1 * xi_y + dv2 * eta_y + dv3 * zeta_y) +
               (dw1 * xi_z + dw2 * eta_z + dw3 * zeta_z);
  if (div > 0) return 0;
  const double duDy = du1 * xi_y + du2 * eta_y + du3 * zeta_y, duDz = du1 * xi_z + du2 * eta_z + du3 * zeta_z;
  const double dvDx = dv1 * xi_x + dv2 * eta_x + dv3 * zeta_x, dvDz = dv1 * xi_z + dv2 * eta_z + dv3 * zeta_z;
  const double dwDx = dw1 * xi_x + dw2 * eta_x + dw3 * zeta_x, dwDy = dw1 * xi_y + dw2 * eta_y + dw3 * zeta_y;
  div *= div;
  const double cx = dwDy - dvDz, cy = duDz - dwDx, cz = dvDx - duDy;
  return div / (div + (cx * cx + cy * cy + cz * cz) + eps);
}

__device__ double jameson(const Zone &z, int64_t id, int64_t sz, int64_t sj, int64_t sk) {
  const double *p = z.bv + 4 * sz;
  const double twoP = 2 * p[id];
  const double pI = p[id + 1] + p[id - 1], pJ = p[id + sj] + p[id - sj], pK = p[id + sk] + p[id - sk];
  return abs(pI - twoP) / (pI + twoP) + abs(pJ - twoP) / (pJ + twoP) + abs(pK - twoP) / (pK + twoP);
}

__device__ double jump(const Zone &z, int64_t id, int64_t sz, int64_t sj, int64_t sk) {
  const double *rho = z.bv, *p = z.bv + 4 * sz;
  const double r0 = rho[id], rI = 1.0 / r0, p0 = p[id], pI = 1.0 / p0;
  double s = 0;
  s = max(s, abs(rho[id + 1] - r0) * rI);
  s = max(s, abs(rho[id + sj] - r0) * rI);
  s = max(s, abs(rho[id + sk] - r0) * rI);
  s = max(s, abs(p[id + 1] - p0) * pI);
  s = max(s, abs(p[id + sj] - p0) * pI);
  s = max(s, abs(p[id + sk] - p0) * pI);
  return s;
}

__global__ void __launch_bounds__(128) shock_sensor_kernel(Zone z, int type, double eps) {
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= d.mx) return;
  const int g = d.ngg;
  const int64_t id = d.idx(g, i, j, k), sz = d.plane(g), sj = d.stride(g, 1), sk = d.stride(g, 2);
  double s;
  if (type == 1) s = jameson(z, id, sz, sj, sk);
  else if (type == 2) s = jump(z, id, sz, sj, sk);
  else s = ducros(z, id, sz, sj, sk, eps);
  z.shock_sensor[id] = s;
}

}  // namespace

cudaError_t launch_shock_sensor(const Zone &z, const Param &p, cudaStream_t st) {
  const dim3 grid((z.d.mx + 127) / 128, z.d.my, z.d.mz);
  shock_sensor_kernel<<<grid, 128, 0, st>>>(z, p.shock_sensor, p.sensor_eps);
  return cudaGetLastError();
}

}  // namespace cfk
