// cv from bv at one node (reference src/FieldOperation.cuh:16-37, 66-84),
// shared by the node-local kernels and the halo assignment.
#pragma once

#include "cfk_common.cuh"
#include "thermo.cuh"

namespace cfk {

template <bool MIX>
__device__ __forceinline__ void cv_from_bv_point(const Zone &z, const Param &p, const Thermo *th, int64_t id) {
  const int64_t sz = z.d.plane(z.d.ngg);
  const double rho = z.bv[id], u = z.bv[id + sz], v = z.bv[id + 2 * sz], w = z.bv[id + 3 * sz];
  z.cv[id] = rho;
  z.cv[id + sz] = rho * u;
  z.cv[id + 2 * sz] = rho * v;
  z.cv[id + 3 * sz] = rho * w;
  for (int l = 0; l < p.n_scalar; ++l) z.cv[id + (5 + l) * sz] = rho * z.sv[id + l * sz];
  const double V2 = u * u + v * v + w * w;
  double total_energy = 0.5 * V2;
  if (MIX) {
    double h[kMaxSpec];
    compute_enthalpy(th, z.bv[id + 5 * sz], h);
    for (int l = 0; l < p.n_spec; ++l) total_energy += h[l] * z.sv[id + l * sz];
    total_energy *= rho;
    total_energy -= z.bv[id + 4 * sz];
  } else {
    total_energy *= rho;
    total_energy += z.bv[id + 4 * sz] / (kGammaAir - 1);
  }
  z.cv[id + 4 * sz] = total_energy;
}


}  // namespace cfk
