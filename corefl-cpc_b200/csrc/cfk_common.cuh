// Shared device-side definitions: physical constants, the zone view passed to
// every kernel by value, and the VectorField3D indexing of the reference
// (reference src/gxl_lib/Array.cuh:246-322).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "corefl_b200.h"

namespace cfk {

// reference src/Constants.h
constexpr double kRu = 8314.462618;
constexpr double kMwAir = 28.9647;
constexpr double kGammaAir = 1.4;
constexpr double kRAir = kRu / kMwAir;
constexpr double kEpsWeno = 1e-40;  // reference src/WENO.cu:8

constexpr int kMaxSpec = 9;   // H2/O2 mechanisms of the configurations: 9 species
constexpr int kMaxVar = 5 + kMaxSpec;

// Geometry of one ghost-padded block.  All plane arrays share (mx,my,mz) and
// differ only in ghost width g.
struct Dims {
  int mx, my, mz, ngg;
  __host__ __device__ int sx(int g) const { return mx + 2 * g; }
  __host__ __device__ int sy(int g) const { return my + 2 * g; }
  __host__ __device__ int64_t plane(int g) const { return (int64_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g); }
  __host__ __device__ int64_t idx(int g, int i, int j, int k) const {
    return ((int64_t)(k + g) * (my + 2 * g) + (j + g)) * (mx + 2 * g) + (i + g);
  }
  __host__ __device__ int64_t stride(int g, int dir) const {
    return dir == 0 ? 1 : (dir == 1 ? (int64_t)(mx + 2 * g) : (int64_t)(mx + 2 * g) * (my + 2 * g));
  }
  __host__ __device__ int ext(int dir) const { return dir == 0 ? mx : (dir == 1 ? my : mz); }
};

// Kernel-side copy of the bound zone (device pointers).
struct Zone {
  Dims d;
  double *jac, *metric, *cv, *bv, *sv, *qn, *mul, *mach;
  double *acoustic_speed, *gamma, *thermal_conductivity, *rho_D, *reaction_timeScale;
  double *dq, *dt_local, *Cn;
  double *shock_sensor;  // ngg ghosts, zero outside the interior; hybrid WENO only
  double *fvis8;         // node viscous fluxes of the 8th-order scheme, 3 x (n_var - 1) planes, ngg ghosts
  const double *y;       // node y coordinate, ngg ghosts (mixing-layer inflow only)
  unsigned long long *inflow_draws;  // applications of a fluctuating inflow so far (context-owned counter)
};

// Kernel-side scalar settings.
struct Param {
  int dim, n_var, n_spec, n_scalar, n_reac;
  int inviscid_scheme, reconstruction, limiter, viscous_order;
  int positive_preserving, gradPInDiffusionFlux, fixed_dt, chem_advance_method;
  double entropy_fix_factor, Pr, Sc, cfl;
  double weno_eps_scale, v_ref, rho_ref;
  int shock_sensor;                 // 0 modified Ducros, 1 modified Jameson, 2 density/pressure jump
  double sensor_eps, sensor_threshold;
  int limit_flow;                   // limit_flow after every stage update
  double limit_ll[5], limit_ul[5];  // bounds of rho, u, v, w, p
};

}  // namespace cfk
