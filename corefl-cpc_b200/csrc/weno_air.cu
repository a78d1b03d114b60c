// Fused characteristic WENO flux + flux difference, calorically perfect air.
//
// Restates compute_convective_term_weno_{x,y,z} with the air characteristic
// helpers (reference src/WENO.cu:831-1138, 10-244, 414-654) followed by
// compute_derivative_{x,y,z} (reference src/WENO.cu:1544, 2219, 2885), as one
// kernel per direction:
//
//   stage   — each CTA stages the stencil points of a tile (a segment of TN
//             nodes along the sweep direction times C columns) into shared
//             memory: conserved Q[5], the Euler flux G[5] along the face
//             normal, p, J/2 and the spectral radius |U_k| + c|grad k|;
//   faces   — each thread projects the 2R+2 stencil points of one face onto
//             the Roe-averaged left eigenvectors, splits them with the local
//             Lax-Friedrichs bound, reconstructs with WENO5-JS / WENO7-Z (or,
//             for the hybrid scheme, with the linear UD5 / UD7 weights where no
//             stencil node is shocked) and projects back; the face fluxes stay
//             in shared memory;
//   diff    — dq(n) -= F(n+1/2) - F(n-1/2) for the tile's nodes.
//
// The face flux never goes to HBM and dq is read-modified-written once per
// direction instead of through a separate derivative pass.  Loads are
// coalesced along i in every direction: x tiles put consecutive faces on
// consecutive lanes, y/z tiles put consecutive i columns on them.
#include "cfk_common.cuh"
#include "weno.cuh"

namespace cfk {

namespace {

constexpr int kNQ = 13;  // staged values per point: Q0..4, G0..4, p, J/2, lambda

// Tile shapes of a sweep: VAR selects one of the CFK_TILE_VARIANTS shapes
// (nodes per column TN x columns C), chosen per direction by the tile
// autotuner.  x tiles run along the lanes, y/z tiles put C consecutive i
// columns on the lanes.
template <int DIR, int VAR>
struct TileShape {
  static constexpr int TN = DIR == 0 ? (VAR == 0 ? 63 : VAR == 1 ? 15 : 31) : (VAR == 0 ? 15 : VAR == 1 ? 31 : 63);
  static constexpr int C = DIR == 0 ? (VAR == 0 ? 4 : VAR == 1 ? 16 : 8) : (VAR == 0 ? 32 : VAR == 1 ? 16 : 8);
};

template <int DIR, int ORD, int VAR = 0>
struct AirTile {
  static constexpr int R = ORD == 7 ? 3 : 2;          // stencil reach left of the face node
  static constexpr int NPF = 2 * R + 2;               // points per face
  static constexpr int TN = TileShape<DIR, VAR>::TN;  // nodes per column
  static constexpr int C = TileShape<DIR, VAR>::C;    // columns per CTA
  static constexpr int NF = TN + 1;             // faces per column
  static constexpr int NPT = TN + 2 * R + 2;    // staged points per column
  static constexpr int NT = 256;                // threads
  // shared-memory offset of (value q, column c, point/face t): x tiles are
  // column-major in t (lanes run along t), y/z tiles are row-major in c.
  __device__ static int spt(int q, int c, int t) {
    return DIR == 0 ? (q * C + c) * NPT + t : (q * NPT + t) * C + c;
  }
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(kNQ * C * NPT + 5 * C * NF); }
};

}  // namespace

// The 13 staged values of one stencil point from its conserved variables,
// p, T, the sweep's metric row and J.
template <class T>
__device__ __forceinline__ void air_stage_point(double *s, int c, int t, double q0, double q1, double q2, double q3,
                                                double q4, double pk, double tk, double m0, double m1, double m2,
                                                double jac) {
  const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
  const double cGradK = norm3d(m0, m1, m2) * sqrt(kGammaAir * kRAir * tk);
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
  s[T::spt(10, c, t)] = pk;
  s[T::spt(11, c, t)] = 0.5 * jac;
  s[T::spt(12, c, t)] = abs(Uk) + cGradK;
}

// Flux of the face between local points t + R and t + R + 1 of column c:
// Roe average, characteristic basis, Lax-Friedrichs split of the 2R + 2
// staged points, WENO (or, away from shocks in the hybrid scheme, the linear
// upwind stencils) and back projection into sflx.  kx, ky, kz: the face
// normal before normalisation.
template <int ORD, class T>
__device__ __forceinline__ void air_face(const double *s, double *sflx, int c, int t, double kx, double ky, double kz,
                                         double eps_ref, bool shock) {
  constexpr int R = T::R, NPF = T::NPF;
  constexpr double gm1 = kGammaAir - 1;
  const int pc = t + R;  // local point of node f
    const double rho_l = s[T::spt(0, c, pc)], rho_r = s[T::spt(0, c, pc + 1)];
    double temp1 = sqrt(rho_l * rho_r);
    const double rlc = 1 / (rho_l + temp1);
    const double rrc = 1 / (temp1 + rho_r);
    const double um = rlc * s[T::spt(1, c, pc)] + rrc * s[T::spt(1, c, pc + 1)];
    const double vm = rlc * s[T::spt(2, c, pc)] + rrc * s[T::spt(2, c, pc + 1)];
    const double wm = rlc * s[T::spt(3, c, pc)] + rrc * s[T::spt(3, c, pc + 1)];
    double temp3 = (rlc * s[T::spt(10, c, pc)] + rrc * s[T::spt(10, c, pc + 1)]) / kRAir;
    const double cm = sqrt(kGammaAir * kRAir * temp3);

    temp1 = rnorm3d(kx, ky, kz);
    kx *= temp1; ky *= temp1; kz *= temp1;
    const double Uk_bar = kx * um + ky * vm + kz * wm;
    double nx = 0, ny = 0, nz = 0;
    if (abs(kx) > 0.8) { nx = -kz; nz = kx; }
    else { ny = kz; nz = -ky; }
    temp1 = rnorm3d(nx, ny, nz);
    nx *= temp1; ny *= temp1; nz *= temp1;
    double qx = ky * nz - kz * ny, qy = kz * nx - kx * nz, qz = kx * ny - ky * nx;
    temp1 = rnorm3d(qx, qy, qz);
    qx *= temp1; qy *= temp1; qz *= temp1;
    const double Un = nx * um + ny * vm + nz * wm;
    const double Uq = qx * um + qy * vm + qz * wm;
    const double ic2 = 1.0 / (cm * cm);
    const double alpha = 0.5 * gm1 * (um * um + vm * vm + wm * wm);

    double lam = 0;
#pragma unroll
    for (int q = 0; q < NPF; ++q) lam = max(lam, s[T::spt(12, c, t + q)]);

    double fChar[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      // keep the stencil in shared memory across the five fields instead of
      // letting the compiler hoist all 2R+2 points into registers
      asm volatile("" ::: "memory");
      double L0, L1, L2, L3, L4;
      if (l == 0) {
        L0 = (alpha + Uk_bar * cm) * ic2 * 0.5;
        L1 = -(gm1 * um + kx * cm) * ic2 * 0.5;
        L2 = -(gm1 * vm + ky * cm) * ic2 * 0.5;
        L3 = -(gm1 * wm + kz * cm) * ic2 * 0.5;
        L4 = gm1 * ic2 * 0.5;
      } else if (l == 1) {
        L0 = -Un; L1 = nx; L2 = ny; L3 = nz; L4 = 0;
      } else if (l == 2) {
        L0 = -Uq; L1 = qx; L2 = qy; L3 = qz; L4 = 0;
      } else if (l == 3) {
        L0 = 1 - alpha * ic2;
        L1 = gm1 * um * ic2;
        L2 = gm1 * vm * ic2;
        L3 = gm1 * wm * ic2;
        L4 = -gm1 * ic2;
      } else {
        L0 = (alpha - Uk_bar * cm) * ic2 * 0.5;
        L1 = -(gm1 * um - kx * cm) * ic2 * 0.5;
        L2 = -(gm1 * vm - ky * cm) * ic2 * 0.5;
        L3 = -(gm1 * wm - kz * cm) * ic2 * 0.5;
        L4 = gm1 * ic2 * 0.5;
      }
      double vp[NPF - 1], vmn[NPF - 1];
#pragma unroll
      for (int q = 0; q < NPF; ++q) {
        const int tq = t + q;
        double LF = L0 * s[T::spt(5, c, tq)] + L1 * s[T::spt(6, c, tq)] + L2 * s[T::spt(7, c, tq)] +
                    L3 * s[T::spt(8, c, tq)];
        double LQ = L0 * s[T::spt(0, c, tq)] + L1 * s[T::spt(1, c, tq)] + L2 * s[T::spt(2, c, tq)] +
                    L3 * s[T::spt(3, c, tq)];
        if (l != 1 && l != 2) {  // the rows of fields 1 and 2 have no energy term
          LF += L4 * s[T::spt(9, c, tq)];
          LQ += L4 * s[T::spt(4, c, tq)];
        }
        const double hj = s[T::spt(11, c, tq)];
        if (q < NPF - 1) vp[q] = hj * (LF + lam * LQ);
        if (q > 0) vmn[q - 1] = hj * (LF - lam * LQ);
      }
      if constexpr (ORD == 7) fChar[l] = shock ? weno7_z(vp, vmn, eps_ref) : weno7_linear(vp, vmn);
      else fChar[l] = shock ? weno5_js(vp, vmn, eps_ref) : weno5_linear(vp, vmn);
    }
    // project back (right eigenvectors written out, reference src/WENO.cu:229-243)
    const double f034 = fChar[0] + fChar[3] + fChar[4];
    const double f04 = fChar[0] - fChar[4];
    const double H = rlc * (s[T::spt(4, c, pc)] + s[T::spt(10, c, pc)]) +
                     rrc * (s[T::spt(4, c, pc + 1)] + s[T::spt(10, c, pc + 1)]);
    sflx[T::sfl(0, c, t)] = f034;
    sflx[T::sfl(1, c, t)] = um * f034 - kx * cm * f04 + nx * fChar[1] + qx * fChar[2];
    sflx[T::sfl(2, c, t)] = vm * f034 - ky * cm * f04 + ny * fChar[1] + qy * fChar[2];
    sflx[T::sfl(3, c, t)] = wm * f034 - kz * cm * f04 + nz * fChar[1] + qz * fChar[2];
    sflx[T::sfl(4, c, t)] = H * f034 - Uk_bar * cm * f04 + Un * fChar[1] + Uq * fChar[2] - cm * cm / gm1 * fChar[3];
  }

// HYB: hybrid UD/WENO scheme, the face switches on the shock sensor.
// VAR: tile shape (TileShape).
template <int DIR, int ORD, bool HYB, int VAR>
__global__ void __launch_bounds__(256, 2) weno_air_flux_diff(Zone z, double eps_ref, const double *sensor,
                                                              double threshold) {
  using T = AirTile<DIR, ORD, VAR>;
  constexpr int R = T::R, NPF = T::NPF, TN = T::TN, C = T::C, NF = T::NF, NPT = T::NPT;
  extern __shared__ double sm[];
  double *spts = sm;
  double *sflx = sm + kNQ * C * NPT;

  const Dims d = z.d;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int m = d.ext(DIR);

  // tile origin: n0 along DIR, column origin across
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

  const int mmo = 3 * DIR;  // metric offset of this direction's grad(xi_dir)
  // ---- stage ------------------------------------------------------------
  for (int item = threadIdx.x; item < NPT * C; item += T::NT) {
    int c, t;
    split(item, NPT, c, t);
    const int a = n0 - 1 - R + t;
    if (cbase + c >= ncol_max || a > m + R) continue;
    const int64_t id = node_idx(g, c, a);
    const double q0 = z.cv[id], q1 = z.cv[id + sz], q2 = z.cv[id + 2 * sz], q3 = z.cv[id + 3 * sz],
                 q4 = z.cv[id + 4 * sz];
    const double pk = z.bv[id + 4 * sz], tk = z.bv[id + 5 * sz];
    const double m0 = z.metric[id + mmo * sz], m1 = z.metric[id + (mmo + 1) * sz],
                 m2 = z.metric[id + (mmo + 2) * sz];
    const double jac = z.jac[id];
    air_stage_point<T>(spts, c, t, q0, q1, q2, q3, q4, pk, tk, m0, m1, m2, jac);
  }
  __syncthreads();

  // ---- face fluxes ------------------------------------------------------
  for (int item = threadIdx.x; item < NF * C; item += T::NT) {
    int c, t;
    split(item, NF, c, t);
    const int f = n0 - 1 + t;  // face between node f and f+1 along DIR
    if (cbase + c >= ncol_max || f > m - 1) continue;
    // face normal, averaged with the (i+1) node in every direction as the
    // reference does (reference src/WENO.cu:886-888, 1627-1629, 2303-2305)
    const int64_t idf = node_idx(g, c, f);
    double kx = 0.5 * (z.metric[idf + mmo * sz] + z.metric[idf + 1 + mmo * sz]);
    double ky = 0.5 * (z.metric[idf + (mmo + 1) * sz] + z.metric[idf + 1 + (mmo + 1) * sz]);
    double kz = 0.5 * (z.metric[idf + (mmo + 2) * sz] + z.metric[idf + 1 + (mmo + 2) * sz]);

    const bool shock = !HYB || face_shocked(sensor, idf, d.stride(g, DIR), g, threshold);
    air_face<ORD, T>(spts, sflx, c, t, kx, ky, kz, eps_ref, shock);
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
    for (int v = 0; v < 5; ++v) z.dq[iq + v * szq] -= sflx[T::sfl(v, c, t + 1)] - sflx[T::sfl(v, c, t)];
  }
}

template <int DIR, int ORD, int VAR>
static cudaError_t launch_var(const Zone &z, double eps_ref, const double *sensor, double threshold,
                              cudaStream_t st) {
  using T = AirTile<DIR, ORD, VAR>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  const size_t smem = T::smem_bytes();
  if (sensor) weno_air_flux_diff<DIR, ORD, true, VAR><<<grid, T::NT, smem, st>>>(z, eps_ref, sensor, threshold);
  else weno_air_flux_diff<DIR, ORD, false, VAR><<<grid, T::NT, smem, st>>>(z, eps_ref, nullptr, threshold);
  return cudaGetLastError();
}

template <int DIR, int ORD>
static cudaError_t launch_dir(const Zone &z, double eps_ref, const double *sensor, double threshold, int var,
                              cudaStream_t st) {
  if (var == 1) return launch_var<DIR, ORD, 1>(z, eps_ref, sensor, threshold, st);
  if (var == 2) return launch_var<DIR, ORD, 2>(z, eps_ref, sensor, threshold, st);
  return launch_var<DIR, ORD, 0>(z, eps_ref, sensor, threshold, st);
}

template <int DIR, int ORD, int VAR>
static cudaError_t set_smem_attr() {
  const int b = (int)AirTile<DIR, ORD, VAR>::smem_bytes();
  cudaError_t e = cudaFuncSetAttribute(weno_air_flux_diff<DIR, ORD, false, VAR>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(weno_air_flux_diff<DIR, ORD, true, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              b);
}

template <int DIR, int ORD>
static cudaError_t set_smem_attrs() {
  cudaError_t e;
  if ((e = set_smem_attr<DIR, ORD, 0>()) != cudaSuccess) return e;
  if ((e = set_smem_attr<DIR, ORD, 1>()) != cudaSuccess) return e;
  return set_smem_attr<DIR, ORD, 2>();
}

// Opt every instantiation in to its dynamic shared-memory size (> 48 KB for
// the y/z tiles).  Called once per device at context creation, outside any
// stream capture.
cudaError_t weno_air_init_attributes() {
  cudaError_t e;
  if ((e = set_smem_attrs<0, 5>()) != cudaSuccess) return e;
  if ((e = set_smem_attrs<1, 5>()) != cudaSuccess) return e;
  if ((e = set_smem_attrs<2, 5>()) != cudaSuccess) return e;
  if ((e = set_smem_attrs<0, 7>()) != cudaSuccess) return e;
  if ((e = set_smem_attrs<1, 7>()) != cudaSuccess) return e;
  return set_smem_attrs<2, 7>();
}

// One sweep (dir 0/1/2) with tile variant var.
cudaError_t launch_weno_air_dir(const Zone &z, const Param &p, int dir, int var, cudaStream_t st) {
  const double eps_ref = kEpsWeno * p.weno_eps_scale;
  // hybrid UD5/UD7 + WENO when a sensor threshold is set (reference src/Parameter.cpp:236-252)
  const double th = p.sensor_threshold;
  const double *sn = th > 1e-10 ? z.shock_sensor : nullptr;
  const bool w7 = p.inviscid_scheme == 72;
  if (dir == 0) return w7 ? launch_dir<0, 7>(z, eps_ref, sn, th, var, st) : launch_dir<0, 5>(z, eps_ref, sn, th, var, st);
  if (dir == 1) return w7 ? launch_dir<1, 7>(z, eps_ref, sn, th, var, st) : launch_dir<1, 5>(z, eps_ref, sn, th, var, st);
  return w7 ? launch_dir<2, 7>(z, eps_ref, sn, th, var, st) : launch_dir<2, 5>(z, eps_ref, sn, th, var, st);
}

// Host launcher: x, y and (3-D) z sweeps in the reference's order; var[d]
// is the tile variant of sweep d.
cudaError_t launch_weno_air(const Zone &z, const Param &p, const int *var, cudaStream_t st, int *n_launch) {
  const int nd = z.d.mz > 1 ? 3 : 2;
  for (int dir = 0; dir < nd; ++dir) {
    cudaError_t e = launch_weno_air_dir(z, p, dir, var[dir], st);
    if (e != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
