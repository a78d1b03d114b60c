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
// Tile: TN nodes along the sweep x C columns; faces n0-1 .. n0+TN-1 need the
// TN + 2 nodes n0-1 .. n0+TN, whose per-node values are staged once.
template <int DIR>
struct VisTile {
  static constexpr int TN = DIR == 0 ? 63 : 15;
  static constexpr int C = DIR == 0 ? 4 : 16;
  static constexpr int NF = TN + 1;
  static constexpr int NP = TN + 2;  // staged nodes per column
  static constexpr int NT = 256;
  // per node: u v w T (4), transverse differences f(+1)-f(-1) of u v w T along
  // the two other directions (8), metric (9), metric row of DIR times J (3), mu
  static constexpr int NQ = 25;
  static constexpr int QV = 0, QD = 4, QM = 12, QK = 21, QMU = 24;
  __device__ static int spt(int q, int c, int t) {
    return DIR == 0 ? (q * C + c) * NP + t : (q * NP + t) * C + c;
  }
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(NQ * C * NP + 4 * C * NF); }
};
}  // namespace

// Three phases, as in the WENO kernels: stage the per-node values of the
// tile (each node's bv, transverse differences, metrics and mu are loaded
// once instead of once per adjacent face), compute the face fluxes into
// shared memory, difference them into dq.  The face arithmetic is the
// reference's except that its transverse derivative
// 0.25 * (f(A+) - f(A-) + f(B+) - f(B-)) is summed as
// 0.25 * ((f(A+) - f(A-)) + (f(B+) - f(B-))) from the staged node differences.
template <int DIR>
__global__ void __launch_bounds__(256, 3) viscous_air_flux_diff(Zone z, double Pr) {
  using T = VisTile<DIR>;
  constexpr int TN = T::TN, C = T::C, NF = T::NF, NP = T::NP;
  extern __shared__ double sm[];
  double *spts = sm;
  double *sflx = sm + T::NQ * C * NP;
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
  // the two transverse directions, lower-numbered first
  constexpr int TLO = DIR == 0 ? 1 : 0, THI = DIR == 2 ? 1 : 2;
  const int64_t slo = d.stride(g, TLO), shi = d.stride(g, THI);
  const int mo = 3 * DIR;

  // ---- stage: nodes n0-1 .. n0+TN ----------------------------------------
  for (int item = threadIdx.x; item < NP * C; item += T::NT) {
    int c, t;
    split(item, NP, c, t);
    const int a = n0 - 1 + t;
    if (cbase + c >= ncol_max || a > m) continue;
    const int64_t id = node_idx(g, c, a);
    const int slots[4] = {1, 2, 3, 5};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double *f = z.bv + slots[q] * sz + id;
      spts[T::spt(T::QV + q, c, t)] = f[0];
      spts[T::spt(T::QD + 2 * q, c, t)] = f[slo] - f[-slo];
      spts[T::spt(T::QD + 2 * q + 1, c, t)] = f[shi] - f[-shi];
    }
    const double jac = z.jac[id];
#pragma unroll
    for (int l = 0; l < 9; ++l) spts[T::spt(T::QM + l, c, t)] = z.metric[id + l * sz];
#pragma unroll
    for (int l = 0; l < 3; ++l) spts[T::spt(T::QK + l, c, t)] = z.metric[id + (mo + l) * sz] * jac;
    spts[T::spt(T::QMU, c, t)] = z.mul[id];
  }
  __syncthreads();

  // ---- faces -------------------------------------------------------------
  for (int item = threadIdx.x; item < NF * C; item += T::NT) {
    int c, t;
    split(item, NF, c, t);
    const int f = n0 - 1 + t;
    if (cbase + c >= ncol_max || f > m - 1) continue;
    const double *s = spts;
    auto A = [&](int q) { return s[T::spt(q, c, t)]; };
    auto B = [&](int q) { return s[T::spt(q, c, t + 1)]; };
    double gm[9];
#pragma unroll
    for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (A(T::QM + l) + B(T::QM + l));
    double dd[4][3];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dd[q][DIR] = B(T::QV + q) - A(T::QV + q);
      dd[q][TLO] = 0.25 * (A(T::QD + 2 * q) + B(T::QD + 2 * q));
      dd[q][THI] = 0.25 * (A(T::QD + 2 * q + 1) + B(T::QD + 2 * q + 1));
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
    const double mul = 0.5 * (A(T::QMU) + B(T::QMU));
    const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
    const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
    const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
    const double tau_xy = mul * (u_y + v_x);
    const double tau_xz = mul * (u_z + w_x);
    const double tau_yz = mul * (v_z + w_y);
    const double gk0 = 0.5 * (A(T::QK) + B(T::QK));
    const double gk1 = 0.5 * (A(T::QK + 1) + B(T::QK + 1));
    const double gk2 = 0.5 * (A(T::QK + 2) + B(T::QK + 2));
    const double f0 = gk0 * tau_xx + gk1 * tau_xy + gk2 * tau_xz;
    const double f1 = gk0 * tau_xy + gk1 * tau_yy + gk2 * tau_yz;
    const double f2 = gk0 * tau_xz + gk1 * tau_yz + gk2 * tau_zz;
    const double um = 0.5 * (A(T::QV) + B(T::QV));
    const double vm = 0.5 * (A(T::QV + 1) + B(T::QV + 1));
    const double wm = 0.5 * (A(T::QV + 2) + B(T::QV + 2));
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

// Column march for the y and z sweeps: one thread per i column walks TM
// nodes along the sweep, keeping the previous node's values and face flux in
// registers, so every node is loaded once, loads stay coalesced along i and
// no block barrier separates load and compute.  Same face arithmetic as the
// staged kernel above.
namespace {
struct VisNode {
  double v[4];     // u, v, w, T
  double dlo[4];   // f(+1) - f(-1) along the lower-numbered transverse direction
  double dhi[4];   // ... along the higher-numbered one
  double mt[9];    // metric
  double mk[3];    // metric row of the sweep times J
  double mu;
};

template <int DIR>
__device__ __forceinline__ void load_node(const Zone &z, int64_t id, int64_t sz, int64_t slo, int64_t shi,
                                          VisNode &n) {
  const int slots[4] = {1, 2, 3, 5};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double *f = z.bv + slots[q] * sz + id;
    n.v[q] = __ldg(f);
    n.dlo[q] = __ldg(f + slo) - __ldg(f - slo);
    n.dhi[q] = __ldg(f + shi) - __ldg(f - shi);
  }
  const double jac = __ldg(z.jac + id);
#pragma unroll
  for (int l = 0; l < 9; ++l) n.mt[l] = __ldg(z.metric + id + l * sz);
#pragma unroll
  for (int l = 0; l < 3; ++l) n.mk[l] = n.mt[3 * DIR + l] * jac;
  n.mu = __ldg(z.mul + id);
}

template <int DIR>
__device__ __forceinline__ void face_flux(const VisNode &A, const VisNode &B, double Pr, double F[4]) {
  constexpr int TLO = DIR == 0 ? 1 : 0, THI = DIR == 2 ? 1 : 2;
  double gm[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (A.mt[l] + B.mt[l]);
  double dd[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    dd[q][DIR] = B.v[q] - A.v[q];
    dd[q][TLO] = 0.25 * (A.dlo[q] + B.dlo[q]);
    dd[q][THI] = 0.25 * (A.dhi[q] + B.dhi[q]);
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
  const double mul = 0.5 * (A.mu + B.mu);
  const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double tau_xy = mul * (u_y + v_x);
  const double tau_xz = mul * (u_z + w_x);
  const double tau_yz = mul * (v_z + w_y);
  const double gk0 = 0.5 * (A.mk[0] + B.mk[0]);
  const double gk1 = 0.5 * (A.mk[1] + B.mk[1]);
  const double gk2 = 0.5 * (A.mk[2] + B.mk[2]);
  F[0] = gk0 * tau_xx + gk1 * tau_xy + gk2 * tau_xz;
  F[1] = gk0 * tau_xy + gk1 * tau_yy + gk2 * tau_yz;
  F[2] = gk0 * tau_xz + gk1 * tau_yz + gk2 * tau_zz;
  const double um = 0.5 * (A.v[0] + B.v[0]);
  const double vm = 0.5 * (A.v[1] + B.v[1]);
  const double wm = 0.5 * (A.v[2] + B.v[2]);
  const double t_x = dd[3][0] * gm[0] + dd[3][1] * gm[3] + dd[3][2] * gm[6];
  const double t_y = dd[3][0] * gm[1] + dd[3][1] * gm[4] + dd[3][2] * gm[7];
  const double t_z = dd[3][0] * gm[2] + dd[3][1] * gm[5] + dd[3][2] * gm[8];
  constexpr double cp = kGammaAir * kRAir / (kGammaAir - 1);
  const double conductivity = mul / Pr * cp;
  F[3] = um * F[0] + vm * F[1] + wm * F[2] + conductivity * (gk0 * t_x + gk1 * t_y + gk2 * t_z);
}

constexpr int kMarchTM = 32;   // nodes per thread
constexpr int kMarchNT = 128;  // threads (i columns) per CTA
}  // namespace

template <int DIR>
__global__ void __launch_bounds__(kMarchNT) viscous_air_march(Zone z, double Pr) {
  static_assert(DIR == 1 || DIR == 2, "the x sweep uses the staged kernel");
  const Dims d = z.d;
  const int i = blockIdx.x * kMarchNT + threadIdx.x;
  if (i >= d.mx) return;
  const int n0 = blockIdx.y * kMarchTM, other = blockIdx.z;
  const int m = d.ext(DIR);
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int64_t sd = d.stride(g, DIR), sdq = d.stride(0, DIR);
  constexpr int TLO = DIR == 0 ? 1 : 0, THI = DIR == 2 ? 1 : 2;
  const int64_t slo = d.stride(g, TLO), shi = d.stride(g, THI);
  int64_t id = DIR == 1 ? d.idx(g, i, n0 - 1, other) : d.idx(g, i, other, n0 - 1);
  int64_t iq = DIR == 1 ? d.idx(0, i, n0, other) : d.idx(0, i, other, n0);
  VisNode A, B;
  load_node<DIR>(z, id, sz, slo, shi, A);
  load_node<DIR>(z, id + sd, sz, slo, shi, B);
  double Fp[4];
  face_flux<DIR>(A, B, Pr, Fp);  // face n0 - 1/2
  const int n_end = min(n0 + kMarchTM, m);
  for (int n = n0; n < n_end; ++n) {
    // face n + 1/2 between node n (B) and node n + 1
    id += sd;
    A = B;
    load_node<DIR>(z, id + sd, sz, slo, shi, B);
    double F[4];
    face_flux<DIR>(A, B, Pr, F);
#pragma unroll
    for (int v = 0; v < 4; ++v) z.dq[iq + (v + 1) * szq] += F[v] - Fp[v];
#pragma unroll
    for (int v = 0; v < 4; ++v) Fp[v] = F[v];
    iq += sdq;
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
  if (DIR == 0) {
    viscous_air_flux_diff<DIR><<<grid, T::NT, T::smem_bytes(), st>>>(z, Pr);
  } else {
    const dim3 gm((d.mx + kMarchNT - 1) / kMarchNT, (d.ext(DIR) + kMarchTM - 1) / kMarchTM,
                  DIR == 1 ? d.mz : d.my);
    viscous_air_march<DIR == 0 ? 1 : DIR><<<gm, kMarchNT, 0, st>>>(z, Pr);
  }
  return cudaGetLastError();
}

// Opt the three sweeps in to their dynamic shared-memory size (> 48 KB).
cudaError_t viscous_air_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(viscous_air_flux_diff<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)VisTile<0>::smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(viscous_air_flux_diff<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VisTile<1>::smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(viscous_air_flux_diff<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VisTile<2>::smem_bytes());
  return e;
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
