// Primitive-variable schemes, calorically perfect air: first-order / MUSCL /
// NND2 reconstruction with the Lax-Friedrichs, Roe, AUSM+ or HLLC flux and
// the flux difference, fused per direction.
//
// Restates compute_convective_term_pv_1D (reference
// src/InviscidScheme.cu:61-169) and Roe_compute_inviscid_flux_1D with
// compute_entropy_fix_delta (:269-395) as one kernel per direction and
// scheme:
//   stage — a CTA stages the primitive variables rho, u, v, w, p of the
//           TN + 4 stencil points of each of its C columns (and, for Roe, the
//           entropy-fix width of each point, computed there from the point's
//           nine metric terms instead of in a separate pass);
//   faces — one thread per face reconstructs the left/right states from four
//           points, reads the two nodes' metric row and Jacobian (coalesced
//           along i) and evaluates the Riemann flux into shared memory;
//   diff  — dq(n) -= F(n+1/2) - F(n-1/2).
// Memory-bound: per node and direction it reads bv[5], metric[3], jac (Roe:
// metric[9]) and read-modify-writes dq[5].
#include "cfk_common.cuh"
#include "riemann.cuh"

namespace cfk {

namespace {

template <int DIR, int SCH>
struct PvTile {
  static constexpr int TN = DIR == 0 ? 124 : 28;  // nodes per column
  static constexpr int C = DIR == 0 ? 2 : 32;     // columns per CTA
  static constexpr int NF = TN + 1;               // faces per column
  static constexpr int NPT = TN + 4;              // staged points per column (i-2 .. i+TN+1)
  static constexpr int NQ = SCH == 2 ? 6 : 5;     // rho, u, v, w, p (+ entropy-fix width)
  static constexpr int NT = 256;
  __device__ static int spt(int q, int c, int t) {
    return DIR == 0 ? (q * C + c) * NPT + t : (q * NPT + t) * C + c;
  }
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(NQ * C * NPT + 5 * C * NF); }
};

}  // namespace

template <int DIR, int SCH, int RECON>
__global__ void __launch_bounds__(256) pv_air_flux_diff(Zone z, int dim, double entropy_fix_factor) {
  using T = PvTile<DIR, SCH>;
  constexpr int TN = T::TN, C = T::C, NF = T::NF, NPT = T::NPT;
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

  // ---- stage: nodes n0-2 .. n0+TN+1 -----------------------------------
  for (int item = threadIdx.x; item < NPT * C; item += T::NT) {
    int c, t;
    split(item, NPT, c, t);
    const int a = n0 - 2 + t;
    if (cbase + c >= ncol_max || a > m + 1) continue;
    const int64_t id = node_idx(g, c, a);
    double pv[5];
#pragma unroll
    for (int l = 0; l < 5; ++l) {
      pv[l] = z.bv[id + l * sz];
      spts[T::spt(l, c, t)] = pv[l];
    }
    if (SCH == 2) {
      double mt[9];
#pragma unroll
      for (int l = 0; l < 9; ++l) mt[l] = z.metric[id + l * sz];
      spts[T::spt(5, c, t)] = entropy_fix_delta_air(pv[0], pv[1], pv[2], pv[3], pv[4], mt, dim, entropy_fix_factor);
    }
  }
  __syncthreads();

  // ---- faces: n0-1 .. n0+TN-1 -------------------------------------------
  const int mmo = 3 * DIR;
  for (int item = threadIdx.x; item < NF * C; item += T::NT) {
    int c, t;
    split(item, NF, c, t);
    const int f = n0 - 1 + t;  // face between node f and f+1
    if (cbase + c >= ncol_max || f > m - 1) continue;
    const int pc = t + 1;  // local point of node f
    double pl[6], pr[6];
#pragma unroll
    for (int l = 0; l < 5; ++l)
      reconstruct_var<RECON>(spts[T::spt(l, c, pc - 1)], spts[T::spt(l, c, pc)], spts[T::spt(l, c, pc + 1)],
                             spts[T::spt(l, c, pc + 2)], pl[l], pr[l]);
    add_energy_air(pl);
    add_energy_air(pr);
    const int64_t idf = node_idx(g, c, f);
    const int64_t sd = d.stride(g, DIR);
    double mtr[2][3], jac[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
#pragma unroll
      for (int l = 0; l < 3; ++l) mtr[q][l] = z.metric[idf + q * sd + (mmo + l) * sz];
      jac[q] = z.jac[idf + q * sd];
    }
    double fc[5];
    if (SCH == 1) {
      lax_friedrichs_air(pl, pr, mtr, jac, fc);
    } else if (SCH == 2) {
      const double delta[2] = {spts[T::spt(5, c, pc)], spts[T::spt(5, c, pc + 1)]};
      roe_air(pl, pr, mtr, jac, delta, fc);
    } else if (SCH == 4) {
      hllc_air(pl, pr, mtr, jac, fc);
    } else {
      ausm_plus_air(pl, pr, mtr, jac, fc);
    }
#pragma unroll
    for (int l = 0; l < 5; ++l) sflx[T::sfl(l, c, t)] = fc[l];
  }
  __syncthreads();

  // ---- difference -------------------------------------------------------
  for (int item = threadIdx.x; item < TN * C; item += T::NT) {
    int c, t;
    split(item, TN, c, t);
    const int a = n0 + t;
    if (cbase + c >= ncol_max || a >= m) continue;
    const int64_t iq = node_idx(0, c, a);
#pragma unroll
    for (int l = 0; l < 5; ++l) z.dq[iq + l * szq] -= sflx[T::sfl(l, c, t + 1)] - sflx[T::sfl(l, c, t)];
  }
}

namespace {

template <int DIR, int SCH, int RECON>
cudaError_t launch_pv_dir(const Zone &z, const Param &p, cudaStream_t st) {
  using T = PvTile<DIR, SCH>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  pv_air_flux_diff<DIR, SCH, RECON><<<grid, T::NT, T::smem_bytes(), st>>>(z, p.dim, p.entropy_fix_factor);
  return cudaGetLastError();
}

template <int DIR, int SCH>
cudaError_t launch_pv_recon(const Zone &z, const Param &p, cudaStream_t st) {
  if (p.reconstruction == 2) return launch_pv_dir<DIR, SCH, 2>(z, p, st);
  if (p.reconstruction == 3) return launch_pv_dir<DIR, SCH, 3>(z, p, st);
  return launch_pv_dir<DIR, SCH, 1>(z, p, st);
}

template <int DIR>
cudaError_t launch_pv_scheme(const Zone &z, const Param &p, cudaStream_t st) {
  switch (p.inviscid_scheme) {
    case 1: return launch_pv_recon<DIR, 1>(z, p, st);
    case 2: return launch_pv_recon<DIR, 2>(z, p, st);
    case 4: return launch_pv_recon<DIR, 4>(z, p, st);
    default: return launch_pv_recon<DIR, 3>(z, p, st);
  }
}

template <int DIR, int SCH, int RECON>
cudaError_t set_pv_attr() {
  return cudaFuncSetAttribute(pv_air_flux_diff<DIR, SCH, RECON>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)PvTile<DIR, SCH>::smem_bytes());
}

template <int DIR, int SCH>
cudaError_t set_pv_attr_recon() {
  cudaError_t e;
  if ((e = set_pv_attr<DIR, SCH, 1>()) != cudaSuccess) return e;
  if ((e = set_pv_attr<DIR, SCH, 2>()) != cudaSuccess) return e;
  return set_pv_attr<DIR, SCH, 3>();
}

template <int DIR>
cudaError_t set_pv_attr_dir() {
  cudaError_t e;
  if ((e = set_pv_attr_recon<DIR, 1>()) != cudaSuccess) return e;
  if ((e = set_pv_attr_recon<DIR, 2>()) != cudaSuccess) return e;
  if ((e = set_pv_attr_recon<DIR, 3>()) != cudaSuccess) return e;
  return set_pv_attr_recon<DIR, 4>();
}

}  // namespace

cudaError_t pv_air_init_attributes() {
  cudaError_t e;
  if ((e = set_pv_attr_dir<0>()) != cudaSuccess) return e;
  if ((e = set_pv_attr_dir<1>()) != cudaSuccess) return e;
  return set_pv_attr_dir<2>();
}

// x, y and (3-D) z sweeps, as the reference's pv and Roe drivers order them.
cudaError_t launch_pv_air(const Zone &z, const Param &p, cudaStream_t st, int *n_launch) {
  cudaError_t e;
  if ((e = launch_pv_scheme<0>(z, p, st)) != cudaSuccess) return e;
  if ((e = launch_pv_scheme<1>(z, p, st)) != cudaSuccess) return e;
  *n_launch += 2;
  if (z.d.mz > 1) {
    if ((e = launch_pv_scheme<2>(z, p, st)) != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
