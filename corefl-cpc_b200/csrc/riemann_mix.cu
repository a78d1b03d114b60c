// Primitive-variable schemes for a reacting mixture (9 species): first-order
// / MUSCL / NND2 reconstruction of rho, u, v, w, p and the mass fractions,
// side energies and gamma from NASA-7 thermo, the Roe, AUSM+ or HLLC flux
// with its species terms, and the flux difference, fused per direction.
//
// Restates compute_convective_term_pv_1D and Roe_compute_inviscid_flux_1D
// with compute_entropy_fix_delta (reference src/InviscidScheme.cu:61-395,
// mixture branches) in the stage / faces / diff structure of riemann_air.cu:
//   stage — rho, u, v, w, p and Y_1..Y_9 of the TN + 4 stencil points of each
//           column (Roe: + the entropy-fix width from the nine metric terms
//           and the acoustic-speed array);
//   faces — one thread per face: reconstruction of 14 variables from four
//           points, two thermo evaluations for the side states (and one at
//           the Roe-averaged temperature for Roe and HLLC), the flux of all
//           14 variables into shared memory;
//   diff  — dq(n) -= F(n+1/2) - F(n-1/2).
#include "cfk_common.cuh"
#include "riemann.cuh"
#include "riemann_mix.cuh"

namespace cfk {

namespace {

template <int DIR, int SCH, int NS>
struct PvMixTile {
  static constexpr int TN = DIR == 0 ? 124 : 28;  // nodes per column
  static constexpr int C = DIR == 0 ? 2 : 16;     // columns per CTA
  static constexpr int NF = TN + 1;
  static constexpr int NPT = TN + 4;              // staged points (i-2 .. i+TN+1)
  static constexpr int NV = 5 + NS;
  static constexpr int NQ = NV + (SCH == 2 ? 1 : 0);  // primitives (+ entropy-fix width)
  static constexpr int NT = 256;
  __device__ static int spt(int q, int c, int t) {
    return DIR == 0 ? (q * C + c) * NPT + t : (q * NPT + t) * C + c;
  }
  __device__ static int sfl(int v, int c, int t) {
    return DIR == 0 ? (v * C + c) * NF + t : (v * NF + t) * C + c;
  }
  static constexpr size_t smem_bytes() { return sizeof(double) * (size_t)(NQ * C * NPT + NV * C * NF); }
};

}  // namespace

template <int DIR, int SCH, int RECON, int NS>
__global__ void __launch_bounds__(256) pv_mix_flux_diff(Zone z, int dim, double entropy_fix_factor,
                                                        const __grid_constant__ Thermo thermo) {
  using T = PvMixTile<DIR, SCH, NS>;
  constexpr int TN = T::TN, C = T::C, NF = T::NF, NPT = T::NPT, NV = T::NV;
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

  // ---- stage: nodes n0-2 .. n0+TN+1 -----------------------------------
  for (int item = threadIdx.x; item < NPT * C; item += T::NT) {
    int c, t;
    split(item, NPT, c, t);
    const int a = n0 - 2 + t;
    if (cbase + c >= ncol_max || a > m + 1) continue;
    const int64_t id = node_idx(g, c, a);
#pragma unroll
    for (int l = 0; l < 5; ++l) spts[T::spt(l, c, t)] = z.bv[id + l * sz];
#pragma unroll
    for (int l = 0; l < NS; ++l) spts[T::spt(5 + l, c, t)] = z.sv[id + l * sz];
    if (SCH == 2) {
      double mt[9];
#pragma unroll
      for (int l = 0; l < 9; ++l) mt[l] = z.metric[id + l * sz];
      spts[T::spt(NV, c, t)] = entropy_fix_delta_mix(spts[T::spt(1, c, t)], spts[T::spt(2, c, t)],
                                                     spts[T::spt(3, c, t)], z.acoustic_speed[id], mt, dim,
                                                     entropy_fix_factor);
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
    double pl[NV + 2], pr[NV + 2];
#pragma unroll
    for (int l = 0; l < NV; ++l)
      reconstruct_var<RECON>(spts[T::spt(l, c, pc - 1)], spts[T::spt(l, c, pc)], spts[T::spt(l, c, pc + 1)],
                             spts[T::spt(l, c, pc + 2)], pl[l], pr[l]);
    add_energy_mix<NS>(th, pl);
    add_energy_mix<NS>(th, pr);
    const int64_t idf = node_idx(g, c, f);
    const int64_t sd = d.stride(g, DIR);
    double mtr[2][3], jac[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
#pragma unroll
      for (int l = 0; l < 3; ++l) mtr[q][l] = z.metric[idf + q * sd + (mmo + l) * sz];
      jac[q] = z.jac[idf + q * sd];
    }
    double fc[NV];
    if (SCH == 2) {
      const double delta[2] = {spts[T::spt(NV, c, pc)], spts[T::spt(NV, c, pc + 1)]};
      roe_mix<NS>(th, pl, pr, mtr, jac, delta, fc);
    } else if (SCH == 4) {
      hllc_mix<NS>(th, pl, pr, mtr, jac, fc);
    } else {
      ausm_plus_mix<NS>(pl, pr, mtr, jac, fc);
    }
#pragma unroll
    for (int l = 0; l < NV; ++l) sflx[T::sfl(l, c, t)] = fc[l];
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
    for (int l = 0; l < NV; ++l) z.dq[iq + l * szq] -= sflx[T::sfl(l, c, t + 1)] - sflx[T::sfl(l, c, t)];
  }
}

namespace {

template <int DIR, int SCH, int RECON>
cudaError_t launch_pv_mix_dir(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st) {
  using T = PvMixTile<DIR, SCH, kMaxSpec>;
  const Dims &d = z.d;
  dim3 grid;
  if (DIR == 0) grid = dim3((d.mx + T::TN - 1) / T::TN, (d.my + T::C - 1) / T::C, d.mz);
  else if (DIR == 1) grid = dim3((d.mx + T::C - 1) / T::C, (d.my + T::TN - 1) / T::TN, d.mz);
  else grid = dim3((d.mx + T::C - 1) / T::C, (d.mz + T::TN - 1) / T::TN, d.my);
  pv_mix_flux_diff<DIR, SCH, RECON, kMaxSpec>
      <<<grid, T::NT, T::smem_bytes(), st>>>(z, p.dim, p.entropy_fix_factor, th);
  return cudaGetLastError();
}

template <int DIR, int SCH>
cudaError_t launch_pv_mix_recon(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st) {
  if (p.reconstruction == 2) return launch_pv_mix_dir<DIR, SCH, 2>(z, p, th, st);
  if (p.reconstruction == 3) return launch_pv_mix_dir<DIR, SCH, 3>(z, p, th, st);
  return launch_pv_mix_dir<DIR, SCH, 1>(z, p, th, st);
}

template <int DIR>
cudaError_t launch_pv_mix_scheme(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st) {
  switch (p.inviscid_scheme) {
    case 2: return launch_pv_mix_recon<DIR, 2>(z, p, th, st);
    case 4: return launch_pv_mix_recon<DIR, 4>(z, p, th, st);
    default: return launch_pv_mix_recon<DIR, 3>(z, p, th, st);
  }
}

template <int DIR, int SCH, int RECON>
cudaError_t set_pv_mix_attr() {
  return cudaFuncSetAttribute(pv_mix_flux_diff<DIR, SCH, RECON, kMaxSpec>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)PvMixTile<DIR, SCH, kMaxSpec>::smem_bytes());
}

template <int DIR, int SCH>
cudaError_t set_pv_mix_attr_recon() {
  cudaError_t e;
  if ((e = set_pv_mix_attr<DIR, SCH, 1>()) != cudaSuccess) return e;
  if ((e = set_pv_mix_attr<DIR, SCH, 2>()) != cudaSuccess) return e;
  return set_pv_mix_attr<DIR, SCH, 3>();
}

template <int DIR>
cudaError_t set_pv_mix_attr_dir() {
  cudaError_t e;
  if ((e = set_pv_mix_attr_recon<DIR, 2>()) != cudaSuccess) return e;
  if ((e = set_pv_mix_attr_recon<DIR, 3>()) != cudaSuccess) return e;
  return set_pv_mix_attr_recon<DIR, 4>();
}

}  // namespace

cudaError_t pv_mix_init_attributes() {
  cudaError_t e;
  if ((e = set_pv_mix_attr_dir<0>()) != cudaSuccess) return e;
  if ((e = set_pv_mix_attr_dir<1>()) != cudaSuccess) return e;
  return set_pv_mix_attr_dir<2>();
}

// x, y and (3-D) z sweeps; Roe (2), AUSM+ (3), HLLC (4).
cudaError_t launch_pv_mix(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st, int *n_launch) {
  cudaError_t e;
  if ((e = launch_pv_mix_scheme<0>(z, p, th, st)) != cudaSuccess) return e;
  if ((e = launch_pv_mix_scheme<1>(z, p, th, st)) != cudaSuccess) return e;
  *n_launch += 2;
  if (z.d.mz > 1) {
    if ((e = launch_pv_mix_scheme<2>(z, p, th, st)) != cudaSuccess) return e;
    *n_launch += 1;
  }
  return cudaSuccess;
}

}  // namespace cfk
