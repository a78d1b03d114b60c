// Second-order viscous flux of calorically perfect air, all three directions
// fused, with the flux differences added to dq.
//
// Restates compute_{f,g,h}v_2nd_order (air branch, reference
// src/ViscousScheme.cu:614-1173) and compute_dFv_dx / dGv_dy / dHv_dz
// (reference src/ViscousScheme.cu:75-127).  The staggered face fluxes stay in
// registers and shared memory, so the vis_flux array of the reference never
// reaches HBM, and every node's inputs are read once per stage.
#include "cfk_common.cuh"

namespace cfk {

// All three directions in one kernel: a CTA owns a 32 x 8 tile of (i, j)
// columns and marches along k through a chunk of planes, keeping two planes
// of per-node values (u, v, w, T, mu, J, metric) with a one-node halo in
// shared memory plus the k-differences f(k+1) - f(k-1) of the current plane.
// Per plane it computes the x and y faces of the plane and the z face above
// each node; the z face below comes from the previous plane.  dq gets the x,
// y and z differences added in that order, the order of the reference's
// per-direction derivative kernels.  Every node's inputs are read from HBM
// once per stage and dq once instead of three times.
namespace {
constexpr int kFX = 32, kFY = 8, kFZ = 32;     // tile and planes per chunk
constexpr int kPX = kFX + 2, kPY = kFY + 2;    // staged points per plane
constexpr int kNV = 15;                        // u v w T mu J metric[9]
constexpr int kFT = kFX * kFY;                 // threads
// the flux's constant factors as products: 1/3 of the normal stresses and
// cp / Pr of the conductivity, formed once (the reference divides by 3 and
// by Pr at every face; the results differ in the last bits)
constexpr double kThird = 1.0 / 3.0;
constexpr double kCpAir = kGammaAir * kRAir / (kGammaAir - 1);

struct FusedSmem {
  double pl[2][kNV][kPY][kPX];   // planes k and k+1 (slots swap)
  double dzp[4][kPY][kPX];       // f(k+1) - f(k-1) of u, v, w, T on plane k
  double fx[4][kFY][kFX + 1];    // x faces of plane k
  double fy[4][kFY + 1][kFX];    // y faces of plane k
};

// Face flux between staged points A = (pa, qa) of slot sa and B = (pb, qb)
// of slot sb, normal to DIR (reference src/ViscousScheme.cu:614-700 and the
// g/h analogues), read straight from shared memory: values are fetched where
// they are used so that the two nodes are never held in registers at once.
// The transverse derivative 0.25 (f(A+) - f(A-) + f(B+) - f(B-)) is summed
// as 0.25 ((f(A+) - f(A-)) + (f(B+) - f(B-))).
template <int DIR>
__device__ __forceinline__ void staged_face(const FusedSmem &S, int sa, int pa, int qa, int sb, int pb, int qb,
                                            double cp_pr, double F[4]) {
  const auto &A = S.pl[sa];
  const auto &B = S.pl[sb];
  // transverse difference of variable q at a point along direction D (0 x, 1 y, 2 z)
  auto tdiff = [&](const double (&p)[kNV][kPY][kPX], int D, int q, int px, int py) -> double {
    if (D == 0) return p[q][py][px + 1] - p[q][py][px - 1];
    if (D == 1) return p[q][py + 1][px] - p[q][py - 1][px];
    return S.dzp[q][py][px];
  };
  constexpr int TLO = DIR == 0 ? 1 : 0, THI = DIR == 2 ? 1 : 2;
  double gm[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (A[6 + l][qa][pa] + B[6 + l][qb][pb]);
  double dd[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    dd[q][DIR] = B[q][qb][pb] - A[q][qa][pa];
    dd[q][TLO] = 0.25 * (tdiff(A, TLO, q, pa, qa) + tdiff(B, TLO, q, pb, qb));
    dd[q][THI] = 0.25 * (tdiff(A, THI, q, pa, qa) + tdiff(B, THI, q, pb, qb));
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
  const double t_x = dd[3][0] * gm[0] + dd[3][1] * gm[3] + dd[3][2] * gm[6];
  const double t_y = dd[3][0] * gm[1] + dd[3][1] * gm[4] + dd[3][2] * gm[7];
  const double t_z = dd[3][0] * gm[2] + dd[3][1] * gm[5] + dd[3][2] * gm[8];
  const double mul = 0.5 * (A[4][qa][pa] + B[4][qb][pb]);
  const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) * kThird;
  const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) * kThird;
  const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) * kThird;
  const double tau_xy = mul * (u_y + v_x);
  const double tau_xz = mul * (u_z + w_x);
  const double tau_yz = mul * (v_z + w_y);
  const double ja = A[5][qa][pa], jb = B[5][qb][pb];
  const double gk0 = 0.5 * (A[6 + 3 * DIR][qa][pa] * ja + B[6 + 3 * DIR][qb][pb] * jb);
  const double gk1 = 0.5 * (A[7 + 3 * DIR][qa][pa] * ja + B[7 + 3 * DIR][qb][pb] * jb);
  const double gk2 = 0.5 * (A[8 + 3 * DIR][qa][pa] * ja + B[8 + 3 * DIR][qb][pb] * jb);
  F[0] = gk0 * tau_xx + gk1 * tau_xy + gk2 * tau_xz;
  F[1] = gk0 * tau_xy + gk1 * tau_yy + gk2 * tau_yz;
  F[2] = gk0 * tau_xz + gk1 * tau_yz + gk2 * tau_zz;
  const double um = 0.5 * (A[0][qa][pa] + B[0][qb][pb]);
  const double vm = 0.5 * (A[1][qa][pa] + B[1][qb][pb]);
  const double wm = 0.5 * (A[2][qa][pa] + B[2][qb][pb]);
  const double conductivity = mul * cp_pr;
  F[3] = um * F[0] + vm * F[1] + wm * F[2] + conductivity * (gk0 * t_x + gk1 * t_y + gk2 * t_z);
}
}  // namespace

__global__ void __launch_bounds__(kFT, 2) viscous_air_fused(Zone z, double Pr) {
  extern __shared__ __align__(16) double fsm[];
  const double cp_pr = kCpAir / Pr;
  FusedSmem &S = *reinterpret_cast<FusedSmem *>(fsm);
  const Dims d = z.d;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int i0 = blockIdx.x * kFX, j0 = blockIdx.y * kFY, k0 = blockIdx.z * kFZ;
  const int tx = threadIdx.x % kFX, ty = threadIdx.x / kFX;
  const bool three_d = d.mz > 1;
  const int k_end = min(k0 + kFZ, d.mz);

  // per-thread share of a plane's staged points: p = threadIdx.x, + kFT
  auto point_ok = [&](int p, int &px, int &py) {
    py = p / kPX;
    px = p - py * kPX;
    return p < kPX * kPY && i0 - 1 + px <= d.mx && j0 - 1 + py <= d.my;
  };
  // the 15 staged values of point (px, py) of plane k into slot sl
  auto load_point = [&](int k, int px, int py, int sl) {
    const int64_t id = d.idx(g, i0 - 1 + px, j0 - 1 + py, k);
    double v[kNV];
    v[0] = z.bv[id + sz];
    v[1] = z.bv[id + 2 * sz];
    v[2] = z.bv[id + 3 * sz];
    v[3] = z.bv[id + 5 * sz];
    v[4] = z.mul[id];
    v[5] = z.jac[id];
#pragma unroll
    for (int l = 0; l < 9; ++l) v[6 + l] = z.metric[id + l * sz];
#pragma unroll
    for (int q = 0; q < kNV; ++q) S.pl[sl][q][py][px] = v[q];
  };

  // planes k0-1 (slot 0) and k0 (slot 1); the z face k0-1/2 between them
  for (int sl = 0; sl < 2; ++sl)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int px, py;
      if (point_ok(threadIdx.x + r * kFT, px, py)) load_point(k0 - 1 + sl, px, py, sl);
    }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = i < d.mx && j < d.my;
  double fzp[4] = {0, 0, 0, 0};
  if (three_d && mine) {
    staged_face<2>(S, 0, tx + 1, ty + 1, 1, tx + 1, ty + 1, cp_pr, fzp);
  }
  // the first iteration refills slot 0, which the z faces above read at
  // neighbouring points
  __syncthreads();
  int cur = 1;  // slot of plane k
  for (int k = k0; k < k_end; ++k) {
    const int nxt = cur ^ 1;  // holds plane k-1, receives plane k+1
    // dq of this node for plane k: loaded now, used after the faces
    double acc[4];
    const int64_t iq = d.idx(0, i, j, k);
    if (mine) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = z.dq[iq + (q + 1) * szq];
    }
    // plane k+1 replaces plane k-1 point by point: every point is read and
    // written by the thread that loads it, so the k-differences
    // f(k+1) - f(k-1) of u, v, w, T come from the old slot value before the
    // new one overwrites it, with no barrier between the two
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int px, py;
      if (!point_ok(threadIdx.x + r * kFT, px, py)) continue;
      const int64_t id = d.idx(g, i0 - 1 + px, j0 - 1 + py, k + 1);
      double v[kNV];
      v[0] = z.bv[id + sz];
      v[1] = z.bv[id + 2 * sz];
      v[2] = z.bv[id + 3 * sz];
      v[3] = z.bv[id + 5 * sz];
      v[4] = z.mul[id];
      v[5] = z.jac[id];
#pragma unroll
      for (int l = 0; l < 9; ++l) v[6 + l] = z.metric[id + l * sz];
#pragma unroll
      for (int q = 0; q < 4; ++q) S.dzp[q][py][px] = v[q] - S.pl[nxt][q][py][px];
#pragma unroll
      for (int q = 0; q < kNV; ++q) S.pl[nxt][q][py][px] = v[q];
    }
    __syncthreads();
    // x faces (33 per row) and y faces (9 per column) of plane k as one work
    // list, the y part starting on a warp boundary, so that the faces beyond
    // one per thread spread over two warps instead of piling onto the first
    constexpr int kNXF = kFY * (kFX + 1), kNYF = (kFY + 1) * kFX;
    constexpr int kYF0 = (kNXF + 31) / 32 * 32;
    for (int f = threadIdx.x; f < kYF0 + kNYF; f += kFT) {
      if (f < kYF0) {
        if (f >= kNXF) continue;
        const int fy_ = f / (kFX + 1), fx_ = f - fy_ * (kFX + 1);
        if (i0 - 1 + fx_ > d.mx - 1 || j0 + fy_ >= d.my) continue;
        double F[4];
        staged_face<0>(S, cur, fx_, fy_ + 1, cur, fx_ + 1, fy_ + 1, cp_pr, F);
#pragma unroll
        for (int q = 0; q < 4; ++q) S.fx[q][fy_][fx_] = F[q];
      } else {
        const int e = f - kYF0;
        const int fy_ = e / kFX, fx_ = e - fy_ * kFX;
        if (i0 + fx_ >= d.mx || j0 - 1 + fy_ > d.my - 1) continue;
        double F[4];
        staged_face<1>(S, cur, fx_ + 1, fy_, cur, fx_ + 1, fy_ + 1, cp_pr, F);
#pragma unroll
        for (int q = 0; q < 4; ++q) S.fy[q][fy_][fx_] = F[q];
      }
    }
    double fzn[4] = {0, 0, 0, 0};
    if (three_d && mine) {
      staged_face<2>(S, cur, tx + 1, ty + 1, nxt, tx + 1, ty + 1, cp_pr, fzn);
    }
    __syncthreads();
    if (mine) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double a = acc[q];
        a += S.fx[q][ty][tx + 1] - S.fx[q][ty][tx];
        a += S.fy[q][ty + 1][tx] - S.fy[q][ty][tx];
        if (three_d) a += fzn[q] - fzp[q];
        z.dq[iq + (q + 1) * szq] = a;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) fzp[q] = fzn[q];
    cur = nxt;
  }
}

// Ring variant: the same tile, march and arithmetic, with only the dynamic
// values (u, v, w, T, mu) staged in shared memory, in a ring of three plane
// slots filled by cp.async: plane k+2 is requested before the faces of plane
// k are computed and lands while they run, so the loads never stall a warp.
// The metric and J (read-only) come through L1 from global memory.  70 KB of
// shared memory per CTA, two CTAs per SM, two barriers per plane.  The face
// flux is term for term that of staged_face (the compiler may contract its
// products into FMAs differently, so the two agree to the last bits).
namespace {
constexpr int kRV = 5;  // u v w T mu

struct RingSmem {
  double dyn[3][kRV][kPY][kPX];  // planes k-1, k, k+1 (slots rotate; one is refilled with k+2)
  double dzp[4][kPY][kPX];       // f(k+1) - f(k-1) of u, v, w, T on plane k
  double fx[4][kFY][kFX + 1];
  double fy[4][kFY + 1][kFX];
};

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void prefetch_l2(const double *p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// staged_face with the metric and J of the two nodes (global indices ida, idb) read from global memory.
template <int DIR>
__device__ __forceinline__ void ring_face(const RingSmem &S, const double *__restrict__ met,
                                          const double *__restrict__ jac, int64_t sz, int sa, int pa, int qa,
                                          int64_t ida, int sb, int pb, int qb, int64_t idb, double cp_pr,
                                          double F[4]) {
  const auto &A = S.dyn[sa];
  const auto &B = S.dyn[sb];
  auto tdiff = [&](const double (&p)[kRV][kPY][kPX], int D, int q, int px, int py) -> double {
    if (D == 0) return p[q][py][px + 1] - p[q][py][px - 1];
    if (D == 1) return p[q][py + 1][px] - p[q][py - 1][px];
    return S.dzp[q][py][px];
  };
  constexpr int TLO = DIR == 0 ? 1 : 0, THI = DIR == 2 ? 1 : 2;
  double gm[9];
#pragma unroll
  for (int l = 0; l < 9; ++l) gm[l] = 0.5 * (__ldg(met + ida + l * sz) + __ldg(met + idb + l * sz));
  double dd[4][3];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    dd[q][DIR] = B[q][qb][pb] - A[q][qa][pa];
    dd[q][TLO] = 0.25 * (tdiff(A, TLO, q, pa, qa) + tdiff(B, TLO, q, pb, qb));
    dd[q][THI] = 0.25 * (tdiff(A, THI, q, pa, qa) + tdiff(B, THI, q, pb, qb));
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
  const double t_x = dd[3][0] * gm[0] + dd[3][1] * gm[3] + dd[3][2] * gm[6];
  const double t_y = dd[3][0] * gm[1] + dd[3][1] * gm[4] + dd[3][2] * gm[7];
  const double t_z = dd[3][0] * gm[2] + dd[3][1] * gm[5] + dd[3][2] * gm[8];
  const double mul = 0.5 * (A[4][qa][pa] + B[4][qb][pb]);
  const double tau_xx = mul * (4 * u_x - 2 * v_y - 2 * w_z) * kThird;
  const double tau_yy = mul * (4 * v_y - 2 * u_x - 2 * w_z) * kThird;
  const double tau_zz = mul * (4 * w_z - 2 * u_x - 2 * v_y) * kThird;
  const double tau_xy = mul * (u_y + v_x);
  const double tau_xz = mul * (u_z + w_x);
  const double tau_yz = mul * (v_z + w_y);
  const double ja = __ldg(jac + ida), jb = __ldg(jac + idb);
  const double gk0 = 0.5 * (__ldg(met + ida + (3 * DIR) * sz) * ja + __ldg(met + idb + (3 * DIR) * sz) * jb);
  const double gk1 = 0.5 * (__ldg(met + ida + (3 * DIR + 1) * sz) * ja + __ldg(met + idb + (3 * DIR + 1) * sz) * jb);
  const double gk2 = 0.5 * (__ldg(met + ida + (3 * DIR + 2) * sz) * ja + __ldg(met + idb + (3 * DIR + 2) * sz) * jb);
  F[0] = gk0 * tau_xx + gk1 * tau_xy + gk2 * tau_xz;
  F[1] = gk0 * tau_xy + gk1 * tau_yy + gk2 * tau_yz;
  F[2] = gk0 * tau_xz + gk1 * tau_yz + gk2 * tau_zz;
  const double um = 0.5 * (A[0][qa][pa] + B[0][qb][pb]);
  const double vm = 0.5 * (A[1][qa][pa] + B[1][qb][pb]);
  const double wm = 0.5 * (A[2][qa][pa] + B[2][qb][pb]);
  const double conductivity = mul * cp_pr;
  F[3] = um * F[0] + vm * F[1] + wm * F[2] + conductivity * (gk0 * t_x + gk1 * t_y + gk2 * t_z);
}
}  // namespace

// MINB: CTAs per SM the register budget is sized for (2: no spills; 3: about
// 80 registers with a few spills, 24 warps per SM).  PF: with the request of
// plane k+2's dynamic values, also ask L2 for its metric and J (the faces of
// plane k+2 read them through L1 two planes later), so that those loads no
// longer wait on DRAM.
template <int MINB, bool PF>
__global__ void __launch_bounds__(kFT, MINB) viscous_air_ring(Zone z, double Pr) {
  extern __shared__ __align__(16) double rsm[];
  const double cp_pr = kCpAir / Pr;
  RingSmem &S = *reinterpret_cast<RingSmem *>(rsm);
  const Dims d = z.d;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int64_t srow = d.stride(g, 1), spl = d.stride(g, 2);
  const int i0 = blockIdx.x * kFX, j0 = blockIdx.y * kFY, k0 = blockIdx.z * kFZ;
  const int tx = threadIdx.x % kFX, ty = threadIdx.x / kFX;
  const bool three_d = d.mz > 1;
  const int k_end = min(k0 + kFZ, d.mz);
  const double *__restrict__ met = z.metric;
  const double *__restrict__ jac = z.jac;

  auto point_ok = [&](int p, int &px, int &py) {
    py = p / kPX;
    px = p - py * kPX;
    return p < kPX * kPY && i0 - 1 + px <= d.mx && j0 - 1 + py <= d.my;
  };
  // this thread's points of plane k into slot sl (the same points every plane)
  auto request = [&](int k, int sl) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int px, py;
      if (!point_ok(threadIdx.x + r * kFT, px, py)) continue;
      const int64_t id = d.idx(g, i0 - 1 + px, j0 - 1 + py, k);
      cp_async8(&S.dyn[sl][0][py][px], z.bv + id + sz);
      cp_async8(&S.dyn[sl][1][py][px], z.bv + id + 2 * sz);
      cp_async8(&S.dyn[sl][2][py][px], z.bv + id + 3 * sz);
      cp_async8(&S.dyn[sl][3][py][px], z.bv + id + 5 * sz);
      cp_async8(&S.dyn[sl][4][py][px], z.mul + id);
    }
  };
  request(k0 - 1, 0);
  request(k0, 1);
  request(k0 + 1, 2);
  cp_async_commit();
  cp_async_wait_all();
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = i < d.mx && j < d.my;
  double fzp[4] = {0, 0, 0, 0};
  if (three_d && mine) {
    const int64_t ida = d.idx(g, i, j, k0 - 1);
    ring_face<2>(S, met, jac, sz, 0, tx + 1, ty + 1, ida, 1, tx + 1, ty + 1, ida + spl, cp_pr, fzp);
  }
  // the first iteration refills slot 0, which the z faces above read at
  // neighbouring points
  __syncthreads();
  int sp = 0, sc = 1, sn = 2;  // slots of planes k-1, k, k+1
  for (int k = k0; k < k_end; ++k) {
    double acc[4];
    const int64_t iq = d.idx(0, i, j, k);
    if (mine) {
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = z.dq[iq + (q + 1) * szq];
    }
    // k-differences at this thread's points: its own copies of planes k-1
    // and k+1 are complete, and no other thread reads these points of
    // slot sp before the next barrier
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      int px, py;
      if (!point_ok(threadIdx.x + r * kFT, px, py)) continue;
#pragma unroll
      for (int q = 0; q < 4; ++q) S.dzp[q][py][px] = S.dyn[sn][q][py][px] - S.dyn[sp][q][py][px];
    }
    if (k + 2 <= k_end) request(k + 2, sp);  // plane k+2 into the slot of plane k-1
    if (PF && k + 2 <= k_end) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        int px, py;
        if (!point_ok(threadIdx.x + r * kFT, px, py)) continue;
        const int64_t id = d.idx(g, i0 - 1 + px, j0 - 1 + py, k + 2);
#pragma unroll
        for (int m = 0; m < 9; ++m) prefetch_l2(met + id + m * sz);
        prefetch_l2(jac + id);
      }
    }
    cp_async_commit();
    __syncthreads();
    constexpr int kNXF = kFY * (kFX + 1), kNYF = (kFY + 1) * kFX;
    constexpr int kYF0 = (kNXF + 31) / 32 * 32;
    for (int f = threadIdx.x; f < kYF0 + kNYF; f += kFT) {
      if (f < kYF0) {
        if (f >= kNXF) continue;
        const int fy_ = f / (kFX + 1), fx_ = f - fy_ * (kFX + 1);
        if (i0 - 1 + fx_ > d.mx - 1 || j0 + fy_ >= d.my) continue;
        const int64_t ida = d.idx(g, i0 - 1 + fx_, j0 + fy_, k);
        double F[4];
        ring_face<0>(S, met, jac, sz, sc, fx_, fy_ + 1, ida, sc, fx_ + 1, fy_ + 1, ida + 1, cp_pr, F);
#pragma unroll
        for (int q = 0; q < 4; ++q) S.fx[q][fy_][fx_] = F[q];
      } else {
        const int e = f - kYF0;
        const int fy_ = e / kFX, fx_ = e - fy_ * kFX;
        if (i0 + fx_ >= d.mx || j0 - 1 + fy_ > d.my - 1) continue;
        const int64_t ida = d.idx(g, i0 + fx_, j0 - 1 + fy_, k);
        double F[4];
        ring_face<1>(S, met, jac, sz, sc, fx_ + 1, fy_, ida, sc, fx_ + 1, fy_ + 1, ida + srow, cp_pr, F);
#pragma unroll
        for (int q = 0; q < 4; ++q) S.fy[q][fy_][fx_] = F[q];
      }
    }
    double fzn[4] = {0, 0, 0, 0};
    if (three_d && mine) {
      const int64_t ida = d.idx(g, i, j, k);
      ring_face<2>(S, met, jac, sz, sc, tx + 1, ty + 1, ida, sn, tx + 1, ty + 1, ida + spl, cp_pr, fzn);
    }
    cp_async_wait_all();
    __syncthreads();
    if (mine) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        double a = acc[q];
        a += S.fx[q][ty][tx + 1] - S.fx[q][ty][tx];
        a += S.fy[q][ty + 1][tx] - S.fy[q][ty][tx];
        if (three_d) a += fzn[q] - fzp[q];
        z.dq[iq + (q + 1) * szq] = a;
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) fzp[q] = fzn[q];
    const int t = sp;
    sp = sc;
    sc = sn;
    sn = t;
  }
}

// Opt the kernel in to its dynamic shared-memory size (108 KB, two CTAs per SM).
cudaError_t viscous_air_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(viscous_air_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(FusedSmem));
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(viscous_air_ring<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(RingSmem));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(viscous_air_ring<2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(RingSmem));
}

// compute_viscous_flux for air (reference src/ViscousScheme.cu:7-40): one
// launch for all directions; var 0 the staged kernel, 1 the ring kernel,
// 2 the ring kernel with the L2 prefetch of the metric two planes ahead.
cudaError_t launch_viscous_air(const Zone &z, const Param &p, cudaStream_t st, int *n_launch, int var) {
  const Dims &d = z.d;
  const dim3 grid((d.mx + kFX - 1) / kFX, (d.my + kFY - 1) / kFY, (d.mz + kFZ - 1) / kFZ);
  if (var == 1) viscous_air_ring<2, false><<<grid, kFT, sizeof(RingSmem), st>>>(z, p.Pr);
  else if (var == 2) viscous_air_ring<2, true><<<grid, kFT, sizeof(RingSmem), st>>>(z, p.Pr);
  else viscous_air_fused<<<grid, kFT, sizeof(FusedSmem), st>>>(z, p.Pr);
  *n_launch += 1;
  return cudaGetLastError();
}

}  // namespace cfk
