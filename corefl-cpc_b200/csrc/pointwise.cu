// Node-local kernels of the stage: SSP-RK3 update, property update, cv from
// bv, local CFL step with its grid minimum, boundary faces and the 2-D
// k-ghost copy.  All are HBM-bound; each touches a node's planes once.
#include "cfk_common.cuh"
#include "thermo.cuh"
#include "cv_point.cuh"
#include "noise.cuh"

namespace cfk {

// Node index of a thread in a launch that flattens the (i, j) plane of an
// nx x ny block into 1-D thread blocks (grid.y = the k planes), so that rows
// shorter than a thread block do not leave most of its lanes idle.
__device__ __forceinline__ bool flat_ij(int nx, int ny, int &i, int &j) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nx * ny) return false;
  j = t / nx;
  i = t - j * nx;
  return true;
}


// SSP-RK3 coefficients (reference src/RK.cuh:11-15)
__constant__ double kRkA[3] = {1.0, 0.75, 1.0 / 3.0};
__constant__ double kRkB[3] = {0.0, 0.25, 2.0 / 3.0};
__constant__ double kRkC[3] = {1.0, 0.25, 2.0 / 3.0};

// ---------------------------------------------------------------------------
// update_physical_properties (reference src/FieldOperation.cuh:86-120) of one
// node: Sutherland viscosity and Mach number for air; the mixture branch also
// computes the mixture-averaged transport properties (reference
// src/Transport.cu:43-165).
// ---------------------------------------------------------------------------
template <bool MIX>
__device__ __forceinline__ void properties_point(const Zone &z, const Param &p, const Thermo *th, int64_t id) {
  const int64_t sz = z.d.plane(z.d.ngg);
  const double t = z.bv[id + 5 * sz];
  const double V = norm3d(z.bv[id + sz], z.bv[id + 2 * sz], z.bv[id + 3 * sz]);
  if (MIX) {
    mixture_properties_point(z, p, th, id, t, V);
  } else {
    constexpr double c_temp = kGammaAir * kRu / kMwAir;
    z.mul[id] = sutherland(t);
    if (z.mach) z.mach[id] = V / sqrt(c_temp * t);
  }
}

// ---------------------------------------------------------------------------
// update_cv_and_bv_rk (reference src/RK.cuh:224-281).  dt comes from the
// device scalar when dt_dev is non-null (CFL step computed on the device).
// ---------------------------------------------------------------------------
// With minus_cn the right-hand side is dq - Cn: update_cv_and_bv_rk_wu
// (reference src/StrangSplitting.cu:504-562).
// PROPS: the node's physical properties (update_physical_properties, below)
// are computed here from the values just written, so that after the boundary
// conditions only the nodes they can change need the separate pass
// (update_physical_properties_kernel with shell = true).
template <bool MIX, bool PROPS>
__global__ void __launch_bounds__(256) update_cv_and_bv_rk_kernel(Zone z, Param p, const Thermo *th, double dt_host,
                                                                  const double *dt_dev, int rk, int *err,
                                                                  bool minus_cn) {
  const Dims d = z.d;
  int i, j;
  if (!flat_ij(d.mx, d.my, i, j)) return;
  const int k = blockIdx.y;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), szq = d.plane(0);
  const int64_t id = d.idx(g, i, j, k), iq = d.idx(0, i, j, k);
  const double dt = dt_dev ? *dt_dev : dt_host;
  const double a = kRkA[rk], b = kRkB[rk], c = kRkC[rk];
  const double dt_div_jac = dt / z.jac[id];
  double cvl[kMaxVar];
  const int nv = p.n_var;
  auto rhs = [&](int l) { return minus_cn ? z.dq[iq + l * szq] - z.Cn[iq + l * szq] : z.dq[iq + l * szq]; };
#pragma unroll
  for (int l = 0; l < 5; ++l) cvl[l] = a * z.qn[id + l * sz] + b * z.cv[id + l * sz] + c * dt_div_jac * rhs(l);
  if (MIX) {
    for (int l = 5; l < nv; ++l) cvl[l] = a * z.qn[id + l * sz] + b * z.cv[id + l * sz] + c * dt_div_jac * rhs(l);
  }
  if (d.mz == 1) cvl[3] = 0;
  const double rho = cvl[0];
  const double density_inv = 1.0 / rho;
  const double u = cvl[1] * density_inv, v = cvl[2] * density_inv, w = cvl[3] * density_inv;
  z.bv[id] = rho;
  z.bv[id + sz] = u;
  z.bv[id + 2 * sz] = v;
  z.bv[id + 3 * sz] = w;
  const double V2 = u * u + v * v + w * w;
  if (MIX) {
    const int ns = p.n_spec;
    double sum_part_den = 0;
    for (int l = 0; l < ns; ++l) {
      if (cvl[5 + l] < 0) cvl[5 + l] = 0;
      else sum_part_den += cvl[5 + l];
    }
    sum_part_den = 1.0 / sum_part_den;
    const double den_ratio = rho * sum_part_den;
    double yk[kMaxSpec];
    for (int l = 0; l < ns; ++l) {
      yk[l] = cvl[5 + l] * sum_part_den;
      z.sv[id + l * sz] = yk[l];
      cvl[5 + l] *= den_ratio;
    }
    for (int l = ns; l < p.n_scalar; ++l) z.sv[id + l * sz] = cvl[5 + l] * density_inv;
    double T = z.bv[id + 5 * sz];
    double pres;
    if (!temperature_newton(th, ns, yk, cvl[4], rho, V2, T, pres)) atomicOr(err, 1);
    z.bv[id + 4 * sz] = pres;
    z.bv[id + 5 * sz] = T;
  } else {
    const double pres = (kGammaAir - 1) * (cvl[4] - 0.5 * rho * V2);
    z.bv[id + 4 * sz] = pres;
    z.bv[id + 5 * sz] = pres * kMwAir * density_inv / kRu;
  }
  for (int l = 0; l < nv; ++l) z.cv[id + l * sz] = cvl[l];
  if (PROPS) properties_point<MIX>(z, p, th, id);
}

template <bool MIX>
__global__ void cv_from_bv_kernel(Zone z, Param p, const Thermo *th) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j;
  if (!flat_ij(d.mx + 2 * g, d.my + 2 * g, i, j)) return;
  i -= g;
  j -= g;
  const int k = blockIdx.y - g;
  cv_from_bv_point<MIX>(z, p, th, d.idx(g, i, j, k));
}

// ---------------------------------------------------------------------------
// limit_flow (reference src/TimeAdvanceFunc.cuh:117-220) in two passes, so
// that every decision is taken on the values before the call: the first marks
// the interior nodes whose density, velocity or pressure is NaN or outside the
// bounds; the second replaces each marked node's rho, u, v, w, p by the mean
// over the unmarked nodes of its 3 x 3 x 3 interior neighbourhood (k, j, i
// loops from -1 to 1, the reference's order), or clamps them to the bounds
// when there is none, then sets T from the state equation and cv from bv.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool out_of_bounds(const double *bv, int64_t id, int64_t sz, const Param &p) {
  for (int l = 0; l < 5; ++l) {
    const double v = bv[id + l * sz];
    if (isnan(v) || v < p.limit_ll[l] || v > p.limit_ul[l]) return true;
  }
  return false;
}

__global__ void limit_flow_mark_kernel(Zone z, Param p, unsigned char *bad) {
  const Dims d = z.d;
  int i, j;
  if (!flat_ij(d.mx, d.my, i, j)) return;
  const int k = blockIdx.y;
  const int64_t sz = d.plane(d.ngg);
  bad[((int64_t)k * d.my + j) * d.mx + i] = out_of_bounds(z.bv, d.idx(d.ngg, i, j, k), sz, p) ? 1 : 0;
}

template <bool MIX>
__global__ void limit_flow_fix_kernel(Zone z, Param p, const Thermo *th, const unsigned char *bad,
                                      unsigned long long *n_fixed) {
  const Dims d = z.d;
  int i, j;
  if (!flat_ij(d.mx, d.my, i, j)) return;
  const int k = blockIdx.y;
  if (!bad[((int64_t)k * d.my + j) * d.mx + i]) return;
  const int g = d.ngg;
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  double upd[5] = {0, 0, 0, 0, 0};
  int kn = 0;
  for (int ka = -1; ka < 2; ++ka) {
    const int k1 = k + ka;
    if (k1 < 0 || k1 >= d.mz) continue;
    for (int ja = -1; ja < 2; ++ja) {
      const int j1 = j + ja;
      if (j1 < 0 || j1 >= d.my) continue;
      for (int ia = -1; ia < 2; ++ia) {
        const int i1 = i + ia;
        if (i1 < 0 || i1 >= d.mx) continue;
        if (bad[((int64_t)k1 * d.my + j1) * d.mx + i1]) continue;
        const int64_t n1 = d.idx(g, i1, j1, k1);
        for (int l = 0; l < 5; ++l) upd[l] += z.bv[n1 + l * sz];
        ++kn;
      }
    }
  }
  if (kn > 0) {
    const double kn_inv = 1.0 / kn;
    for (int l = 0; l < 5; ++l) upd[l] *= kn_inv;
  } else {
    // fmax(NaN, ll) = ll, as the reference's max(var, ll) gives
    for (int l = 0; l < 5; ++l) upd[l] = fmin(fmax(z.bv[id + l * sz], p.limit_ll[l]), p.limit_ul[l]);
  }
  for (int l = 0; l < 5; ++l) z.bv[id + l * sz] = upd[l];
  if (MIX) {
    double R = 0;
    for (int l = 0; l < p.n_spec; ++l) R += z.sv[id + l * sz] * th->gas_const[l];
    z.bv[id + 5 * sz] = upd[4] / (upd[0] * R);
  } else {
    z.bv[id + 5 * sz] = upd[4] * kMwAir / (upd[0] * kRu);
  }
  cv_from_bv_point<MIX>(z, p, th, id);
  atomicAdd(n_fixed, 1ull);
}

// ---------------------------------------------------------------------------
// update_physical_properties (reference src/FieldOperation.cuh:86-120) over
// the padded block.  The mixture branch also computes the mixture-averaged
// transport properties (reference src/Transport.cu:43-165).
// ---------------------------------------------------------------------------
// planar (2-D blocks, inside the step drivers, after the k-ghost copy): the
// k-ghost planes hold copies of plane k = 0, so their properties are those of
// plane 0 — computed once on plane 0 and copied, instead of 2 ngg + 1 times.
template <bool MIX>
__global__ void update_physical_properties_kernel(Zone z, Param p, const Thermo *th, bool shell, bool planar) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j;
  if (!flat_ij(d.mx + 2 * g, d.my + 2 * g, i, j)) return;
  i -= g;
  j -= g;
  const int k = planar ? 0 : (int)blockIdx.y - g;
  // shell: only the nodes the boundary conditions, the inner-face and halo
  // assignments and the 2-D k-ghost copy can write — the ghost layers and the
  // outermost interior layer; the update computed the others' properties
  const bool inner = i >= 1 && i <= d.mx - 2 && j >= 1 && j <= d.my - 2 &&
                     (d.mz == 1 ? k == 0 : (k >= 1 && k <= d.mz - 2));
  const int64_t id = d.idx(g, i, j, k);
  if (!(shell && inner)) properties_point<MIX>(z, p, th, id);
  if (!planar) return;
  const int64_t sz = d.plane(g), sk = d.stride(g, 2);
  for (int q = -g; q <= g; ++q) {
    if (q == 0) continue;
    const int64_t o = id + q * sk;
    z.mul[o] = z.mul[id];
    if (z.mach) z.mach[o] = z.mach[id];
    if (MIX) {
      z.gamma[o] = z.gamma[id];
      z.acoustic_speed[o] = z.acoustic_speed[id];
      z.thermal_conductivity[o] = z.thermal_conductivity[id];
      for (int l = 0; l < p.n_spec; ++l) z.rho_D[o + l * sz] = z.rho_D[id + l * sz];
    }
  }
}

// ---------------------------------------------------------------------------
// local_time_step (reference src/TimeAdvanceFunc.cuh:28-115) fused with the
// grid minimum of global_time_step (reference src/TimeAdvanceFunc.cu:102-152):
// a warp/CTA min reduction and one atomicMin on the bit pattern (dt > 0, so
// the unsigned order of the bits is the order of the values).
// ---------------------------------------------------------------------------
// with_reaction = false: local_time_step_without_reaction (reference
// src/TimeAdvanceFunc.cu:21-100), the step of Wu's splitting.
template <bool MIX>
// Each CTA walks the planes k = blockIdx.y, + gridDim.y, ... so that the
// grid minimum costs one atomic per CTA of several planes, not per plane.
__global__ void __launch_bounds__(256) local_time_step_kernel(Zone z, Param p, const Thermo *th,
                                                              unsigned long long *dt_min_bits, bool with_reaction) {
  const Dims d = z.d;
  int i, j;
  const bool node = flat_ij(d.mx, d.my, i, j);
  double dt_cta = 1e6;
  for (int k = blockIdx.y; k < d.mz; k += gridDim.y) {
  double dt = 1e6;
  if (node) {
    const int g = d.ngg;
    const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
    const double *mt = z.metric;
    const int dim = d.mz == 1 ? 2 : 3;
    const double grad_xi = norm3d(mt[id], mt[id + sz], mt[id + 2 * sz]);
    const double grad_eta = norm3d(mt[id + 3 * sz], mt[id + 4 * sz], mt[id + 5 * sz]);
    const double grad_zeta = norm3d(mt[id + 6 * sz], mt[id + 7 * sz], mt[id + 8 * sz]);
    const double u = z.bv[id + sz], v = z.bv[id + 2 * sz], w = z.bv[id + 3 * sz];
    const double U = u * mt[id] + v * mt[id + sz] + w * mt[id + 2 * sz];
    const double V = u * mt[id + 3 * sz] + v * mt[id + 4 * sz] + w * mt[id + 5 * sz];
    const double W = u * mt[id + 6 * sz] + v * mt[id + 7 * sz] + w * mt[id + 8 * sz];
    double a;
    if (MIX) a = z.acoustic_speed[id];
    else a = sqrt(kGammaAir * kRAir * z.bv[id + 5 * sz]);
    double msr = max(abs(U) + a * grad_xi, abs(V) + a * grad_eta);
    if (dim == 3) msr = max(msr, abs(W) + a * grad_zeta);
    if (p.viscous_order > 0) {
      double max_length = max(grad_xi, grad_eta);
      if (dim == 3) max_length = max(max_length, grad_zeta);
      const double iRho = 1.0 / z.bv[id];
      double mdv;
      if (MIX) {
        mdv = mixture_max_diffuse_vel(z, p, th, id, iRho);
      } else {
        mdv = max(kGammaAir, 4.0 / 3.0) * iRho;
        mdv *= z.mul[id] / p.Pr;
      }
      msr = max(msr, max_length * max_length * mdv);
    }
    dt = p.cfl / msr;
    if (MIX && with_reaction && p.n_reac > 0) {
      const double reaction_dt = p.cfl * z.reaction_timeScale[id];
      if (reaction_dt > 1e-20 && reaction_dt < 1e-5) dt = min(dt, reaction_dt);
    }
    if (z.dt_local) z.dt_local[d.idx(0, i, j, k)] = dt;
  }
  dt_cta = min(dt_cta, dt);
  }
  double dt = dt_cta;
  for (int o = 16; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  __shared__ double wmin[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wmin[wid] = dt;
  __syncthreads();
  if (wid == 0) {
    dt = lane < (int)(blockDim.x >> 5) ? wmin[lane] : 1e6;
    for (int o = 4; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    if (lane == 0) atomicMin(dt_min_bits, (unsigned long long)__double_as_longlong(dt));
  }
}

__global__ void reset_dt_kernel(unsigned long long *bits) { *bits = (unsigned long long)__double_as_longlong(1e6); }

// ---------------------------------------------------------------------------
// Boundary faces (reference src/BoundCond.cu:2002-2171, 3033-3080), each
// over the face widened by ngg ghosts tangentially (reference
// src/Mesh.cpp:14-31).  One thread per face node.
// ---------------------------------------------------------------------------
struct FaceGeom {
  int face, direction;
  int lo[3], n[3];  // range start and extent per axis
};

__device__ __forceinline__ void face_node(const FaceGeom &fg, int t, int &i, int &j, int &k) {
  const int a = t % fg.n[0], r = t / fg.n[0];
  const int b = r % fg.n[1], c = r / fg.n[1];
  i = fg.lo[0] + a; j = fg.lo[1] + b; k = fg.lo[2] + c;
}

// Work split of a boundary-face kernel.  On i faces the ghost layers of a
// face node are consecutive in memory, so ngg + 1 threads share a node: part
// 0 does the face node's own work, part gg fills ghost layer gg (the ghost
// fills read interior nodes only, never the face node, so the parts are
// independent); the lanes of a warp then cover whole runs of ghost cells
// instead of one cell per row.  On j and k faces one thread does the node and
// all its ghost layers, the lanes running along i.
__device__ __forceinline__ bool face_work(const FaceGeom &fg, int g, int &i, int &j, int &k, int &gg_lo,
                                          int &gg_hi, bool &face_part) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int parts = fg.face == 0 ? g + 1 : 1;
  const int node = t / parts, part = t - node * parts;
  if (node >= fg.n[0] * fg.n[1] * fg.n[2]) return false;
  face_node(fg, node, i, j, k);
  face_part = fg.face != 0 || part == 0;
  gg_lo = fg.face == 0 ? part : 1;
  gg_hi = fg.face == 0 ? part : g;
  if (fg.face == 0 && part == 0) { gg_lo = 1; gg_hi = 0; }
  return true;
}

// apply_outflow (reference src/BoundCond.cu:2065-2188).  Plain outflow: the
// ghost layers copy the face node.  With a back pressure: where the face's
// normal Mach number (gamma from the mixture's cp at the face) is below 1,
// the state at the face is the characteristic one at the back pressure,
// rho_b = rho1 + (p_b - p1)/c1^2, V_b = V1 - (p_b - p1)/(rho1 c1) n from the
// inner node, and the ghosts reflect the inner nodes about it (mass
// fractions about the face's); otherwise the ghosts copy the face state.  The
// face node itself is left as it is, as in the reference, so every thread
// reads only the face node and inner nodes and the i-face split is safe.
template <bool MIX>
__global__ void bc_outflow_kernel(Zone z, Param p, const Thermo *th, FaceGeom fg, cfk_outflow of) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j, k, gg_lo, gg_hi;
  bool face_part;
  if (!face_work(fg, g, i, j, k, gg_lo, gg_hi, face_part)) return;
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  const int64_t s = d.stride(g, fg.face) * fg.direction;
  if (!of.back_pressure_on) {
    for (int gg = gg_lo; gg <= gg_hi; ++gg) {
      const int64_t gi = id + gg * s;
      for (int l = 0; l < 6; ++l) z.bv[gi + l * sz] = z.bv[id + l * sz];
      for (int l = 0; l < p.n_scalar; ++l) z.sv[gi + l * sz] = z.sv[id + l * sz];
      cv_from_bv_point<MIX>(z, p, th, gi);
    }
    return;
  }
  if (gg_lo > gg_hi) return;
  const int mf = 3 * fg.face;
  double nx = z.metric[id + mf * sz], ny = z.metric[id + (mf + 1) * sz], nz = z.metric[id + (mf + 2) * sz];
  const double grad_n_inv = fg.direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= grad_n_inv;
  ny *= grad_n_inv;
  nz *= grad_n_inv;
  double u_b = z.bv[id + sz], v_b = z.bv[id + 2 * sz], w_b = z.bv[id + 3 * sz];
  const double u_face = nx * u_b + ny * v_b + nz * w_b;
  double p_b = z.bv[id + 4 * sz], rho_b = z.bv[id];
  double gamma = kGammaAir;
  double yk_b[kMaxSpec];
  if (MIX) {
    double cpk[kMaxSpec];
    compute_cp(th, z.bv[id + 5 * sz], cpk);
    double cp = 0, R = 0;
    for (int l = 0; l < p.n_spec; ++l) {
      yk_b[l] = z.sv[id + l * sz];
      cp += z.sv[id + l * sz] * cpk[l];
      R += z.sv[id + l * sz] * th->gas_const[l];
    }
    gamma = cp / (cp - R);
  }
  const double a_b = sqrt(gamma * p_b / rho_b);
  const double mach_b = fabs(u_face / a_b);
  if (mach_b < 1) {
    p_b = of.back_pressure;
    const int64_t i1 = id - s;
    const double d1 = z.bv[i1], u1 = z.bv[i1 + sz], v1 = z.bv[i1 + 2 * sz], w1 = z.bv[i1 + 3 * sz];
    const double p1 = z.bv[i1 + 4 * sz];
    gamma = kGammaAir;
    if (MIX) {
      double cpk[kMaxSpec];
      compute_cp(th, z.bv[i1 + 5 * sz], cpk);
      double cp = 0, R = 0;
      for (int l = 0; l < p.n_spec; ++l) {
        cp += z.sv[i1 + l * sz] * cpk[l];
        R += z.sv[i1 + l * sz] * th->gas_const[l];
      }
      gamma = cp / (cp - R);
    }
    const double c1 = sqrt(gamma * p1 / d1);
    const double temp = (p_b - p1) / c1;
    rho_b = d1 + temp / c1;
    u_b = u1 - nx * temp / d1;
    v_b = v1 - ny * temp / d1;
    w_b = w1 - nz * temp / d1;
    for (int gg = gg_lo; gg <= gg_hi; ++gg) {
      const int64_t gi = id + gg * s, ii = id - gg * s;
      const double p_g = 2 * p_b - z.bv[ii + 4 * sz], rho_g = 2 * rho_b - z.bv[ii];
      z.bv[gi] = rho_g;
      z.bv[gi + sz] = 2 * u_b - z.bv[ii + sz];
      z.bv[gi + 2 * sz] = 2 * v_b - z.bv[ii + 2 * sz];
      z.bv[gi + 3 * sz] = 2 * w_b - z.bv[ii + 3 * sz];
      z.bv[gi + 4 * sz] = p_g;
      double R = kRAir;
      if (MIX) {
        R = 0;
        for (int l = 0; l < p.n_spec; ++l) {
          z.sv[gi + l * sz] = 2 * yk_b[l] - z.sv[ii + l * sz];
          R += z.sv[gi + l * sz] * th->gas_const[l];
        }
      }
      z.bv[gi + 5 * sz] = p_g / (rho_g * R);
      cv_from_bv_point<MIX>(z, p, th, gi);
    }
  } else {
    for (int gg = gg_lo; gg <= gg_hi; ++gg) {
      const int64_t gi = id + gg * s;
      z.bv[gi] = rho_b;
      z.bv[gi + sz] = u_b;
      z.bv[gi + 2 * sz] = v_b;
      z.bv[gi + 3 * sz] = w_b;
      z.bv[gi + 4 * sz] = p_b;
      z.bv[gi + 5 * sz] = z.bv[id + 5 * sz];
      for (int l = 0; l < p.n_scalar; ++l) z.sv[gi + l * sz] = z.sv[id + l * sz];
      cv_from_bv_point<MIX>(z, p, th, gi);
    }
  }
}

template <bool MIX>
__global__ void bc_symmetry_kernel(Zone z, Param p, const Thermo *th, FaceGeom fg) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j, k, gg_lo, gg_hi;
  bool face_part;
  if (!face_work(fg, g, i, j, k, gg_lo, gg_hi, face_part)) return;
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  const int64_t s = d.stride(g, fg.face) * fg.direction;
  const int64_t in = id - s;
  const int mf = 3 * fg.face;
  double k_x = z.metric[id + mf * sz], k_y = z.metric[id + (mf + 1) * sz], k_z = z.metric[id + (mf + 2) * sz];
  const double k_magnitude = sqrt(k_x * k_x + k_y * k_y + k_z * k_z);
  k_x /= k_magnitude; k_y /= k_magnitude; k_z /= k_magnitude;
  if (face_part) {
    const double u1 = z.bv[in + sz], v1 = z.bv[in + 2 * sz], w1 = z.bv[in + 3 * sz];
    const double u_k = k_x * u1 + k_y * v1 + k_z * w1;
    z.bv[id + sz] = u1 - k_x * u_k;
    z.bv[id + 2 * sz] = v1 - k_y * u_k;
    z.bv[id + 3 * sz] = w1 - k_z * u_k;
    z.bv[id] = z.bv[in];
    z.bv[id + 4 * sz] = z.bv[in + 4 * sz];
    z.bv[id + 5 * sz] = z.bv[in + 5 * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = z.sv[in + l * sz];
  }
  for (int gg = gg_lo; gg <= gg_hi; ++gg) {
    const int64_t gi = id + gg * s, ii = id - gg * s;
    z.bv[gi] = z.bv[ii];
    const double u = z.bv[ii + sz], v = z.bv[ii + 2 * sz], w = z.bv[ii + 3 * sz];
    const double u_k = k_x * u + k_y * v + k_z * w;
    z.bv[gi + sz] = u - 2 * u_k * k_x;
    z.bv[gi + 2 * sz] = v - 2 * u_k * k_y;
    z.bv[gi + 3 * sz] = w - 2 * u_k * k_z;
    z.bv[gi + 4 * sz] = z.bv[ii + 4 * sz];
    z.bv[gi + 5 * sz] = z.bv[ii + 5 * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gi + l * sz] = z.sv[ii + l * sz];
    cv_from_bv_point<MIX>(z, p, th, gi);
  }
}

template <bool MIX>
__global__ void bc_periodic_kernel(Zone z, Param p, const Thermo *th, FaceGeom fg) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j, k, gg_lo, gg_hi;
  bool face_part;
  if (!face_work(fg, g, i, j, k, gg_lo, gg_hi, face_part)) return;
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  const int64_t sd = d.stride(g, fg.face);
  const int64_t s = sd * fg.direction;
  const int mface = d.ext(fg.face);
  const int64_t io = id + (int64_t)(fg.direction < 0 ? (mface - 1) : -(mface - 1)) * sd;
  if (face_part) {
    for (int l = 0; l < 6; ++l) {
      const double ave = 0.5 * (z.bv[id + l * sz] + z.bv[io + l * sz]);
      z.bv[id + l * sz] = ave;
      z.bv[io + l * sz] = ave;
    }
    for (int l = 0; l < p.n_scalar; ++l) {
      const double ave = 0.5 * (z.sv[id + l * sz] + z.sv[io + l * sz]);
      z.sv[id + l * sz] = ave;
      z.sv[io + l * sz] = ave;
    }
    cv_from_bv_point<MIX>(z, p, th, id);
  }
  for (int gg = gg_lo; gg <= gg_hi; ++gg) {
    const int64_t gi = id + gg * s, ii = io + gg * s;
    for (int l = 0; l < 6; ++l) z.bv[gi + l * sz] = z.bv[ii + l * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gi + l * sz] = z.sv[ii + l * sz];
    cv_from_bv_point<MIX>(z, p, th, gi);
  }
}

// apply_inflow (reference src/BoundCond.cu:2190-2705), constant inflow
// without fluctuations.  The face node takes the inflow state, or — subsonic
// inflow whose normal Mach number, from the face node's current velocity, is
// not below -1 — the characteristic combination of the inflow state and the
// inner node: p = (p1 + p_in - rho1 c1 (V_in - V1).n) / 2, rho = rho_in +
// (p - p_in) / c1^2, V = V_in - (p - p_in) / (rho1 c1) n, T from the state
// equation.  Ghost layer g takes the face values (supersonic) or reflects
// inner node g about them with p and rho held above 0.1 of the face values
// (subsonic).  One thread per face node and its ghost line: the face values
// depend on the face node's values before they are overwritten.
// Index of a face node in its face plane, padded, as the reference numbers
// its per-node random states (src/BoundCond.cu:2485-2496).
__device__ __forceinline__ uint64_t inflow_noise_node(const Dims &d, int face, int i, int j, int k) {
  const int g = d.ngg;
  if (face == 1) return (uint64_t)(k + g) * (d.mx + 2 * g) + (i + g);
  if (face == 2) return (uint64_t)(j + g) * (d.mx + 2 * g) + (i + g);
  return (uint64_t)(k + g) * (d.my + 2 * g) + (j + g);
}

template <bool MIX>
__global__ void bc_inflow_kernel(Zone z, Param p, const Thermo *th, FaceGeom fg, cfk_inflow in) {
  const Dims d = z.d;
  const int g = d.ngg;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= fg.n[0] * fg.n[1] * fg.n[2]) return;
  int i, j, k;
  face_node(fg, t, i, j, k);
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  const int64_t s = d.stride(g, fg.face) * fg.direction;
  double density = in.density, u = in.u, v = in.v, w = in.w, pr = in.pressure, T = in.temperature;
  const double *svb = in.sv;
  if (in.inflow_type == 2) {
    // mixing layer (src/BoundCond.cu:2455-2506)
    const double y = z.y[id];
    u = 0.5 * (in.u + in.u_lower) + 0.5 * (in.u - in.u_lower) * tanh(2 * y / in.delta_omega);
    if (!(y >= 0)) {
      density = in.density_lower;
      v = in.v_lower;
      w = in.w_lower;
      pr = in.p_lower;
      T = in.t_lower;
      svb = in.sv_lower;
    }
    if (in.fluctuation_type == 1) {
      const uint64_t node = inflow_noise_node(d, fg.face, i, j, k), call = *z.inflow_draws;
      const double rms = in.fluctuation_intensity * u * exp(-y * y);
      double n0, n1, n2, n3;
      noise_normal_pair(in.seed, call, node, 0, n0, n1);
      noise_normal_pair(in.seed, call, node, 1, n2, n3);
      u += n0 * rms;
      v += n1 * rms;
      w += n2 * rms;
    }
  } else if (in.subsonic) {
    const int mf = 3 * fg.face;
    double nx = z.metric[id + mf * sz], ny = z.metric[id + (mf + 1) * sz], nz = z.metric[id + (mf + 2) * sz];
    const double grad_n_inv = fg.direction / sqrt(nx * nx + ny * ny + nz * nz);
    nx *= grad_n_inv;
    ny *= grad_n_inv;
    nz *= grad_n_inv;
    const double c0 = MIX ? z.acoustic_speed[id] : sqrt(kGammaAir * kRAir * z.bv[id + 5 * sz]);
    const double Mn = (z.bv[id + sz] * nx + z.bv[id + 2 * sz] * ny + z.bv[id + 3 * sz] * nz) / c0;
    if (!(Mn < -1.0)) {
      const int64_t i1 = id - s;
      const double c1 = MIX ? z.acoustic_speed[i1] : sqrt(kGammaAir * kRAir * z.bv[i1 + 5 * sz]);
      const double rho1 = z.bv[i1], p1 = z.bv[i1 + 4 * sz];
      pr = 0.5 * (p1 + in.pressure - rho1 * c1 * ((in.u - z.bv[i1 + sz]) * nx + (in.v - z.bv[i1 + 2 * sz]) * ny +
                                                  (in.w - z.bv[i1 + 3 * sz]) * nz));
      density = in.density + (pr - in.pressure) / (c1 * c1);
      u = in.u - (pr - in.pressure) / (rho1 * c1) * nx;
      v = in.v - (pr - in.pressure) / (rho1 * c1) * ny;
      w = in.w - (pr - in.pressure) / (rho1 * c1) * nz;
      T = MIX ? pr * in.mw / (density * kRu) : pr / (density * kRAir);
    }
  } else if (in.fluctuation_type == 1) {
    // white noise on u of a constant inflow (src/BoundCond.cu:2573-2596)
    const uint64_t node = inflow_noise_node(d, fg.face, i, j, k), call = *z.inflow_draws;
    double n0, n1;
    noise_normal_pair(in.seed, call, node, 0, n0, n1);
    u += n0 * in.fluctuation_intensity * sqrt(in.u * in.u + in.v * in.v + in.w * in.w);
  }
  z.bv[id] = density;
  z.bv[id + sz] = u;
  z.bv[id + 2 * sz] = v;
  z.bv[id + 3 * sz] = w;
  z.bv[id + 4 * sz] = pr;
  z.bv[id + 5 * sz] = T;
  for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = svb[l];
  cv_from_bv_point<MIX>(z, p, th, id);
  for (int gg = 1; gg <= g; ++gg) {
    const int64_t gi = id + gg * s;
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gi + l * sz] = svb[l];
    if (in.subsonic) {
      const int64_t ii = id - gg * s;
      double rho2 = 2 * density - z.bv[ii], p2 = 2 * pr - z.bv[ii + 4 * sz];
      if (p2 <= 0.1 * pr) p2 = 0.1 * pr;
      if (rho2 <= 0.1 * density) rho2 = 0.1 * density;
      z.bv[gi] = rho2;
      z.bv[gi + sz] = 2 * u - z.bv[ii + sz];
      z.bv[gi + 2 * sz] = 2 * v - z.bv[ii + 2 * sz];
      z.bv[gi + 3 * sz] = 2 * w - z.bv[ii + 3 * sz];
      z.bv[gi + 4 * sz] = p2;
      z.bv[gi + 5 * sz] = MIX ? p2 * in.mw / (rho2 * kRu) : p2 / (rho2 * kRAir);
    } else {
      z.bv[gi] = density;
      z.bv[gi + sz] = u;
      z.bv[gi + 2 * sz] = v;
      z.bv[gi + 3 * sz] = w;
      z.bv[gi + 4 * sz] = pr;
      z.bv[gi + 5 * sz] = T;
    }
    cv_from_bv_point<MIX>(z, p, th, gi);
  }
}

// One more application of the fluctuating inflow: the next one draws new deviates.
__global__ void inflow_draw_advance_kernel(unsigned long long *draws) { *draws += 1; }

// apply_wall (reference src/BoundCond.cu:2761-3031) without its jet,
// shock-blowing and wall-fluctuation branches (so v_blow = 0).  The face node
// takes zero velocity, its inner neighbour's pressure, the wall temperature
// (isothermal) or the inner neighbour's temperature (adiabatic), the inner
// neighbour's mass fractions (non-catalytic) or the wall's (catalytic) and
// rho = p / (R T).  Ghost layer gg mirrors inner node gg: velocity reversed,
// pressure copied, temperature copied (adiabatic) or reflected about the wall
// temperature, T_g = 2 T_w - T_i, replaced by T_w at or below 0.1 T_w
// (isothermal).  A catalytic ghost's gas constant is the wall's, summed from
// yk in the order the reference sums the face node's fractions, so the ghost
// parts never read the face node that part 0 writes.
template <bool MIX>
__global__ void bc_wall_kernel(Zone z, Param p, const Thermo *th, FaceGeom fg, cfk_wall wall) {
  const Dims d = z.d;
  const int g = d.ngg;
  int i, j, k, gg_lo, gg_hi;
  bool face_part;
  if (!face_work(fg, g, i, j, k, gg_lo, gg_hi, face_part)) return;
  const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
  const int64_t s = d.stride(g, fg.face) * fg.direction;
  const bool isothermal = wall.thermal_type == 0;
  const bool catalytic = MIX && wall.catalytic_type == 1;
  if (face_part) {
    const int64_t in = id - s;
    const double t_wall = isothermal ? wall.temperature : z.bv[in + 5 * sz];
    const double pw = z.bv[in + 4 * sz];
    double R = kRAir;
    if (MIX) {
      R = 0;
      for (int l = 0; l < p.n_spec; ++l) {
        const double y = catalytic ? wall.yk[l] : z.sv[in + l * sz];
        z.sv[id + l * sz] = y;
        R += y * th->gas_const[l];
      }
    }
    z.bv[id] = pw / (t_wall * R);
    z.bv[id + sz] = 0;
    z.bv[id + 2 * sz] = 0;
    z.bv[id + 3 * sz] = 0;
    z.bv[id + 4 * sz] = pw;
    z.bv[id + 5 * sz] = t_wall;
    cv_from_bv_point<MIX>(z, p, th, id);
  }
  const double v_blow = 0;
  for (int gg = gg_lo; gg <= gg_hi; ++gg) {
    const int64_t gi = id + gg * s, ii = id - gg * s;
    const double p_i = z.bv[ii + 4 * sz], t_i = z.bv[ii + 5 * sz];
    double t_g = t_i;
    if (isothermal) {
      t_g = 2 * wall.temperature - t_i;
      if (t_g <= 0.1 * wall.temperature) t_g = wall.temperature;
    }
    double R = kRAir;
    if (MIX) {
      R = 0;
      for (int l = 0; l < p.n_spec; ++l) {
        const double y = catalytic ? wall.yk[l] : z.sv[ii + l * sz];
        z.sv[gi + l * sz] = y;
        R += y * th->gas_const[l];
      }
    }
    z.bv[gi] = p_i / (t_g * R);
    z.bv[gi + sz] = -z.bv[ii + sz];
    z.bv[gi + 2 * sz] = v_blow * 2 - z.bv[ii + 2 * sz];
    z.bv[gi + 3 * sz] = -z.bv[ii + 3 * sz];
    z.bv[gi + 4 * sz] = p_i;
    z.bv[gi + 5 * sz] = t_g;
    cv_from_bv_point<MIX>(z, p, th, gi);
  }
}

// inner_communication (reference src/DataCommunication.cu:36-102): one thread
// per node of the face's loop (face node + ghost layers along the normal, the
// face's own nodes across it).  Ghost nodes take the target block's primitive
// variables.  A face node moving faster than 1e-15 is averaged with the
// target's face node, both sides written, or takes the target's values when
// the target node is at rest (a wall on the other side); a face node at rest
// is left as it is.  This block's cv is recomputed at every visited node.
// Threads write distinct nodes: ghost reads touch target nodes behind the
// target face (at least one layer in, never a face node) and the host checks
// that both blocks are thicker than ngg along the face normal.
template <bool MIX>
__global__ void inner_face_kernel(Zone z, Zone tz, Param p, const Thermo *th, cfk_inner_face f, int n_total) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_total) return;
  const int r = t / f.n_point[0];
  const int n[3] = {t - r * f.n_point[0], r % f.n_point[1], r / f.n_point[1]};
  int idx[3], d_idx[3], idt[3];
  for (int a = 0; a < 3; ++a) {
    d_idx[a] = f.loop_dir[a] * n[a];
    idx[a] = f.range_start[a] + d_idx[a];
  }
  for (int a = 0; a < 3; ++a) idt[a] = f.target_start[a] + f.target_loop_dir[a] * d_idx[f.src_tar[a]];
  const int g = z.d.ngg;
  const int64_t sz = z.d.plane(g), tsz = tz.d.plane(g);
  const int64_t id = z.d.idx(g, idx[0], idx[1], idx[2]), it = tz.d.idx(g, idt[0], idt[1], idt[2]);
  const int face_node = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
  if (idx[f.face] == face_node) {
    const double u_this = norm3d(z.bv[id + sz], z.bv[id + 2 * sz], z.bv[id + 3 * sz]);
    if (fabs(u_this) > 1e-15) {
      const double u_that = norm3d(tz.bv[it + tsz], tz.bv[it + 2 * tsz], tz.bv[it + 3 * tsz]);
      if (fabs(u_that) < 1e-15) {
        for (int l = 0; l < 6; ++l) z.bv[id + l * sz] = tz.bv[it + l * tsz];
        for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = tz.sv[it + l * tsz];
      } else {
        for (int l = 0; l < 6; ++l) {
          const double ave = 0.5 * (tz.bv[it + l * tsz] + z.bv[id + l * sz]);
          z.bv[id + l * sz] = ave;
          tz.bv[it + l * tsz] = ave;
        }
        for (int l = 0; l < p.n_scalar; ++l) {
          const double ave = 0.5 * (tz.sv[it + l * tsz] + z.sv[id + l * sz]);
          z.sv[id + l * sz] = ave;
          tz.sv[it + l * tsz] = ave;
        }
      }
    }
  } else {
    for (int l = 0; l < 6; ++l) z.bv[id + l * sz] = tz.bv[it + l * tsz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = tz.sv[it + l * tsz];
  }
  cv_from_bv_point<MIX>(z, p, th, id);
}

// eliminate_k_gradient (reference src/FieldOperation.cu:47-72)
__global__ void eliminate_k_gradient_kernel(Zone z, Param p) {
  const Dims d = z.d;
  const int g = d.ngg;
  const int i = blockIdx.x * blockDim.x + threadIdx.x - g;
  const int j = blockIdx.y - g;
  if (i >= d.mx + g) return;
  const int64_t sz = d.plane(g), i0 = d.idx(g, i, j, 0);
  for (int k = 1; k <= g; ++k) {
    const int64_t ip = d.idx(g, i, j, k), im = d.idx(g, i, j, -k);
    for (int l = 0; l < 6; ++l) { z.bv[ip + l * sz] = z.bv[i0 + l * sz]; z.bv[im + l * sz] = z.bv[i0 + l * sz]; }
    for (int l = 0; l < p.n_scalar; ++l) { z.sv[ip + l * sz] = z.sv[i0 + l * sz]; z.sv[im + l * sz] = z.sv[i0 + l * sz]; }
    for (int l = 0; l < p.n_var; ++l) { z.cv[ip + l * sz] = z.cv[i0 + l * sz]; z.cv[im + l * sz] = z.cv[i0 + l * sz]; }
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// grids for flat_ij: the (i, j) plane flattened along x, one k plane per grid.y
static dim3 interior_grid(const Dims &d, int tpb) {
  return dim3((unsigned)(((int64_t)d.mx * d.my + tpb - 1) / tpb), d.mz);
}
static dim3 padded_grid(const Dims &d, int tpb) {
  return dim3((unsigned)(((int64_t)(d.mx + 2 * d.ngg) * (d.my + 2 * d.ngg) + tpb - 1) / tpb), d.mz + 2 * d.ngg);
}

cudaError_t launch_update_rk(const Zone &z, const Param &p, const Thermo *th, double dt, const double *dt_dev,
                             int rk, int *err, cudaStream_t st, bool minus_cn, bool with_props) {
  const dim3 grid = interior_grid(z.d, 128);
  if (p.n_spec > 0) {
    if (with_props) update_cv_and_bv_rk_kernel<true, true><<<grid, 128, 0, st>>>(z, p, th, dt, dt_dev, rk, err, minus_cn);
    else update_cv_and_bv_rk_kernel<true, false><<<grid, 128, 0, st>>>(z, p, th, dt, dt_dev, rk, err, minus_cn);
  } else {
    if (with_props) update_cv_and_bv_rk_kernel<false, true><<<grid, 128, 0, st>>>(z, p, th, dt, dt_dev, rk, err, minus_cn);
    else update_cv_and_bv_rk_kernel<false, false><<<grid, 128, 0, st>>>(z, p, th, dt, dt_dev, rk, err, minus_cn);
  }
  return cudaGetLastError();
}

cudaError_t launch_limit_flow(const Zone &z, const Param &p, const Thermo *th, unsigned char *bad,
                              unsigned long long *n_fixed, cudaStream_t st) {
  limit_flow_mark_kernel<<<interior_grid(z.d, 256), 256, 0, st>>>(z, p, bad);
  if (p.n_spec > 0) limit_flow_fix_kernel<true><<<interior_grid(z.d, 256), 256, 0, st>>>(z, p, th, bad, n_fixed);
  else limit_flow_fix_kernel<false><<<interior_grid(z.d, 256), 256, 0, st>>>(z, p, th, bad, n_fixed);
  return cudaGetLastError();
}

cudaError_t launch_cv_from_bv(const Zone &z, const Param &p, const Thermo *th, cudaStream_t st) {
  if (p.n_spec > 0) cv_from_bv_kernel<true><<<padded_grid(z.d, 128), 128, 0, st>>>(z, p, th);
  else cv_from_bv_kernel<false><<<padded_grid(z.d, 128), 128, 0, st>>>(z, p, th);
  return cudaGetLastError();
}

cudaError_t launch_update_properties(const Zone &z, const Param &p, const Thermo *th, cudaStream_t st, bool shell,
                                     bool planar) {
  dim3 grid = padded_grid(z.d, 128);
  planar = planar && z.d.mz == 1;
  if (planar) grid.y = 1;
  if (p.n_spec > 0) update_physical_properties_kernel<true><<<grid, 128, 0, st>>>(z, p, th, shell, planar);
  else update_physical_properties_kernel<false><<<grid, 128, 0, st>>>(z, p, th, shell, planar);
  return cudaGetLastError();
}

cudaError_t launch_local_dt(const Zone &z, const Param &p, const Thermo *th, unsigned long long *dt_bits,
                            cudaStream_t st, bool with_reaction) {
  reset_dt_kernel<<<1, 1, 0, st>>>(dt_bits);
  dim3 grid = interior_grid(z.d, 256);
  grid.y = grid.y < 16 ? grid.y : 16;  // planes per CTA: ceil(mz / 16)
  if (p.n_spec > 0)
    local_time_step_kernel<true><<<grid, 256, 0, st>>>(z, p, th, dt_bits, with_reaction);
  else
    local_time_step_kernel<false><<<grid, 256, 0, st>>>(z, p, th, dt_bits, with_reaction);
  return cudaGetLastError();
}

// A face's node range: its tangential extent widened by ngg ghosts only with
// the 2nd-order viscous scheme, as the reference registers its boundaries
// (src/Mesh.cpp:14-31, 637: need_extend_boundary = viscous_order == 2); for a
// 2-D block the k range is then [-ngg, ngg], else [0, 0].
static FaceGeom make_face(const Dims &d, const cfk_face &f, int viscous_order) {
  const int g = viscous_order == 2 ? d.ngg : 0;
  FaceGeom fg;
  fg.face = f.face;
  fg.direction = f.direction;
  const int m[3] = {d.mx, d.my, d.mz};
  for (int a = 0; a < 3; ++a) {
    if (a == f.face) {
      fg.lo[a] = f.direction < 0 ? 0 : m[a] - 1;
      fg.n[a] = 1;
    } else {
      fg.lo[a] = -g;
      fg.n[a] = m[a] + 2 * g;
    }
  }
  if (d.mz == 1) { fg.lo[2] = -g; fg.n[2] = 2 * g + 1; }
  return fg;
}

cudaError_t launch_boundary_conditions(const Zone &z, const Param &p, const Thermo *th, const cfk_face *faces,
                                       int n_face, const cfk_wall &wall, const cfk_inflow &inflow,
                                       const cfk_outflow &outflow, cudaStream_t st, int *n_launch) {
  // reference priority order: outflow, inflow, symmetry, wall, periodic
  static const int order[5] = {6, 5, 3, 2, 8};
  for (int o = 0; o < 5; ++o) {
    for (int n = 0; n < n_face; ++n) {
      if (faces[n].label != order[o]) continue;
      const FaceGeom fg = make_face(z.d, faces[n], p.viscous_order);
      const bool split = order[o] != 5;  // the inflow kernel keeps a face node's line in one thread
      const int cnt = fg.n[0] * fg.n[1] * fg.n[2] * (split && fg.face == 0 ? z.d.ngg + 1 : 1);
      const int blocks = (cnt + 127) / 128;
      const bool mix = p.n_spec > 0;
      if (order[o] == 6) {
        if (mix) bc_outflow_kernel<true><<<blocks, 128, 0, st>>>(z, p, th, fg, outflow);
        else bc_outflow_kernel<false><<<blocks, 128, 0, st>>>(z, p, th, fg, outflow);
      } else if (order[o] == 3) {
        if (mix) bc_symmetry_kernel<true><<<blocks, 128, 0, st>>>(z, p, th, fg);
        else bc_symmetry_kernel<false><<<blocks, 128, 0, st>>>(z, p, th, fg);
      } else if (order[o] == 5) {
        if (mix) bc_inflow_kernel<true><<<blocks, 128, 0, st>>>(z, p, th, fg, inflow);
        else bc_inflow_kernel<false><<<blocks, 128, 0, st>>>(z, p, th, fg, inflow);
        if (inflow.fluctuation_type == 1) {
          inflow_draw_advance_kernel<<<1, 1, 0, st>>>(z.inflow_draws);
          ++*n_launch;
        }
      } else if (order[o] == 2) {
        if (mix) bc_wall_kernel<true><<<blocks, 128, 0, st>>>(z, p, th, fg, wall);
        else bc_wall_kernel<false><<<blocks, 128, 0, st>>>(z, p, th, fg, wall);
      } else {
        if (mix) bc_periodic_kernel<true><<<blocks, 128, 0, st>>>(z, p, th, fg);
        else bc_periodic_kernel<false><<<blocks, 128, 0, st>>>(z, p, th, fg);
      }
      ++*n_launch;
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
    }
  }
  if (z.d.mz == 1) {
    eliminate_k_gradient_kernel<<<dim3((z.d.mx + 2 * z.d.ngg + 127) / 128, z.d.my + 2 * z.d.ngg), 128, 0, st>>>(z, p);
    ++*n_launch;
  }
  return cudaGetLastError();
}

cudaError_t launch_eliminate_k_gradient(const Zone &z, const Param &p, cudaStream_t st) {
  eliminate_k_gradient_kernel<<<dim3((z.d.mx + 2 * z.d.ngg + 127) / 128, z.d.my + 2 * z.d.ngg), 128, 0, st>>>(z, p);
  return cudaGetLastError();
}

cudaError_t launch_inner_communication(const Zone &z, const Zone &tz, const Param &p, const Thermo *th,
                                       const cfk_inner_face &f, cudaStream_t st) {
  const int n_total = f.n_point[0] * f.n_point[1] * f.n_point[2];
  const int blocks = (n_total + 127) / 128;
  if (p.n_spec > 0) inner_face_kernel<true><<<blocks, 128, 0, st>>>(z, tz, p, th, f, n_total);
  else inner_face_kernel<false><<<blocks, 128, 0, st>>>(z, tz, p, th, f, n_total);
  return cudaGetLastError();
}

}  // namespace cfk
