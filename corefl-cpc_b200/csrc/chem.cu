// Chemistry kernels: the explicit finite-rate source of the RK3 path and the
// substepped 0-D reaction step of Wu's splitting (explicit or point
// implicit), the latter in two schedules — one thread per node, and a
// persistent work-queue kernel for nodes with uneven substep counts.
#include "cfk_common.cuh"
#include "chem.cuh"
#include "chem_fast.cuh"
#include "thermo.cuh"

namespace cfk {

constexpr int kMaxSubsteps = 100000;

// ---------------------------------------------------------------------------
// finite_rate_chemistry (reference src/FiniteRateChem.cu:1388-1464), explicit
// treatment: dq[5+l] += J * omega_l; reaction time scale = min rhoY/omega_d.
// The rates are evaluated in an out-of-line call: with nvcc 12.9 for sm_100a
// the fully inlined form of this kernel returned wrong sources (NaN/1e24 on
// the parity test's inputs) while the out-of-line form matches the oracle.
// ---------------------------------------------------------------------------
__device__ __noinline__ void sources_at(const Mech *mc, double T, const double *c, double *omega, double *omega_d) {
  double q1[kMaxReac], q2[kMaxReac];
  rates_of_progress(mc, T, c, q1, q2);
  species_sources(mc, q1, q2, omega, omega_d);
}

__global__ void __launch_bounds__(128) finite_rate_chemistry_kernel(Zone z, const Mech *mc) {
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= d.mx) return;
  const int g = d.ngg, ns = mc->th.n_spec;
  const int64_t sz = d.plane(g), szq = d.plane(0), id = d.idx(g, i, j, k), iq = d.idx(0, i, j, k);
  const double density = z.bv[id];
  double c[kMaxSpec];
  for (int l = 0; l < ns; ++l) c[l] = density * z.sv[id + l * sz] * mc->th.imw[l] * 1e-3;
  double omega[kMaxSpec], omega_d[kMaxSpec];
  sources_at(mc, z.bv[id + 5 * sz], c, omega, omega_d);
  double time_scale = 1e6;
  const double jac = z.jac[id];
  for (int l = 0; l < ns; ++l) {
    z.dq[iq + (l + 5) * szq] += jac * omega[l];
    const double y = z.sv[id + l * sz];
    if (y > 1e-25 && abs(omega_d[l]) > 1e-25) time_scale = min(time_scale, abs(density * y / omega_d[l]));
  }
  z.reaction_timeScale[id] = time_scale;
}

// ---------------------------------------------------------------------------
// One node of the Wu reaction step.  State in registers across substeps:
// cv[0..4], rhoY[ns], T; written back once at the end.
// ---------------------------------------------------------------------------
struct NodeState {
  double q[5];
  double rY[kMaxSpec];
  double T;
  double cn[5], cnY[kMaxSpec];
  double iJac;
  double ts;  // reaction time scale
};

__device__ __forceinline__ void load_node(const Zone &z, int ns, int64_t id, int64_t iq, NodeState &s) {
  const int64_t sz = z.d.plane(z.d.ngg), szq = z.d.plane(0);
#pragma unroll
  for (int l = 0; l < 5; ++l) s.q[l] = z.cv[id + l * sz];
  for (int l = 0; l < ns; ++l) s.rY[l] = z.cv[id + (5 + l) * sz];
  s.T = z.bv[id + 5 * sz];
  if (z.Cn) {
#pragma unroll
    for (int l = 0; l < 5; ++l) s.cn[l] = z.Cn[iq + l * szq];
    for (int l = 0; l < ns; ++l) s.cnY[l] = z.Cn[iq + (5 + l) * szq];
  } else {
#pragma unroll
    for (int l = 0; l < 5; ++l) s.cn[l] = 0;
    for (int l = 0; l < ns; ++l) s.cnY[l] = 0;
  }
  s.iJac = 1.0 / z.jac[id];
  s.ts = z.reaction_timeScale[id];
}

__device__ __forceinline__ void store_node(const Zone &z, const Param &p, int ns, int64_t id, const NodeState &s,
                                           const double *yk, double pres) {
  const int64_t sz = z.d.plane(z.d.ngg);
#pragma unroll
  for (int l = 0; l < 5; ++l) z.cv[id + l * sz] = s.q[l];
  for (int l = 0; l < ns; ++l) {
    z.cv[id + (5 + l) * sz] = s.rY[l];
    z.sv[id + l * sz] = yk[l];
  }
  const double rho_inv = 1.0 / s.q[0];
  for (int l = ns; l < p.n_scalar; ++l) z.sv[id + l * sz] = z.cv[id + (5 + l) * sz] * rho_inv;
  z.bv[id] = s.q[0];
  z.bv[id + sz] = s.q[1] * rho_inv;
  z.bv[id + 2 * sz] = s.q[2] * rho_inv;
  z.bv[id + 3 * sz] = s.q[3] * rho_inv;
  z.bv[id + 4 * sz] = pres;
  z.bv[id + 5 * sz] = s.T;
  z.reaction_timeScale[id] = s.ts;
}

// wu_zeroDReaction (reference src/StrangSplitting.cu:43-224), methods 0 and 1.
// yk and pres receive the mass fractions and pressure after the substep.
__device__ __forceinline__ bool zero_d_substep(const Mech *mc, int method, double dt, NodeState &s, double *yk,
                                               double &pres) {
  const Thermo *th = &mc->th;
  const Kinetics &kn = mc->kn;
  const int ns = th->n_spec;
  double c[kMaxSpec];
  for (int l = 0; l < ns; ++l) c[l] = s.rY[l] * th->imw[l] * 1e-3;
  double q1[kMaxReac], q2[kMaxReac], omega[kMaxSpec], omega_d[kMaxSpec];
  rates_of_progress(mc, s.T, c, q1, q2);
  species_sources(mc, q1, q2, omega, omega_d);
  for (int l = 0; l < ns; ++l) c[l] *= 1e+3 / th->imw[l];
  if (method == 1) {
    double jac[kMaxSpec * kMaxSpec];
    for (int a = 0; a < ns * ns; ++a) jac[a] = 0;
    for (int r = 0; r < kn.n_reac; ++r)
      for (int qa = 0; qa < kn.n_inv[r]; ++qa) {
        const double net = kn.inv_b[r][qa] - kn.inv_f[r][qa];
        if (net == 0) continue;
        const int m = kn.inv_sp[r][qa];
        for (int qb = 0; qb < kn.n_inv[r]; ++qb) {
          const int n = kn.inv_sp[r][qb];
          jac[m * ns + n] += net * (kn.inv_f[r][qb] * q1[r] - kn.inv_b[r][qb] * q2[r]);
        }
      }
    for (int m = 0; m < ns; ++m)
      for (int n = 0; n < ns; ++n) {
        const double rhoY = c[n];
        const double zz = rhoY > 1e-25 ? jac[m * ns + n] / rhoY : 0.0;
        jac[m * ns + n] = (m == n ? 1 : 0) - dt * (zz * 1e+3 / th->imw[m]);
      }
    solve_chem_system(jac, omega, ns);
  }
#pragma unroll
  for (int l = 0; l < 5; ++l) s.q[l] += s.cn[l] * dt * s.iJac;
  double time_scale = 1e6;
  for (int l = 0; l < ns; ++l) {
    if (s.rY[l] > 1e-25 && abs(omega_d[l]) > 1e-25) time_scale = min(time_scale, abs(s.rY[l] / omega_d[l]));
    s.rY[l] += (omega[l] + s.cnY[l] * s.iJac) * dt;
  }
  s.ts = time_scale;
  const double rho = s.q[0];
  const double rho_inv = 1.0 / rho;
  const double u = s.q[1] * rho_inv, v = s.q[2] * rho_inv, w = s.q[3] * rho_inv;
  double sum = 0;
  for (int l = 0; l < ns; ++l) {
    if (s.rY[l] < 0) s.rY[l] = 0;
    else sum += s.rY[l];
  }
  sum = 1.0 / sum;
  const double ratio = rho * sum;
  for (int l = 0; l < ns; ++l) {
    yk[l] = s.rY[l] * sum;
    s.rY[l] *= ratio;
  }
  return temperature_newton(th, ns, yk, s.q[4], rho, u * u + v * v + w * w, s.T, pres);
}

// Substep plan of wu_reaction_step (reference src/StrangSplitting.cu:392-420).
__device__ __forceinline__ void substep_plan(double dt, double ts, int &n_sub, double &h, double &h_last,
                                             bool &capped) {
  if (ts < 1e-15) ts = 0.2 * dt;
  const double nd = dt / ts;
  capped = nd >= (double)kMaxSubsteps;
  n_sub = capped ? kMaxSubsteps : (int)nd;
  h = dt / (n_sub + 1);
  h_last = dt - h * n_sub;
}

__global__ void __launch_bounds__(128) wu_reaction_plain_kernel(Zone z, Param p, const Mech *mc, double dt,
                                                                int *nsub_out, int *err) {
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= d.mx) return;
  const int ns = mc->th.n_spec;
  const int64_t id = d.idx(d.ngg, i, j, k), iq = d.idx(0, i, j, k);
  NodeState s;
  load_node(z, ns, id, iq, s);
  int n_sub;
  double h, h_last;
  bool capped;
  substep_plan(dt, s.ts, n_sub, h, h_last, capped);
  if (capped) atomicOr(err, 2);
  double yk[kMaxSpec], pres = z.bv[id + 4 * z.d.plane(d.ngg)];
  for (int l = 0; l < ns; ++l) yk[l] = z.sv[id + l * z.d.plane(d.ngg)];
  bool ok = true;
  for (int n = 0; n < n_sub; ++n) ok &= zero_d_substep(mc, p.chem_advance_method, h, s, yk, pres);
  int taken = n_sub;
  if (abs(h_last) > 1e-12) {
    ok &= zero_d_substep(mc, p.chem_advance_method, h_last, s, yk, pres);
    ++taken;
  }
  if (!ok) atomicOr(err, 1);
  store_node(z, p, ns, id, s, yk, pres);
  if (nsub_out) nsub_out[iq] = taken;
}

// Persistent work queue.  Every lane owns one node at a time and runs one
// substep per loop trip; a lane whose node is finished writes it back and
// takes the next node index from a global counter (one atomicAdd per warp,
// shared out with a prefix over the lanes that need work).  All lanes of a
// warp execute the same substep code in every trip, whatever substep their
// node is at, so nodes with many substeps do not leave the rest of the warp
// idle.  The loop ends when the counter passes the node count.  With a node
// list, the queue runs over list[0 .. *list_count) instead of all nodes.
__global__ void __launch_bounds__(128) wu_reaction_queue_kernel(Zone z, Param p, const Mech *mc, double dt,
                                                                int *nsub_out, int *err, unsigned int *counter,
                                                                const unsigned int *list,
                                                                const unsigned int *list_count) {
  const Dims d = z.d;
  const int ns = mc->th.n_spec;
  const unsigned int total = list ? *list_count : (unsigned int)d.mx * d.my * d.mz;
  const int64_t szp = d.plane(d.ngg);
  const int lane = threadIdx.x & 31;
  NodeState s;
  double yk[kMaxSpec], pres = 0, h = 0, h_last = 0;
  int n_sub = 0, done = 0, taken = 0;
  unsigned int node = 0xffffffffu;
  int64_t id = 0, iq = 0;
  bool ok = true, have = false, exhausted = false;
  for (;;) {
    // lanes without a node take one (until the queue has run dry for them)
    const bool need = !have && !exhausted;
    const unsigned int mask = __ballot_sync(0xffffffffu, need);
    if (mask) {
      unsigned int base = 0;
      const int leader = __ffs(mask) - 1;
      if (lane == leader) base = atomicAdd(counter, (unsigned int)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        node = base + __popc(mask & ((1u << lane) - 1));
        if (node < total) {
          if (list) node = list[node];
          const int i = node % d.mx, rem = node / d.mx, j = rem % d.my, k = rem / d.my;
          id = d.idx(d.ngg, i, j, k);
          iq = d.idx(0, i, j, k);
          load_node(z, ns, id, iq, s);
          for (int l = 0; l < ns; ++l) yk[l] = z.sv[id + l * szp];
          pres = z.bv[id + 4 * szp];
          bool capped;
          substep_plan(dt, s.ts, n_sub, h, h_last, capped);
          if (capped) atomicOr(err, 2);
          done = 0;
          taken = 0;
          ok = true;
          have = true;
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, have)) break;
    if (have) {
      // substeps 0..n_sub-1 use h, the last one h_last (skipped if ~0)
      double hh = done < n_sub ? h : h_last;
      const bool run = done < n_sub || abs(h_last) > 1e-12;
      if (run) {
        ok &= zero_d_substep(mc, p.chem_advance_method, hh, s, yk, pres);
        ++taken;
      }
      ++done;
      if (done > n_sub) {
        if (!ok) atomicOr(err, 1);
        store_node(z, p, ns, id, s, yk, pres);
        if (nsub_out) nsub_out[iq] = taken;
        have = false;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Compile-time species count (NS = 9, the bundled H2 mechanisms): the same
// two schedules over zero_d_substep_ns, with each lane's NS x NS system in
// shared memory.
// ---------------------------------------------------------------------------
constexpr int kFastBlock = 64;

template <int NS>
__host__ __device__ constexpr int fast_smem_bytes() { return (NS * NS + NS) * kFastBlock * (int)sizeof(double); }

template <int NS>
__global__ void __launch_bounds__(kFastBlock) wu_reaction_plain_ns_kernel(Zone z, Param p,
                                                                         const __grid_constant__ Mech mech, double dt,
                                                                         int *nsub_out, int *err) {
  const Mech *mc = &mech;
  extern __shared__ double sys[];
  const LaneSlot L{sys + threadIdx.x, kFastBlock}, R{sys + NS * NS * kFastBlock + threadIdx.x, kFastBlock};
  const Dims d = z.d;
  const long long q = (long long)blockIdx.x * kFastBlock + threadIdx.x;
  if (q >= (long long)d.mx * d.my * d.mz) return;
  const int i = (int)(q % d.mx), rem = (int)(q / d.mx), j = rem % d.my, k = rem / d.my;
  const int64_t id = d.idx(d.ngg, i, j, k), iq = d.idx(0, i, j, k);
  NodeStateN<NS> s;
  double yk[NS], pres;
  load_node_ns<NS>(z, id, iq, s, yk, pres);
  int n_sub;
  double h, h_last;
  bool capped;
  substep_plan(dt, s.ts, n_sub, h, h_last, capped);
  if (capped) atomicOr(err, 2);
  bool ok = true;
  for (int n = 0; n < n_sub; ++n) ok &= zero_d_substep_ns<NS>(mc, p.chem_advance_method, h, s, yk, pres, L, R);
  int taken = n_sub;
  if (abs(h_last) > 1e-12) {
    ok &= zero_d_substep_ns<NS>(mc, p.chem_advance_method, h_last, s, yk, pres, L, R);
    ++taken;
  }
  if (!ok) atomicOr(err, 1);
  store_node_ns<NS>(z, p.n_scalar, id, s, yk, pres);
  if (nsub_out) nsub_out[iq] = taken;
}

// Work-queue schedule (see wu_reaction_queue_kernel), optionally over a node list.
template <int NS>
__global__ void __launch_bounds__(kFastBlock) wu_reaction_queue_ns_kernel(Zone z, Param p,
                                                                         const __grid_constant__ Mech mech, double dt,
                                                                         int *nsub_out, int *err,
                                                                         unsigned int *counter,
                                                                         const unsigned int *list,
                                                                         const unsigned int *list_count) {
  const Mech *mc = &mech;
  extern __shared__ double sys[];
  const LaneSlot L{sys + threadIdx.x, kFastBlock}, R{sys + NS * NS * kFastBlock + threadIdx.x, kFastBlock};
  const Dims d = z.d;
  const unsigned int total = list ? *list_count : (unsigned int)d.mx * d.my * d.mz;
  const int lane = threadIdx.x & 31;
  NodeStateN<NS> s;
  double yk[NS], pres = 0, h = 0, h_last = 0;
  int n_sub = 0, done = 0, taken = 0;
  int64_t id = 0, iq = 0;
  bool ok = true, have = false, exhausted = false;
  for (;;) {
    const bool need = !have && !exhausted;
    const unsigned int mask = __ballot_sync(0xffffffffu, need);
    if (mask) {
      unsigned int base = 0;
      const int leader = __ffs(mask) - 1;
      if (lane == leader) base = atomicAdd(counter, (unsigned int)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        unsigned int node = base + __popc(mask & ((1u << lane) - 1));
        if (node < total) {
          if (list) node = list[node];
          const int i = node % d.mx, rem = node / d.mx, j = rem % d.my, k = rem / d.my;
          id = d.idx(d.ngg, i, j, k);
          iq = d.idx(0, i, j, k);
          load_node_ns<NS>(z, id, iq, s, yk, pres);
          bool capped;
          substep_plan(dt, s.ts, n_sub, h, h_last, capped);
          if (capped) atomicOr(err, 2);
          done = 0;
          taken = 0;
          ok = true;
          have = true;
        } else {
          exhausted = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, have)) break;
    if (have) {
      const double hh = done < n_sub ? h : h_last;
      const bool run = done < n_sub || abs(h_last) > 1e-12;
      if (run) {
        ok &= zero_d_substep_ns<NS>(mc, p.chem_advance_method, hh, s, yk, pres, L, R);
        ++taken;
      }
      ++done;
      if (done > n_sub) {
        if (!ok) atomicOr(err, 1);
        store_node_ns<NS>(z, p.n_scalar, id, s, yk, pres);
        if (nsub_out) nsub_out[iq] = taken;
        have = false;
      }
    }
  }
}

// Persistent grid of the work-queue kernels: resident blocks per SM x SMs.
template <class K>
static long long queue_blocks(K kernel, int block, int smem, int n_sm, long long nodes) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  long long blocks = (long long)n_sm * per_sm;
  const long long need = (nodes + block - 1) / block;
  if (blocks > need) blocks = need;
  return blocks < 1 ? 1 : blocks;
}

cudaError_t launch_finite_rate_chemistry(const Zone &z, const Mech *mc, cudaStream_t st) {
  finite_rate_chemistry_kernel<<<dim3((z.d.mx + 127) / 128, z.d.my, z.d.mz), 128, 0, st>>>(z, mc);
  return cudaGetLastError();
}

cudaError_t launch_wu_reaction(const Zone &z, const Param &p, const Mech *mc, const Mech &mc_host, double dt,
                               int schedule, int *nsub_out, int *err, unsigned int *counter, int n_sm,
                               cudaStream_t st) {
  const long long total = (long long)z.d.mx * z.d.my * z.d.mz;
  if (p.n_spec == kMaxSpec) {
    constexpr int smem = fast_smem_bytes<kMaxSpec>();
    if (schedule == 0) {
      wu_reaction_plain_ns_kernel<kMaxSpec><<<(unsigned)((total + kFastBlock - 1) / kFastBlock), kFastBlock, smem, st>>>(
          z, p, mc_host, dt, nsub_out, err);
    } else {
      cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
      if (e != cudaSuccess) return e;
      const long long blocks = queue_blocks(wu_reaction_queue_ns_kernel<kMaxSpec>, kFastBlock, smem, n_sm, total);
      wu_reaction_queue_ns_kernel<kMaxSpec><<<(unsigned)blocks, kFastBlock, smem, st>>>(
          z, p, mc_host, dt, nsub_out, err, counter, nullptr, nullptr);
    }
    return cudaGetLastError();
  }
  if (schedule == 0) {
    wu_reaction_plain_kernel<<<dim3((z.d.mx + 127) / 128, z.d.my, z.d.mz), 128, 0, st>>>(z, p, mc, dt, nsub_out, err);
  } else {
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    long long blocks = (long long)n_sm * 8;
    const long long need = (total + 127) / 128;
    if (blocks > need) blocks = need;
    wu_reaction_queue_kernel<<<(unsigned)blocks, 128, 0, st>>>(z, p, mc, dt, nsub_out, err, counter, nullptr, nullptr);
  }
  return cudaGetLastError();
}

// Work-queue reaction step over the nodes list[0 .. *list_count); the count
// lives on the device, so the grid covers max_nodes.
cudaError_t launch_wu_reaction_list(const Zone &z, const Param &p, const Mech *mc, const Mech &mc_host, double dt,
                                    const unsigned int *list, const unsigned int *list_count, long long max_nodes,
                                    int *err, unsigned int *counter, int n_sm, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return e;
  if (p.n_spec == kMaxSpec) {
    constexpr int smem = fast_smem_bytes<kMaxSpec>();
    const long long blocks = queue_blocks(wu_reaction_queue_ns_kernel<kMaxSpec>, kFastBlock, smem, n_sm, max_nodes);
    wu_reaction_queue_ns_kernel<kMaxSpec><<<(unsigned)blocks, kFastBlock, smem, st>>>(z, p, mc_host, dt, nullptr, err,
                                                                                    counter, list, list_count);
    return cudaGetLastError();
  }
  long long blocks = (long long)n_sm * 8;
  const long long need = (max_nodes + 127) / 128;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  wu_reaction_queue_kernel<<<(unsigned)blocks, 128, 0, st>>>(z, p, mc, dt, nullptr, err, counter, list, list_count);
  return cudaGetLastError();
}

}  // namespace cfk
