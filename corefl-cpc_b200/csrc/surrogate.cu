// MLP chemistry surrogate kernels on the sm_100a tensor cores.
//
//  * sg_step_kernel: the gated surrogate reaction step.  Persistent CTAs of
//    two 128-thread groups; each group takes tiles of 128 nodes, one node per
//    thread: FP64 state -> standardised features (BF16) -> four tcgen05 GEMMs
//    (M=128 nodes; accumulators in TMEM; tanh epilogues written back to shared
//    memory as the next layer's operand) -> FP64 post-processing: inverse
//    transform, element-conservation projection, energy-consistent
//    temperature by Newton iteration, gate.  Nodes that fail the gate, and a
//    rotating sample judged against the plain integrator, are appended to a
//    node list that the FP64 work-queue kernel integrates afterwards.
//  * sg_train_kernel: fused forward + backward of one minibatch.  Weight
//    gradients accumulate in TMEM over a CTA's tiles (bias gradients come out
//    of the same GEMMs through the constant-1 columns) and are written as
//    per-CTA partial sums; sg_adam_kernel reduces them and updates the FP32
//    master weights and their BF16 copy.
#include <cuda_bf16.h>

#include "surrogate.cuh"
#include "tc_ptx.cuh"

namespace cfk {
using namespace tc;

namespace {

constexpr long long kWaitCycles = 4LL << 30;  // about 2 s of SM clock
constexpr int kTileA0 = 128 * 16 * 2;        // 128 x 16 BF16 operand tile
constexpr int kTileH = 128 * 144 * 2;        // 128 x 144 BF16 operand tile
constexpr int kRowA0 = 16 * 16;              // bytes per 8-row group, 16 columns
constexpr int kRowH = 144 * 16;              // bytes per 8-row group, 144 columns

// step kernel shared memory: weights | per group: a0, act | 2 mbarriers | TMEM slot
constexpr int kStepGroup = kTileA0 + kTileH;
constexpr int kStepMbar = kSgWBytes + 2 * kStepGroup;
constexpr int kStepSmem = kStepMbar + 64;

// train kernel shared memory: weights | a0 | h1 | h2 | h3 | dy | db3 | mbarrier | TMEM slot
constexpr int kTrA0 = kSgWBytes;
constexpr int kTrH1 = kTrA0 + kTileA0;
constexpr int kTrH2 = kTrH1 + kTileH;
constexpr int kTrH3 = kTrH2 + kTileH;
constexpr int kTrDY = kTrH3 + kTileH;
constexpr int kTrDB = kTrDY + kTileA0;
constexpr int kTrMbar = kTrDB + 64;
constexpr int kTrainSmem = kTrMbar + 64;
static_assert(kTrainSmem <= 227 * 1024, "train kernel shared memory");

// TMEM columns of the train kernel (512 allocated)
constexpr uint32_t kTmScratch = 0, kTmDW1 = 128, kTmDW2 = 288, kTmDW0 = 448, kTmDW3 = 480;

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ float bf_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf_hi(uint32_t u) { return __uint_as_float(u & 0xffff0000u); }

// Descriptors over a core-matrix tile with `cols` columns.
__device__ __forceinline__ uint64_t dK(uint32_t a, int cols) { return smem_desc(a, 128, cols * 16); }
__device__ __forceinline__ uint64_t dMN(uint32_t a, int cols) { return smem_desc(a, cols * 16, 128); }

// D (+)= A * B over `ksteps` K=16 slices.  A K-major operand steps 256 bytes
// (two core matrices) per slice; an MN-major one steps 16 rows.
__device__ __forceinline__ void gemm(uint32_t tm, uint32_t a, int a_cols, bool a_mn, uint32_t b, int b_cols,
                                     bool b_mn, int ksteps, uint32_t idesc, bool acc) {
  for (int kk = 0; kk < ksteps; ++kk) {
    const uint64_t da = a_mn ? dMN(a + kk * a_cols * 32, a_cols) : dK(a + kk * 256, a_cols);
    const uint64_t db = b_mn ? dMN(b + kk * b_cols * 32, b_cols) : dK(b + kk * 256, b_cols);
    mma_bf16(tm, da, db, idesc, (acc || kk > 0) ? 1u : 0u);
  }
}

__device__ __forceinline__ uint8_t *row_ptr_h(uint8_t *tile, int row) { return tile + (row >> 3) * kRowH + (row & 7) * 16; }
__device__ __forceinline__ uint8_t *row_ptr_a0(uint8_t *tile, int row) { return tile + (row >> 3) * kRowA0 + (row & 7) * 16; }

// Constant columns 128..143 of a hidden tile row: (1, 0, ..., 0).
__device__ __forceinline__ void init_const_cols(uint8_t *tile, int row) {
  uint8_t *rp = row_ptr_h(tile, row);
  *reinterpret_cast<uint4 *>(rp + 16 * 128) = make_uint4(pack2(1.f, 0.f), 0u, 0u, 0u);
  *reinterpret_cast<uint4 *>(rp + 17 * 128) = make_uint4(0u, 0u, 0u, 0u);
}

__device__ __forceinline__ void write_a0_row(uint8_t *tile, int row, const float *x, float one) {
  uint8_t *rp = row_ptr_a0(tile, row);
  *reinterpret_cast<uint4 *>(rp) = make_uint4(pack2(x[0], x[1]), pack2(x[2], x[3]), pack2(x[4], x[5]), pack2(x[6], x[7]));
  *reinterpret_cast<uint4 *>(rp + 128) = make_uint4(pack2(x[8], x[9]), pack2(x[10], x[11]), 0u, pack2(0.f, one));
}

// tanh of this lane's 128 accumulator columns -> columns 0..127 of its tile row.
__device__ __forceinline__ void epi_tanh(uint32_t tl, uint8_t *tile, int row) {
  uint8_t *rp = row_ptr_h(tile, row);
#pragma unroll
  for (int cb = 0; cb < 4; ++cb) {
    float v[32];
    tmem_ld32(tl + cb * 32, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float *w = v + 8 * q;
      const uint4 u = make_uint4(pack2(tanh_approx(w[0]), tanh_approx(w[1])), pack2(tanh_approx(w[2]), tanh_approx(w[3])),
                                 pack2(tanh_approx(w[4]), tanh_approx(w[5])), pack2(tanh_approx(w[6]), tanh_approx(w[7])));
      *reinterpret_cast<uint4 *>(rp + (cb * 4 + q) * 128) = u;
    }
  }
}

// dz = dh * (1 - h^2): dh from TMEM, h read from the tile row, dz written in place.
__device__ __forceinline__ void epi_dtanh(uint32_t tl, uint8_t *tile, int row) {
  uint8_t *rp = row_ptr_h(tile, row);
#pragma unroll
  for (int cb = 0; cb < 4; ++cb) {
    float v[32];
    tmem_ld32(tl + cb * 32, v);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint4 *p = reinterpret_cast<uint4 *>(rp + (cb * 4 + q) * 128);
      const uint4 h = *p;
      const float *w = v + 8 * q;
      float hv[8] = {bf_lo(h.x), bf_hi(h.x), bf_lo(h.y), bf_hi(h.y), bf_lo(h.z), bf_hi(h.z), bf_lo(h.w), bf_hi(h.w)};
      *p = make_uint4(pack2(w[0] * (1.f - hv[0] * hv[0]), w[1] * (1.f - hv[1] * hv[1])),
                      pack2(w[2] * (1.f - hv[2] * hv[2]), w[3] * (1.f - hv[3] * hv[3])),
                      pack2(w[4] * (1.f - hv[4] * hv[4]), w[5] * (1.f - hv[5] * hv[5])),
                      pack2(w[6] * (1.f - hv[6] * hv[6]), w[7] * (1.f - hv[7] * hv[7])));
    }
  }
}

__device__ __forceinline__ void warp_count(unsigned long long *ctr, bool pred) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  if (m && (int)(threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(ctr, (unsigned long long)__popc(m));
}

// Slot of this lane in a warp-aggregated append (valid where pred).
__device__ __forceinline__ unsigned warp_append(unsigned *count, bool pred) {
  const unsigned m = __ballot_sync(0xffffffffu, pred);
  const int lane = threadIdx.x & 31;
  unsigned base = 0;
  if (m) {
    const int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(count, (unsigned)__popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
  }
  return base + __popc(m & ((1u << lane) - 1));
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Block, row and column of master element e; cols of its block.
__host__ __device__ inline void sg_locate(int e, int &blk, int &row, int &col, int &cols) {
  int base;
  if (e < kSgW1) { blk = 0; base = kSgW0; cols = 16; }
  else if (e < kSgW2) { blk = 1; base = kSgW1; cols = 144; }
  else if (e < kSgW3) { blk = 2; base = kSgW2; cols = 144; }
  else { blk = 3; base = kSgW3; cols = 144; }
  row = (e - base) / cols;
  col = (e - base) % cols;
}

__device__ __forceinline__ int sg_cm_byte(int e) {
  int blk, row, col, cols;
  sg_locate(e, blk, row, col, cols);
  const int base = blk == 0 ? kSgW0 : blk == 1 ? kSgW1 : blk == 2 ? kSgW2 : kSgW3;
  return 2 * base + (int)cm_offset(row, col, cols);
}

}  // namespace

// ---------------------------------------------------------------------------
// Gated surrogate reaction step
// ---------------------------------------------------------------------------
struct SgStepArgs {
  Zone z;
  const Mech *mc;
  const uint8_t *w16;
  SgNorm nrm;
  SgGate gate;
  SgProj proj;
  double dt;
  int n_nodes;
  unsigned *list, *list_count;
  SgJudge *judge;
  unsigned *judge_count;
  unsigned short *revert;
  SgCounters *cnt;
  int *err;
};

__global__ void __launch_bounds__(256, 1) sg_step_kernel(const __grid_constant__ SgStepArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, g = warp >> 2, row = tid & 127;
  uint8_t *sw = smem;
  uint8_t *sa0 = smem + kSgWBytes + g * kStepGroup;
  uint8_t *sact = sa0 + kTileA0;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kStepMbar);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + kStepMbar + 16);

  for (int o = tid * 16; o < kSgWBytes; o += 256 * 16)
    *reinterpret_cast<uint4 *>(sw + o) = __ldg(reinterpret_cast<const uint4 *>(a.w16 + o));
  init_const_cols(sact, row);
  if (tid == 0) {
    mbar_init(smem_addr(&mbar[0]), 1);
    mbar_init(smem_addr(&mbar[1]), 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(smem_addr(tslot), 256);
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tcol = *tslot + g * 128;
  const uint32_t tl = tcol + ((uint32_t)(32 * (warp & 3)) << 16);
  const uint32_t mb = smem_addr(&mbar[g]);
  const uint32_t a0s = smem_addr(sa0), acts = smem_addr(sact), ws = smem_addr(sw);
  const int bar_id = 1 + g;
  uint32_t phase = 0;
  bool bad = false;

  const Dims d = a.z.d;
  const Thermo *th = &a.mc->th;
  const int ns = th->n_spec;
  const int64_t szp = d.plane(d.ngg), szq = d.plane(0);
  const int n_tiles = (a.n_nodes + 127) / 128;
  const uint32_t id_h = idesc_bf16(128, 128, 0, 0), id_o = idesc_bf16(128, 16, 0, 0);

  auto run = [&](int layer) -> bool {
    fence_proxy_async();
    fence_before_sync();
    group_bar(bar_id);
    if (row == 0) {
      fence_after_sync();
      if (layer == 0) gemm(tcol, a0s, 16, false, ws + 2 * kSgW0, 16, false, 1, id_h, false);
      else if (layer == 1) gemm(tcol, acts, 144, false, ws + 2 * kSgW1, 144, false, 9, id_h, false);
      else if (layer == 2) gemm(tcol, acts, 144, false, ws + 2 * kSgW2, 144, false, 9, id_h, false);
      else gemm(tcol, acts, 144, false, ws + 2 * kSgW3, 144, false, 9, id_o, false);
      mma_commit(mb);
    }
    const bool ok = mbar_wait(mb, phase, kWaitCycles);
    phase ^= 1u;
    const bool any_bad = group_any(bar_id, !ok);
    fence_after_sync();
    return !any_bad;
  };

  for (int t = blockIdx.x * 2 + g; t < n_tiles; t += gridDim.x * 2) {
    const int q = t * 128 + row;
    const bool valid = q < a.n_nodes;
    int64_t id = 0, iq = 0;
    // Y0: composition the predicted change applies to; Te, qe: temperature and
    // conserved variables it starts from (the node's own, or with the frozen
    // transport term Cn the state that term alone reaches by the step's end)
    double T0 = 0, p0 = 0, Y0[kMaxSpec], Te = 0, qe[5] = {0, 0, 0, 0, 0};
    int reason = valid ? 0 : -1;
    float x[kSgIn];
    if (valid) {
      const int i = q % d.mx, r = q / d.mx, j = r % d.my, k = r / d.my;
      id = d.idx(d.ngg, i, j, k);
      iq = d.idx(0, i, j, k);
      T0 = a.z.bv[id + 5 * szp];
      p0 = a.z.bv[id + 4 * szp];
      for (int l = 0; l < kMaxSpec; ++l) Y0[l] = l < ns ? a.z.sv[id + l * szp] : 0.0;
#pragma unroll
      for (int l = 0; l < 5; ++l) qe[l] = a.z.cv[id + l * szp];
      Te = T0;
      double Tf = T0, pf = p0, Yf[kMaxSpec];
      for (int l = 0; l < kMaxSpec; ++l) Yf[l] = Y0[l];
      if (a.z.Cn) {
        // features at the mid-step state of the frozen transport, the change
        // applied to its end-of-step state
        double q0[5], rY0[kMaxSpec], cq[5], crY[kMaxSpec], qm[5];
        const double s = a.dt / a.z.jac[id];
#pragma unroll
        for (int l = 0; l < 5; ++l) {
          q0[l] = qe[l];
          cq[l] = a.z.Cn[iq + l * szq] * s;
        }
        bool moved = false;
#pragma unroll
        for (int l = 0; l < 5; ++l) moved |= cq[l] != 0.0;
        for (int l = 0; l < ns; ++l) {
          rY0[l] = a.z.cv[id + (5 + l) * szp];
          crY[l] = a.z.Cn[iq + (5 + l) * szq] * s;
          moved |= crY[l] != 0.0;
        }
        // a node the transport term leaves unchanged keeps its own state
        if (moved) {
          double pe = 0;
          const bool ok = sg_transported_pair(th, ns, q0, rY0, cq, crY, T0, qm, Yf, Tf, pf, qe, Y0, Te, pe);
          if (!ok) {
            reason = SG_NEWTON_FAILED;
            Tf = T0;
            pf = p0;
          }
        }
      }
      double f[kSgIn];
      sg_raw_features(Tf, pf, Yf, ns, a.dt, f);
      // the range check runs in raw feature units, with an excursion of
      // 1e-3 max(1, |mean|) allowed beyond the training range (a feature that
      // sits at an end of its range in most rows, such as a mass fraction at
      // zero, must not fall out by the rounding of the stored bounds), plus
      // ood_margin standard deviations
      bool ood = false;
      for (int c = 0; c < kSgIn; ++c) {
        const double mean = (double)a.nrm.in_mean[c], rs = (double)a.nrm.in_rstd[c];
        const double dev = f[c] - mean;
        x[c] = (float)(dev * rs);
        const double tol = 1e-3 * fmax(1.0, fabs(mean));
        if (rs == 0.0) {
          ood |= fabs(dev) > tol;
        } else {
          const double m = a.gate.ood_margin / rs + tol;
          ood |= dev < (double)a.nrm.in_lo[c] / rs - m || dev > (double)a.nrm.in_hi[c] / rs + m;
        }
      }
      // expected substeps of the plain integrator (its substep plan)
      double tau = a.z.reaction_timeScale[id];
      if (tau < 1e-15) tau = 0.2 * a.dt;
      if (a.revert[q] > 0) {
        a.revert[q] -= 1;
        reason = SG_REVERT;
      } else if (ood) {
        reason = SG_OOD;
      } else if (a.dt / tau < a.gate.min_substeps) {
        reason = SG_CHEAP;
      }
    } else {
      for (int c = 0; c < kSgIn; ++c) x[c] = 0.f;
      for (int l = 0; l < kMaxSpec; ++l) Y0[l] = 0.0;
    }
    write_a0_row(sa0, row, x, valid ? 1.f : 0.f);

    if (!run(0)) { bad = true; break; }
    epi_tanh(tl, sact, row);
    if (!run(1)) { bad = true; break; }
    epi_tanh(tl, sact, row);
    if (!run(2)) { bad = true; break; }
    epi_tanh(tl, sact, row);
    if (!run(3)) { bad = true; break; }
    float o[16];
    tmem_ld16(tl, o);

    bool judged = false;
    double Tn = 0, Yn[kMaxSpec];
    if (reason == 0) {
      double rr[kSgOut];
      for (int c = 0; c < kSgOut; ++c)
        rr[c] = sg_target_inv((double)a.nrm.out_mean[c] + (double)a.nrm.out_std[c] * (double)o[c], a.nrm.out_scale[c]);
      double Z0[4];
      for (int e = 0; e < a.proj.n_elem; ++e) {
        double s = 0;
        for (int l = 0; l < ns; ++l) s += a.proj.mu[e][l] * Y0[l];
        Z0[e] = s;
      }
      for (int l = 0; l < ns; ++l) Yn[l] = sg_boxcox_inv(sg_boxcox(Y0[l]) + rr[l]);
      const bool projected = sg_project(a.proj, ns, Z0, Yn);
      double qv[5], rY[kMaxSpec];
#pragma unroll
      for (int l = 0; l < 5; ++l) qv[l] = qe[l];
      for (int l = 0; l < ns; ++l) rY[l] = qv[0] * Yn[l];
      const double rinv = 1.0 / qv[0];
      const double u = qv[1] * rinv, v = qv[2] * rinv, w = qv[3] * rinv;
      double guess = Te + rr[9];
      guess = fmin(fmax(guess, fmax(Te - 500.0, 200.0)), Te + 3000.0);
      Tn = guess;
      double pn = 0;
      const bool ok = projected && temperature_newton(th, ns, Yn, qv[4], qv[0], u * u + v * v + w * w, Tn, pn);
      if (!ok) reason = SG_NEWTON_FAILED;
      else if (fabs(Tn - Te) > a.gate.dT_max) reason = SG_IGNITION;
      else if (fabs(Te + rr[9] - Tn) > a.gate.dT_consistency) reason = SG_CONSISTENCY;
      judged = reason == 0 && a.gate.judge_stride > 0 &&
               ((unsigned)q + (unsigned)a.gate.judge_salt) % (unsigned)a.gate.judge_stride == 0;
      if (reason == 0 && !judged) {
        if (a.z.Cn) {
#pragma unroll
          for (int l = 0; l < 5; ++l) a.z.cv[id + l * szp] = qv[l];
        }
        for (int l = 0; l < ns; ++l) {
          a.z.cv[id + (5 + l) * szp] = rY[l];
          a.z.sv[id + l * szp] = Yn[l];
        }
        a.z.bv[id] = qv[0];
        a.z.bv[id + szp] = u;
        a.z.bv[id + 2 * szp] = v;
        a.z.bv[id + 3 * szp] = w;
        a.z.bv[id + 4 * szp] = pn;
        a.z.bv[id + 5 * szp] = Tn;
        a.z.reaction_timeScale[id] = fmin(fmax(exp(rr[10]), 1e-20), 1e6);
      }
    }
    // bookkeeping (every lane of the warp takes part)
    warp_count(&a.cnt->n[SG_CELLS], valid);
    warp_count(&a.cnt->n[SG_SURROGATE], reason == 0 && !judged);
    warp_count(&a.cnt->n[SG_OOD], reason == SG_OOD);
    warp_count(&a.cnt->n[SG_IGNITION], reason == SG_IGNITION);
    warp_count(&a.cnt->n[SG_CONSISTENCY], reason == SG_CONSISTENCY);
    warp_count(&a.cnt->n[SG_REVERT], reason == SG_REVERT);
    warp_count(&a.cnt->n[SG_NEWTON_FAILED], reason == SG_NEWTON_FAILED);
    warp_count(&a.cnt->n[SG_CHEAP], reason == SG_CHEAP);
    warp_count(&a.cnt->n[SG_JUDGED], judged);
    const bool to_plain = reason > 0 || judged;
    const unsigned slot = warp_append(a.list_count, to_plain);
    if (to_plain) a.list[slot] = (unsigned)q;
    const unsigned js = warp_append(a.judge_count, judged);
    if (judged) {
      SgJudge &jr = a.judge[js];
      jr.cell = (unsigned)q;
      jr.T = (float)Tn;
      for (int l = 0; l < kMaxSpec; ++l) jr.Y[l] = l < ns ? (float)Yn[l] : 0.f;
    }
  }

  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(*tslot, 256);
  }
  if (bad && row == 0) atomicOr(a.err, 4);
}

// Judged nodes: compare the plain integrator's result (now in the zone) with
// the surrogate's prediction — temperature in K, species in Box-Cox units
// (relative for trace species) — and put failures on the plain integrator
// for revert_steps steps.
__global__ void sg_judge_kernel(Zone z, int ns, const SgJudge *judge, const unsigned *judge_count, SgGate gate,
                                unsigned short *revert, SgCounters *cnt) {
  const unsigned n = *judge_count;
  const Dims d = z.d;
  const int64_t szp = d.plane(d.ngg);
  for (unsigned s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    const SgJudge jr = judge[s];
    const int q = (int)jr.cell;
    const int i = q % d.mx, r = q / d.mx, j = r % d.my, k = r / d.my;
    const int64_t id = d.idx(d.ngg, i, j, k);
    const double dT = fabs(z.bv[id + 5 * szp] - (double)jr.T);
    double dbc = 0;
    for (int l = 0; l < ns; ++l) dbc = fmax(dbc, fabs(sg_boxcox(z.sv[id + l * szp]) - sg_boxcox((double)jr.Y[l])));
    atomicMax(&cnt->judge_max_dT_bits, (unsigned long long)__double_as_longlong(dT));
    atomicMax(&cnt->judge_max_dbc_bits, (unsigned long long)__double_as_longlong(dbc));
    atomicAdd(&cnt->judge_sum_dT, dT);
    if (dT > gate.judge_tol_T || dbc > gate.judge_tol_bc) {
      atomicAdd(&cnt->n[SG_JUDGE_FAILED], 1ull);
      revert[q] = (unsigned short)min(gate.revert_steps, 65535);
    }
  }
}

// ---------------------------------------------------------------------------
// Training data: a snapshot of (T, p, Y) before a plain reaction step, then
// the raw features and targets after it.
// ---------------------------------------------------------------------------
// Training rows from the plain integrator.  Before its step: the state the
// features are read at and the state the change applies to (sg_transported:
// the node's own without a transport term, else the frozen transport term's
// mid-step and end-of-step states), 21 doubles per node: T, p, Y[9] of the
// first, T, Y[9] of the second.  After it: one row of raw features and
// targets per node, the targets the changes from the second state.
constexpr int kSnap = 21;

__global__ void sg_snapshot_kernel(Zone z, const Thermo *th, int n_nodes, double dt, double *snap) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_nodes) return;
  const Dims d = z.d;
  const int ns = th->n_spec;
  const int i = q % d.mx, r = q / d.mx, j = r % d.my, k = r / d.my;
  const int64_t id = d.idx(d.ngg, i, j, k), szp = d.plane(d.ngg);
  double *s = snap + (int64_t)q * kSnap;
  double T0 = z.bv[id + 5 * szp], p0 = z.bv[id + 4 * szp], Y0[kMaxSpec];
  for (int l = 0; l < kMaxSpec; ++l) Y0[l] = l < ns ? z.sv[id + l * szp] : 0.0;
  double Tf = T0, pf = p0, Yf[kMaxSpec], Te = T0, Ye[kMaxSpec];
  for (int l = 0; l < kMaxSpec; ++l) Yf[l] = Ye[l] = Y0[l];
  if (z.Cn) {
    const int64_t iq = d.idx(0, i, j, k), szq = d.plane(0);
    double q0[5], rY0[kMaxSpec], cq[5], crY[kMaxSpec], qt[5], pe = 0;
    const double sc = dt / z.jac[id];
    bool moved = false;
    for (int l = 0; l < 5; ++l) {
      q0[l] = z.cv[id + l * szp];
      cq[l] = z.Cn[iq + l * szq] * sc;
      moved |= cq[l] != 0.0;
    }
    for (int l = 0; l < ns; ++l) {
      rY0[l] = z.cv[id + (5 + l) * szp];
      crY[l] = z.Cn[iq + (5 + l) * szq] * sc;
      moved |= crY[l] != 0.0;
    }
    double qm[5];
    if (moved && !sg_transported_pair(th, ns, q0, rY0, cq, crY, T0, qm, Yf, Tf, pf, qt, Ye, Te, pe)) {
      // no transported state: the row falls back to the node's own (a
      // training sample of the reaction alone)
      Tf = Te = T0;
      pf = p0;
      for (int l = 0; l < kMaxSpec; ++l) Yf[l] = Ye[l] = Y0[l];
    }
  }
  s[0] = Tf;
  s[1] = pf;
  for (int l = 0; l < kMaxSpec; ++l) s[2 + l] = Yf[l];
  s[11] = Te;
  for (int l = 0; l < kMaxSpec; ++l) s[12 + l] = Ye[l];
}

__global__ void sg_record_kernel(Zone z, int ns, int n_nodes, const double *snap, double dt, float *X, float *G) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_nodes) return;
  const Dims d = z.d;
  const int i = q % d.mx, r = q / d.mx, j = r % d.my, k = r / d.my;
  const int64_t id = d.idx(d.ngg, i, j, k), szp = d.plane(d.ngg);
  const double *s = snap + (int64_t)q * kSnap;
  double f[kSgIn];
  sg_raw_features(s[0], s[1], s + 2, ns, dt, f);
  for (int c = 0; c < kSgIn; ++c) X[(int64_t)q * kSgIn + c] = (float)f[c];
  float *gq = G + (int64_t)q * kSgOut;
  for (int l = 0; l < kMaxSpec; ++l)
    gq[l] = l < ns ? (float)(sg_boxcox(z.sv[id + l * szp]) - sg_boxcox(s[12 + l])) : 0.f;
  gq[9] = (float)(z.bv[id + 5 * szp] - s[11]);
  gq[10] = (float)log(fmin(fmax(z.reaction_timeScale[id], 1e-20), 1e6));
}

// Column sums, sums of squares, minima and maxima of X (12 columns) and G
// (11 columns).  mm holds order-preserving unsigned keys of the floats.
__device__ __forceinline__ unsigned float_key(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

struct SgScales {
  float s[kSgOut];
};

__global__ void sg_colstats_kernel(const float *X, const float *G, long long n, SgScales sc, double *acc,
                                   unsigned *mm) {
  constexpr int C = kSgIn + kSgOut;
  double s[C], s2[C];
  unsigned lo[C], hi[C];
  for (int c = 0; c < C; ++c) { s[c] = 0; s2[c] = 0; lo[c] = 0xffffffffu; hi[c] = 0u; }
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < C; ++c) {
      float v;
      if (c < kSgIn) {
        v = X[r * kSgIn + c];
      } else {
        v = G[r * kSgOut + c - kSgIn];
        if (sc.s[c - kSgIn] > 0.f) v = asinhf(v / sc.s[c - kSgIn]);
      }
      s[c] += v;
      s2[c] += (double)v * v;
      const unsigned kk = float_key(v);
      lo[c] = min(lo[c], kk);
      hi[c] = max(hi[c], kk);
    }
  }
  for (int c = 0; c < C; ++c) {
    double a1 = s[c], a2 = s2[c];
    unsigned l = lo[c], h = hi[c];
    for (int o = 16; o > 0; o >>= 1) {
      a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      l = min(l, __shfl_xor_sync(0xffffffffu, l, o));
      h = max(h, __shfl_xor_sync(0xffffffffu, h, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(&acc[2 * c], a1);
      atomicAdd(&acc[2 * c + 1], a2);
      atomicMin(&mm[2 * c], l);
      atomicMax(&mm[2 * c + 1], h);
    }
  }
}

// ---------------------------------------------------------------------------
// Training: fused forward + backward of one minibatch
// ---------------------------------------------------------------------------
struct SgTrainArgs {
  const float *X, *G;
  long long n;               // rows in the data set
  long long perm_a, perm_b;  // row of minibatch entry i: (perm_a * i + perm_b) mod n
  long long start;           // first minibatch entry
  int count;                 // minibatch rows
  int mode;                  // 0: gradients, 1: forward outputs only
  SgNorm nrm;
  const uint8_t *w16;
  float *partials;           // [gridDim.x][kSgNParam]
  double *loss;
  float *Yout;               // mode 1: [n][16] standardised outputs
  int *err;
};

__global__ void __launch_bounds__(128, 1) sg_train_kernel(const __grid_constant__ SgTrainArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, row = tid;
  uint8_t *sw = smem;
  uint8_t *sa0 = smem + kTrA0, *sh1 = smem + kTrH1, *sh2 = smem + kTrH2, *sh3 = smem + kTrH3, *sdy = smem + kTrDY;
  float *db3 = reinterpret_cast<float *>(smem + kTrDB);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + kTrMbar);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + kTrMbar + 8);

  for (int o = tid * 16; o < kSgWBytes; o += 128 * 16)
    *reinterpret_cast<uint4 *>(sw + o) = __ldg(reinterpret_cast<const uint4 *>(a.w16 + o));
  init_const_cols(sh1, row);
  init_const_cols(sh2, row);
  init_const_cols(sh3, row);
  if (tid < 16) db3[tid] = 0.f;
  if (tid == 0) {
    mbar_init(smem_addr(mbar), 1);
    mbar_init_fence();
  }
  if (warp == 0) tmem_alloc(smem_addr(tslot), 512);
  fence_proxy_async();
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tb = *tslot;
  const uint32_t lane_off = (uint32_t)(32 * warp) << 16;
  const uint32_t tsc = tb + kTmScratch;
  const uint32_t mb = smem_addr(mbar);
  const uint32_t a0s = smem_addr(sa0), h1s = smem_addr(sh1), h2s = smem_addr(sh2), h3s = smem_addr(sh3);
  const uint32_t dys = smem_addr(sdy), ws = smem_addr(sw);
  const uint32_t id_h = idesc_bf16(128, 128, 0, 0), id_o = idesc_bf16(128, 16, 0, 0);
  const uint32_t id_dh = idesc_bf16(128, 128, 0, 1);     // dz (K-major) x W (MN-major)
  const uint32_t id_dw = idesc_bf16(128, 144, 1, 1);     // dz^T x a (both MN-major), 144 incl. bias column
  const uint32_t id_dw0 = idesc_bf16(128, 16, 1, 1);     // dz1^T x a0 / a3^T x dy
  uint32_t phase = 0;
  bool bad = false, first = true;
  double loss_acc = 0;
  const float scale = 2.f / ((float)a.count * (float)kSgOut);
  const int n_tiles = (a.count + 127) / 128;

  auto run = [&](int stage) -> bool {
    fence_proxy_async();
    fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      fence_after_sync();
      switch (stage) {
        case 0: gemm(tsc, a0s, 16, false, ws + 2 * kSgW0, 16, false, 1, id_h, false); break;
        case 1: gemm(tsc, h1s, 144, false, ws + 2 * kSgW1, 144, false, 9, id_h, false); break;
        case 2: gemm(tsc, h2s, 144, false, ws + 2 * kSgW2, 144, false, 9, id_h, false); break;
        case 3: gemm(tsc, h3s, 144, false, ws + 2 * kSgW3, 144, false, 9, id_o, false); break;
        case 4:  // dW3^T += a3^T dy ; dh3 = dy W3
          gemm(tb + kTmDW3, h3s, 144, true, dys, 16, true, 8, id_dw0, !first);
          gemm(tsc, dys, 16, false, ws + 2 * kSgW3, 144, true, 1, id_dh, false);
          break;
        case 5:  // dW2 += dz3^T a2 ; dh2 = dz3 W2
          gemm(tb + kTmDW2, h3s, 144, true, h2s, 144, true, 8, id_dw, !first);
          gemm(tsc, h3s, 144, false, ws + 2 * kSgW2, 144, true, 8, id_dh, false);
          break;
        case 6:  // dW1 += dz2^T a1 ; dh1 = dz2 W1
          gemm(tb + kTmDW1, h2s, 144, true, h1s, 144, true, 8, id_dw, !first);
          gemm(tsc, h2s, 144, false, ws + 2 * kSgW1, 144, true, 8, id_dh, false);
          break;
        default:  // dW0 += dz1^T a0
          gemm(tb + kTmDW0, h1s, 144, true, a0s, 16, true, 8, id_dw0, !first);
          break;
      }
      mma_commit(mb);
    }
    const bool ok = mbar_wait(mb, phase, kWaitCycles);
    phase ^= 1u;
    const bool any_bad = __syncthreads_or(!ok) != 0;
    fence_after_sync();
    return !any_bad;
  };

  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int r = t * 128 + row;
    const bool valid = r < a.count;
    long long s = 0;
    float x[kSgIn], tgt[kSgOut];
    if (valid) {
      s = (long long)(((unsigned long long)a.perm_a * (unsigned long long)(a.start + r) + (unsigned long long)a.perm_b) %
                      (unsigned long long)a.n);
      for (int c = 0; c < kSgIn; ++c) x[c] = (a.X[s * kSgIn + c] - a.nrm.in_mean[c]) * a.nrm.in_rstd[c];
      if (a.mode == 0)
        for (int c = 0; c < kSgOut; ++c) {
          const float g = a.G[s * kSgOut + c], sc = a.nrm.out_scale[c];
          tgt[c] = ((sc > 0.f ? asinhf(g / sc) : g) - a.nrm.out_mean[c]) / a.nrm.out_std[c];
        }
    } else {
      for (int c = 0; c < kSgIn; ++c) x[c] = 0.f;
      for (int c = 0; c < kSgOut; ++c) tgt[c] = 0.f;
    }
    write_a0_row(sa0, row, x, valid ? 1.f : 0.f);
    if (!run(0)) { bad = true; break; }
    epi_tanh(tsc + lane_off, sh1, row);
    if (!run(1)) { bad = true; break; }
    epi_tanh(tsc + lane_off, sh2, row);
    if (!run(2)) { bad = true; break; }
    epi_tanh(tsc + lane_off, sh3, row);
    if (!run(3)) { bad = true; break; }
    float y[16];
    tmem_ld16(tsc + lane_off, y);
    if (a.mode == 1) {
      if (valid)
        for (int c = 0; c < 16; ++c) a.Yout[s * 16 + c] = y[c];
      continue;
    }
    float dy[16];
    for (int c = 0; c < 16; ++c) {
      const float e = (valid && c < kSgOut) ? y[c] - tgt[c] : 0.f;
      loss_acc += (double)e * e;
      dy[c] = e * scale;
    }
    {
      uint8_t *rp = row_ptr_a0(sdy, row);
      *reinterpret_cast<uint4 *>(rp) = make_uint4(pack2(dy[0], dy[1]), pack2(dy[2], dy[3]), pack2(dy[4], dy[5]), pack2(dy[6], dy[7]));
      *reinterpret_cast<uint4 *>(rp + 128) =
          make_uint4(pack2(dy[8], dy[9]), pack2(dy[10], dy[11]), pack2(dy[12], dy[13]), pack2(dy[14], dy[15]));
    }
    for (int c = 0; c < kSgOut; ++c) {
      const float sum = warp_sum(dy[c]);
      if (lane == 0) atomicAdd(&db3[c], sum);
    }
    if (!run(4)) { bad = true; break; }
    epi_dtanh(tsc + lane_off, sh3, row);
    if (!run(5)) { bad = true; break; }
    epi_dtanh(tsc + lane_off, sh2, row);
    if (!run(6)) { bad = true; break; }
    epi_dtanh(tsc + lane_off, sh1, row);
    if (!run(7)) { bad = true; break; }
    first = false;
  }

  if (a.mode == 0 && !bad) {
    float *part = a.partials + (long long)blockIdx.x * kSgNParam;
    const int o = row;  // TMEM lane = output row (dW0, dW1, dW2) or input row (dW3^T)
    if (first) {
      // no tile processed by this CTA: zero partial
      for (int e = tid; e < kSgNParam; e += 128) part[e] = 0.f;
    } else {
      float v[32];
      for (int cb = 0; cb < 4; ++cb) {
        tmem_ld32(tb + kTmDW1 + lane_off + cb * 32, v);
        for (int c = 0; c < 32; ++c) part[kSgW1 + o * 144 + cb * 32 + c] = v[c];
        tmem_ld32(tb + kTmDW2 + lane_off + cb * 32, v);
        for (int c = 0; c < 32; ++c) part[kSgW2 + o * 144 + cb * 32 + c] = v[c];
      }
      tmem_ld16(tb + kTmDW1 + lane_off + 128, v);
      for (int c = 0; c < 16; ++c) part[kSgW1 + o * 144 + 128 + c] = v[c];
      tmem_ld16(tb + kTmDW2 + lane_off + 128, v);
      for (int c = 0; c < 16; ++c) part[kSgW2 + o * 144 + 128 + c] = v[c];
      tmem_ld16(tb + kTmDW0 + lane_off, v);
      for (int c = 0; c < 16; ++c) part[kSgW0 + o * 16 + c] = v[c];
      tmem_ld16(tb + kTmDW3 + lane_off, v);
      for (int c = 0; c < 16; ++c) part[kSgW3 + c * 144 + o] = v[c];
      __syncthreads();
      if (tid < 16) {
        part[kSgW3 + tid * 144 + 128] = tid < kSgOut ? db3[tid] : 0.f;
        for (int c = 129; c < 144; ++c) part[kSgW3 + tid * 144 + c] = 0.f;
      }
    }
  }
  if (a.mode == 0) {
    double l = loss_acc;
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if (lane == 0) atomicAdd(a.loss, l);
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    fence_after_sync();
    tmem_dealloc(tb, 512);
  }
  if (bad && tid == 0) atomicOr(a.err, 4);
}

// Sum of the per-CTA partial gradients; optional export; Adam update of the
// FP32 master weights and their BF16 core-matrix copy.  Once a training
// kernel has flagged a tensor-core wait timeout (value 4 in err) its partials
// are incomplete, so the update is skipped: the weights stay as they were
// until the host reads the flag and reports the error.
__global__ void sg_adam_kernel(float *master, float *m, float *v, const float *partials, int n_part, uint8_t *w16,
                               float lr, float b1, float b2, float eps, float bc1, float bc2, float *grad_out,
                               int update, const int *err) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kSgNParam) return;
  float g = 0.f;
  for (int p = 0; p < n_part; ++p) g += partials[(long long)p * kSgNParam + e];
  if (grad_out) grad_out[e] = g;
  if (!update) return;
  if (err && (*(volatile const int *)err & 4)) return;
  const float mm = b1 * m[e] + (1.f - b1) * g;
  const float vv = b2 * v[e] + (1.f - b2) * g * g;
  m[e] = mm;
  v[e] = vv;
  const float w = master[e] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
  master[e] = w;
  *reinterpret_cast<__nv_bfloat16 *>(w16 + sg_cm_byte(e)) = __float2bfloat16_rn(w);
}

// Master weights -> BF16 copy.
__global__ void sg_publish_kernel(const float *master, uint8_t *w16) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kSgNParam) return;
  *reinterpret_cast<__nv_bfloat16 *>(w16 + sg_cm_byte(e)) = __float2bfloat16_rn(master[e]);
}

// Xavier-uniform weights, zero biases and padding, zero optimiser moments.
__global__ void sg_init_kernel(float *master, float *m, float *v, unsigned long long seed) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kSgNParam) return;
  int blk, row, col, cols;
  sg_locate(e, blk, row, col, cols);
  const int fan_in = blk == 0 ? kSgIn : kSgH;
  const int fan_out = blk == 3 ? kSgOut : kSgH;
  const bool real = col < fan_in && row < fan_out;
  float w = 0.f;
  if (real) {
    const double u = (double)(splitmix64(seed * 0x100000001B3ull + (unsigned long long)e) >> 11) * (1.0 / 9007199254740992.0);
    w = (float)((2.0 * u - 1.0) * sqrt(6.0 / (fan_in + fan_out)));
  }
  master[e] = w;
  m[e] = 0.f;
  v[e] = 0.f;
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t sg_init_attributes() {
  cudaError_t e = cudaFuncSetAttribute(sg_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStepSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(sg_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
}

cudaError_t launch_sg_step(const Zone &z, const Mech *mc, const uint8_t *w16, const SgNorm &nrm, const SgGate &gate,
                           const SgProj &proj, double dt, unsigned *list, unsigned *list_count, SgJudge *judge,
                           unsigned *judge_count, unsigned short *revert, SgCounters *cnt, int *err, int n_sm,
                           cudaStream_t st) {
  SgStepArgs a;
  a.z = z; a.mc = mc; a.w16 = w16; a.nrm = nrm; a.gate = gate; a.proj = proj; a.dt = dt;
  a.n_nodes = z.d.mx * z.d.my * z.d.mz;
  a.list = list; a.list_count = list_count; a.judge = judge; a.judge_count = judge_count;
  a.revert = revert; a.cnt = cnt; a.err = err;
  const int n_tiles = (a.n_nodes + 127) / 128;
  int grid = (n_tiles + 1) / 2;
  if (grid > n_sm) grid = n_sm;
  if (grid < 1) grid = 1;
  sg_step_kernel<<<grid, 256, kStepSmem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sg_judge(const Zone &z, int ns, const SgJudge *judge, const unsigned *judge_count,
                            const SgGate &gate, unsigned short *revert, SgCounters *cnt, int n_sm, cudaStream_t st) {
  sg_judge_kernel<<<n_sm, 128, 0, st>>>(z, ns, judge, judge_count, gate, revert, cnt);
  return cudaGetLastError();
}

cudaError_t launch_sg_snapshot(const Zone &z, const Thermo *th, double dt, double *snap, cudaStream_t st) {
  const int n = z.d.mx * z.d.my * z.d.mz;
  sg_snapshot_kernel<<<(n + 127) / 128, 128, 0, st>>>(z, th, n, dt, snap);
  return cudaGetLastError();
}

cudaError_t launch_sg_record(const Zone &z, int ns, const double *snap, double dt, float *X, float *G, cudaStream_t st) {
  const int n = z.d.mx * z.d.my * z.d.mz;
  sg_record_kernel<<<(n + 127) / 128, 128, 0, st>>>(z, ns, n, snap, dt, X, G);
  return cudaGetLastError();
}

cudaError_t launch_sg_colstats(const float *X, const float *G, long long n, const float *scales, double *acc,
                               unsigned *mm, int n_sm, cudaStream_t st) {
  long long blocks = (n + 255) / 256;
  if (blocks > 4LL * n_sm) blocks = 4LL * n_sm;
  if (blocks < 1) blocks = 1;
  SgScales sc;
  for (int c = 0; c < kSgOut; ++c) sc.s[c] = scales[c];
  sg_colstats_kernel<<<(unsigned)blocks, 256, 0, st>>>(X, G, n, sc, acc, mm);
  return cudaGetLastError();
}

cudaError_t launch_sg_train(const float *X, const float *G, long long n, long long perm_a, long long perm_b,
                            long long start, int count, int mode, const SgNorm &nrm, const uint8_t *w16,
                            float *partials, int max_ctas, double *loss, float *Yout, int *err, int *n_ctas,
                            cudaStream_t st) {
  SgTrainArgs a;
  a.X = X; a.G = G; a.n = n; a.perm_a = perm_a; a.perm_b = perm_b; a.start = start; a.count = count; a.mode = mode;
  a.nrm = nrm; a.w16 = w16; a.partials = partials; a.loss = loss; a.Yout = Yout; a.err = err;
  int grid = (count + 127) / 128;
  if (grid > max_ctas) grid = max_ctas;
  if (grid < 1) grid = 1;
  *n_ctas = grid;
  sg_train_kernel<<<grid, 128, kTrainSmem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_sg_adam(float *master, float *m, float *v, const float *partials, int n_part, uint8_t *w16,
                           float lr, float b1, float b2, float eps, float bc1, float bc2, float *grad_out, int update,
                           const int *err, cudaStream_t st) {
  sg_adam_kernel<<<(kSgNParam + 255) / 256, 256, 0, st>>>(master, m, v, partials, n_part, w16, lr, b1, b2, eps, bc1,
                                                          bc2, grad_out, update, err);
  return cudaGetLastError();
}

cudaError_t launch_sg_publish(const float *master, uint8_t *w16, cudaStream_t st) {
  sg_publish_kernel<<<(kSgNParam + 255) / 256, 256, 0, st>>>(master, w16);
  return cudaGetLastError();
}

cudaError_t launch_sg_init(float *master, float *m, float *v, unsigned long long seed, cudaStream_t st) {
  sg_init_kernel<<<(kSgNParam + 255) / 256, 256, 0, st>>>(master, m, v, seed);
  return cudaGetLastError();
}

}  // namespace cfk
