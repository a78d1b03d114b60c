// C ABI of the MLP chemistry surrogate: training-data recording from the
// plain integrator, normalisation, training on the device (fused
// forward/backward tcgen05 kernels + Adam), parameter exchange, and the gated
// surrogate reaction step with the plain FP64 work-queue integrator as
// fallback and judge.  None of these has a counterpart in the reference.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "ctx.cuh"
#include "surrogate.cuh"

namespace cfk {
cudaError_t sg_init_attributes();
cudaError_t launch_sg_step(const Zone &z, const Mech *mc, const uint8_t *w16, const SgNorm &nrm, const SgGate &gate,
                           const SgProj &proj, double dt, unsigned *list, unsigned *list_count, SgJudge *judge,
                           unsigned *judge_count, unsigned short *revert, SgCounters *cnt, int *err, int n_sm,
                           cudaStream_t st);
cudaError_t launch_sg_judge(const Zone &z, int ns, const SgJudge *judge, const unsigned *judge_count,
                            const SgGate &gate, unsigned short *revert, SgCounters *cnt, int n_sm, cudaStream_t st);
cudaError_t launch_sg_snapshot(const Zone &z, const Thermo *th, double dt, double *snap, cudaStream_t st);
cudaError_t launch_sg_record(const Zone &z, int ns, const double *snap, double dt, float *X, float *G, cudaStream_t st);
cudaError_t launch_sg_colstats(const float *X, const float *G, long long n, const float *scales, double *acc,
                               unsigned *mm, int n_sm, cudaStream_t st);
cudaError_t launch_sg_train(const float *X, const float *G, long long n, long long perm_a, long long perm_b,
                            long long start, int count, int mode, const SgNorm &nrm, const uint8_t *w16,
                            float *partials, int max_ctas, double *loss, float *Yout, int *err, int *n_ctas,
                            cudaStream_t st);
cudaError_t launch_sg_adam(float *master, float *m, float *v, const float *partials, int n_part, uint8_t *w16,
                           float lr, float b1, float b2, float eps, float bc1, float bc2, float *grad_out, int update,
                           const int *err, cudaStream_t st);
cudaError_t launch_sg_publish(const float *master, uint8_t *w16, cudaStream_t st);
cudaError_t launch_sg_init(float *master, float *m, float *v, unsigned long long seed, cudaStream_t st);
cudaError_t launch_wu_reaction_list(const Zone &z, const Param &p, const Mech *mc, const Mech &mc_host, double dt,
                                    const unsigned int *list, const unsigned int *list_count, long long max_nodes,
                                    int *err, unsigned int *counter, int n_sm, cudaStream_t st);

struct Surrogate {
  uint8_t *w16 = nullptr;
  float *master = nullptr, *m = nullptr, *v = nullptr, *partials = nullptr;
  double *loss = nullptr;
  double *col_acc = nullptr;  // 2 x 23 sums
  unsigned *col_mm = nullptr; // 2 x 23 min/max keys
  SgCounters *cnt = nullptr;
  unsigned *counts = nullptr;  // [0] fallback list length, [1] judged, [2] work-queue counter
  unsigned *list = nullptr;
  SgJudge *judge = nullptr;
  unsigned short *revert = nullptr;
  double *snap = nullptr;
  long long cap = 0;
  SgNorm norm{};
  SgProj proj{};
  bool have_norm = false;
  long long adam_t = 0;
};

void surrogate_destroy(Surrogate *s) {
  if (!s) return;
  void *ptrs[] = {s->w16, s->master, s->m, s->v, s->partials, s->loss, s->col_acc, s->col_mm, s->cnt,
                  s->counts, s->list, s->judge, s->revert, s->snap};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete s;
}

}  // namespace cfk

using namespace cfk_detail;

namespace {

cudaError_t ensure_nodes(Surrogate *s, long long n) {
  if (s->cap >= n) return cudaSuccess;
  cudaFree(s->list);
  cudaFree(s->judge);
  cudaFree(s->revert);
  cudaFree(s->snap);
  s->list = nullptr; s->judge = nullptr; s->revert = nullptr; s->snap = nullptr; s->cap = 0;
  cudaError_t e;
  if ((e = cudaMalloc(&s->list, n * sizeof(unsigned))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&s->judge, n * sizeof(SgJudge))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&s->revert, n * sizeof(unsigned short))) != cudaSuccess) return e;
  if ((e = cudaMemset(s->revert, 0, n * sizeof(unsigned short))) != cudaSuccess) return e;
  if ((e = cudaMalloc(&s->snap, n * 21 * sizeof(double))) != cudaSuccess) return e;
  s->cap = n;
  return cudaSuccess;
}

long long zone_nodes(const cfk_ctx *c) { return (long long)c->z.d.mx * c->z.d.my * c->z.d.mz; }

int need_surrogate(cfk_ctx *c, bool need_norm) {
  if (!c->sg) return fail(c, CFK_ERR_STATE, "surrogate not initialised (cfk_surrogate_init)");
  if (need_norm && !c->sg->have_norm)
    return fail(c, CFK_ERR_STATE, "surrogate normalisation not set (cfk_surrogate_fit_normalization or set_params)");
  return CFK_OK;
}

int check_err_flags(cfk_ctx *c) {
  int h = 0;
  CFK_CHECK(c, cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
  if (h & 4) {
    cudaMemset(c->d_err, 0, sizeof(int));
    return fail(c, CFK_ERR_CUDA, "surrogate kernel: tensor-core completion wait timed out");
  }
  return CFK_OK;
}

}  // namespace

extern "C" {

int cfk_surrogate_init(cfk_ctx *c, unsigned long long seed, int n_elem, const double *elem_mu) {
  if (!c) return CFK_ERR_ARG;
  if (n_elem < 1 || n_elem > 4 || !elem_mu) return fail(c, CFK_ERR_ARG, "n_elem must be 1..4 with an element matrix");
  if (c->hp.n_spec < 1) return fail(c, CFK_ERR_STATE, "the surrogate needs a reacting mixture context");
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  CFK_CHECK(c, sg_init_attributes(), "surrogate kernel attributes");
  if (!c->sg) {
    Surrogate *s = new Surrogate();
    c->sg = s;
    cudaError_t e = cudaSuccess;
    auto al = [&](void **p, size_t bytes) {
      if (e == cudaSuccess) e = cudaMalloc(p, bytes);
      if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    al((void **)&s->w16, kSgWBytes);
    al((void **)&s->master, kSgNParam * sizeof(float));
    al((void **)&s->m, kSgNParam * sizeof(float));
    al((void **)&s->v, kSgNParam * sizeof(float));
    al((void **)&s->partials, (size_t)c->n_sm * kSgNParam * sizeof(float));
    al((void **)&s->loss, 64);
    al((void **)&s->col_acc, 2 * 23 * sizeof(double));
    al((void **)&s->col_mm, 2 * 23 * sizeof(unsigned));
    al((void **)&s->cnt, sizeof(SgCounters));
    al((void **)&s->counts, 64);
    if (e != cudaSuccess) return cuda_fail(c, e, "surrogate allocation");
  }
  Surrogate *s = c->sg;
  s->proj.n_elem = n_elem;
  for (int e = 0; e < 4; ++e)
    for (int k = 0; k < kMaxSpec; ++k)
      s->proj.mu[e][k] = (e < n_elem && k < c->hp.n_spec) ? elem_mu[e * c->hp.n_spec + k] : 0.0;
  CFK_CHECK(c, launch_sg_init(s->master, s->m, s->v, seed, 0), "surrogate init");
  CFK_CHECK(c, launch_sg_publish(s->master, s->w16, 0), "surrogate publish");
  CFK_CHECK(c, cudaDeviceSynchronize(), "surrogate init");
  s->adam_t = 0;
  return CFK_OK;
}

int cfk_surrogate_record(cfk_ctx *c, int phase, double dt, float *X, float *G, void *stream) {
  NEED_ZONE(c);
  int r = need_surrogate(c, false);
  if (r) return r;
  Surrogate *s = c->sg;
  CFK_CHECK(c, ensure_nodes(s, zone_nodes(c)), "surrogate node buffers");
  if (!(dt > 0)) return fail(c, CFK_ERR_ARG, "record needs dt > 0");
  if (phase == 0) {
    CFK_CHECK(c, launch_sg_snapshot(c->z, &c->d_mech->th, dt, s->snap, S(stream)), "surrogate snapshot");
  } else if (phase == 1) {
    if (!X || !G) return fail(c, CFK_ERR_ARG, "record needs X and G");
    CFK_CHECK(c, launch_sg_record(c->z, c->hp.n_spec, s->snap, dt, X, G, S(stream)), "surrogate record");
  } else {
    return fail(c, CFK_ERR_ARG, "phase must be 0 (before the step) or 1 (after it)");
  }
  c->launches += 1;
  return CFK_OK;
}

int cfk_surrogate_fit_normalization(cfk_ctx *c, const float *X, const float *G, long long n) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, false);
  if (r) return r;
  if (!X || !G || n < 2) return fail(c, CFK_ERR_ARG, "need X, G and n >= 2 rows");
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  Surrogate *s = c->sg;
  SgNorm &nm = s->norm;
  // asinh scales of the increments: the median |g| of each output over an
  // evenly strided sample of at most 2^18 rows (floors as below); none for
  // the log time scale
  {
    const long long stride = std::max(1LL, n / 262144);
    const long long m = (n + stride - 1) / stride;
    std::vector<float> sample((size_t)m * kSgOut);
    CFK_CHECK(c, cudaMemcpy2D(sample.data(), kSgOut * sizeof(float), G, stride * kSgOut * sizeof(float),
                              kSgOut * sizeof(float), (size_t)m, cudaMemcpyDeviceToHost),
              "target sample read");
    std::vector<float> col((size_t)m);
    for (int o = 0; o < kSgOut; ++o) {
      if (o == 10) { nm.out_scale[o] = 0.f; continue; }
      for (long long r = 0; r < m; ++r) col[r] = std::fabs(sample[r * kSgOut + o]);
      std::nth_element(col.begin(), col.begin() + m / 2, col.end());
      const double floor = o < 9 ? 1e-8 : 1e-4;
      nm.out_scale[o] = (float)std::max((double)col[m / 2], floor);
    }
  }
  CFK_CHECK(c, cudaMemset(s->col_acc, 0, 2 * 23 * sizeof(double)), "stats reset");
  std::vector<unsigned> mm0(46);
  for (int i = 0; i < 23; ++i) { mm0[2 * i] = 0xffffffffu; mm0[2 * i + 1] = 0u; }
  CFK_CHECK(c, cudaMemcpy(s->col_mm, mm0.data(), 46 * sizeof(unsigned), cudaMemcpyHostToDevice), "stats reset");
  CFK_CHECK(c, launch_sg_colstats(X, G, n, nm.out_scale, s->col_acc, s->col_mm, c->n_sm, 0), "column statistics");
  std::vector<double> acc(46);
  std::vector<unsigned> mm(46);
  CFK_CHECK(c, cudaMemcpy(acc.data(), s->col_acc, 46 * sizeof(double), cudaMemcpyDeviceToHost), "stats read");
  CFK_CHECK(c, cudaMemcpy(mm.data(), s->col_mm, 46 * sizeof(unsigned), cudaMemcpyDeviceToHost), "stats read");
  c->launches += 1;
  auto unkey = [](unsigned k) {
    const unsigned b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &b, 4);
    return (double)f;
  };
  for (int col = 0; col < 23; ++col) {
    const double mean = acc[2 * col] / n;
    const double var = std::max(acc[2 * col + 1] / n - mean * mean, 0.0);
    const double sd = std::sqrt(var);
    const double lo = unkey(mm[2 * col]), hi = unkey(mm[2 * col + 1]);
    if (col < kSgIn) {
      // a feature that is constant over the training set (up to rounding)
      // carries no information: rstd 0, and the gate compares it raw
      const bool constant = sd <= 1e-6 * std::max(1.0, std::fabs(mean));
      nm.in_mean[col] = (float)mean;
      nm.in_rstd[col] = constant ? 0.f : (float)(1.0 / sd);
      nm.in_lo[col] = constant ? 0.f : (float)((lo - mean) / sd);
      nm.in_hi[col] = constant ? 0.f : (float)((hi - mean) / sd);
    } else {
      const int o = col - kSgIn;
      // floors of the standard deviation of the learnt variable: 1e-6 for the
      // increments of unscaled columns, 1e-3 for ln tau and asinh columns
      const double floor = (o < 10 && nm.out_scale[o] == 0.f) ? 1e-6 : 1e-3;
      nm.out_mean[o] = (float)mean;
      nm.out_std[o] = (float)std::max(sd, floor);
    }
  }
  s->have_norm = true;
  return CFK_OK;
}

int cfk_surrogate_train(cfk_ctx *c, const float *X, const float *G, long long n, int epochs, int batch, double lr0,
                        double lr1, unsigned long long seed, double *loss_per_epoch) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, true);
  if (r) return r;
  if (!X || !G || n < 1 || n > 2147483647LL || epochs < 1 || batch < 1 || !(lr0 >= 0) || !(lr1 >= 0))
    return fail(c, CFK_ERR_ARG, "bad training arguments");
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  Surrogate *s = c->sg;
  std::mt19937_64 rng(seed);
  const long long steps_per_epoch = (n + batch - 1) / batch;
  const long long total = steps_per_epoch * epochs;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  long long step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    long long pa = 1, pb = 0;
    if (n > 1) {
      do { pa = (long long)(rng() % (unsigned long long)(n - 1)) + 1; } while (std::gcd(pa, n) != 1);
      pb = (long long)(rng() % (unsigned long long)n);
    }
    CFK_CHECK(c, cudaMemsetAsync(s->loss, 0, sizeof(double), 0), "loss reset");
    for (long long st = 0; st < n; st += batch, ++step) {
      const int count = (int)std::min<long long>(batch, n - st);
      int n_ctas = 0;
      CFK_CHECK(c, launch_sg_train(X, G, n, pa, pb, st, count, 0, s->norm, s->w16, s->partials, c->n_sm, s->loss,
                                   nullptr, c->d_err, &n_ctas, 0),
                "surrogate train");
      const double lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + std::cos(M_PI * (double)step / (double)total));
      s->adam_t += 1;
      const float bc1 = 1.f - std::pow(b1, (float)s->adam_t), bc2 = 1.f - std::pow(b2, (float)s->adam_t);
      CFK_CHECK(c, launch_sg_adam(s->master, s->m, s->v, s->partials, n_ctas, s->w16, (float)lr, b1, b2, eps, bc1,
                                  bc2, nullptr, 1, c->d_err, 0),
                "surrogate adam");
      c->launches += 2;
    }
    double l = 0;
    CFK_CHECK(c, cudaMemcpy(&l, s->loss, sizeof(double), cudaMemcpyDeviceToHost), "loss read");
    if (loss_per_epoch) loss_per_epoch[ep] = l / ((double)n * kSgOut);
    r = check_err_flags(c);
    if (r) return r;
  }
  return CFK_OK;
}

int cfk_surrogate_gradients(cfk_ctx *c, const float *X, const float *G, long long n, float *grad_out,
                            double *loss_out) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, true);
  if (r) return r;
  if (!X || !G || !grad_out || n < 1 || n > 2147483647LL) return fail(c, CFK_ERR_ARG, "bad gradient arguments");
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  Surrogate *s = c->sg;
  CFK_CHECK(c, cudaMemset(s->loss, 0, sizeof(double)), "loss reset");
  int n_ctas = 0;
  CFK_CHECK(c, launch_sg_train(X, G, n, 1, 0, 0, (int)n, 0, s->norm, s->w16, s->partials, c->n_sm, s->loss, nullptr,
                               c->d_err, &n_ctas, 0),
            "surrogate gradients");
  CFK_CHECK(c, launch_sg_adam(s->master, s->m, s->v, s->partials, n_ctas, s->w16, 0.f, 0.9f, 0.999f, 1e-8f, 1.f, 1.f,
                              grad_out, 0, nullptr, 0),
            "gradient reduction");
  c->launches += 2;
  CFK_CHECK(c, cudaDeviceSynchronize(), "surrogate gradients");
  if (loss_out) {
    double l = 0;
    CFK_CHECK(c, cudaMemcpy(&l, s->loss, sizeof(double), cudaMemcpyDeviceToHost), "loss read");
    *loss_out = l / ((double)n * kSgOut);
  }
  return check_err_flags(c);
}

int cfk_surrogate_forward(cfk_ctx *c, const float *X, long long n, float *Y) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, true);
  if (r) return r;
  if (!X || !Y || n < 1 || n > 2147483647LL) return fail(c, CFK_ERR_ARG, "bad forward arguments");
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  Surrogate *s = c->sg;
  int n_ctas = 0;
  CFK_CHECK(c, launch_sg_train(X, X, n, 1, 0, 0, (int)n, 1, s->norm, s->w16, s->partials, c->n_sm, s->loss, Y,
                               c->d_err, &n_ctas, 0),
            "surrogate forward");
  c->launches += 1;
  CFK_CHECK(c, cudaDeviceSynchronize(), "surrogate forward");
  return check_err_flags(c);
}

int cfk_surrogate_get_params(cfk_ctx *c, float *weights, float *norm) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, false);
  if (r) return r;
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  if (weights)
    CFK_CHECK(c, cudaMemcpy(weights, c->sg->master, kSgNParam * sizeof(float), cudaMemcpyDeviceToHost), "weights read");
  if (norm) std::memcpy(norm, &c->sg->norm, sizeof(SgNorm));
  return CFK_OK;
}

int cfk_surrogate_set_params(cfk_ctx *c, const float *weights, const float *norm) {
  if (!c) return CFK_ERR_ARG;
  int r = need_surrogate(c, false);
  if (r) return r;
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  Surrogate *s = c->sg;
  if (weights) {
    CFK_CHECK(c, cudaMemcpy(s->master, weights, kSgNParam * sizeof(float), cudaMemcpyHostToDevice), "weights write");
    CFK_CHECK(c, cudaMemset(s->m, 0, kSgNParam * sizeof(float)), "moments reset");
    CFK_CHECK(c, cudaMemset(s->v, 0, kSgNParam * sizeof(float)), "moments reset");
    CFK_CHECK(c, launch_sg_publish(s->master, s->w16, 0), "surrogate publish");
    CFK_CHECK(c, cudaDeviceSynchronize(), "surrogate publish");
    s->adam_t = 0;
  }
  if (norm) {
    std::memcpy(&s->norm, norm, sizeof(SgNorm));
    for (int i = 0; i < kSgOut; ++i)
      if (!(s->norm.out_std[i] > 0)) return fail(c, CFK_ERR_ARG, "output standard deviations must be positive");
    s->have_norm = true;
  }
  return CFK_OK;
}

int cfk_surrogate_default_gate(cfk_surrogate_gate *g) {
  if (!g) return CFK_ERR_ARG;
  g->ood_margin = 0.0;
  g->dT_max = 5.0;
  g->dT_consistency = 0.5;
  g->judge_tol_T = 1.0;
  g->judge_tol_bc = 5e-3;
  g->min_substeps = 50.0;
  g->judge_stride = 64;
  g->revert_steps = 50;
  return CFK_OK;
}

int cfk_surrogate_reaction_step(cfk_ctx *c, double dt, const cfk_surrogate_gate *gate, int step_index,
                                cfk_surrogate_stats *stats, void *stream) {
  NEED_ZONE(c);
  int r = need_surrogate(c, true);
  if (r) return r;
  if (!c->have_mech || c->hp.n_reac == 0) return fail(c, CFK_ERR_STATE, "no reacting mechanism loaded");
  if (!gate || !(dt > 0)) return fail(c, CFK_ERR_ARG, "need a gate and dt > 0");
  if (gate->judge_stride < 0 || gate->revert_steps < 0) return fail(c, CFK_ERR_ARG, "bad gate");
  if (c->hp.chem_advance_method != 0 && c->hp.chem_advance_method != 1)
    return fail(c, CFK_ERR_ARG, "chem_advance_method must be 0 (explicit) or 1 (point implicit)");
  Surrogate *s = c->sg;
  const long long n = zone_nodes(c);
  CFK_CHECK(c, ensure_nodes(s, n), "surrogate node buffers");
  cudaStream_t st = S(stream);
  SgGate g;
  g.ood_margin = gate->ood_margin;
  g.dT_max = gate->dT_max;
  g.dT_consistency = gate->dT_consistency;
  g.judge_tol_T = gate->judge_tol_T;
  g.judge_tol_bc = gate->judge_tol_bc;
  g.min_substeps = gate->min_substeps;
  g.judge_stride = gate->judge_stride;
  g.judge_salt = gate->judge_stride > 0 ? (int)((unsigned)step_index * 40503u % (unsigned)gate->judge_stride) : 0;
  g.revert_steps = gate->revert_steps;
  CFK_CHECK(c, cudaMemsetAsync(s->counts, 0, 16, st), "surrogate counters");
  CFK_CHECK(c, cudaMemsetAsync(s->cnt, 0, sizeof(SgCounters), st), "surrogate counters");
  CFK_CHECK(c, launch_sg_step(c->z, c->d_mech, s->w16, s->norm, g, s->proj, dt, s->list, s->counts, s->judge,
                              s->counts + 1, s->revert, s->cnt, c->d_err, c->n_sm, st),
            "surrogate step");
  CFK_CHECK(c, launch_wu_reaction_list(c->z, c->p, c->d_mech, c->h_mech, dt, s->list, s->counts, n, c->d_err,
                                       s->counts + 2, c->n_sm, st),
            "fallback reaction step");
  c->launches += 2;
  if (g.judge_stride > 0) {
    CFK_CHECK(c, launch_sg_judge(c->z, c->hp.n_spec, s->judge, s->counts + 1, g, s->revert, s->cnt, c->n_sm, st),
              "surrogate judge");
    c->launches += 1;
  }
  if (stats) {
    SgCounters h;
    CFK_CHECK(c, cudaMemcpyAsync(&h, s->cnt, sizeof(SgCounters), cudaMemcpyDeviceToHost, st), "stats read");
    CFK_CHECK(c, cudaStreamSynchronize(st), "stats read");
    stats->cells = (long long)h.n[SG_CELLS];
    stats->surrogate = (long long)h.n[SG_SURROGATE];
    stats->fallback_ood = (long long)h.n[SG_OOD];
    stats->fallback_ignition = (long long)h.n[SG_IGNITION];
    stats->fallback_consistency = (long long)h.n[SG_CONSISTENCY];
    stats->fallback_revert = (long long)h.n[SG_REVERT];
    stats->fallback_newton = (long long)h.n[SG_NEWTON_FAILED];
    stats->fallback_cheap = (long long)h.n[SG_CHEAP];
    stats->judged = (long long)h.n[SG_JUDGED];
    stats->judge_failed = (long long)h.n[SG_JUDGE_FAILED];
    double mx, my;
    std::memcpy(&mx, &h.judge_max_dT_bits, 8);
    std::memcpy(&my, &h.judge_max_dbc_bits, 8);
    stats->judge_max_dT = mx;
    stats->judge_max_dbc = my;
    stats->judge_mean_dT = h.n[SG_JUDGED] ? h.judge_sum_dT / (double)h.n[SG_JUDGED] : 0.0;
    return check_err_flags(c);
  }
  return CFK_OK;
}

}  // extern "C"
