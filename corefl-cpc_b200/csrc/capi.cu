// C ABI of the library: context, zone binding, per-stage entry points, whole
// RK3 steps (plain and CUDA-graph replayed) and host<->device helpers.
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "ctx.cuh"

namespace cfk {
cudaError_t launch_weno_air(const Zone &z, const Param &p, const int *var, cudaStream_t st, int *n_launch);
cudaError_t launch_weno_air_dir(const Zone &z, const Param &p, int dir, int var, cudaStream_t st);
cudaError_t weno_air_init_attributes();
cudaError_t launch_pv_air(const Zone &z, const Param &p, cudaStream_t st, int *n_launch);
cudaError_t launch_pv_mix(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st, int *n_launch);
cudaError_t pv_mix_init_attributes();
cudaError_t pv_air_init_attributes();
cudaError_t launch_weno_mix(const Zone &z, const Param &p, const Thermo &th, const double *dt_dev, double dt_host,
                            const int *var, cudaStream_t st, int *n_launch);
cudaError_t launch_weno_mix_dir(const Zone &z, const Param &p, const Thermo &th, const double *dt_dev,
                                double dt_host, int dir, int var, cudaStream_t st);
cudaError_t weno_mix_init_attributes();
cudaError_t launch_viscous_mix(const Zone &z, const Param &p, const Thermo &th, cudaStream_t st, int *n_launch);
cudaError_t viscous_mix_init_attributes();
cudaError_t launch_viscous_air(const Zone &z, const Param &p, cudaStream_t st, int *n_launch, int var);
cudaError_t viscous_air_init_attributes();
cudaError_t launch_update_rk(const Zone &z, const Param &p, const Thermo *th, double dt, const double *dt_dev,
                             int rk, int *err, cudaStream_t st, bool minus_cn = false, bool with_props = false);
cudaError_t launch_cv_from_bv(const Zone &z, const Param &p, const Thermo *th, cudaStream_t st);
cudaError_t launch_update_properties(const Zone &z, const Param &p, const Thermo *th, cudaStream_t st,
                                     bool shell = false, bool planar = false);
cudaError_t launch_local_dt(const Zone &z, const Param &p, const Thermo *th, unsigned long long *dt_bits,
                            cudaStream_t st, bool with_reaction = true);
cudaError_t launch_limit_flow(const Zone &z, const Param &p, const Thermo *th, unsigned char *bad,
                              unsigned long long *n_fixed, cudaStream_t st);
cudaError_t launch_boundary_conditions(const Zone &z, const Param &p, const Thermo *th, const cfk_face *faces,
                                       int n_face, const cfk_wall &wall, const cfk_inflow &inflow,
                                       const cfk_outflow &outflow, cudaStream_t st, int *n_launch);
cudaError_t launch_finite_rate_chemistry(const Zone &z, const Mech *mc, cudaStream_t st);
long long halo_doubles(const Dims &d, const Param &p, int face);
cudaError_t launch_halo_pack(const Zone &z, const Param &p, int face, int direction, double *buf, cudaStream_t st);
cudaError_t launch_halo_assign(const Zone &z, const Param &p, const Thermo *th, int face, int direction,
                               const double *buf, cudaStream_t st);
cudaError_t launch_eliminate_k_gradient(const Zone &z, const Param &p, cudaStream_t st);
cudaError_t launch_inner_communication(const Zone &z, const Zone &tz, const Param &p, const Thermo *th,
                                       const cfk_inner_face &f, cudaStream_t st);
cudaError_t launch_shock_sensor(const Zone &z, const Param &p, cudaStream_t st);
cudaError_t launch_viscous8(const Zone &z, const Param &p, const Thermo *th, const cfk_face *faces, int n_face,
                            double *fvis, cudaStream_t st, int *n_launch);
cudaError_t launch_wu_reaction(const Zone &z, const Param &p, const Mech *mc, const Mech &mc_host, double dt,
                               int schedule, int *nsub_out, int *err, unsigned int *counter, int n_sm,
                               cudaStream_t st);
}  // namespace cfk

using namespace cfk;
using namespace cfk_detail;

namespace {
const char *const kPhaseName[CFK_NPHASE] = {"cfk inviscid flux", "cfk viscous flux", "cfk update",
                                            "cfk boundary conditions", "cfk properties", "cfk time step",
                                            "cfk reaction"};

// One phase of a step: an NVTX range named after it (visible to Nsight
// Systems; inert when no tool is attached) and, with profiling on, CUDA
// events around the launches issued in its scope.
struct PhaseScope {
  cfk_ctx *c;
  int phase;
  cudaStream_t st;
  int *n;
  int n0;
  cudaEvent_t a = nullptr;
  PhaseScope(cfk_ctx *c_, int ph, cudaStream_t s, int *n_) : c(c_), phase(ph), st(s), n(n_), n0(*n_) {
    nvtxRangePushA(kPhaseName[ph]);
    if (c->profiling) { a = c->take_event(); cudaEventRecord(a, st); }
  }
  ~PhaseScope() {
    nvtxRangePop();
    if (!c->profiling) return;
    cudaEvent_t b = c->take_event();
    cudaEventRecord(b, st);
    c->recs.push_back({phase, a, b, (long long)(*n - n0)});
  }
};
}  // namespace

namespace {

// Ghost layers the inviscid scheme reads (reference src/Parameter.cpp:196-252):
// 4 for WENO7, 3 for WENO5, 2 for the primitive-variable schemes; none for
// chemistry-only contexts.
int ghost_layers(int scheme, int viscous_order) {
  int g = scheme == 0 ? 0 : 2;
  if (scheme == 71 || scheme == 72) g = 4;
  if (scheme == 51 || scheme == 52) g = 3;
  if (viscous_order == 8 && g < 4) g = 4;  // 8th-order viscous stencil (reference src/Parameter.cpp:298-300)
  return g;
}

// compute_inviscid_flux dispatch (reference src/InviscidScheme.cu:12-26);
// th: host copy of the mixture tables, nullptr for air.  dt_dev / dt_host:
// the step's dt (DParameter::dt) for the positive-preserving limiter.
cudaError_t launch_inviscid(const Zone &z, const Param &p, const Thermo *th, const double *dt_dev, double dt_host,
                            const int *var, cudaStream_t st, int *n) {
  if (p.inviscid_scheme == 52 || p.inviscid_scheme == 72)
    return th ? launch_weno_mix(z, p, *th, dt_dev, dt_host, var, st, n) : launch_weno_air(z, p, var, st, n);
  return th ? launch_pv_mix(z, p, *th, st, n) : launch_pv_air(z, p, st, n);
}

// compute_viscous_flux dispatch (reference src/ViscousScheme.cu:7-73): the
// 2nd-order face scheme or the 8th-order collocated one.
cudaError_t launch_viscous(const Zone &z, const Param &p, const Thermo *th, const cfk_face *faces, int n_face,
                           cudaStream_t st, int *n, int visc_var = 0) {
  if (p.viscous_order == 8 || p.viscous_order == 4) return launch_viscous8(z, p, th, faces, n_face, z.fvis8, st, n);
  return th ? launch_viscous_mix(z, p, *th, st, n) : launch_viscous_air(z, p, st, n, visc_var);
}

int validate(const cfk_param *p, std::string &why) {
  if (p->dim != 2 && p->dim != 3) { why = "dim must be 2 or 3"; return -1; }
  if (p->n_spec < 0 || p->n_spec > kMaxSpec) { why = "n_spec out of range (0..9)"; return -1; }
  if (p->n_var != 5 + p->n_scalar) { why = "n_var must equal 5 + n_scalar"; return -1; }
  if (p->n_scalar < p->n_spec) { why = "n_scalar must be >= n_spec"; return -1; }
  const int s = p->inviscid_scheme;
  if (!(s == 52 || s == 72 || s == 0 || (s >= 1 && s <= 4))) {
    why = "inviscid_scheme " + std::to_string(s) + " is not supported by this build";
    return -1;
  }
  if (s >= 1 && s <= 4 && !(p->reconstruction >= 1 && p->reconstruction <= 3)) {
    why = "reconstruction must be 1 (first order), 2 (MUSCL) or 3 (NND2) for inviscid_scheme 1-4";
    return -1;
  }
  if (s >= 1 && s <= 4 && !(p->limiter == 0 || p->limiter == 1)) { why = "limiter must be 0 or 1"; return -1; }
  if (s == 2 && !(p->entropy_fix_factor >= 0)) { why = "entropy_fix_factor must be >= 0"; return -1; }
  if (p->viscous_order != 0 && p->viscous_order != 2 && p->viscous_order != 4 && p->viscous_order != 8) {
    why = "viscous_order must be 0, 2, 4 or 8";
    return -1;
  }
  if (p->sensor_threshold > 1e-10 && !(s == 52 || s == 72)) {
    why = "shockSensor_threshold > 0 (hybrid scheme) needs inviscid_scheme 52 or 72";
    return -1;
  }
  if (p->sensor_threshold > 1e-10 && !(p->shock_sensor >= 0 && p->shock_sensor <= 2)) {
    why = "shock_sensor must be 0 (Ducros), 1 (Jameson) or 2 (density/pressure jump)";
    return -1;
  }
  if (p->positive_preserving && p->n_spec > 0 && !(s == 52 || s == 72 || s == 0)) {
    why = "positive_preserving is supported with the WENO schemes (52, 72)";
    return -1;
  }
  if (p->n_spec > 0 && s == 1) {
    why = "the Lax-Friedrichs flux has no mixture form (the reference leaves it unimplemented); use 2, 3 or 4";
    return -1;
  }
  if (p->n_spec > 0 && s != 0 && p->n_spec != kMaxSpec) {
    why = "the mixture flux kernels are built for 9 species";
    return -1;
  }
  if (p->n_spec > 0 && p->n_scalar != p->n_spec) {
    why = "passive scalars beside the species are not supported (n_scalar must equal n_spec)";
    return -1;
  }
  if (p->gradPInDiffusionFlux != 0 && p->gradPInDiffusionFlux != 1) {
    why = "gradPInDiffusionFlux must be 0 or 1";
    return -1;
  }
  if (s == 0 && p->n_spec == 0) { why = "inviscid_scheme 0 (no flux) is for reacting mixtures only"; return -1; }
  if (p->n_face < 0 || p->n_face > 6) { why = "n_face must be 0..6"; return -1; }
  // The WENO weights are normalised through products of two (eps + beta)^2
  // terms; eps = 1e-40 * weno_eps_scale must stay above 1e-70 so that those
  // products (>= eps^4) remain normal numbers.
  if ((s == 52 || s == 72) && !(p->weno_eps_scale >= 1e-30)) {
    why = "weno_eps_scale must be >= 1e-30 ((rho_ref*v_ref)^2)";
    return -1;
  }
  for (int n = 0; n < p->n_face; ++n) {
    const cfk_face &f = p->faces[n];
    if (f.face < 0 || f.face > 2 || (f.direction != -1 && f.direction != 1) ||
        !(f.label == 6 || f.label == 8 || f.label == 3 || f.label == 2 || f.label == 5)) {
      why = "unsupported boundary face description";
      return -1;
    }
    if (f.label == 6 && p->outflow.back_pressure_on) {
      if (p->outflow.back_pressure_on != 1 || !(p->outflow.back_pressure > 0)) {
        why = "outflow back pressure: back_pressure_on must be 0 or 1 and back_pressure > 0";
        return -1;
      }
    }
    if (f.label == 5) {
      const cfk_inflow &q = p->inflow;
      if (!(q.density > 0) || !(q.pressure > 0) || !(q.temperature > 0) || (p->n_spec > 0 && !(q.mw > 0)) ||
          (q.subsonic != 0 && q.subsonic != 1)) {
        why = "inflow needs density, pressure, temperature (and mw for mixtures) > 0 and subsonic 0 or 1";
        return -1;
      }
      if (q.inflow_type != 0 && q.inflow_type != 2) {
        why = "inflow_type must be 0 (constant) or 2 (mixing layer); profile inflows are not supported";
        return -1;
      }
      if (q.inflow_type == 2 && (!(q.density_lower > 0) || !(q.p_lower > 0) || !(q.t_lower > 0) ||
                                 !(q.delta_omega > 0))) {
        why = "mixing-layer inflow needs density_lower, p_lower, t_lower and delta_omega > 0";
        return -1;
      }
      if (q.fluctuation_type != 0 && q.fluctuation_type != 1) {
        why = "inflow fluctuation_type must be 0 or 1 (white noise)";
        return -1;
      }
    }
    if (f.label == 2) {
      const cfk_wall &w = p->wall;
      if (w.thermal_type != 0 && w.thermal_type != 1) {
        why = "wall thermal_type must be 0 (isothermal) or 1 (adiabatic); equilibrium radiation needs the "
              "wall-distance field, which this path does not carry";
        return -1;
      }
      if (w.thermal_type == 0 && !(w.temperature > 0)) { why = "isothermal wall needs temperature > 0"; return -1; }
      if (p->n_spec > 0 && w.catalytic_type != 0 && w.catalytic_type != 1) {
        why = "wall catalytic_type must be 0 (non-catalytic) or 1 (fully catalytic)";
        return -1;
      }
    }
  }
  return 0;
}

}  // namespace

extern "C" {

int cfk_create(const cfk_param *param, cfk_ctx **out) {
  if (!param || !out) return CFK_ERR_ARG;
  *out = nullptr;
  std::string why;
  if (validate(param, why) != 0) {
    fprintf(stderr, "cfk_create: %s\n", why.c_str());
    return CFK_ERR_ARG;
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    fprintf(stderr, "cfk_create: no CUDA device (%s)\n", cudaGetErrorString(e));
    return CFK_ERR_CUDA;
  }
  if (param->device < 0 || param->device >= ndev) {
    fprintf(stderr, "cfk_create: device %d out of range (%d devices)\n", param->device, ndev);
    return CFK_ERR_ARG;
  }
  e = cudaSetDevice(param->device);
  if (e != cudaSuccess) return CFK_ERR_CUDA;
  e = weno_air_init_attributes();
  if (e == cudaSuccess) e = pv_air_init_attributes();
  if (e == cudaSuccess) e = pv_mix_init_attributes();
  if (e == cudaSuccess) e = viscous_air_init_attributes();
  if (e == cudaSuccess) e = weno_mix_init_attributes();
  if (e == cudaSuccess) e = viscous_mix_init_attributes();
  if (e != cudaSuccess) {
    fprintf(stderr, "cfk_create: kernel attribute setup failed (%s)\n", cudaGetErrorString(e));
    return CFK_ERR_CUDA;
  }
  cfk_ctx *c = new cfk_ctx();
  c->hp = *param;
  Param &p = c->p;
  p.dim = param->dim; p.n_var = param->n_var; p.n_spec = param->n_spec; p.n_scalar = param->n_scalar;
  p.n_reac = param->n_reac; p.inviscid_scheme = param->inviscid_scheme; p.reconstruction = param->reconstruction;
  p.limiter = param->limiter; p.viscous_order = param->viscous_order;
  p.positive_preserving = param->positive_preserving; p.gradPInDiffusionFlux = param->gradPInDiffusionFlux;
  p.fixed_dt = param->fixed_dt; p.entropy_fix_factor = param->entropy_fix_factor; p.Pr = param->Pr;
  p.Sc = param->Sc; p.cfl = param->cfl; p.weno_eps_scale = param->weno_eps_scale; p.v_ref = param->v_ref;
  p.rho_ref = param->rho_ref;
  p.chem_advance_method = param->chem_advance_method;
  p.shock_sensor = param->shock_sensor; p.sensor_eps = param->sensor_eps;
  p.sensor_threshold = param->sensor_threshold;
  p.limit_flow = param->limit_flow;
  for (int l = 0; l < 5; ++l) {
    p.limit_ll[l] = param->limit_ll[l];
    p.limit_ul[l] = param->limit_ul[l];
  }
  // starting tile shapes and viscous form (cfk_autotune_tiles may change
  // them): for air the ones the tuner picks on large 3-D blocks (x 31x8,
  // y/z 31x16; the ring form with the L2 prefetch), for mixtures the first
  // shape of each sweep
  if (p.n_spec == 0) {
    c->tile_var[0] = 2;
    c->tile_var[1] = 1;
    c->tile_var[2] = 1;
  }
  c->visc_var = 2;
  e = cudaMalloc(&c->d_dt_bits, 64);
  if (e != cudaSuccess) { delete c; return CFK_ERR_CUDA; }
  c->d_err = reinterpret_cast<int *>(reinterpret_cast<char *>(c->d_dt_bits) + 8);
  cudaMemset(c->d_dt_bits, 0, 64);
  e = cudaMalloc(&c->d_mech, sizeof(Mech));
  if (e != cudaSuccess) { cudaFree(c->d_dt_bits); delete c; return CFK_ERR_CUDA; }
  cudaMemset(c->d_mech, 0, sizeof(Mech));
  cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, param->device);
  *out = c;
  return CFK_OK;
}

int cfk_destroy(cfk_ctx *c) {
  if (!c) return CFK_OK;
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->sg) surrogate_destroy(c->sg);
  for (auto &r : c->recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  for (auto e : c->pool) cudaEventDestroy(e);
  for (void *ptr : c->owned) cudaFree(ptr);
  if (c->own_sensor) cudaFree(c->own_sensor);
  if (c->own_fvis8) cudaFree(c->own_fvis8);
  if (c->own_limit) cudaFree(c->own_limit);
  cudaFree(c->d_dt_bits);
  cudaFree(c->d_mech);
  delete c;
  return CFK_OK;
}

const char *cfk_last_error(const cfk_ctx *c) { return c ? c->err.c_str() : "null context"; }

// limit_flow's flag per interior node, owned by the context.
static int ensure_limit_flags(cfk_ctx *c) {
  const size_t n = (size_t)c->z.d.plane(0);
  if (c->own_limit_n >= n) return CFK_OK;
  if (c->own_limit) cudaFree(c->own_limit);
  c->own_limit = nullptr;
  c->own_limit_n = 0;
  CFK_CHECK(c, cudaMalloc(&c->own_limit, n), "limit_flow flag allocation");
  c->own_limit_n = n;
  return CFK_OK;
}

// Device counter of the nodes limit_flow repaired (in the context's scratch line).
static unsigned long long *limit_counter(cfk_ctx *c) {
  return reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(c->d_dt_bits) + 24);
}

int cfk_bind_zone(cfk_ctx *c, const cfk_zone *zn) {
  if (!c || !zn) return CFK_ERR_ARG;
  if (zn->mx < 1 || zn->my < 1 || zn->mz < 1) return fail(c, CFK_ERR_ARG, "zone extents must be positive");
  const int need_g = ghost_layers(c->hp.inviscid_scheme, c->hp.viscous_order);
  if (zn->ngg < need_g) return fail(c, CFK_ERR_ARG, "ngg too small for the inviscid or viscous scheme");
  if ((c->hp.dim == 2) != (zn->mz == 1)) return fail(c, CFK_ERR_ARG, "dim does not match mz");
  if (c->hp.inviscid_scheme != 0 && (!zn->cv || !zn->bv || !zn->qn || !zn->dq || !zn->metric || !zn->jac))
    return fail(c, CFK_ERR_ARG, "cv, bv, qn, dq, metric and jac are required");
  if (c->hp.n_spec > 0 && (!zn->cv || !zn->bv || !zn->sv || !zn->jac || !zn->reaction_timeScale))
    return fail(c, CFK_ERR_ARG, "cv, bv, sv, jac and reaction_timeScale are required for reacting mixtures");
  if (c->hp.n_spec > 0 && c->hp.inviscid_scheme != 0 &&
      (!zn->acoustic_speed || !zn->gamma || !zn->mul || !zn->thermal_conductivity || !zn->rho_D))
    return fail(c, CFK_ERR_ARG,
                "acoustic_speed, gamma, mul, thermal_conductivity and rho_D are required for the mixture flow path");
  if (c->hp.viscous_order > 0 && !zn->mul) return fail(c, CFK_ERR_ARG, "mul is required for viscous runs");
  if (c->hp.positive_preserving && c->hp.n_spec > 0 && !zn->dt_local)
    return fail(c, CFK_ERR_ARG, "dt_local is required with positive_preserving");
  if (c->hp.n_scalar > 0 && !zn->sv) return fail(c, CFK_ERR_ARG, "sv is required when n_scalar > 0");
  // 32-bit plane extents, as in the reference's int indexing
  const double P = (double)(zn->mx + 2 * zn->ngg) * (zn->my + 2 * zn->ngg) * (zn->mz + 2 * zn->ngg);
  if (P * c->hp.n_var > 2147483647.0) return fail(c, CFK_ERR_ARG, "block too large for 32-bit plane indexing");
  Zone &z = c->z;
  z.d = Dims{zn->mx, zn->my, zn->mz, zn->ngg};
  z.jac = zn->jac; z.metric = zn->metric; z.cv = zn->cv; z.bv = zn->bv; z.sv = zn->sv; z.qn = zn->qn;
  z.mul = zn->mul; z.mach = zn->mach; z.acoustic_speed = zn->acoustic_speed; z.gamma = zn->gamma;
  z.thermal_conductivity = zn->thermal_conductivity; z.rho_D = zn->rho_D;
  z.reaction_timeScale = zn->reaction_timeScale; z.dq = zn->dq; z.dt_local = zn->dt_local; z.Cn = zn->Cn;
  z.shock_sensor = zn->shock_sensor;
  z.fvis8 = nullptr;
  z.y = zn->y;
  z.inflow_draws = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(c->d_dt_bits) + 32);
  for (int n = 0; n < c->hp.n_face; ++n)
    if (c->hp.faces[n].label == 5 && c->hp.inflow.inflow_type == 2 && !zn->y)
      return fail(c, CFK_ERR_ARG, "the mixing-layer inflow needs the zone's y plane");
  if (c->hp.viscous_order == 8 || c->hp.viscous_order == 4) {
    // node fluxes of the collocated viscous schemes, owned by the context
    const size_t n8 = (size_t)z.d.plane(z.d.ngg) * 3 * (c->hp.n_var - 1);
    if (c->own_fvis8_n < n8) {
      if (c->own_fvis8) cudaFree(c->own_fvis8);
      c->own_fvis8 = nullptr;
      c->own_fvis8_n = 0;
      CFK_CHECK(c, cudaMalloc(&c->own_fvis8, n8 * sizeof(double)), "8th-order viscous flux allocation");
      c->own_fvis8_n = n8;
    }
    CFK_CHECK(c, cudaMemset(c->own_fvis8, 0, n8 * sizeof(double)), "8th-order viscous flux reset");
    z.fvis8 = c->own_fvis8;
  }
  if (c->p.sensor_threshold > 1e-10 && !z.shock_sensor) {
    // the hybrid scheme needs a sensor array whose ghost layers are zero
    // (reference src/Field.cu:526, allocated with cudaMemset 0)
    const size_t P = (size_t)z.d.plane(z.d.ngg);
    if (c->own_sensor_n < P) {
      if (c->own_sensor) cudaFree(c->own_sensor);
      c->own_sensor = nullptr;
      c->own_sensor_n = 0;
      CFK_CHECK(c, cudaMalloc(&c->own_sensor, P * sizeof(double)), "shock sensor allocation");
      c->own_sensor_n = P;
    }
    CFK_CHECK(c, cudaMemset(c->own_sensor, 0, P * sizeof(double)), "shock sensor reset");
    z.shock_sensor = c->own_sensor;
  }
  if (c->p.limit_flow) {
    if (int r = ensure_limit_flags(c)) return r;
  }
  c->bound = true;
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  return CFK_OK;
}

int cfk_alloc_zone(cfk_ctx *c, int mx, int my, int mz, cfk_zone *out) {
  if (!c || !out) return CFK_ERR_ARG;
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  const int g = ghost_layers(c->hp.inviscid_scheme, c->hp.viscous_order);
  cfk_zone zn{};
  zn.mx = mx; zn.my = my; zn.mz = mz; zn.ngg = g;
  const size_t P = (size_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g), N = (size_t)mx * my * mz;
  const int nv = c->hp.n_var, ns = c->hp.n_spec, nsc = c->hp.n_scalar;
  auto al = [&](double **ptr, size_t n) -> bool {
    if (n == 0) { *ptr = nullptr; return true; }
    void *v = nullptr;
    if (cudaMalloc(&v, n * sizeof(double)) != cudaSuccess) return false;
    cudaMemset(v, 0, n * sizeof(double));
    c->owned.push_back(v);
    *ptr = static_cast<double *>(v);
    return true;
  };
  bool ok = al(&zn.jac, P) && al(&zn.metric, 9 * P) && al(&zn.cv, nv * P) && al(&zn.bv, 6 * P) &&
            al(&zn.sv, nsc * P) && al(&zn.qn, nv * P) && al(&zn.mul, P) && al(&zn.mach, P) &&
            al(&zn.dq, nv * N) && al(&zn.dt_local, N) && al(&zn.y, P);
  if (ok && c->hp.sensor_threshold > 1e-10) ok = al(&zn.shock_sensor, P);
  if (ok && ns > 0)
    ok = al(&zn.acoustic_speed, P) && al(&zn.gamma, P) && al(&zn.thermal_conductivity, P) && al(&zn.rho_D, ns * P) &&
         al(&zn.reaction_timeScale, P) && al(&zn.Cn, nv * N);
  if (!ok) return fail(c, CFK_ERR_CUDA, "cudaMalloc failed in cfk_alloc_zone");
  *out = zn;
  return cfk_bind_zone(c, &zn);
}

static const Thermo *thermo_of(cfk_ctx *c) { return c->have_mech ? &c->d_mech->th : nullptr; }
// host copy of the mixture tables for kernels that take them by value
static const Thermo *thermo_host(cfk_ctx *c) { return c->have_mech ? &c->h_mech.th : nullptr; }
static int need_mech_for_mixture(cfk_ctx *c) {
  if (c->hp.n_spec > 0 && !c->have_mech) return fail(c, CFK_ERR_STATE, "mixture context without a mechanism");
  return CFK_OK;
}

int cfk_set_mechanism(cfk_ctx *c, const cfk_mechanism *m) {
  if (!c || !m) return CFK_ERR_ARG;
  if (m->n_spec != c->hp.n_spec) return fail(c, CFK_ERR_ARG, "mechanism n_spec differs from the context's n_spec");
  if (m->n_spec < 1 || m->n_spec > kMaxSpec || m->n_reac < 0 || m->n_reac > kMaxReac)
    return fail(c, CFK_ERR_ARG, "mechanism size out of range");
  if (m->n_reac != c->hp.n_reac) return fail(c, CFK_ERR_ARG, "mechanism n_reac differs from the context's n_reac");
  Mech h;
  std::memset(&h, 0, sizeof(h));
  Thermo &th = h.th;
  const int ns = m->n_spec;
  th.n_spec = ns;
  const double R_u = 8314.462618;
  for (int l = 0; l < ns; ++l) {
    th.mw[l] = m->mw[l];
    th.imw[l] = 1.0 / m->mw[l];
    th.gas_const[l] = R_u / m->mw[l];
    th.t_low[l] = m->t_low[l]; th.t_mid[l] = m->t_mid[l]; th.t_high[l] = m->t_high[l];
    for (int q = 0; q < 7; ++q) { th.low[l][q] = m->low[l][q]; th.high[l][q] = m->high[l][q]; }
    th.geometry[l] = m->geometry[l];
    th.LJ_potent_inv[l] = m->LJ_potent_inv[l];
    th.vis_coeff[l] = m->vis_coeff[l];
    th.ZRotF298[l] = m->ZRotF298[l];
    for (int n = 0; n < ns; ++n) {
      th.WjDivWi_to_One4th[l][n] = m->WjDivWi_to_One4th[l][n];
      th.sqrt_WiDivWjPl1Mul8[l][n] = m->sqrt_WiDivWjPl1Mul8[l][n];
      th.binary_diffusivity_coeff[l][n] = m->binary_diffusivity_coeff[l][n];
      th.kb_over_eps_jk[l][n] = m->kb_over_eps_jk[l][n];
    }
  }
  Kinetics &kn = h.kn;
  kn.n_reac = m->n_reac;
  for (int r = 0; r < m->n_reac; ++r) {
    kn.type[r] = m->reac_type[r];
    kn.rev[r] = m->rev_type[r];
    kn.order[r] = m->order[r];
    kn.A[r] = m->A[r]; kn.b[r] = m->b[r]; kn.Ea[r] = m->Ea[r];
    kn.A2[r] = m->A2[r]; kn.b2[r] = m->b2[r]; kn.Ea2[r] = m->Ea2[r];
    kn.troe_alpha[r] = m->troe_alpha[r]; kn.troe_t3[r] = m->troe_t3[r];
    kn.troe_t1[r] = m->troe_t1[r]; kn.troe_t2[r] = m->troe_t2[r];
    int n = 0;
    for (int l = 0; l < ns; ++l) {
      kn.tb[r][l] = m->third_body_coeff[r][l];
      if (m->stoi_f[r][l] != 0 || m->stoi_b[r][l] != 0) {
        if (n == kMaxInvolved) return fail(c, CFK_ERR_ARG, "a reaction involves more than 6 species");
        if (m->stoi_f[r][l] < 0 || m->stoi_b[r][l] < 0 || m->stoi_f[r][l] > 127 || m->stoi_b[r][l] > 127)
          return fail(c, CFK_ERR_ARG, "stoichiometric coefficient out of range");
        kn.inv_sp[r][n] = l;
        kn.inv_f[r][n] = m->stoi_f[r][l];
        kn.inv_b[r][n] = m->stoi_b[r][l];
        kn.stf[r][l] = (signed char)m->stoi_f[r][l];
        kn.stb[r][l] = (signed char)m->stoi_b[r][l];
        kn.inv_mask[r] |= 1u << l;
        if (m->stoi_f[r][l] != m->stoi_b[r][l]) kn.net_mask[r] |= 1u << l;
        ++n;
      }
    }
    kn.n_inv[r] = n;
  }
  CFK_CHECK(c, cudaSetDevice(c->hp.device), "cudaSetDevice");
  CFK_CHECK(c, cudaMemcpy(c->d_mech, &h, sizeof(Mech), cudaMemcpyHostToDevice), "mechanism upload");
  c->h_mech = h;
  c->have_mech = true;
  return CFK_OK;
}

int cfk_finite_rate_chemistry(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (!c->have_mech || c->hp.n_reac == 0) return fail(c, CFK_ERR_STATE, "no reacting mechanism loaded");
  if (!c->z.dq) return fail(c, CFK_ERR_ARG, "dq is required");
  CFK_CHECK(c, launch_finite_rate_chemistry(c->z, c->d_mech, S(stream)), "finite_rate_chemistry");
  c->launches += 1;
  return CFK_OK;
}

int cfk_wu_reaction_step(cfk_ctx *c, double dt, int schedule, int *nsub_out, void *stream) {
  NEED_ZONE(c);
  if (!c->have_mech || c->hp.n_reac == 0) return fail(c, CFK_ERR_STATE, "no reacting mechanism loaded");
  if (schedule != 0 && schedule != 1) return fail(c, CFK_ERR_ARG, "schedule must be 0 or 1");
  if (c->hp.chem_advance_method != 0 && c->hp.chem_advance_method != 1)
    return fail(c, CFK_ERR_ARG, "chem_advance_method must be 0 (explicit) or 1 (point implicit)");
  unsigned int *counter = reinterpret_cast<unsigned int *>(reinterpret_cast<char *>(c->d_dt_bits) + 16);
  CFK_CHECK(c, launch_wu_reaction(c->z, c->p, c->d_mech, c->h_mech, dt, schedule, nsub_out, c->d_err, counter,
                                  c->n_sm, S(stream)),
            "wu_reaction_step");
  c->launches += 1;
  return CFK_OK;
}

int cfk_compute_viscous_flux(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (c->hp.viscous_order == 0) return CFK_OK;
  if (int r = need_mech_for_mixture(c)) return r;
  int n = 0;
  CFK_CHECK(c, launch_viscous(c->z, c->p, thermo_host(c), c->hp.faces, c->hp.n_face, S(stream), &n, c->visc_var),
            "viscous flux");
  c->launches += n;
  return CFK_OK;
}

int cfk_compute_inviscid_flux(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (c->hp.inviscid_scheme == 0) return fail(c, CFK_ERR_STATE, "inviscid_scheme 0 has no flux");
  if (int r = need_mech_for_mixture(c)) return r;
  int n = 0;
  // the limiter's dt: the fixed dt, else the last CFL dt on the device
  const double *dt_dev = c->p.fixed_dt ? nullptr : reinterpret_cast<const double *>(c->d_dt_bits);
  CFK_CHECK(c, launch_inviscid(c->z, c->p, thermo_host(c), dt_dev, c->hp.dt, c->tile_var, S(stream), &n),
            "inviscid flux");
  c->launches += n;
  return CFK_OK;
}

int cfk_compute_shock_sensor(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (!(c->p.sensor_threshold > 1e-10)) return CFK_OK;
  CFK_CHECK(c, launch_shock_sensor(c->z, c->p, S(stream)), "compute_shock_sensor");
  c->launches += 1;
  return CFK_OK;
}

// Tile autotuner: times every tile variant of each WENO sweep on the bound
// zone (into a scratch dq, so the caller's arrays are untouched) and keeps
// the fastest per direction.  The primitive-variable kernels have one tile
// shape per direction and are left as they are.
int cfk_autotune_tiles(cfk_ctx *c, int reps, double *ms_out, int *choice_out, void *stream) {
  NEED_ZONE(c);
  const int s = c->hp.inviscid_scheme;
  if (ms_out)
    for (int n = 0; n < 3 * CFK_TILE_VARIANTS; ++n) ms_out[n] = 0;
  if (!(s == 52 || s == 72)) {
    if (choice_out) for (int d = 0; d < 3; ++d) choice_out[d] = c->tile_var[d];
    return CFK_OK;
  }
  if (int r = need_mech_for_mixture(c)) return r;
  if (reps < 1) reps = 1;
  cudaStream_t st = S(stream);
  const Zone &z0 = c->z;
  const size_t N = (size_t)z0.d.plane(0);
  double *scratch = nullptr;
  CFK_CHECK(c, cudaMalloc(&scratch, N * c->p.n_var * sizeof(double)), "autotune scratch");
  Zone zt = z0;
  zt.dq = scratch;
  Param pt = c->p;
  pt.positive_preserving = 0;  // the limiter is a rare branch; tune the flux itself
  const Thermo *th = thermo_host(c);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaError_t e = cudaMemsetAsync(scratch, 0, N * c->p.n_var * sizeof(double), st);
  const int nd = z0.d.mz > 1 ? 3 : 2;
  int choice[3] = {c->tile_var[0], c->tile_var[1], c->tile_var[2]};
  auto sweep = [&](int dir, int var) -> cudaError_t {
    return th ? launch_weno_mix_dir(zt, pt, *th, nullptr, c->hp.dt, dir, var, st)
              : launch_weno_air_dir(zt, pt, dir, var, st);
  };
  for (int dir = 0; dir < nd && e == cudaSuccess; ++dir) {
    double best = 1e300;
    for (int var = 0; var < CFK_TILE_VARIANTS && e == cudaSuccess; ++var) {
      e = sweep(dir, var);  // warm-up
      if (e == cudaSuccess) e = cudaEventRecord(a, st);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = sweep(dir, var);
      if (e == cudaSuccess) e = cudaEventRecord(b, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(b);
      float ms = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
      const double avg = (double)ms / reps;
      if (ms_out) ms_out[dir * CFK_TILE_VARIANTS + var] = avg;
      if (e == cudaSuccess && avg < best) { best = avg; choice[dir] = var; }
      c->launches += reps + 1;
    }
  }
  // the two forms of the fused air viscous kernel (staged, ring)
  int visc_choice = c->visc_var;
  if (e == cudaSuccess && !th && c->p.viscous_order == 2) {
    double best = 1e300;
    for (int var = 0; var < 3 && e == cudaSuccess; ++var) {
      int nl = 0;
      e = launch_viscous_air(zt, pt, st, &nl, var);  // warm-up
      if (e == cudaSuccess) e = cudaEventRecord(a, st);
      for (int r = 0; r < reps && e == cudaSuccess; ++r) e = launch_viscous_air(zt, pt, st, &nl, var);
      if (e == cudaSuccess) e = cudaEventRecord(b, st);
      if (e == cudaSuccess) e = cudaEventSynchronize(b);
      float ms = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
      if (e == cudaSuccess && ms / reps < best) { best = ms / reps; visc_choice = var; }
      c->visc_ms[var] = ms / reps;
      c->launches += nl;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(scratch);
  if (e != cudaSuccess) return cuda_fail(c, e, "autotune");
  c->visc_var = visc_choice;
  for (int d = 0; d < 3; ++d) c->tile_var[d] = choice[d];
  if (choice_out) for (int d = 0; d < 3; ++d) choice_out[d] = choice[d];
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  return CFK_OK;
}

int cfk_viscous_variant(cfk_ctx *c, int set, int *var, double *ms) {
  if (!c || !var) return CFK_ERR_ARG;
  if (set) {
    if (*var < 0 || *var > 2) return fail(c, CFK_ERR_ARG, "viscous variant must be 0, 1 or 2");
    c->visc_var = *var;
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  } else {
    *var = c->visc_var;
  }
  if (ms) { ms[0] = c->visc_ms[0]; ms[1] = c->visc_ms[1]; ms[2] = c->visc_ms[2]; }
  return CFK_OK;
}

int cfk_set_tile_variants(cfk_ctx *c, const int *var) {
  if (!c || !var) return CFK_ERR_ARG;
  for (int d = 0; d < 3; ++d)
    if (var[d] < 0 || var[d] >= CFK_TILE_VARIANTS) return fail(c, CFK_ERR_ARG, "tile variant out of range");
  for (int d = 0; d < 3; ++d) c->tile_var[d] = var[d];
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  return CFK_OK;
}

int cfk_update_cv_and_bv_rk(cfk_ctx *c, double dt, int rk, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  if (rk < 0 || rk > 2) return fail(c, CFK_ERR_ARG, "rk must be 0, 1 or 2");
  CFK_CHECK(c, launch_update_rk(c->z, c->p, thermo_of(c), dt, nullptr, rk, c->d_err, S(stream)), "update_cv_and_bv_rk");
  c->launches += 1;
  return CFK_OK;
}

int cfk_limit_flow(cfk_ctx *c, long long *n_repaired, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  if (int r = ensure_limit_flags(c)) return r;
  cudaStream_t st = S(stream);
  CFK_CHECK(c, cudaMemsetAsync(limit_counter(c), 0, sizeof(unsigned long long), st), "limit_flow counter");
  CFK_CHECK(c, launch_limit_flow(c->z, c->p, thermo_of(c), c->own_limit, limit_counter(c), st), "limit_flow");
  c->launches += 2;
  if (n_repaired) {
    unsigned long long v = 0;
    CFK_CHECK(c, cudaMemcpyAsync(&v, limit_counter(c), sizeof v, cudaMemcpyDeviceToHost, st), "limit_flow count");
    CFK_CHECK(c, cudaStreamSynchronize(st), "limit_flow sync");
    *n_repaired = (long long)v;
  }
  return CFK_OK;
}

static int halo_face_ok(cfk_ctx *c, int face, int direction) {
  if (face < 0 || face > 2 || (direction != -1 && direction != 1))
    return fail(c, CFK_ERR_ARG, "face must be 0, 1 or 2 and direction -1 or +1");
  if (face == 2 && c->z.d.mz == 1) return fail(c, CFK_ERR_ARG, "a 2-D block has no k faces to share");
  return CFK_OK;
}

int cfk_halo_size(cfk_ctx *c, int face, long long *n_doubles) {
  NEED_ZONE(c);
  if (int r = halo_face_ok(c, face, -1)) return r;
  if (!n_doubles) return fail(c, CFK_ERR_ARG, "n_doubles is NULL");
  *n_doubles = halo_doubles(c->z.d, c->p, face);
  return CFK_OK;
}

int cfk_halo_pack(cfk_ctx *c, int face, int direction, double *buf, void *stream) {
  NEED_ZONE(c);
  if (int r = halo_face_ok(c, face, direction)) return r;
  if (!buf) return fail(c, CFK_ERR_ARG, "buf is NULL");
  CFK_CHECK(c, launch_halo_pack(c->z, c->p, face, direction, buf, S(stream)), "halo pack");
  c->launches += 1;
  return CFK_OK;
}

int cfk_halo_assign(cfk_ctx *c, int face, int direction, const double *buf, void *stream) {
  NEED_ZONE(c);
  if (int r = halo_face_ok(c, face, direction)) return r;
  if (int r = need_mech_for_mixture(c)) return r;
  if (!buf) return fail(c, CFK_ERR_ARG, "buf is NULL");
  CFK_CHECK(c, launch_halo_assign(c->z, c->p, thermo_of(c), face, direction, buf, S(stream)), "halo assign");
  c->launches += 1;
  return CFK_OK;
}

int cfk_update_physical_properties(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  CFK_CHECK(c, launch_update_properties(c->z, c->p, thermo_of(c), S(stream)), "update_physical_properties");
  c->launches += 1;
  return CFK_OK;
}

int cfk_compute_cv_from_bv(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  CFK_CHECK(c, launch_cv_from_bv(c->z, c->p, thermo_of(c), S(stream)), "compute_cv_from_bv");
  c->launches += 1;
  return CFK_OK;
}

int cfk_apply_boundary_conditions(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  int n = 0;
  CFK_CHECK(c, launch_boundary_conditions(c->z, c->p, thermo_of(c), c->hp.faces, c->hp.n_face, c->hp.wall,
                                          c->hp.inflow, c->hp.outflow, S(stream), &n),
            "boundary conditions");
  c->launches += n;
  return CFK_OK;
}

int cfk_eliminate_k_gradient(cfk_ctx *c, void *stream) {
  NEED_ZONE(c);
  if (c->z.d.mz != 1) return fail(c, CFK_ERR_ARG, "eliminate_k_gradient is for 2-D blocks (mz == 1)");
  CFK_CHECK(c, launch_eliminate_k_gradient(c->z, c->p, S(stream)), "eliminate_k_gradient");
  c->launches += 1;
  return CFK_OK;
}

// Host checks of an inner face: a well-formed loop, and every node it maps —
// in this block and in the target — inside the padded arrays.  The index maps
// are affine, so the two ends of each axis bound them.
static int check_inner_face(const Dims &d, const Dims &td, const cfk_inner_face &f, std::string &why) {
  if (f.face < 0 || f.face > 2 || (f.direction != 1 && f.direction != -1)) { why = "bad face/direction"; return -1; }
  int seen = 0;
  long long total = 1;
  for (int a = 0; a < 3; ++a) {
    if (f.src_tar[a] < 0 || f.src_tar[a] > 2) { why = "src_tar must map onto axes 0..2"; return -1; }
    seen |= 1 << f.src_tar[a];
    if ((f.loop_dir[a] != 1 && f.loop_dir[a] != -1) || (f.target_loop_dir[a] != 1 && f.target_loop_dir[a] != -1)) {
      why = "loop directions must be +1 or -1";
      return -1;
    }
    if (f.n_point[a] < 1) { why = "n_point must be >= 1"; return -1; }
    total *= f.n_point[a];
  }
  if (seen != 7) { why = "src_tar must be a permutation of the axes"; return -1; }
  if (total > (1LL << 30)) { why = "face loop too large"; return -1; }
  const int m[3] = {d.mx, d.my, d.mz}, tm[3] = {td.mx, td.my, td.mz};
  for (int a = 0; a < 3; ++a) {
    const int last = f.range_start[a] + f.loop_dir[a] * (f.n_point[a] - 1);
    const int lo = std::min(f.range_start[a], last), hi = std::max(f.range_start[a], last);
    if (lo < -d.ngg || hi > m[a] - 1 + d.ngg) { why = "inner face leaves this block's padded range"; return -1; }
    const int b = f.src_tar[a];
    const int t0 = f.target_start[a], t1 = f.target_start[a] + f.target_loop_dir[a] * f.loop_dir[b] * (f.n_point[b] - 1);
    if (std::min(t0, t1) < -td.ngg || std::max(t0, t1) > tm[a] - 1 + td.ngg) {
      why = "inner face leaves the target block's padded range";
      return -1;
    }
    if (b == f.face && tm[a] <= td.ngg) { why = "target block not thicker than ngg along the face normal"; return -1; }
  }
  if (m[f.face] <= d.ngg) { why = "block not thicker than ngg along the face normal"; return -1; }
  return 0;
}

int cfk_inner_communication(cfk_ctx *c, cfk_ctx *t, const cfk_inner_face *f, void *stream) {
  NEED_ZONE(c);
  if (!t || !f) return fail(c, CFK_ERR_ARG, "inner_communication: null target or face");
  if (!t->bound) return fail(c, CFK_ERR_STATE, "inner_communication: target has no zone bound");
  if (int r = need_mech_for_mixture(c)) return r;
  if (t->hp.device != c->hp.device) return fail(c, CFK_ERR_ARG, "inner_communication: blocks on different devices");
  if (t->z.d.ngg != c->z.d.ngg || (t->z.d.mz == 1) != (c->z.d.mz == 1) || t->p.n_var != c->p.n_var ||
      t->p.n_scalar != c->p.n_scalar || t->p.n_spec != c->p.n_spec)
    return fail(c, CFK_ERR_ARG, "inner_communication: blocks differ in ngg, dimension or variables");
  std::string why;
  if (check_inner_face(c->z.d, t->z.d, *f, why) != 0) return fail(c, CFK_ERR_ARG, "inner_communication: " + why);
  CFK_CHECK(c, launch_inner_communication(c->z, t->z, c->p, thermo_of(c), *f, S(stream)), "inner_communication");
  c->launches += 1;
  return CFK_OK;
}

int cfk_local_time_step(cfk_ctx *c, double *dt_out, void *stream) {
  NEED_ZONE(c);
  if (int r = need_mech_for_mixture(c)) return r;
  CFK_CHECK(c, launch_local_dt(c->z, c->p, thermo_of(c), c->d_dt_bits, S(stream)), "local_time_step");
  c->launches += 2;
  if (dt_out) {
    CFK_CHECK(c, cudaMemcpyAsync(dt_out, c->d_dt_bits, sizeof(double), cudaMemcpyDeviceToHost, S(stream)), "dt copy");
    CFK_CHECK(c, cudaStreamSynchronize(S(stream)), "dt sync");
  }
  return CFK_OK;
}

// The body of one RK3 step, issued on one stream with no host synchronisation.
static int rk3_step_async(cfk_ctx *c, cudaStream_t st) {
  if (c->hp.inviscid_scheme == 0) return fail(c, CFK_ERR_STATE, "inviscid_scheme 0 contexts have no RK3 step");
  if (int r = need_mech_for_mixture(c)) return r;
  const Zone &z = c->z;
  const Param &p = c->p;
  const Thermo *th = thermo_of(c);
  const size_t P = (size_t)z.d.plane(z.d.ngg), N = (size_t)z.d.plane(0);
  int n = 0;
  CFK_CHECK(c, cudaMemcpyAsync(z.qn, z.cv, P * p.n_var * sizeof(double), cudaMemcpyDeviceToDevice, st), "qn copy");
  if (p.sensor_threshold > 1e-10) {
    // once per step, before the stages (reference src/RK.cuh:112-117)
    PhaseScope ps(c, CFK_PH_INVISCID, st, &n);
    CFK_CHECK(c, launch_shock_sensor(z, p, st), "compute_shock_sensor");
    ++n;
  }
  const double *dt_dev = nullptr;
  if (!p.fixed_dt) {
    PhaseScope ps(c, CFK_PH_DT, st, &n);
    CFK_CHECK(c, launch_local_dt(z, p, th, c->d_dt_bits, st), "local_time_step");
    n += 2;
    dt_dev = reinterpret_cast<const double *>(c->d_dt_bits);
  }
  // the properties of the nodes the boundary conditions cannot change are
  // computed by the update kernel; the pass after the boundary conditions
  // covers the rest (the ghost layers and the outermost interior layer).
  // limit_flow rewrites interior nodes after the update, and the subsonic
  // inflow of a mixture reads the acoustic speed of the stage before, so with
  // either the properties stay one pass over the padded block after the
  // boundary conditions.
  bool bc_reads_props = false;
  for (int f = 0; f < c->hp.n_face; ++f)
    if (c->hp.faces[f].label == 5 && c->hp.inflow.subsonic && p.n_spec > 0) bc_reads_props = true;
  const bool fuse_props = !p.limit_flow && !bc_reads_props;
  for (int rk = 0; rk < 3; ++rk) {
    CFK_CHECK(c, cudaMemsetAsync(z.dq, 0, N * p.n_var * sizeof(double), st), "dq memset");
    if (p.viscous_order > 0) {
      PhaseScope ps(c, CFK_PH_VISCOUS, st, &n);
      CFK_CHECK(c, launch_viscous(z, p, thermo_host(c), c->hp.faces, c->hp.n_face, st, &n, c->visc_var), "viscous flux");
    }
    if (c->have_mech && p.n_reac > 0) {
      // explicit chemical source of a reacting mixture (reference src/RK.cuh:147-149)
      CFK_CHECK(c, launch_finite_rate_chemistry(z, c->d_mech, st), "finite_rate_chemistry");
      ++n;
    }
    {
      PhaseScope ps(c, CFK_PH_INVISCID, st, &n);
      CFK_CHECK(c, launch_inviscid(z, p, thermo_host(c), dt_dev, c->hp.dt, c->tile_var, st, &n), "inviscid flux");
    }
    {
      PhaseScope ps(c, CFK_PH_UPDATE, st, &n);
      CFK_CHECK(c, launch_update_rk(z, p, th, c->hp.dt, dt_dev, rk, c->d_err, st, false, fuse_props), "update");
      ++n;
      if (p.limit_flow) {
        // limit_flow<M> after the update (reference src/RK.cuh:163-164)
        CFK_CHECK(c, launch_limit_flow(z, p, th, c->own_limit, limit_counter(c), st), "limit_flow");
        n += 2;
      }
    }
    {
      PhaseScope ps(c, CFK_PH_BC, st, &n);
      CFK_CHECK(c, launch_boundary_conditions(z, p, th, c->hp.faces, c->hp.n_face, c->hp.wall, c->hp.inflow,
                                              c->hp.outflow, st, &n),
                "boundary conditions");
    }
    {
      PhaseScope ps(c, CFK_PH_PROPS, st, &n);
      CFK_CHECK(c, launch_update_properties(z, p, th, st, fuse_props, true), "properties");
      ++n;
    }
  }
  c->launches += n;
  return CFK_OK;
}

// One step of Wu's splitting (the loop body of wu_splitting, reference
// src/StrangSplitting.cu:683-861).  With the CFL step the dt is read back to
// the host once (the reaction kernels take it by value).
// The reaction sub-step of a Wu step: the plain integrator (schedule 0/1),
// optionally bracketed by the surrogate's training-row snapshot and record,
// or the gated surrogate step.
struct WuReaction {
  int mode = 0;  // 0 plain, 1 plain with training rows, 2 surrogate
  float *X = nullptr, *G = nullptr;
  const cfk_surrogate_gate *gate = nullptr;
  int step_index = 0;
  cfk_surrogate_stats *stats = nullptr;
};

static int wu_splitting(cfk_ctx *c, int schedule, const WuReaction &rx, double *dt_used, void *stream);

int cfk_wu_splitting_step(cfk_ctx *c, int schedule, double *dt_used, void *stream) {
  return wu_splitting(c, schedule, WuReaction{}, dt_used, stream);
}

int cfk_wu_splitting_step_record(cfk_ctx *c, int schedule, float *X, float *G, double *dt_used, void *stream) {
  if (!X || !G) return fail(c, CFK_ERR_ARG, "recording needs X and G");
  WuReaction rx;
  rx.mode = 1;
  rx.X = X;
  rx.G = G;
  return wu_splitting(c, schedule, rx, dt_used, stream);
}

int cfk_wu_splitting_step_surrogate(cfk_ctx *c, const cfk_surrogate_gate *gate, int step_index,
                                    cfk_surrogate_stats *stats, double *dt_used, void *stream) {
  WuReaction rx;
  rx.mode = 2;
  rx.gate = gate;
  rx.step_index = step_index;
  rx.stats = stats;
  return wu_splitting(c, 1, rx, dt_used, stream);
}

static int wu_splitting(cfk_ctx *c, int schedule, const WuReaction &rx, double *dt_used, void *stream) {
  NEED_ZONE(c);
  if (c->hp.inviscid_scheme == 0) return fail(c, CFK_ERR_STATE, "inviscid_scheme 0 contexts have no transport step");
  if (!c->have_mech || c->hp.n_reac == 0) return fail(c, CFK_ERR_STATE, "no reacting mechanism loaded");
  if (!c->z.Cn) return fail(c, CFK_ERR_ARG, "Cn is required for Wu's splitting");
  if (schedule != 0 && schedule != 1) return fail(c, CFK_ERR_ARG, "schedule must be 0 or 1");
  const Zone &z = c->z;
  const Param &p = c->p;
  const Thermo *th = thermo_of(c);
  cudaStream_t st = S(stream);
  const size_t P = (size_t)z.d.plane(z.d.ngg), N = (size_t)z.d.plane(0);
  int n = 0;
  double dt = c->hp.dt;
  if (!p.fixed_dt) {
    PhaseScope ps(c, CFK_PH_DT, st, &n);
    CFK_CHECK(c, launch_local_dt(z, p, th, c->d_dt_bits, st, false), "local_time_step_without_reaction");
    n += 2;
    CFK_CHECK(c, cudaMemcpyAsync(&dt, c->d_dt_bits, sizeof(double), cudaMemcpyDeviceToHost, st), "dt copy");
    CFK_CHECK(c, cudaStreamSynchronize(st), "dt sync");
  }
  // compute_cn (:15-41): shock sensor, then Cn = transport right-hand side
  if (p.sensor_threshold > 1e-10) {
    PhaseScope ps(c, CFK_PH_INVISCID, st, &n);
    CFK_CHECK(c, launch_shock_sensor(z, p, st), "compute_shock_sensor");
    ++n;
  }
  CFK_CHECK(c, cudaMemsetAsync(z.dq, 0, N * p.n_var * sizeof(double), st), "dq memset");
  if (p.viscous_order > 0) {
    PhaseScope ps(c, CFK_PH_VISCOUS, st, &n);
    CFK_CHECK(c, launch_viscous(z, p, thermo_host(c), c->hp.faces, c->hp.n_face, st, &n, c->visc_var), "viscous flux");
  }
  {
    PhaseScope ps(c, CFK_PH_INVISCID, st, &n);
    CFK_CHECK(c, launch_inviscid(z, p, thermo_host(c), nullptr, dt, c->tile_var, st, &n), "inviscid flux");
    CFK_CHECK(c, cudaMemcpyAsync(z.Cn, z.dq, N * p.n_var * sizeof(double), cudaMemcpyDeviceToDevice, st),
              "Cn copy");
  }
  // wu_reaction_subStep (:475-502)
  {
    PhaseScope ps(c, CFK_PH_REACTION, st, &n);
    if (rx.mode == 2) {
      const long long before = c->launches;
      if (int r = cfk_surrogate_reaction_step(c, dt, rx.gate, rx.step_index, rx.stats, stream)) return r;
      n += (int)(c->launches - before);
      c->launches = before;
    } else {
      if (rx.mode == 1) {
        if (int r = cfk_surrogate_record(c, 0, dt, nullptr, nullptr, stream)) return r;
      }
      unsigned int *counter = reinterpret_cast<unsigned int *>(reinterpret_cast<char *>(c->d_dt_bits) + 16);
      CFK_CHECK(c, launch_wu_reaction(z, p, c->d_mech, c->h_mech, dt, schedule, nullptr, c->d_err, counter, c->n_sm,
                                      st),
                "wu_reaction_step");
      ++n;
      if (rx.mode == 1) {
        if (int r = cfk_surrogate_record(c, 1, dt, rx.X, rx.G, stream)) return r;
      }
    }
  }
  {
    PhaseScope ps(c, CFK_PH_BC, st, &n);
    CFK_CHECK(c, launch_boundary_conditions(z, p, th, c->hp.faces, c->hp.n_face, c->hp.wall, c->hp.inflow,
                                            c->hp.outflow, st, &n),
              "boundary conditions");
  }
  {
    PhaseScope ps(c, CFK_PH_PROPS, st, &n);
    CFK_CHECK(c, launch_update_properties(z, p, th, st, false, true), "properties");
    ++n;
  }
  // wu_RK_subStep (:564-634): SSP-RK3 over dt/2 on dq - Cn, no property update
  CFK_CHECK(c, cudaMemcpyAsync(z.qn, z.cv, P * p.n_var * sizeof(double), cudaMemcpyDeviceToDevice, st), "qn copy");
  for (int rk = 0; rk < 3; ++rk) {
    CFK_CHECK(c, cudaMemsetAsync(z.dq, 0, N * p.n_var * sizeof(double), st), "dq memset");
    if (p.viscous_order > 0) {
      PhaseScope ps(c, CFK_PH_VISCOUS, st, &n);
      CFK_CHECK(c, launch_viscous(z, p, thermo_host(c), c->hp.faces, c->hp.n_face, st, &n, c->visc_var), "viscous flux");
    }
    {
      PhaseScope ps(c, CFK_PH_INVISCID, st, &n);
      CFK_CHECK(c, launch_inviscid(z, p, thermo_host(c), nullptr, dt, c->tile_var, st, &n), "inviscid flux");
    }
    {
      PhaseScope ps(c, CFK_PH_UPDATE, st, &n);
      CFK_CHECK(c, launch_update_rk(z, p, th, 0.5 * dt, nullptr, rk, c->d_err, st, true), "update (dq - Cn)");
      ++n;
      if (p.limit_flow) {
        // limit_flow<M> after the update (reference src/StrangSplitting.cu:602-604)
        CFK_CHECK(c, launch_limit_flow(z, p, th, c->own_limit, limit_counter(c), st), "limit_flow");
        n += 2;
      }
    }
    {
      PhaseScope ps(c, CFK_PH_BC, st, &n);
      CFK_CHECK(c, launch_boundary_conditions(z, p, th, c->hp.faces, c->hp.n_face, c->hp.wall, c->hp.inflow,
                                              c->hp.outflow, st, &n),
                "boundary conditions");
    }
  }
  c->launches += n;
  if (dt_used) *dt_used = dt;
  return CFK_OK;
}

int cfk_rk3_step(cfk_ctx *c, double *dt_used, void *stream) {
  NEED_ZONE(c);
  int r = rk3_step_async(c, S(stream));
  if (r != CFK_OK) return r;
  if (dt_used) {
    if (c->p.fixed_dt) *dt_used = c->hp.dt;
    else {
      CFK_CHECK(c, cudaMemcpyAsync(dt_used, c->d_dt_bits, sizeof(double), cudaMemcpyDeviceToHost, S(stream)), "dt copy");
      CFK_CHECK(c, cudaStreamSynchronize(S(stream)), "dt sync");
    }
  }
  return CFK_OK;
}

int cfk_rk3_step_graph(cfk_ctx *c, double *dt_used, void *stream) {
  NEED_ZONE(c);
  cudaStream_t st = S(stream);
  if (!c->graph_exec) {
    // capture on a private stream so that the caller's legacy stream is never in capture mode
    cudaStream_t cap;
    CFK_CHECK(c, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
    cudaGraph_t graph;
    CFK_CHECK(c, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    const long long before = c->launches;
    const bool prof = c->profiling;
    c->profiling = false;
    int r = rk3_step_async(c, cap);
    c->profiling = prof;
    cudaError_t e = cudaStreamEndCapture(cap, &graph);
    cudaStreamDestroy(cap);
    c->graph_kernels = c->launches - before;
    c->launches = before;
    if (r != CFK_OK) return r;
    if (e != cudaSuccess) return cuda_fail(c, e, "end capture");
    e = cudaGraphInstantiate(&c->graph_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(c, e, "graph instantiate");
  }
  CFK_CHECK(c, cudaGraphLaunch(c->graph_exec, st), "graph launch");
  c->launches += c->graph_kernels;
  if (dt_used) {
    if (c->p.fixed_dt) *dt_used = c->hp.dt;
    else {
      CFK_CHECK(c, cudaMemcpyAsync(dt_used, c->d_dt_bits, sizeof(double), cudaMemcpyDeviceToHost, st), "dt copy");
      CFK_CHECK(c, cudaStreamSynchronize(st), "dt sync");
    }
  }
  return CFK_OK;
}

int cfk_memcpy_h2d(cfk_ctx *c, void *dst, const void *src, size_t bytes, void *stream) {
  CFK_CHECK(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S(stream)), "h2d");
  return CFK_OK;
}
int cfk_memcpy_d2h(cfk_ctx *c, void *dst, const void *src, size_t bytes, void *stream) {
  CFK_CHECK(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, S(stream)), "d2h");
  return CFK_OK;
}
int cfk_memcpy_d2d(cfk_ctx *c, void *dst, const void *src, size_t bytes, void *stream) {
  CFK_CHECK(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, S(stream)), "d2d");
  return CFK_OK;
}
int cfk_stream_sync(cfk_ctx *c, void *stream) {
  CFK_CHECK(c, cudaStreamSynchronize(S(stream)), "stream sync");
  int h_err = 0;
  if (c && c->d_err) {
    CFK_CHECK(c, cudaMemcpy(&h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
    if (h_err) {
      cudaMemset(c->d_err, 0, sizeof(int));
      std::string msg;
      if (h_err & 1) msg += "temperature Newton iteration reached its 1000-iteration cap; ";
      if (h_err & 4) msg += "surrogate kernel: tensor-core completion wait timed out; ";
      if (h_err & 2) msg += "a node needed more than 100000 reaction substeps (capped); ";
      return fail(c, CFK_ERR_NUMERIC, msg);
    }
  }
  return CFK_OK;
}
int cfk_host_alloc(size_t bytes, void **out) {
  if (!out) return CFK_ERR_ARG;
  return cudaMallocHost(out, bytes) == cudaSuccess ? CFK_OK : CFK_ERR_CUDA;
}
int cfk_host_free(void *ptr) { return cudaFreeHost(ptr) == cudaSuccess ? CFK_OK : CFK_ERR_CUDA; }

long long cfk_kernel_launches(const cfk_ctx *c) { return c ? c->launches : 0; }

int cfk_set_profiling(cfk_ctx *c, int on) {
  if (!c) return CFK_ERR_ARG;
  c->profiling = on != 0;
  return CFK_OK;
}

int cfk_profile_read(cfk_ctx *c, double *ms, long long *kernels) {
  if (!c || !ms || !kernels) return CFK_ERR_ARG;
  for (int k = 0; k < CFK_NPHASE; ++k) { ms[k] = 0; kernels[k] = 0; }
  for (auto &r : c->recs) {
    CFK_CHECK(c, cudaEventSynchronize(r.b), "profile sync");
    float t = 0;
    CFK_CHECK(c, cudaEventElapsedTime(&t, r.a, r.b), "profile elapsed");
    ms[r.phase] += t;
    kernels[r.phase] += r.kernels;
    c->pool.push_back(r.a);
    c->pool.push_back(r.b);
  }
  c->recs.clear();
  return CFK_OK;
}

}  // extern "C"
