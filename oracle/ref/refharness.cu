// Driver of the reference solver's own per-step kernels, for recording its
// outputs as test fixtures (test infrastructure; built with the reference's
// sources by oracle/ref/Makefile, never part of the library).
//
// It builds the reference's Parameter, Mesh and Driver from a case directory
// in the reference's input format (input/setup.txt, input/grid/grid   0.grd,
// input/boundary_condition/boundary   0.txt), optionally replaces the initial
// basic and scalar variables with input/init_bv.bin / input/init_sv.bin
// (padded planes, the reference's VectorField3D layout), runs the
// reference's Driver::initialize_computation and then advances step by step
// with the same call sequence as the reference's time loops, writing the
// device arrays after every step:
//
//   refharness <case dir> rk3 <steps>   SSP-RK3 steps   (src/RK.cuh:84-216)
//   refharness <case dir> wu  <steps>   Wu splitting    (src/StrangSplitting.cu:683-861)
//   refharness <case dir> visc 0        one compute_viscous_flux into a zeroed
//        dq from the initialised state (src/ViscousScheme.cu:7-73): writes
//        out/visc_dq.bin and the flux arrays out/visc_{f,g,h}.bin
//   refharness <case dir> react <steps> <dt>
//        reaction steps only: wu_reaction_step with Cn = 0 on every node
//        (src/StrangSplitting.cu:373-421, constant-volume reactors)
//   refharness <case dir> rk3last <steps>
//   refharness <case dir> wulast <steps>
//   refharness <case dir> reactlast <steps> <dt>
//        the same steps, writing only the state after the last one
//   refharness <case dir> rk3time <steps> <warm-up>
//   refharness <case dir> wutime <steps> <warm-up>
//   refharness <case dir> reacttime <steps> <dt> <warm-up>
//        the same steps timed with CUDA events, without any file output:
//        one JSON line on stdout with the per-step times
//
// Output, under <case dir>/out/: state_<s>_<name>.bin for s = 0 (after
// initialisation and compute_cv_from_bv) .. steps, name in cv, bv, sv
// (and reaction_timeScale for mixtures); dt_<s>.bin; and at s = 0 the
// grid arrays metric, jac, mul.  Every file is the raw padded device array,
// float64, variable planes one after another.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include <unistd.h>

#include "Parameter.h"
#include "Mesh.h"
#include "Driver.cuh"
#include "FieldOperation.cuh"
#include "TimeAdvanceFunc.cuh"
#include "InviscidScheme.cuh"
#include "ViscousScheme.cuh"
#include "DataCommunication.cuh"
#include "FiniteRateChem.cuh"
#include "Fluctuation.cuh"
#include "RK.cuh"
#include "StrangSplitting.cuh"

namespace cfd {
// Instantiated (with external linkage) in the reference's StrangSplitting.cu.
template<MixtureModel mix_model> void wu_reaction_subStep(std::vector<Field> &field, DParameter *param,
  Parameter &parameter, const Mesh &mesh, DBoundCond &bound_cond, int n_block, dim3 tpb, dim3 *bpg, real dt, int step);
template<MixtureModel mix_model> void wu_RK_subStep(std::vector<Field> &field, DParameter *param, Parameter &parameter,
  const Mesh &mesh, DBoundCond &bound_cond, int n_block, int step, dim3 tpb, dim3 *bpg, real dt);
__global__ void wu_reaction_step(DZone *zone, const DParameter *param, real dt);
}

namespace {

// Timed runs (rk3time, wutime, reacttime) check launches without synchronising, so
// the timed region holds only the reference's own synchronisation points.
bool g_sync_checks = true;

void check(const char *what) {
  cudaError_t e = g_sync_checks ? cudaDeviceSynchronize() : cudaSuccess;
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "refharness: %s: %s\n", what, cudaGetErrorString(e));
    std::exit(3);
  }
}

void write_device(const std::string &path, const void *dptr, size_t bytes) {
  std::vector<char> h(bytes);
  if (bytes) {
    const cudaError_t e = cudaMemcpy(h.data(), dptr, bytes, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      std::fprintf(stderr, "refharness: copy for %s: %s\n", path.c_str(), cudaGetErrorString(e));
      std::exit(3);
    }
  }
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::fprintf(stderr, "refharness: cannot write %s\n", path.c_str());
    std::exit(2);
  }
  std::fwrite(h.data(), 1, bytes, f);
  std::fclose(f);
}

void write_value(const std::string &path, double v) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) std::exit(2);
  std::fwrite(&v, sizeof v, 1, f);
  std::fclose(f);
}

// Replaces a padded device array (n planes) with the contents of a file, if
// the file exists; its size must match exactly.
bool load_into(const std::string &path, void *dptr, size_t bytes) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) return false;
  const size_t n = static_cast<size_t>(in.tellg());
  if (n != bytes) {
    std::fprintf(stderr, "refharness: %s holds %zu bytes, the array %zu\n", path.c_str(), n, bytes);
    std::exit(2);
  }
  in.seekg(0);
  std::vector<char> h(n);
  in.read(h.data(), static_cast<std::streamsize>(n));
  if (cudaMemcpy(dptr, h.data(), n, cudaMemcpyHostToDevice) != cudaSuccess) {
    std::fprintf(stderr, "refharness: upload of %s failed\n", path.c_str());
    std::exit(3);
  }
  return true;
}

template<MixtureModel M> struct Run {
  cfd::Parameter &parameter;
  cfd::Mesh &mesh;
  cfd::Driver<M> driver;
  int n_var;
  int n_scalar;

  Run(cfd::Parameter &p, cfd::Mesh &m) : parameter(p), mesh(m), driver(p, m) {
    n_var = parameter.get_int("n_var");
    n_scalar = parameter.get_int("n_scalar");
  }

  cfd::DZone &zone() { return *driver.field[0].h_ptr; }

  void dump_state(int s) {
    cfd::DZone &z = zone();
    const std::string pre = "out/state_" + std::to_string(s) + "_";
    const size_t sz = static_cast<size_t>(z.cv.size());
    write_device(pre + "cv.bin", z.cv.data(), sz * n_var * sizeof(real));
    write_device(pre + "bv.bin", z.bv.data(), sz * 6 * sizeof(real));
    if (n_scalar > 0) write_device(pre + "sv.bin", z.sv.data(), sz * n_scalar * sizeof(real));
    if constexpr (M == MixtureModel::Mixture) {
      if (parameter.get_int("reaction") == 1)
        write_device(pre + "reaction_timeScale.bin", z.reaction_timeScale.data(), sz * sizeof(real));
    }
  }

  void dump_grid() {
    cfd::DZone &z = zone();
    const size_t sz = static_cast<size_t>(z.jac.size());
    write_device("out/metric.bin", z.metric.data(), sz * 9 * sizeof(real));
    write_device("out/jac.bin", z.jac.data(), sz * sizeof(real));
    write_device("out/mul.bin", z.mul.data(), sz * sizeof(real));
  }

  // The scalar settings the reference derived from setup.txt (reference
  // state scaling, entropy fix, ...), as "name value" lines.
  void dump_param() {
    std::vector<char> raw(sizeof(cfd::DParameter));
    if (cudaMemcpy(raw.data(), driver.param, raw.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
      std::fprintf(stderr, "refharness: DParameter copy failed\n");
      std::exit(3);
    }
    const auto *p = reinterpret_cast<const cfd::DParameter *>(raw.data());
    FILE *f = std::fopen("out/param.txt", "w");
    if (!f) std::exit(2);
    std::fprintf(f, "weno_eps_scale %.17g\nrho_ref %.17g\nv_ref %.17g\na_ref2 %.17g\n", p->weno_eps_scale, p->rho_ref,
                 p->v_ref, p->a_ref2);
    std::fprintf(f, "entropy_fix_factor %.17g\ncfl %.17g\nPr %.17g\nSc %.17g\nsensor_eps %.17g\n",
                 p->entropy_fix_factor, p->cfl, p->Pr, p->Sc, p->sensor_eps);
    std::fprintf(f, "ngg %d\nn_var %d\nn_scalar %d\n", mesh[0].ngg, n_var, n_scalar);
    std::fclose(f);
  }

  // Initial-state override, then the reference's own initialisation.
  void initialise() {
    cfd::DZone &z = zone();
    const size_t sz = static_cast<size_t>(z.bv.size());
    const bool bv = load_into("input/init_bv.bin", z.bv.data(), sz * 6 * sizeof(real));
    bool sv = false;
    if (n_scalar > 0) sv = load_into("input/init_sv.bin", z.sv.data(), sz * n_scalar * sizeof(real));
    std::printf("refharness: initial bv %s, sv %s\n", bv ? "from input/init_bv.bin" : "from setup.txt",
                n_scalar > 0 ? (sv ? "from input/init_sv.bin" : "from setup.txt") : "none");
    check("override");
    driver.initialize_computation();
    check("initialize_computation");
  }

  dim3 tpb() const { return mesh.dimension == 2 ? dim3{16, 16, 1} : dim3{8, 8, 4}; }
  dim3 bpg() const {
    const dim3 t = tpb();
    return {(mesh[0].mx - 1) / t.x + 1, (mesh[0].my - 1) / t.y + 1, (mesh[0].mz - 1) / t.z + 1};
  }
  dim3 bpg_padded() const {
    const dim3 t = tpb();
    const int ng_1 = 2 * mesh[0].ngg - 1;
    return {(mesh[0].mx + ng_1) / t.x + 1, (mesh[0].my + ng_1) / t.y + 1, (mesh[0].mz + ng_1) / t.z + 1};
  }

  // As the reference's time loops do before their first step.
  void start() {
    cfd::DZone *d = driver.field[0].d_ptr;
    cfd::store_last_step<<<bpg(), tpb()>>>(d);
    cfd::compute_cv_from_bv<M><<<bpg_padded(), tpb()>>>(d, driver.param);
    check("compute_cv_from_bv");
  }

  real time_step(bool with_reaction_limit) {
    if (parameter.get_bool("fixed_time_step")) return parameter.get_real("dt");
    cfd::DZone *d = driver.field[0].d_ptr;
    if (with_reaction_limit)
      cfd::local_time_step<M><<<bpg(), tpb()>>>(d, driver.param);
    else
      cfd::local_time_step_without_reaction<<<bpg(), tpb()>>>(d, driver.param);
    const real dt = cfd::global_time_step(mesh, parameter, driver.field);
    cfd::update_dt_global<<<1, 1>>>(driver.param, dt);
    check("time step");
    return dt;
  }

  // One SSP-RK3 step: the body of the reference's RK3 loop (src/RK.cuh:89-206)
  // for one block, without its residual and file output.
  real rk3_step(int step) {
    auto &field = driver.field;
    cfd::DParameter *param = driver.param;
    cfd::DZone &z = zone();
    const size_t sz = static_cast<size_t>(z.cv.size());
    cudaMemcpy(z.qn.data(), z.cv.data(), sz * sizeof(real) * n_var, cudaMemcpyDeviceToDevice);
    if (parameter.get_string("hybrid_inviscid_scheme") != "NO")
      cfd::compute_shock_sensor<<<bpg(), tpb()>>>(field[0].d_ptr, param);
    const real dt = time_step(true);
    for (int rk = 0; rk < 3; ++rk) {
      cudaMemset(z.dq.data(), 0, static_cast<size_t>(z.dq.size()) * n_var * sizeof(real));
      cfd::compute_viscous_flux<M>(mesh, field, param, parameter);
      if (parameter.get_int("reaction") == 1) cfd::finite_rate_chemistry<<<bpg(), tpb()>>>(field[0].d_ptr, param);
      cfd::compute_inviscid_flux<M>(mesh[0], field[0].d_ptr, param, n_var, parameter);
      driver.bound_cond.template nonReflectingBoundary<M>(mesh[0], field[0], param);
      cfd::update_cv_and_bv_rk<M><<<bpg(), tpb()>>>(field[0].d_ptr, param, dt, rk);
      if (parameter.get_bool("limit_flow")) cfd::limit_flow<M><<<bpg(), tpb()>>>(field[0].d_ptr, param);
      driver.bound_cond.template apply_boundary_conditions<M>(mesh[0], field[0], param, step);
      cfd::update_values_with_fluctuations<<<bpg(), tpb()>>>(field[0].d_ptr, param);
      cfd::data_communication<M>(mesh, field, parameter, step, param);
      if (mesh.dimension == 2) {
        const dim3 t = tpb();
        const int ng_1 = 2 * mesh[0].ngg - 1;
        const dim3 b{(mesh[0].mx + ng_1) / t.x + 1, (mesh[0].my + ng_1) / t.y + 1, 1};
        cfd::eliminate_k_gradient<<<b, t>>>(field[0].d_ptr, param);
      }
      cfd::update_physical_properties<M><<<bpg_padded(), tpb()>>>(field[0].d_ptr, param);
      check("rk stage");
    }
    return dt;
  }

  // One Wu splitting step: the body of the reference's wu_splitting loop
  // (src/StrangSplitting.cu:756-771) for one block.
  real wu_step(int step) {
    dim3 b = bpg();
    const real dt = time_step(false);
    cfd::compute_cn<M>(driver.field, driver.param, parameter, mesh, 1, tpb(), &b);
    check("compute_cn");
    cfd::wu_reaction_subStep<M>(driver.field, driver.param, parameter, mesh, driver.bound_cond, 1, tpb(), &b, dt, step);
    check("reaction sub-step");
    cfd::wu_RK_subStep<M>(driver.field, driver.param, parameter, mesh, driver.bound_cond, 1, step, tpb(), &b, 0.5 * dt);
    check("transport sub-step");
    return dt;
  }

  // One viscous-flux evaluation (compute_viscous_flux, src/ViscousScheme.cu:7-73)
  // into a zeroed dq, from the initialised state: dq and the node/face flux
  // arrays it leaves behind.
  void viscous_once() {
    cfd::DZone &z = zone();
    const size_t nq = static_cast<size_t>(z.dq.size()) * n_var * sizeof(real);
    const size_t nf = static_cast<size_t>(z.fFlux.size()) * n_var * sizeof(real);
    cudaMemset(z.dq.data(), 0, nq);
    cfd::compute_viscous_flux<M>(mesh, driver.field, driver.param, parameter);
    check("compute_viscous_flux");
    write_device("out/visc_dq.bin", z.dq.data(), nq);
    write_device("out/visc_f.bin", z.fFlux.data(), nf);
    write_device("out/visc_g.bin", z.gFlux.data(), nf);
    write_device("out/visc_h.bin", z.hFlux.data(), nf);
  }

  // Reaction only, Cn = 0: a batch of constant-volume reactors.  Timed runs
  // zero Cn once before their first step (zero_cn = false afterwards).
  real react_step(real dt, bool zero_cn = true) {
    cfd::DZone &z = zone();
    if (zero_cn) cudaMemset(z.Cn.data(), 0, static_cast<size_t>(z.Cn.size()) * n_var * sizeof(real));
    cfd::wu_reaction_step<<<bpg(), tpb()>>>(driver.field[0].d_ptr, driver.param, dt);
    check("wu_reaction_step");
    return dt;
  }
};

// Timed steps of the reference's own kernels: `warmup` untimed steps, then
// `steps` steps, each between two CUDA events on the legacy default stream,
// which is where every reference kernel driven here is launched.  Prints one
// JSON line: the total and the per-step times (ms) and the node count.
template<MixtureModel M> int timed(Run<M> &r, const std::string &mode, int steps, int warmup, double react_dt) {
  const bool rk3 = mode == "rk3time", wu = mode == "wutime";
  if (!rk3 && !wu) r.react_step(react_dt, true);  // zero Cn; this step counts as a warm-up step
  auto one = [&](int s) -> real {
    if (rk3) return r.rk3_step(s);
    if (wu) return r.wu_step(s);
    return r.react_step(react_dt, false);
  };
  g_sync_checks = false;
  for (int s = 1; s <= warmup; ++s) one(s);
  g_sync_checks = true;
  check("warm-up steps");
  g_sync_checks = false;
  std::vector<cudaEvent_t> ev(static_cast<size_t>(steps) + 1);
  for (auto &e : ev) cudaEventCreate(&e);
  real dt = 0;
  cudaEventRecord(ev[0]);
  for (int s = 1; s <= steps; ++s) {
    dt = one(warmup + s);
    cudaEventRecord(ev[static_cast<size_t>(s)]);
  }
  cudaEventSynchronize(ev.back());
  g_sync_checks = true;
  check("timed steps");
  float total = 0;
  cudaEventElapsedTime(&total, ev[0], ev.back());
  std::printf("{\"mode\": \"%s\", \"steps\": %d, \"warmup\": %d, \"ms_total\": %.6f, \"ms_per_step\": [",
              mode.c_str(), steps, warmup, total);
  for (int s = 1; s <= steps; ++s) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[static_cast<size_t>(s) - 1], ev[static_cast<size_t>(s)]);
    std::printf("%s%.6f", s > 1 ? ", " : "", ms);
  }
  const auto &b = r.mesh[0];
  std::printf("], \"nodes\": %lld, \"mx\": %d, \"my\": %d, \"mz\": %d, \"dt\": %.17g}\n",
              static_cast<long long>(b.mx) * b.my * b.mz, b.mx, b.my, b.mz, dt);
  for (auto &e : ev) cudaEventDestroy(e);
  return 0;
}

template<MixtureModel M> int run(cfd::Parameter &parameter, cfd::Mesh &mesh, const std::string &mode, int steps,
                                 double react_dt, int warmup) {
  Run<M> r(parameter, mesh);
  r.initialise();
  r.start();
  if (mode == "rk3time" || mode == "wutime" || mode == "reacttime") return timed(r, mode, steps, warmup, react_dt);
  // reactlast, rk3last: the state after the last step only (large blocks)
  const bool last_only = mode == "reactlast" || mode == "rk3last" || mode == "wulast";
  if (!last_only) {
    r.dump_grid();
    r.dump_param();
    r.dump_state(0);
  }
  if (mode == "visc") {
    r.viscous_once();
    return 0;
  }
  for (int s = 1; s <= steps; ++s) {
    real dt = 0;
    if (mode == "rk3" || mode == "rk3last")
      dt = r.rk3_step(s);
    else if (mode == "wu" || mode == "wulast")
      dt = r.wu_step(s);
    else
      dt = r.react_step(react_dt);
    if (!last_only || s == steps) {
      write_value("out/dt_" + std::to_string(s) + ".bin", dt);
      r.dump_state(s);
    }
    std::printf("refharness: step %d dt %.17g\n", s, dt);
  }
  return 0;
}

}  // namespace

int main(int argc, char *argv[]) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: refharness <case dir> rk3|rk3last|wu|wulast|react|reactlast|visc <steps> [dt]\n"
                         "       refharness <case dir> rk3time|wutime <steps> <warm-up steps>\n"
                         "       refharness <case dir> reacttime <steps> <dt> <warm-up steps>\n");
    return 2;
  }
  const std::string mode = argv[2];
  const int steps = std::atoi(argv[3]);
  const bool react = mode == "react" || mode == "reactlast" || mode == "reacttime";
  const double react_dt = react && argc > 4 ? std::atof(argv[4]) : 0.0;
  const int warmup = (mode == "rk3time" || mode == "wutime") ? (argc > 4 ? std::atoi(argv[4]) : 0)
                                       : (mode == "reacttime" && argc > 5 ? std::atoi(argv[5]) : 0);
  if (mode != "rk3" && mode != "rk3last" && mode != "wu" && mode != "wulast" && mode != "react" &&
      mode != "reactlast" && mode != "visc" && mode != "rk3time" && mode != "wutime" &&
      mode != "reacttime") {
    std::fprintf(stderr, "refharness: unknown mode %s\n", mode.c_str());
    return 2;
  }
  if ((mode == "rk3time" || mode == "wutime" || mode == "reacttime") && (steps < 1 || warmup < 0)) {
    std::fprintf(stderr, "refharness: a timed run needs steps >= 1 and warm-up steps >= 0\n");
    return 2;
  }
  if (react && !(react_dt > 0)) {
    std::fprintf(stderr, "refharness: react needs a positive dt\n");
    return 2;
  }
  if (chdir(argv[1]) != 0) {
    std::fprintf(stderr, "refharness: cannot enter %s\n", argv[1]);
    return 2;
  }
  int pargc = 1;
  char **pargv = argv;
  cfd::Parameter parameter(&pargc, &pargv);
  cfd::Mesh mesh(parameter);
  if (mesh.n_block != 1) {
    std::fprintf(stderr, "refharness: one block expected, the mesh has %d\n", mesh.n_block);
    return 2;
  }
  const int species = parameter.get_int("species");
  if (!parameter.get_bool("turbulence")) parameter.update_parameter("turbulence_method", 0);
  if (species == 1) return run<MixtureModel::Mixture>(parameter, mesh, mode, steps, react_dt, warmup);
  return run<MixtureModel::Air>(parameter, mesh, mode, steps, react_dt, warmup);
}
