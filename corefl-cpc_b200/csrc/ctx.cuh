// Internal definition of the library context shared by the translation
// units that implement the C ABI, and the error helpers they use.
#pragma once

#include <string>
#include <vector>

#include "cfk_common.cuh"
#include "chem.cuh"
#include "thermo.cuh"

namespace cfk {
struct Surrogate;
void surrogate_destroy(Surrogate *s);
}  // namespace cfk

using namespace cfk;

struct cfk_ctx {
  cfk_param hp{};
  Param p{};
  Zone z{};
  bool bound = false;
  std::vector<void *> owned;  // device arrays owned by the context
  double *own_sensor = nullptr;  // context-allocated shock sensor (zone without one)
  size_t own_sensor_n = 0;
  double *own_fvis8 = nullptr;   // node viscous fluxes of the 8th-order scheme
  size_t own_fvis8_n = 0;
  unsigned char *own_limit = nullptr;  // limit_flow: out-of-bounds flag per interior node
  size_t own_limit_n = 0;
  Mech *d_mech = nullptr;
  Mech h_mech{};  // host copy, passed by value to the kernels that read it from the constant bank
  bool have_mech = false;
  int n_sm = 148;
  // device scratch: [0] dt bits (u64), [1] error flags (int)
  unsigned long long *d_dt_bits = nullptr;
  int *d_err = nullptr;
  long long launches = 0;
  std::string err;
  // CUDA graph of one RK3 step
  cudaGraphExec_t graph_exec = nullptr;
  long long graph_kernels = 0;
  // tile variant of each sweep of the WENO flux kernels (tile autotuner)
  int tile_var[3] = {0, 0, 0};      // cfk_create sets the air default {2, 1, 1}
  int visc_var = 2;                 // fused air viscous kernel: 0 staged, 1 cp.async ring, 2 ring + L2 prefetch
  double visc_ms[3] = {0, 0, 0};    // their times in the last autotune (ms per launch)
  // phase timing with CUDA events (plain steps only)
  bool profiling = false;
  struct Rec { int phase; cudaEvent_t a, b; long long kernels; };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  // MLP chemistry surrogate (weights, optimiser state, gate bookkeeping)
  Surrogate *sg = nullptr;
  cudaEvent_t take_event() {
    if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
};


namespace cfk_detail {

inline int fail(cfk_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}

inline int cuda_fail(cfk_ctx *c, cudaError_t e, const char *where) {
  return fail(c, CFK_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace cfk_detail

#define CFK_CHECK(ctx, call, where)                                      \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) return cfk_detail::cuda_fail(ctx, e_, where); \
  } while (0)

#define NEED_ZONE(c)                                                              \
  do {                                                                            \
    if (!(c)) return CFK_ERR_ARG;                                                 \
    if (!(c)->bound) return cfk_detail::fail(c, CFK_ERR_STATE, "no zone bound");              \
    CFK_CHECK(c, cudaSetDevice((c)->hp.device), "cudaSetDevice");                 \
  } while (0)

