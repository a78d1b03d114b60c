// Local CFL time step with its grid minimum, in a form that allocates no
// device memory: for callers that cannot call cudaMalloc — a host whose
// memory policy forbids allocations after start-up (a pool sized once), one
// that owns all device memory itself, or a time-critical loop in which a
// cudaMalloc would synchronise the device.  The
// context-based entry point needs a context (whose creation allocates); this
// one takes the settings and the zone directly and keeps its scratch in a
// file-scope device array instead.
//
// Scratch: one partial minimum per CTA of the first pass, in g_dt_partials
// (kStaticDtSlots doubles, 2 MiB, held by every GPU that loads the library
// until the process exits).  Every slot that the second pass reads is written
// by the first pass of the same call, so nothing needs clearing.  All calls
// share the array: calls that overlap on the GPU (different streams, no
// ordering between them) race on it and must be serialised by the caller.
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda.h>  // driver types for the context-id lookup (entry points resolved at run time)

#include "cfk_common.cuh"

namespace cfk {

constexpr int kStaticDtSlots = 1 << 18;  // first-pass CTAs: ceil(mx/256) * my * mz must not exceed this
constexpr int kStaticDtThreads = 256;

static __device__ __align__(256) double g_dt_partials[kStaticDtSlots];

// Same per-node formula as the context entry point's kernel (air model,
// reference src/TimeAdvanceFunc.cuh:28-115), reduced per CTA into the scratch.
__global__ void __launch_bounds__(kStaticDtThreads) local_dt_static_pass1(Zone z, double cfl, double Pr,
                                                                          int viscous, double *partials) {
  const Dims d = z.d;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  double dt = 1e6;
  if (i < d.mx) {
    const int g = d.ngg;
    const int64_t sz = d.plane(g), id = d.idx(g, i, j, k);
    const double *mt = z.metric;
    const bool three_d = d.mz > 1;
    const double grad_xi = norm3d(mt[id], mt[id + sz], mt[id + 2 * sz]);
    const double grad_eta = norm3d(mt[id + 3 * sz], mt[id + 4 * sz], mt[id + 5 * sz]);
    const double grad_zeta = norm3d(mt[id + 6 * sz], mt[id + 7 * sz], mt[id + 8 * sz]);
    const double u = z.bv[id + sz], v = z.bv[id + 2 * sz], w = z.bv[id + 3 * sz];
    const double U = u * mt[id] + v * mt[id + sz] + w * mt[id + 2 * sz];
    const double V = u * mt[id + 3 * sz] + v * mt[id + 4 * sz] + w * mt[id + 5 * sz];
    const double W = u * mt[id + 6 * sz] + v * mt[id + 7 * sz] + w * mt[id + 8 * sz];
    const double a = sqrt(kGammaAir * kRAir * z.bv[id + 5 * sz]);
    double msr = max(abs(U) + a * grad_xi, abs(V) + a * grad_eta);
    if (three_d) msr = max(msr, abs(W) + a * grad_zeta);
    if (viscous) {
      double max_length = max(grad_xi, grad_eta);
      if (three_d) max_length = max(max_length, grad_zeta);
      const double iRho = 1.0 / z.bv[id];
      double mdv = max(kGammaAir, 4.0 / 3.0) * iRho;
      mdv *= z.mul[id] / Pr;
      msr = max(msr, max_length * max_length * mdv);
    }
    dt = cfl / msr;
    if (z.dt_local) z.dt_local[d.idx(0, i, j, k)] = dt;
  }
  for (int o = 16; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  __shared__ double wmin[kStaticDtThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wmin[wid] = dt;
  __syncthreads();
  if (wid == 0) {
    dt = lane < kStaticDtThreads / 32 ? wmin[lane] : 1e6;
    for (int o = 16; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    if (lane == 0) partials[((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = dt;
  }
}

__global__ void __launch_bounds__(1024) local_dt_static_pass2(const double *partials, int n, double *dt_min) {
  double dt = 1e6;
  for (int t = threadIdx.x; t < n; t += blockDim.x) dt = min(dt, partials[t]);
  for (int o = 16; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  __shared__ double wmin[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wmin[wid] = dt;
  __syncthreads();
  if (wid == 0) {
    dt = lane < (int)(blockDim.x >> 5) ? wmin[lane] : 1e6;
    for (int o = 16; o > 0; o >>= 1) dt = min(dt, __shfl_xor_sync(0xffffffffu, dt, o));
    if (lane == 0) *dt_min = dt;
  }
}

namespace {
// Device address of g_dt_partials per device, looked up with that device
// current.  In host code the symbol itself is only a host-side stand-in;
// kernels must be given this address.  The lookup is kept together with the id
// of the context it was made in: cudaDeviceReset destroys the context and the
// module's copy of the array with it, and the context the runtime creates on
// the next call has a new id, so the address is looked up again there.
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
struct ScratchSlot {
  unsigned long long ctx_id;
  double *addr;
};
ScratchSlot g_scratch[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult(CUDAAPI *)(CUcontext *);
using CtxGetIdFn = CUresult(CUDAAPI *)(CUcontext, unsigned long long *);

// Id of the context current on the calling thread (unique over the process's
// lifetime); 0 if the driver cannot report it, in which case every call looks
// the address up afresh.
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  if (!get_current || !get_id) return 0;
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Called with `dev` current (the runtime has made its primary context current).
int scratch_for_device(int dev, double **out, char *err, size_t err_len) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long id = current_context_id();
  ScratchSlot &slot = g_scratch[dev];
  if (!slot.addr || id == 0 || slot.ctx_id != id) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_dt_partials);
    if (e != cudaSuccess || !p) {
      if (err && err_len) std::snprintf(err, err_len, "cudaGetSymbolAddress of the dt scratch failed: %s",
                                        cudaGetErrorString(e));
      return CFK_ERR_CUDA;
    }
    slot.addr = static_cast<double *>(p);
    slot.ctx_id = id;
  }
  *out = slot.addr;
  return CFK_OK;
}

// Restores the calling thread's current device when the entry point returns.
struct DeviceRestore {
  int dev = -1;
  ~DeviceRestore() {
    if (dev >= 0) cudaSetDevice(dev);
  }
};
}  // namespace

}  // namespace cfk

extern "C" int cfk_local_time_step_static(const cfk_param *param, const cfk_zone *zone, double *dt_min_device,
                                          void *stream, char *err, size_t err_len) {
  using namespace cfk;
  auto report = [&](int code, const char *msg) {
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
    return code;
  };
  if (!param || !zone || !dt_min_device) return report(CFK_ERR_ARG, "param, zone and dt_min_device are required");
  if (param->n_spec != 0) return report(CFK_ERR_ARG, "only the air model (n_spec = 0) is supported");
  if (zone->mx < 1 || zone->my < 1 || zone->mz < 1 || zone->ngg < 1)
    return report(CFK_ERR_ARG, "zone extents and ngg must be positive");
  const long long blocks_x = (zone->mx + kStaticDtThreads - 1) / kStaticDtThreads;
  const long long n_blocks = blocks_x * zone->my * zone->mz;
  if (n_blocks > kStaticDtSlots) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "zone too large for the static dt scratch: ceil(mx/%d)*my*mz = %lld CTA minima, maximum %d",
                  kStaticDtThreads, n_blocks, kStaticDtSlots);
    return report(CFK_ERR_ARG, msg);
  }
  if (zone->my > 65535 || zone->mz > 65535) return report(CFK_ERR_ARG, "my and mz must not exceed 65535");
  if (!zone->metric || !zone->bv || (param->viscous_order > 0 && !zone->mul))
    return report(CFK_ERR_ARG, "metric and bv (and mul for viscous runs) are required");
  if (param->device < 0 || param->device >= kMaxDevices) return report(CFK_ERR_ARG, "device ordinal out of range");
  DeviceRestore restore;
  cudaError_t e = cudaGetDevice(&restore.dev);
  if (e != cudaSuccess) return report(CFK_ERR_CUDA, cudaGetErrorString(e));
  if (restore.dev == param->device) restore.dev = -1;  // already current: nothing to restore
  e = cudaSetDevice(param->device);
  if (e != cudaSuccess) return report(CFK_ERR_CUDA, cudaGetErrorString(e));
  double *scratch = nullptr;
  const int rc = scratch_for_device(param->device, &scratch, err, err_len);
  if (rc != CFK_OK) return rc;

  Zone z{};
  z.d = Dims{zone->mx, zone->my, zone->mz, zone->ngg};
  z.metric = zone->metric;
  z.bv = zone->bv;
  z.mul = zone->mul;
  z.dt_local = zone->dt_local;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  local_dt_static_pass1<<<dim3((unsigned)blocks_x, zone->my, zone->mz), kStaticDtThreads, 0, st>>>(
      z, param->cfl, param->Pr, param->viscous_order > 0 ? 1 : 0, scratch);
  local_dt_static_pass2<<<1, 1024, 0, st>>>(scratch, (int)n_blocks, dt_min_device);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(CFK_ERR_CUDA, cudaGetErrorString(e));
  return CFK_OK;
}
