// Halo exchange of a block face shared with a block on another rank (the
// reference's parallel faces, src/DataCommunication.cu:105-307): pack the
// face nodes and the ngg node layers inside them for the neighbour, and
// assign what the neighbour packed — its face nodes averaged into ours (or
// copied where ours is a wall node, |V| <= 1e-15, and theirs is not), its
// inner layers into our ghost layers — with cv from bv at every node written.
//
// The face is a whole block face (face axis 0/1/2, direction -1 min / +1
// max side) over the block's own tangential nodes, as the reference
// registers parallel faces (no ghost extension).  Buffer layout: node t of
// the face (first tangential axis fastest), layer q = 0..ngg (0 the face
// node, q the q-th node inwards), variable l of the 6 basic variables and
// then the n_scalar scalars: buf[(t * (ngg + 1) + q) * (6 + n_scalar) + l] —
// the per-node order of the reference's buffers.  The library does not move
// the buffers between ranks: the host does, with any transport (NCCL, MPI).
#include "cfk_common.cuh"
#include "cv_point.cuh"
#include "thermo.cuh"

namespace cfk {

namespace {

struct HaloFace {
  int face, direction, a, b, na, nb, f0;  // tangential axes a < b, their extents, face node index
};

__device__ __forceinline__ void halo_node(const HaloFace &h, int t, int q_off, int (&idx)[3]) {
  const int ta = t % h.na, tb = t / h.na;
  idx[h.a] = ta;
  idx[h.b] = tb;
  idx[h.face] = h.f0 + q_off;
}

__global__ void halo_pack_kernel(Zone z, Param p, HaloFace h, double *buf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= h.na * h.nb) return;
  const Dims d = z.d;
  const int g = d.ngg, nt = 6 + p.n_scalar;
  const int64_t sz = d.plane(g);
  for (int q = 0; q <= g; ++q) {
    int idx[3];
    halo_node(h, t, -q * h.direction, idx);
    const int64_t id = d.idx(g, idx[0], idx[1], idx[2]);
    double *o = buf + ((int64_t)t * (g + 1) + q) * nt;
    for (int l = 0; l < 6; ++l) o[l] = z.bv[id + l * sz];
    for (int l = 0; l < p.n_scalar; ++l) o[6 + l] = z.sv[id + l * sz];
  }
}

template <bool MIX>
__global__ void halo_assign_kernel(Zone z, Param p, const Thermo *th, HaloFace h, const double *buf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= h.na * h.nb) return;
  const Dims d = z.d;
  const int g = d.ngg, nt = 6 + p.n_scalar;
  const int64_t sz = d.plane(g);
  const double *in = buf + (int64_t)t * (g + 1) * nt;
  int idx[3];
  halo_node(h, t, 0, idx);
  int64_t id = d.idx(g, idx[0], idx[1], idx[2]);
  // the shared face node (reference src/DataCommunication.cu:226-252)
  const double u_this = norm3d(z.bv[id + sz], z.bv[id + 2 * sz], z.bv[id + 3 * sz]);
  if (fabs(u_this) > 1e-15) {
    if (norm3d(in[1], in[2], in[3]) < 1e-15) {
      for (int l = 0; l < 6; ++l) z.bv[id + l * sz] = in[l];
      for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = in[6 + l];
    } else {
      for (int l = 0; l < 6; ++l) z.bv[id + l * sz] = 0.5 * (z.bv[id + l * sz] + in[l]);
      for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = 0.5 * (z.sv[id + l * sz] + in[6 + l]);
    }
    cv_from_bv_point<MIX>(z, p, th, id);
  }
  // ghost layer q from the neighbour's q-th inner layer (:254-265)
  for (int q = 1; q <= g; ++q) {
    halo_node(h, t, q * h.direction, idx);
    id = d.idx(g, idx[0], idx[1], idx[2]);
    const double *v = in + q * nt;
    for (int l = 0; l < 6; ++l) z.bv[id + l * sz] = v[l];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[id + l * sz] = v[6 + l];
    cv_from_bv_point<MIX>(z, p, th, id);
  }
}

HaloFace make_halo(const Dims &d, int face, int direction) {
  HaloFace h;
  h.face = face;
  h.direction = direction;
  h.a = face == 0 ? 1 : 0;
  h.b = face == 2 ? 1 : 2;
  const int m[3] = {d.mx, d.my, d.mz};
  h.na = m[h.a];
  h.nb = m[h.b];
  h.f0 = direction < 0 ? 0 : m[face] - 1;
  return h;
}

}  // namespace

long long halo_doubles(const Dims &d, const Param &p, int face) {
  const HaloFace h = make_halo(d, face, -1);
  return (long long)h.na * h.nb * (d.ngg + 1) * (6 + p.n_scalar);
}

cudaError_t launch_halo_pack(const Zone &z, const Param &p, int face, int direction, double *buf, cudaStream_t st) {
  const HaloFace h = make_halo(z.d, face, direction);
  const int n = h.na * h.nb;
  halo_pack_kernel<<<(n + 127) / 128, 128, 0, st>>>(z, p, h, buf);
  return cudaGetLastError();
}

cudaError_t launch_halo_assign(const Zone &z, const Param &p, const Thermo *th, int face, int direction,
                               const double *buf, cudaStream_t st) {
  const HaloFace h = make_halo(z.d, face, direction);
  const int n = h.na * h.nb;
  if (p.n_spec > 0) halo_assign_kernel<true><<<(n + 127) / 128, 128, 0, st>>>(z, p, th, h, buf);
  else halo_assign_kernel<false><<<(n + 127) / 128, 128, 0, st>>>(z, p, th, h, buf);
  return cudaGetLastError();
}

}  // namespace cfk
