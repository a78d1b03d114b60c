"""Slab decomposition of one block across ranks, the multi-process form of
the reference's RK3 stage loop (src/RK.cuh:84-216 with parallel_communication,
src/DataCommunication.cu:105-208, and the global time step's MPI minimum,
src/TimeAdvanceFunc.cu:102-127).

A block is cut along one axis into slabs that share the node plane at each
cut.  Every slab is a block of its own whose cut faces carry no boundary
condition; once per stage, after the boundary conditions, each slab packs the
face node and the ngg nodes inside each cut face (cfk_halo_pack), the
buffers go to the neighbouring slab, and it assigns them (cfk_halo_assign:
the shared face node averaged, the ghost layers filled).  The CFL step is the
minimum over all slabs.  Slabs may live in one process (LocalTransport) or
one per rank (DistTransport over torch.distributed: NCCL for device buffers,
gloo for host buffers).  The zone operations are those of the C ABI
(LibraryZone); the arithmetic of a decomposed step equals the single block's
wherever the stencils read only exchanged nodes.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def slab_bounds(m: int, n: int):
    """Node ranges [s_r, e_r] of n slabs over m nodes sharing their cut nodes."""
    cuts = [round(r * (m - 1) / n) for r in range(n + 1)]
    return [(cuts[r], cuts[r + 1]) for r in range(n)]


def split_slabs(case, n: int, axis: int, periodic: bool = False):
    """n slab cases of `case` along `axis` (0 i, 1 j, 2 k): every padded
    array is sliced from the whole block's (metrics, state), and the faces of
    each slab are the block's faces on its outer sides only (none on `axis`
    when the axis is a periodic seam)."""
    if n < 1 or (axis == 2 and case.mz == 1):
        raise ValueError("bad slab count or axis")
    g = case.ngg
    shape = case.shape()  # (k, j, i) padded
    ax = 2 - axis         # array axis of `axis`
    m = (case.mx, case.my, case.mz)[axis]
    out = []
    for r, (s, e) in enumerate(slab_bounds(m, n)):
        sl = [slice(None)] * 3
        sl[ax] = slice(s, e + 1 + 2 * g)

        ext = [case.mx, case.my, case.mz]
        ext[axis] = e - s + 1
        n_pad = (ext[0] + 2 * g) * (ext[1] + 2 * g) * (ext[2] + 2 * g)

        def cut(a, sl=sl, n_pad=n_pad):
            a = np.asarray(a)
            lead = a.shape[:-1]
            if a.size == 0:
                return np.zeros(lead + (n_pad,))
            return np.ascontiguousarray(a.reshape(lead + shape)[(Ellipsis,) + tuple(sl)]).reshape(lead + (-1,))

        faces = [(f, d, lab) for f, d, lab in case.faces
                 if f != axis or (not periodic and ((d < 0 and r == 0) or (d > 0 and r == n - 1)))]
        x = cut(case.x) if case.x is not None else None
        out.append(dataclasses.replace(case, mx=ext[0], my=ext[1], mz=ext[2], metric=cut(case.metric),
                                       jac=cut(case.jac), bv=cut(case.bv), sv=cut(case.sv), faces=faces, x=x,
                                       xyz=None, name=f"{case.name}_slab{r}"))
    return out


class LocalTransport:
    """All slabs in this process: buffers pass by reference."""

    def exchange(self, outgoing):
        return {(src, dst, -d): buf for (src, dst, d), buf in outgoing.items()}

    def minimum(self, x: float) -> float:
        return x


class DistTransport:
    """Slabs spread over the ranks of torch.distributed (NCCL for device
    buffers, gloo for host buffers); rank_of[s] is the rank holding slab s.
    exchange takes the buffers this rank's slabs send, keyed (src, dst, d)
    with d the side of the sending face, and returns the buffers they receive,
    keyed (src, dst, side of the receiving face).  Messages between two ranks
    are posted in the sorted order of their keys on both sides, so that the
    point-to-point matching (in posting order per peer) pairs them."""

    def __init__(self, dist, rank_of, make_buffer, group=None):
        self.dist, self.rank_of, self.group = dist, list(rank_of), group
        self.rank = dist.get_rank(group)
        self.make_buffer = make_buffer  # n -> an empty float64 tensor on the transport's device

    def exchange(self, outgoing):
        local = {k: v for k, v in outgoing.items() if self.rank_of[k[1]] == self.rank}
        incoming = {(src, dst, -d): buf for (src, dst, d), buf in local.items()}
        sends = sorted(k for k in outgoing if k not in local)
        # the mirror of every remote send: that neighbour sends back over the same face pair
        recvs = sorted((dst, src, -d) for (src, dst, d) in sends)
        ops = [self.dist.P2POp(self.dist.isend, outgoing[k], self.rank_of[k[1]], self.group) for k in sends]
        for (src, dst, d) in recvs:
            buf = self.make_buffer(outgoing[(dst, src, -d)].numel())
            incoming[(src, dst, -d)] = buf
            ops.append(self.dist.P2POp(self.dist.irecv, buf, self.rank_of[src], self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return incoming

    def minimum(self, x: float) -> float:
        t = self.make_buffer(1)
        t.fill_(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return float(t.item())


class SlabRun:
    """RK3 steps of the slabs `ids` (of n_slabs along `axis`) held by this
    process, zones[q] providing the zone operations of slab ids[q]
    (LibraryZone on the GPU).  periodic: the block's two faces on `axis`
    are one periodic seam, exchanged between the first and last slab like a
    cut (the parallel-face form of periodicity; n_slabs >= 2)."""

    def __init__(self, zones, ids, n_slabs: int, axis: int, transport, two_d: bool, periodic: bool = False):
        if periodic and n_slabs < 2:
            raise ValueError("a periodic seam needs two slabs at least")
        self.zones, self.ids, self.n, self.axis = list(zones), list(ids), n_slabs, axis
        self.tr, self.two_d, self.periodic = transport, two_d, periodic

    def neighbour(self, s: int, d: int):
        t = s + d
        if 0 <= t < self.n:
            return t
        return t % self.n if self.periodic else None

    def exchange(self):
        out = {}
        for z, s in zip(self.zones, self.ids):
            for d in (-1, 1):
                t = self.neighbour(s, d)
                if t is not None:
                    out[(s, t, d)] = z.halo_pack(self.axis, d)
        got = self.tr.exchange(out)
        for z, s in zip(self.zones, self.ids):
            for d in (-1, 1):
                t = self.neighbour(s, d)
                if t is not None:
                    z.halo_assign(self.axis, d, got[(t, s, d)])
        if self.two_d:
            for z in self.zones:
                z.eliminate_k()

    def initialize(self):
        """src/Driver.cu:126-211: properties, BCs, communication, properties;
        then cv from bv over the padded block (src/RK.cuh:37-46)."""
        for z in self.zones:
            z.properties()
        for z in self.zones:
            z.bc()
        self.exchange()
        for z in self.zones:
            z.properties()
            z.cv_from_bv()

    def step(self) -> float:
        """One RK3 step (src/RK.cuh:84-216): qn <- cv, dt the minimum over
        every slab of the local CFL steps, three stages of right-hand side
        and update, boundary conditions, halo exchange, properties."""
        for z in self.zones:
            z.save_qn()
        dt = self.tr.minimum(min(z.local_dt() for z in self.zones))
        for rk in range(3):
            for z in self.zones:
                z.zero_dq()
                z.viscous()
                z.inviscid()
                z.update(dt, rk)
            for z in self.zones:
                z.bc()
            self.exchange()
            for z in self.zones:
                z.properties()
        return dt


class LibraryZone:
    """Zone operations of a slab on the GPU through the C ABI: `ctx` a bound
    corefl_b200.Context, `t` its device arrays (torch tensors, reference
    layout) with at least cv, qn, dq, and `param` the context's parameters.
    The step's start computes the shock sensor where the scheme has one
    (src/RK.cuh:112-116); the right-hand side adds the explicit chemical
    source of a reacting mixture (src/RK.cuh:147-149); the update is followed
    by limit_flow where it is on (src/RK.cuh:162-165)."""

    def __init__(self, ctx, t, param):
        import torch

        self.ctx, self.t, self.torch = ctx, t, torch
        self.sensor = param.get("sensor_threshold", 0.0) > 1e-10
        self.chem = param.get("n_spec", 0) > 0 and param.get("n_reac", 0) > 0
        self.limit = bool(param.get("limit_flow", 0))

    def halo_pack(self, face, direction):
        buf = self.torch.empty(self.ctx.halo_size(face), dtype=self.torch.float64, device=self.t["cv"].device)
        self.ctx.halo_pack(face, direction, buf.data_ptr())
        return buf

    def halo_assign(self, face, direction, buf):
        self.ctx.halo_assign(face, direction, buf.data_ptr())

    def eliminate_k(self):
        self.ctx.eliminate_k_gradient()

    def properties(self):
        self.ctx.properties()

    def bc(self):
        self.ctx.boundary_conditions()

    def cv_from_bv(self):
        self.ctx.cv_from_bv()

    def save_qn(self):
        self.t["qn"].copy_(self.t["cv"])
        if self.sensor:
            self.ctx.shock_sensor()

    def local_dt(self):
        return self.ctx.local_time_step()

    def zero_dq(self):
        self.t["dq"].zero_()

    def viscous(self):
        self.ctx.viscous()
        if self.chem:
            self.ctx.finite_rate_chemistry()

    def inviscid(self):
        self.ctx.inviscid()

    def update(self, dt, rk):
        self.ctx.update_rk(dt, rk)
        if self.limit:
            self.ctx.limit_flow()
