"""Slab zone operations on the CPU oracle (the checker of the slab driver),
and the comparison of decomposed runs against the whole block."""
from __future__ import annotations

import ctypes

import numpy as np

import pyoracle


class OracleSlabZone:
    """The zone operations slabs.SlabRun calls, on one oracle block.  Halo
    buffers are torch CPU tensors so that gloo can carry them."""

    def __init__(self, case):
        import torch

        self.torch = torch
        self.case = case
        self.oz = pyoracle.OracleZone(case)
        self.sensor = case.param.get("sensor_threshold", 0.0) > 1e-10

    def __getitem__(self, k):
        return self.oz[k]

    def halo_pack(self, face, direction):
        return self.torch.from_numpy(self.oz.halo_pack(face, direction))

    def halo_assign(self, face, direction, buf):
        self.oz.halo_assign(face, direction, buf.numpy())

    def eliminate_k(self):
        self.oz.call("orc_eliminate_k_gradient")

    def properties(self):
        self.oz.call("orc_update_physical_properties")

    def bc(self):
        self.oz.call("orc_apply_boundary_conditions")

    def cv_from_bv(self):
        self.oz.call("orc_compute_cv_from_bv")

    def save_qn(self):
        self.oz["qn"][:] = self.oz["cv"]
        if self.sensor:
            self.oz.call("orc_compute_shock_sensor")

    def local_dt(self):
        self.oz.call("orc_local_time_step")
        return self.oz.L.orc_global_time_step(ctypes.byref(self.oz.z))

    def zero_dq(self):
        self.oz["dq"][:] = 0.0

    def viscous(self):
        self.oz.call("orc_compute_viscous_flux")

    def inviscid(self):
        self.oz.call("orc_compute_inviscid_flux")

    def update(self, dt, rk):
        self.oz.z.dt_step = dt
        self.oz.call("orc_update_cv_and_bv_rk", dt, rk)


def interior(case, arr):
    g = case.ngg
    a = arr.reshape((arr.shape[0],) + case.shape())
    return a[:, g:g + case.mz, g:g + case.my, g:g + case.mx]


def assemble(whole, slabs, arrays, axis):
    """The whole block's interior of a (n, P) variable stack put together
    from the slabs' interiors (a shared cut plane taken from the lower
    slab), and the largest difference between the two copies of each cut
    plane."""
    import slabs as sl

    m = (whole.mx, whole.my, whole.mz)[axis]
    ax = 3 - axis  # array axis in (n, k, j, i)
    parts, seam = [], 0.0
    bounds = sl.slab_bounds(m, len(slabs))
    for r, (c, a) in enumerate(zip(slabs, arrays)):
        it = interior(c, a)
        if r > 0:
            prev = np.take(parts[-1], [-1], axis=ax)
            seam = max(seam, float(np.abs(np.take(it, [0], axis=ax) - prev).max()))
            it = np.take(it, range(1, it.shape[ax]), axis=ax)
        parts.append(it)
    out = np.concatenate(parts, axis=ax)
    assert out.shape[ax] == m and bounds[-1][1] == m - 1
    return out, seam


def plane_scale(*arrays):
    """Largest magnitude of each variable plane over all the given (n, ...)
    arrays, the three momentum planes sharing one scale."""
    scale = np.max([np.abs(b).reshape(b.shape[0], -1).max(axis=1) for b in arrays], axis=0)
    if scale.shape[0] >= 4:
        scale[1:4] = scale[1:4].max()
    return np.where(scale == 0, 1.0, scale)


def rel_diff(a, b, scale=None):
    """Largest difference relative to each variable plane's largest magnitude
    in b (the three momentum planes sharing one scale), or to `scale` (per
    plane, e.g. plane_scale over every slab of a decomposition: a slab of gas
    at rest has momenta at round-off level, which are no scale of their own)."""
    if scale is None:
        scale = plane_scale(b)
    return float((np.abs(a - b).reshape(b.shape[0], -1) / np.asarray(scale)[:, None]).max())


def run_rank(rank, world, port, spec, out):
    """One gloo rank of a decomposed run: the slabs rank_of assigns to this
    rank, stepped `steps` times; out[rank] = {slab id: (cv, bv)}."""
    import os

    import torch
    import torch.distributed as dist

    import slabs as sl

    case_fn, n, axis, steps, rank_of, periodic = spec
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        whole = case_fn()
        parts = sl.split_slabs(whole, n, axis, periodic=periodic)
        ids = [s for s in range(n) if rank_of[s] == rank]
        zones = [OracleSlabZone(parts[s]) for s in ids]
        tr = sl.DistTransport(dist, rank_of, lambda k: torch.empty(k, dtype=torch.float64))
        run = sl.SlabRun(zones, ids, n, axis, tr, two_d=whole.mz == 1, periodic=periodic)
        run.initialize()
        dts = [run.step() for _ in range(steps)]
        out[rank] = {s: (z["cv"].copy(), z["bv"].copy(), dts) for s, z in zip(ids, zones)}
    finally:
        dist.destroy_process_group()
