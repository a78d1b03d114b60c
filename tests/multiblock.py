"""Multi-block RK3 stepping for the tests, on the CPU oracle or on the GPU
through the C ABI, in the reference's order across blocks (src/RK.cuh:84-212):
per step qn <- cv and dt = the minimum of the blocks' local CFL steps; per
stage every block's dq reset, viscous and inviscid terms and update, then
every block's boundary conditions, then the inner-face communication of every
block face by face (src/DataCommunication.cu:6-34), then (2-D) the k-ghost
copy, then every block's properties.  The start of a run follows
src/Driver.cu:126-211 (properties, BCs, communication, k-ghost copy,
properties) and then computes cv from bv."""
from __future__ import annotations

import ctypes

import numpy as np

import corefl_b200 as cfk
import pyoracle


class _Blocks:
    def __init__(self, cases_, links):
        self.cases = list(cases_)
        self.two_d = self.cases[0].mz == 1
        self.links = links

    def _communicate(self):
        for b, face in self.faces:
            self.comm(b, face)
        if self.two_d:
            for b in range(len(self.cases)):
                self.elim(b)

    def initialize(self):
        n = len(self.cases)
        for b in range(n):
            self.properties(b)
        for b in range(n):
            self.bc(b)
        self._communicate()
        for b in range(n):
            self.properties(b)
            self.cv_from_bv(b)
        self.sync()

    def step(self) -> float:
        n = len(self.cases)
        for b in range(n):
            self.save_qn(b)
        dt = min(self.local_dt(b) for b in range(n))
        for rk in range(3):
            for b in range(n):
                self.zero_dq(b)
                self.viscous(b)
                self.inviscid(b)
                self.update(b, dt, rk)
            for b in range(n):
                self.bc(b)
            self._communicate()
            for b in range(n):
                self.properties(b)
        self.sync()
        return dt

    def sync(self):
        pass


class OracleBlocks(_Blocks):
    def __init__(self, cases_, links):
        super().__init__(cases_, links)
        self.z = [pyoracle.OracleZone(c) for c in self.cases]
        dim, ngg = self.cases[0].param["dim"], self.cases[0].ngg
        self.faces = [(b, pyoracle.register_inner_face(dim, ngg, s, t, tb)) for b, s, t, tb in links]

    def comm(self, b, face):
        self.z[b].inner_communication(self.z[face.target_block], face)

    def elim(self, b):
        self.z[b].call("orc_eliminate_k_gradient")

    def properties(self, b):
        self.z[b].call("orc_update_physical_properties")

    def cv_from_bv(self, b):
        self.z[b].call("orc_compute_cv_from_bv")

    def bc(self, b):
        self.z[b].call("orc_apply_boundary_conditions")

    def save_qn(self, b):
        self.z[b]["qn"][:] = self.z[b]["cv"]

    def local_dt(self, b):
        oz = self.z[b]
        oz.call("orc_local_time_step")
        return oz.L.orc_global_time_step(ctypes.byref(oz.z))

    def zero_dq(self, b):
        self.z[b]["dq"][:] = 0.0

    def viscous(self, b):
        self.z[b].call("orc_compute_viscous_flux")

    def inviscid(self, b):
        self.z[b].call("orc_compute_inviscid_flux")

    def update(self, b, dt, rk):
        self.z[b].z.dt_step = dt
        self.z[b].call("orc_update_cv_and_bv_rk", dt, rk)


class GpuBlocks(_Blocks):
    def __init__(self, cases_, links):
        from gpuzone import GpuZone

        super().__init__(cases_, links)
        self.g = [GpuZone(c) for c in self.cases]
        dim, ngg = self.cases[0].param["dim"], self.cases[0].ngg
        self.faces = [(b, cfk.register_inner_face(dim, ngg, s, t, tb)) for b, s, t, tb in links]

    def comm(self, b, face):
        self.g[b].ctx.inner_communication(self.g[face.target_block].ctx, face)

    def elim(self, b):
        self.g[b].ctx.eliminate_k_gradient()

    def properties(self, b):
        self.g[b].ctx.properties()

    def cv_from_bv(self, b):
        self.g[b].ctx.cv_from_bv()

    def bc(self, b):
        self.g[b].ctx.boundary_conditions()

    def save_qn(self, b):
        self.g[b].t["qn"].copy_(self.g[b].t["cv"])

    def local_dt(self, b):
        return self.g[b].ctx.local_time_step()

    def zero_dq(self, b):
        self.g[b].t["dq"].zero_()

    def viscous(self, b):
        self.g[b].ctx.viscous()

    def inviscid(self, b):
        self.g[b].ctx.inviscid()

    def update(self, b, dt, rk):
        self.g[b].ctx.update_rk(dt, rk)

    def sync(self):
        self.g[0].torch.cuda.synchronize()


def whole_interior_of(case, arr, lo, hi):
    """Interior nodes i = lo..hi of a padded (n, P) array of `case`, as
    (n, mz, my, hi - lo + 1)."""
    g = case.ngg
    a = arr.reshape(arr.shape[0], case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)
    return a[:, g:g + case.mz, g:g + case.my, g + lo:g + hi + 1]


def interior_of(case, arr):
    return whole_interior_of(case, arr, 0, case.mx - 1)


def split_difference(whole, whole_arr, A, B, arrs, h):
    """Largest difference between the interiors of blocks A and B (cut at
    node plane h) and the matching interior nodes of the whole block,
    relative to each plane's largest magnitude in the whole block; the three
    momentum planes share one scale, as in gpuzone.rel_err."""
    scale = np.abs(whole_arr).max(axis=1)
    scale[1:4] = scale[1:4].max()
    scale = np.where(scale == 0, 1.0, scale)[:, None, None, None]
    ea = np.abs(interior_of(A, arrs[0]) - whole_interior_of(whole, whole_arr, 0, h)) / scale
    eb = np.abs(interior_of(B, arrs[1]) - whole_interior_of(whole, whole_arr, h, whole.mx - 1)) / scale
    return float(max(ea.max(), eb.max()))
