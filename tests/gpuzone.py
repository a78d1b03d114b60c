"""Test helpers: device arrays of one block (torch allocations, reference
layout) bound to a corefl_b200 context, and comparison utilities."""
from __future__ import annotations

import numpy as np

import corefl_b200 as cfk


class GpuZone:
    def __init__(self, case, param_overrides=None, sensor_array=True):
        import torch

        self.torch = torch
        self.case = case
        p = dict(case.param)
        if param_overrides:
            p.update(param_overrides)
        self.param = p
        self.ctx = cfk.Context(p, case.faces)
        c = case
        nv, nsc, ns = p["n_var"], p["n_scalar"], p["n_spec"]
        P, N = c.P, c.N
        dev = torch.device("cuda:0")
        z = lambda *s: torch.zeros(s, dtype=torch.float64, device=dev)
        self.t = {
            "jac": torch.from_numpy(np.ascontiguousarray(c.jac)).to(dev),
            "metric": torch.from_numpy(np.ascontiguousarray(c.metric)).to(dev),
            "cv": z(nv, P), "bv": torch.from_numpy(c.bv.copy()).to(dev), "qn": z(nv, P),
            "mul": z(P), "mach": z(P), "dq": z(nv, N), "dt_local": z(N),
        }
        if nsc:
            self.t["sv"] = torch.from_numpy(np.ascontiguousarray(c.sv)).to(dev) if c.sv.shape[0] else z(nsc, P)
        if ns:
            for k in ("acoustic_speed", "gamma", "thermal_conductivity", "reaction_timeScale"):
                self.t[k] = z(P)
            self.t["rho_D"] = z(ns, P)
            self.t["Cn"] = z(nv, N)
        if getattr(c, "y", None) is not None:
            self.t["y"] = torch.from_numpy(np.ascontiguousarray(c.y)).to(dev)
        if sensor_array and p.get("sensor_threshold", 0.0) > 1e-10:
            self.t["shock_sensor"] = z(P)  # else the context allocates its own
        self.ctx.bind(c.mx, c.my, c.mz, c.ngg, {k: v.data_ptr() for k, v in self.t.items()})
        if ns:
            self.ctx.set_mechanism(c.mech)

    def initialize(self):
        """properties, BCs (with the 2-D k-ghost copy), properties, cv from bv —
        the same start-of-run sequence the oracle helper uses."""
        self.ctx.properties()
        self.ctx.boundary_conditions()
        self.ctx.properties()
        self.ctx.cv_from_bv()
        self.torch.cuda.synchronize()

    def get(self, k) -> np.ndarray:
        self.torch.cuda.synchronize()
        return self.t[k].cpu().numpy()

    def load_from(self, oz, keys=("cv", "bv", "mul", "qn")):
        """Copy the oracle's state arrays into the device arrays."""
        for k in keys:
            self.t[k].copy_(self.torch.from_numpy(oz[k][: self.t[k].shape[0]]).to(self.t[k].device))
        if "sv" in self.t:
            self.t["sv"].copy_(self.torch.from_numpy(oz["sv"][: self.t["sv"].shape[0]]))


def rel_err(a: np.ndarray, b: np.ndarray, momentum=(1, 2, 3)) -> float:
    """Normwise relative difference, maximised over variable planes:
    max|a_l - b_l| / scale_l, where scale_l = max|b_l| except that the three
    momentum planes share one scale (the largest of them), so that a
    component that is zero up to round-off (v in a 1-D problem) is measured
    against the momentum magnitude rather than against its own round-off.
    Pass momentum=() for arrays that are not conserved-variable stacks."""
    a = np.atleast_2d(a)
    b = np.atleast_2d(b)
    mom = [l for l in momentum if l < b.shape[0]]
    mom_scale = max((np.abs(b[l]).max() for l in mom), default=0.0)
    worst = 0.0
    for l in range(b.shape[0]):
        scale = mom_scale if l in mom else np.abs(b[l]).max()
        if scale == 0:
            scale = 1.0
        worst = max(worst, float(np.abs(a[l] - b[l]).max() / scale))
    return worst


def interior_planes(case, arr: np.ndarray) -> np.ndarray:
    """Interior nodes of every plane of a padded (n, P) array, as (n, N)."""
    return np.stack([case.interior(arr[l]).reshape(-1) for l in range(arr.shape[0])])


def pointwise_rel_err(a: np.ndarray, b: np.ndarray, n_spec: int = 0, p: np.ndarray | None = None) -> float:
    """Pointwise relative difference of conserved-variable stacks (n, N),
    maximised over nodes and variables: density and total energy |a - b| / |b|
    at each node; each momentum component |a_l - b_l| / max(|rho V|, rho c) at
    each node, with the node's own momentum magnitude, or, where the flow is
    slower than sound, the acoustic momentum rho c (ideal gas, gamma = 1.4,
    from the node's density, energy and momentum) — a component that is zero
    up to round-off, like v in a 1-D problem, has no relative error of its own;
    the partial densities |a_l - b_l| / rho (mass-fraction units).  For
    mixtures (n_spec > 0), whose energy includes formation enthalpies, the
    momentum floor is 1e-8 of the largest momentum magnitude instead of rho c,
    unless the node pressures p of the reference state are given: then the
    floor is sqrt(p rho), a lower bound of rho c for any gas (gamma >= 1)."""
    a = np.atleast_2d(a)
    b = np.atleast_2d(b)
    worst = 0.0
    for l in (0, 4):
        if l < b.shape[0]:
            worst = max(worst, float((np.abs(a[l] - b[l]) / np.abs(b[l])).max()))
    if b.shape[0] >= 5:
        mag2 = b[1] ** 2 + b[2] ** 2 + b[3] ** 2
        mag = np.sqrt(mag2)
        if p is not None:
            floor = np.sqrt(np.maximum(np.asarray(p) * b[0], 0.0))
        elif n_spec == 0:
            p_air = 0.4 * (b[4] - 0.5 * mag2 / b[0])
            floor = np.sqrt(np.maximum(1.4 * p_air * b[0], 0.0))
        else:
            floor = 1e-8 * max(float(mag.max()), 1e-300)
        den = np.maximum(np.maximum(mag, floor), 1e-300)
        for l in (1, 2, 3):
            worst = max(worst, float((np.abs(a[l] - b[l]) / den).max()))
    for l in range(5, 5 + n_spec):
        if l < b.shape[0]:
            worst = max(worst, float((np.abs(a[l] - b[l]) / np.abs(b[0])).max()))
    return worst
