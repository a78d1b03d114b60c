"""Replays the reference's recorded runs (tests/golden/ref_*.npz, written by
oracle/ref/make_ref_fixtures.py from the reference's own build) through the
CPU oracle or the CUDA library, step by step from the same inputs, and
measures the differences.

Each fixture names its case through the generator's builders, so the inputs
here are the ones the reference ran on: the padded initial basic variables
(or, where the reference initialised itself from setup.txt, this package's
builder of the same state, which the replay checks against the reference's
interior), the same grid, and the reference's own derived scalars (the WENO
epsilon scale of its reference state).
"""
from __future__ import annotations

import dataclasses
import importlib.util
import os
import sys

import numpy as np

from gpuzone import pointwise_rel_err, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden")

_gen = None


def generator():
    """The fixture generator module (its case specifications)."""
    global _gen
    if _gen is None:
        spec = importlib.util.spec_from_file_location("make_ref_fixtures",
                                                      os.path.join(ROOT, "oracle", "ref", "make_ref_fixtures.py"))
        _gen = importlib.util.module_from_spec(spec)
        sys.modules["make_ref_fixtures"] = _gen
        spec.loader.exec_module(_gen)
    return _gen


def names():
    """The recorded runs, by the generator's spec key."""
    return list(generator().SPECS)


def fixture_path(name):
    return os.path.join(GOLDEN, f"ref_{generator().SPECS[name]().name}.npz")


def load(name):
    with np.load(fixture_path(name)) as z:
        return {k: z[k] for k in z.files}


def spec_and_case(name, fx):
    """The generator's spec, with the reference's derived scalars applied."""
    spec = generator().SPECS[name]()
    c = spec.case
    param = dict(c.param)
    param.update(weno_eps_scale=float(fx["param_weno_eps_scale"]), rho_ref=float(fx["param_rho_ref"]),
                 v_ref=float(fx["param_v_ref"]))
    return spec, dataclasses.replace(c, param=param)


def interior(case, a):
    """(n, P) padded planes -> (n, N) interior nodes."""
    a = np.atleast_2d(a)
    return np.stack([case.interior(a[l]).reshape(-1) for l in range(a.shape[0])])


def grid_differences(case, fx):
    """Largest relative differences between the builder's metric and Jacobian
    and the reference's, over the sampled padded nodes it recorded.  Only the
    nodes the reference fills are compared: it leaves the corner ghost nodes
    (outside the block in two or more directions) of its ghost grid unset."""
    idx = fx["grid_idx"]
    mx, my, mz, g = (int(v) for v in fx["shape"])
    shape = (mz + 2 * g, my + 2 * g, mx + 2 * g)
    k, j, i = np.unravel_index(idx, shape)
    outside = ((i < g) | (i >= g + mx)).astype(int) + ((j < g) | (j >= g + my)).astype(int)
    if mz > 1:
        outside += ((k < g) | (k >= g + mz)).astype(int)
    keep = outside <= 1
    m_ref, j_ref = fx["metric"][:, keep], fx["jac"][keep]
    m_b, j_b = case.metric[:, idx][:, keep], case.jac[idx][keep]
    scale = np.maximum(np.abs(m_ref).max(axis=1, keepdims=True), 1e-300)
    e_m = float((np.abs(m_b - m_ref) / scale).max())
    e_j = float((np.abs(j_b - j_ref) / np.abs(j_ref)).max())
    return e_m, e_j


@dataclasses.dataclass
class StepReport:
    step: int
    dt_rel: float
    cv_norm: float
    cv_point: float
    extra: dict


def compare_state(case, fx, s, cv, sv=None, ts=None, n_spec=0):
    ref = fx["cv"][s]
    extra = {}
    if sv is not None and "sv" in fx:
        extra["sv"] = float(np.abs(sv - fx["sv"][s]).max())
    if ts is not None and "reaction_timeScale" in fx:
        r = fx["reaction_timeScale"][s]
        extra["timescale"] = float((np.abs(ts - r) / np.maximum(np.abs(r), 1e-300)).max())
    return rel_err(cv, ref), pointwise_rel_err(cv, ref, n_spec=n_spec, p=fx["p"][s]), extra


class OracleReplay:
    def __init__(self, name):
        import pyoracle

        self.fx = load(name)
        self.spec, self.case = spec_and_case(name, self.fx)
        self.oz = pyoracle.OracleZone(self.case)
        self.n_spec = self.case.param["n_spec"]

    def start(self):
        self.oz.initialize()
        if self.spec.mode == "react":
            self.set_timescale(self.fx["reaction_timeScale"][0])

    def set_timescale(self, ts):
        a = self.oz["reaction_timeScale"]
        self.case.interior(a)[...] = ts.reshape(self.case.mz, self.case.my, self.case.mx)

    def state(self):
        cv = interior(self.case, self.oz["cv"])
        sv = interior(self.case, self.oz["sv"])[: self.n_spec] if self.n_spec else None
        ts = interior(self.case, self.oz["reaction_timeScale"])[0] if self.n_spec else None
        return cv, sv, ts

    def step(self):
        if self.spec.mode == "rk3":
            return self.oz.step()
        if self.spec.mode == "wu":
            return self.oz.wu_splitting_step()
        self.oz["Cn"][...] = 0
        self.oz.reaction_step(self.spec.react_dt)
        return self.spec.react_dt


class GpuReplay(OracleReplay):
    def __init__(self, name):
        from gpuzone import GpuZone

        self.fx = load(name)
        self.spec, self.case = spec_and_case(name, self.fx)
        self.gz = GpuZone(self.case)
        self.n_spec = self.case.param["n_spec"]

    def start(self):
        self.gz.initialize()
        if self.spec.mode == "react":
            import torch

            a = self.gz.get("reaction_timeScale")
            self.case.interior(a)[...] = self.fx["reaction_timeScale"][0].reshape(self.case.mz, self.case.my,
                                                                                 self.case.mx)
            self.gz.t["reaction_timeScale"].copy_(torch.from_numpy(a))

    def state(self):
        cv = interior(self.case, self.gz.get("cv"))
        sv = interior(self.case, self.gz.get("sv"))[: self.n_spec] if self.n_spec else None
        ts = interior(self.case, self.gz.get("reaction_timeScale"))[0] if self.n_spec else None
        return cv, sv, ts

    def step(self):
        if self.spec.mode == "rk3":
            return self.gz.ctx.rk3_step()
        if self.spec.mode == "wu":
            return self.gz.ctx.wu_splitting_step(schedule=1)
        self.gz.t["Cn"].zero_()
        self.gz.ctx.wu_reaction_step(self.spec.react_dt, schedule=1)
        self.gz.ctx.sync()
        return self.spec.react_dt


def replay(r: OracleReplay):
    """Runs every recorded step; returns the reports (step 0 = the state after
    initialisation)."""
    r.start()
    out = []
    cv, sv, ts = r.state()
    e_n, e_p, extra = compare_state(r.case, r.fx, 0, cv, sv, ts, r.n_spec)
    out.append(StepReport(0, 0.0, e_n, e_p, extra))
    for s in range(1, r.fx["cv"].shape[0]):
        dt = r.step()
        ref_dt = float(r.fx["dt"][s - 1])
        cv, sv, ts = r.state()
        e_n, e_p, extra = compare_state(r.case, r.fx, s, cv, sv, ts, r.n_spec)
        out.append(StepReport(s, abs(dt - ref_dt) / abs(ref_dt), e_n, e_p, extra))
    return out
