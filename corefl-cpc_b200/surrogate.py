"""Host-side workflow of the MLP chemistry surrogate over the C ABI.

Training data come from the library's own plain point-implicit reaction step
(cfk_wu_reaction_step), recorded on the device; normalisation, training,
inference and the gated reaction step all run in the library's kernels.
Device buffers are torch tensors (device memory only).
"""
from __future__ import annotations

import numpy as np

import corefl_b200 as cf


def record_trajectories(ctx: "cf.Context", n_nodes: int, steps: int, dt: float, torch, every: int = 1,
                        schedule: int = 1, device: str = "cuda:0"):
    """Run `steps` plain reaction steps of dt on the bound zone and record one
    (features, targets) row per node for every `every`-th step.  Returns
    device tensors X (rows, 12) and G (rows, 11)."""
    n_rec = (steps + every - 1) // every
    X = torch.empty((n_rec * n_nodes, cf.SG_NIN), dtype=torch.float32, device=device)
    G = torch.empty((n_rec * n_nodes, cf.SG_NOUT), dtype=torch.float32, device=device)
    r = 0
    for s in range(steps):
        rec = s % every == 0
        if rec:
            ctx.surrogate_record(0, dt)
        ctx.wu_reaction_step(dt, schedule=schedule)
        if rec:
            ctx.surrogate_record(1, dt, X[r * n_nodes].data_ptr(), G[r * n_nodes].data_ptr())
            r += 1
    ctx.sync()
    return X, G


def fit(ctx: "cf.Context", X, G, epochs: int = 40, batch: int = 8192, lr0: float = 2e-3, lr1: float = 2e-5,
        seed: int = 0):
    """Standardisation from (X, G), then Adam on the device; returns the
    per-epoch mean losses."""
    n = X.shape[0]
    ctx.surrogate_fit_normalization(X.data_ptr(), G.data_ptr(), n)
    return ctx.surrogate_train(X.data_ptr(), G.data_ptr(), n, epochs, batch, lr0, lr1, seed)


def ignition_metrics(dt: float, T0: np.ndarray, T: np.ndarray):
    """Per-cell ignition delay, peak temperature and largest per-step rise.
    T is (steps, cells), the temperature after each step of dt from T0; the
    ignition delay is the midpoint of the step with the largest rise (the
    time of max dT/dt on the per-step trajectory)."""
    dT = np.diff(np.vstack([np.asarray(T0)[None, :], T]), axis=0)
    k = np.argmax(dT, axis=0)
    return (k + 0.5) * dt, T.max(axis=0), dT.max(axis=0)


def record_flow(ctx: "cf.Context", n_nodes: int, steps: int, torch, every: int = 1, schedule: int = 1,
                device: str = "cuda:0"):
    """Run `steps` plain Wu-splitting steps of the bound flow zone and record
    one (features, targets) row per node of the reaction sub-step for every
    `every`-th step (cfk_wu_splitting_step_record: features at the frozen
    transport term's mid-step state, targets from its end state).  Returns
    device tensors X (rows, 12), G (rows, 11) and the step sizes."""
    n_rec = (steps + every - 1) // every
    X = torch.empty((n_rec * n_nodes, cf.SG_NIN), dtype=torch.float32, device=device)
    G = torch.empty((n_rec * n_nodes, cf.SG_NOUT), dtype=torch.float32, device=device)
    dts, r = [], 0
    for s in range(steps):
        if s % every == 0:
            dts.append(ctx.wu_splitting_step_record(X[r * n_nodes].data_ptr(), G[r * n_nodes].data_ptr(), schedule))
            r += 1
        else:
            dts.append(ctx.wu_splitting_step(schedule))
    ctx.sync()
    return X, G, np.array(dts)
