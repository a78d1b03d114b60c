"""The batched-reactor workload node by node: the reference's own build against
this library (a check, not part of the library).

2^20 seeded Li-2004 constant-volume reactors (seed 2026; T ~ U[1000,1600] K,
p log-uniform in [1,10] atm, phi ~ U[0.5,2]) advance `--steps` point-implicit
reaction steps of 1e-7 s twice: with oracle/_ref/refharness in its reactlast
mode (the reference's wu_reaction_step, src/StrangSplitting.cu:373-421, state
written after the last step), and with this library's one-thread-per-node
reaction step through the C ABI (and once more with its work-queue schedule,
for the timing).  Prints one JSON object: the largest relative temperature
difference over all nodes, the number of nodes differing by more than 1e-12,
the same for the reaction time scale, and this library's per-step device
times of both schedules and largest substep counts.  Run on a machine with a GPU
after `make -C oracle/ref REF=<reference checkout>`:

    python oracle/ref/compare_reactors_gpu.py [--steps 13] [--side 1024]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_ref_fixtures as mrf  # noqa: E402
import time_ref_gpu as trg  # noqa: E402
from make_ref_fixtures import cases  # noqa: E402

import corefl_b200 as cfk  # noqa: E402  (on the path through make_ref_fixtures)
import mechanism  # noqa: E402


def library_run(case, mech, steps, schedule=0):
    """This library's reaction steps of 1e-7 s (schedule 0: one thread per
    node, 1: the work queue): final T and reaction time scale (node order),
    per-step ms and max substeps."""
    import torch

    param = dict(case.param)
    param["device"] = 0
    ctx = cfk.Context(param, case.faces)
    zone = ctx.alloc_zone(case.mx, case.my, case.mz)
    ctx.set_mechanism(mech)
    for fld, arr in (("bv", case.bv), ("sv", case.sv), ("jac", case.jac), ("metric", case.metric)):
        a = np.ascontiguousarray(arr)
        ctx.h2d(getattr(zone, fld), a.ctypes.data, a.nbytes)
    ctx.cv_from_bv()
    nsub = torch.zeros(case.N, dtype=torch.int32, device="cuda:0")
    ms, mx = [], []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.wu_reaction_step(1e-7, schedule=schedule, nsub_ptr=nsub.data_ptr())
        e1.record()
        torch.cuda.synchronize()
        ms.append(round(e0.elapsed_time(e1), 3))
        mx.append(int(nsub.max().item()))
    P = case.P
    T = torch.empty(P, dtype=torch.float64, device="cuda:0")
    ts = torch.empty(P, dtype=torch.float64, device="cuda:0")
    ctx.d2d(T.data_ptr(), zone.bv + 5 * P * 8, P * 8)
    ctx.d2d(ts.data_ptr(), zone.reaction_timeScale, P * 8)
    ctx.sync()
    T, ts = T.cpu().numpy(), ts.cpu().numpy()
    ctx.close()
    return case.interior(T).reshape(-1), case.interior(ts).reshape(-1), ms, mx


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=13)
    ap.add_argument("--side", type=int, default=1024, help="reactors = side^2 (default 2^20)")
    a = ap.parse_args()
    if not os.path.exists(mrf.HARNESS):
        sys.exit(f"{mrf.HARNESS} not built (make -C oracle/ref REF=<reference checkout>)")
    work = tempfile.mkdtemp(prefix="cmpreact_")
    try:
        spec = trg._reactor_spec(a.side)
        d = mrf.prepare_case(spec, work)
        r = subprocess.run([mrf.HARNESS, d, "reactlast", str(a.steps), "1e-07"], capture_output=True, text=True,
                           timeout=3600)
        if r.returncode != 0:
            sys.exit(f"refharness exited {r.returncode}\n{r.stderr[-2000:]}")
        g = cases.ghost_layers(52)
        shape = (1 + 2 * g, a.side + 2 * g, a.side + 2 * g)

        def ref_interior(name, planes):
            arr = np.fromfile(os.path.join(d, "out", f"state_{a.steps}_{name}.bin"), dtype=np.float64)
            return arr.reshape(planes, *shape)[:, g, g:g + a.side, g:g + a.side].reshape(planes, -1)

        T_ref = ref_interior("bv", 6)[5]
        ts_ref = ref_interior("reaction_timeScale", 1)[0]
    finally:
        shutil.rmtree(work, ignore_errors=True)
    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, a.side * a.side, seed=2026)
    T, ts, ms, mx = library_run(case, mech, a.steps)
    _, _, ms_q, _ = library_run(case, mech, a.steps, schedule=1)
    rT = np.abs(T - T_ref) / T_ref
    rts = np.abs(ts - ts_ref) / np.maximum(np.abs(ts_ref), 1e-300)
    print(json.dumps({
        "reactors": int(case.N), "steps": a.steps, "dt": 1e-7,
        "T_max_rel_diff": float(rT.max()), "T_nodes_above_1e-12": int((rT > 1e-12).sum()),
        "tau_max_rel_diff": float(rts.max()), "tau_nodes_above_1e-12": int((rts > 1e-12).sum()),
        "nan_ref": int(np.isnan(T_ref).sum()), "nan_library": int(np.isnan(T).sum()),
        "library_ms_per_step": ms, "library_queue_ms_per_step": ms_q, "library_max_substeps": mx}))


if __name__ == "__main__":
    main()
