"""The headline block node by node: the reference's own build against this
library (a check, not part of the library).

The 257^3 curvilinear periodic wave (WENO7 characteristic + 2nd-order viscous
flux, SSP-RK3) advances `--steps` RK3 steps twice from the same inputs: with
oracle/_ref/refharness in its rk3last mode (the reference's RK3 loop body,
src/RK.cuh:89-206, state written after the last step) and with this library's
cfk_rk3_step through the C ABI.  With --fixed-dt the step is fixed, else both
take their own CFL step.  Prints one JSON object: the time step of each and
the normwise and pointwise relative differences of the conserved variables
after the last step.  Run on a machine with a GPU after
`make -C oracle/ref REF=<reference checkout>`:

    python oracle/ref/compare_wave_gpu.py [--n 257] [--steps 2] [--fixed-dt DT]
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
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import make_ref_fixtures as mrf  # noqa: E402
import time_ref_gpu as trg  # noqa: E402
from gpuzone import GpuZone, interior_planes, pointwise_rel_err, rel_err  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=257)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--fixed-dt", type=float, default=0.0, help="fixed time step (0: the CFL step)")
    a = ap.parse_args()
    if not os.path.exists(mrf.HARNESS):
        sys.exit(f"{mrf.HARNESS} not built (make -C oracle/ref REF=<reference checkout>)")
    spec = trg._wave_spec(a.n)
    case = spec.case
    if a.fixed_dt > 0:
        case.param.update(fixed_dt=1, dt=a.fixed_dt)
    work = tempfile.mkdtemp(prefix="cmpwave_")
    try:
        d = mrf.prepare_case(spec, work)
        r = subprocess.run([mrf.HARNESS, d, "rk3last", str(a.steps)], capture_output=True, text=True, timeout=3600)
        if r.returncode != 0:
            sys.exit(f"refharness exited {r.returncode}\n{r.stderr[-2000:]}")
        nv = case.param["n_var"]
        cv_ref = np.fromfile(os.path.join(d, "out", f"state_{a.steps}_cv.bin"), dtype=np.float64)
        cv_ref = interior_planes(case, cv_ref.reshape(nv, -1))
        dt_ref = float(np.fromfile(os.path.join(d, "out", f"dt_{a.steps}.bin"), dtype=np.float64)[0])
    finally:
        shutil.rmtree(work, ignore_errors=True)
    gz = GpuZone(case)
    gz.initialize()
    dt = 0.0
    for _ in range(a.steps):
        dt = gz.ctx.rk3_step()
    cv = interior_planes(case, gz.get("cv"))
    print(json.dumps({
        "block": f"{case.mx}x{case.my}x{case.mz}", "steps": a.steps,
        "dt_mode": "fixed" if a.fixed_dt > 0 else "CFL", "dt_reference": dt_ref, "dt_library": dt,
        "dt_rel_diff": abs(dt - dt_ref) / abs(dt_ref) if dt_ref else None,
        "cv_normwise_rel_diff": rel_err(cv, cv_ref), "cv_pointwise_rel_diff": pointwise_rel_err(cv, cv_ref)}))


if __name__ == "__main__":
    main()
