"""The flow workloads node by node: the reference's own build against this
library (a check, not part of the library).

Two blocks, each advanced `--steps` steps twice from the same inputs, with
oracle/_ref/refharness in a last-state mode and with this library through
the C ABI:

* wave: the 257^3 curvilinear periodic wave (WENO7 characteristic + 2nd-order
  viscous flux), SSP-RK3 (the reference's RK3 loop body, src/RK.cuh:89-206;
  cfk_rk3_step);
* sod: the 400 x 7 Sod tube (WENO5 characteristic, SSP-RK3, CFL 0.5; the
  reference initialises it from setup.txt), `--sod-steps` steps (250 reach
  t ~ 0.2);
* tube: the 2048 x 512 reflected-shock tube (stoichiometric H2-O2 with 70 %
  Ar, PREMIX mechanism, wall-normal stretching 1.02, WENO5 characteristic +
  mixture-averaged viscous fluxes, adiabatic no-slip walls), Wu splitting with
  the point-implicit reaction sub-step (src/StrangSplitting.cu:756-771;
  cfk_wu_splitting_step).

With --fixed-dt the step is fixed, else both take their own CFL step.  Prints
one JSON object per case: the time step of each and the normwise and
pointwise relative differences of the conserved variables (partial densities
included) after the last step.  Run on a machine with a GPU after
`make -C oracle/ref REF=<reference checkout>`:

    python oracle/ref/compare_flow_gpu.py [--case wave|sod|tube|all] [--steps 2] [--fixed-dt DT]
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
from make_ref_fixtures import Spec  # noqa: E402
from gpuzone import GpuZone, interior_planes, pointwise_rel_err, rel_err  # noqa: E402


def compare(name: str, spec: Spec, mode: str, steps: int, fixed_dt: float, with_oracle: bool = False) -> dict:
    case = spec.case
    if fixed_dt > 0:
        case.param.update(fixed_dt=1, dt=fixed_dt)
    work = tempfile.mkdtemp(prefix="cmpflow_")
    try:
        d = mrf.prepare_case(spec, work)
        r = subprocess.run([mrf.HARNESS, d, mode, str(steps)], capture_output=True, text=True, timeout=3600)
        if r.returncode != 0:
            sys.exit(f"{name}: refharness exited {r.returncode}\n{r.stderr[-2000:]}")
        nv = case.param["n_var"]
        cv_ref = np.fromfile(os.path.join(d, "out", f"state_{steps}_cv.bin"), dtype=np.float64)
        cv_ref = interior_planes(case, cv_ref.reshape(nv, -1))
        p_ref = None
        if case.param["n_spec"]:
            bv_ref = np.fromfile(os.path.join(d, "out", f"state_{steps}_bv.bin"), dtype=np.float64)
            p_ref = interior_planes(case, bv_ref.reshape(6, -1))[4]
        dt_ref = float(np.fromfile(os.path.join(d, "out", f"dt_{steps}.bin"), dtype=np.float64)[0])
    finally:
        shutil.rmtree(work, ignore_errors=True)
    gz = GpuZone(case)
    gz.initialize()
    dt = 0.0
    for _ in range(steps):
        dt = gz.ctx.rk3_step() if mode == "rk3last" else gz.ctx.wu_splitting_step(schedule=1)
    cv = interior_planes(case, gz.get("cv"))
    ns = case.param["n_spec"]
    extra = {}
    if with_oracle:
        # the CPU restatement of the same steps, against both
        sys.path.insert(0, os.path.dirname(HERE))
        import pyoracle

        oz = pyoracle.OracleZone(case)
        oz.initialize()
        for _ in range(steps):
            oz.step() if mode == "rk3last" else oz.wu_splitting_step()
        cv_o = interior_planes(case, oz["cv"])
        extra = {"oracle_vs_reference_normwise": rel_err(cv_o, cv_ref),
                 "library_vs_oracle_normwise": rel_err(cv, cv_o)}
    return {**extra, "case": name, "block": f"{case.mx}x{case.my}x{case.mz}", "steps": steps,
            "dt_mode": "fixed" if fixed_dt > 0 else "CFL", "dt_reference": dt_ref, "dt_library": dt,
            "dt_rel_diff": abs(dt - dt_ref) / abs(dt_ref) if dt_ref else None,
            "cv_normwise_rel_diff": rel_err(cv, cv_ref),
            "cv_pointwise_rel_diff": pointwise_rel_err(cv, cv_ref, n_spec=ns, p=p_ref)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["wave", "sod", "tube", "all"], default="all")
    ap.add_argument("--sod-steps", type=int, default=250)
    ap.add_argument("--oracle", action="store_true", help="also run the CPU restatement and compare it with both")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--fixed-dt", type=float, default=0.0, help="fixed time step (0: the CFL step)")
    ap.add_argument("--n", type=int, default=257, help="wave: nodes per direction")
    ap.add_argument("--tube", type=int, nargs=2, default=[2048, 512], help="tube: nodes along x and y")
    a = ap.parse_args()
    if not os.path.exists(mrf.HARNESS):
        sys.exit(f"{mrf.HARNESS} not built (make -C oracle/ref REF=<reference checkout>)")
    if a.case in ("wave", "all"):
        print(json.dumps(compare("wave", trg._wave_spec(a.n), "rk3last", a.steps, a.fixed_dt, a.oracle)), flush=True)
    if a.case in ("sod", "all"):
        print(json.dumps(compare("sod", mrf._sod(), "rk3last", a.sod_steps, a.fixed_dt, a.oracle)), flush=True)
    if a.case in ("tube", "all"):
        print(json.dumps(compare("tube", trg._tube_spec(*a.tube), "wulast", a.steps, a.fixed_dt, a.oracle)), flush=True)


if __name__ == "__main__":
    main()
