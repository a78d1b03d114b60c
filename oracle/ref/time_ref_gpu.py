"""Times the reference solver's own sm_100a build on the GPU (a measurement
of the reference, not part of the library).

Runs oracle/_ref/refharness in its timed modes on the workloads the
library's benchmark measures, written in the reference's input format by the
same case builders:

* wave: the 257^3-node curvilinear periodic wave (x = xi + 0.05 sin 2pi eta
  sin 2pi zeta, rho = 1 + 0.01 sin 2pi x, u = 1, p = 1/gamma, Sutherland at
  Re = 1000), WENO7 characteristic flux + 2nd-order viscous flux, SSP-RK3
  with the CFL step: the reference's RK3 loop body (src/RK.cuh:89-206),
  its own CFL time step included;
* reactors: 2^20 constant-volume H2/air reactors (Li-2004, seed 2026, the
  benchmark's batch) as a 1024 x 1024 block, point-implicit Wu reaction
  steps of 1e-7 s (src/StrangSplitting.cu:373-421);
* tube: the 2048 x 512 reflected-shock tube (H2-O2-Ar, PREMIX mechanism,
  WENO5 characteristic + mixture-averaged viscous fluxes, adiabatic walls),
  Wu-splitting steps with the CFL step (src/StrangSplitting.cu:756-771).

Each is timed with CUDA events after `warm-up` untimed steps; the script
prints one JSON object (per-step times, median, nodes, updates per second).
Run on a machine with a GPU after `make -C oracle/ref REF=<reference
checkout>`:

    python oracle/ref/time_ref_gpu.py [--wave-n 257] [--steps 10] [--warmup 3] [--only wave|reactors|tube]
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import make_ref_fixtures as mrf  # noqa: E402
from make_ref_fixtures import Spec, cases  # noqa: E402

import mechanism  # noqa: E402  (on the path through make_ref_fixtures)


def _wave_spec(n: int) -> Spec:
    c = cases.sine_wave(n=n, scheme=72, viscous=True, cfl=0.5)
    return Spec(f"wave_{n}_weno7_visc", c, "rk3", 0, reference_state=mrf._sine_ref())


def _reactor_spec(n_side: int) -> Spec:
    spec = mrf._reactors(n_side=n_side, steps=0, dt=1e-7, seed=2026)
    spec.name = f"reactors_li2004_{n_side * n_side}"
    return spec


def _tube_spec(nx: int, ny: int) -> Spec:
    mech = mechanism.load("premix_h2_ar")
    c = cases.reflected_shock_tube(mech, nx, ny)
    p = c.param
    # the reference state: the gas behind the incident shock (its density and
    # speed set the WENO epsilon scale, as in the case's own parameters)
    y = {mech.species[k]: float(c.sv[k, 0]) for k in range(mech.n_spec)}
    i2 = int(np.argmin(np.abs(c.bv[0] - p["rho_ref"])))
    st = dict({"type": "inflow", "label": 5, "density": float(p["rho_ref"]), "velocity": float(p["v_ref"]),
               "pressure": float(c.bv[4, i2]), "u": 1.0, "v": 0.0, "w": 0.0}, **y)
    return Spec(f"tube_{nx}x{ny}_wu", c, "wu", 0, mech_name="premix_h2_ar",
                reference_state=mrf._struct("shocked", st) + mrf._ref("shocked"))


def _time(spec: Spec, work: str, steps: int, warmup: int, timeout: int) -> dict:
    t0 = time.time()
    d = mrf.prepare_case(spec, work)
    prep = time.time() - t0
    if spec.mode in ("rk3", "wu"):
        cmd = [mrf.HARNESS, d, spec.mode + "time", str(steps), str(warmup)]
    else:
        cmd = [mrf.HARNESS, d, "reacttime", str(steps), repr(spec.react_dt), str(warmup)]
    t0 = time.time()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    run_s = time.time() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{spec.name}: refharness exited {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    res = json.loads(line)
    ms = np.array(res["ms_per_step"])
    res.update(case=spec.name, ms_median=float(np.median(ms)), ms_mean=float(ms.mean()),
               updates_per_s=res["nodes"] / (float(np.median(ms)) * 1e-3),
               prepare_s=round(prep, 1), harness_s=round(run_s, 1))
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--wave-n", type=int, default=257)
    ap.add_argument("--reactor-side", type=int, default=1024, help="reactors = side^2 (default 2^20)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--only", choices=["wave", "reactors", "tube"], default=None)
    ap.add_argument("--tube", type=int, nargs=2, default=[2048, 512], help="tube: nodes along x and y")
    ap.add_argument("--work", default=None, help="case directory root (default: a temporary directory, removed)")
    ap.add_argument("--timeout", type=int, default=1200)
    a = ap.parse_args()
    if not os.path.exists(mrf.HARNESS):
        sys.exit(f"{mrf.HARNESS} not built (make -C oracle/ref REF=<reference checkout>)")
    work = a.work or tempfile.mkdtemp(prefix="reftime_")
    out = {"what": "reference sources built unmodified for sm_100a (oracle/ref/Makefile), timed by refharness "
                   "with CUDA events on the default stream",
           "steps": a.steps, "warmup": a.warmup}
    try:
        if a.only in (None, "wave"):
            out["wave"] = _time(_wave_spec(a.wave_n), work, a.steps, a.warmup, a.timeout)
        if a.only in (None, "reactors"):
            out["reactors"] = _time(_reactor_spec(a.reactor_side), work, a.steps, a.warmup, a.timeout)
        if a.only in (None, "tube"):
            out["tube"] = _time(_tube_spec(*a.tube), work, a.steps, a.warmup, a.timeout)
    finally:
        if a.work is None:
            shutil.rmtree(work, ignore_errors=True)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
