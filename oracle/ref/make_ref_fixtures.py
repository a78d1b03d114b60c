"""Records the reference solver's own per-step outputs as test fixtures
(test infrastructure).

Runs oracle/_ref/refharness — the reference's sources built unmodified by
oracle/ref/Makefile, driven step by step — on cases written in the
reference's input format from this package's case builders, and stores the
interior of every recorded array in tests/golden/ref_<case>.npz.  Run on a
machine with a GPU, after `make -C oracle/ref REF=<reference checkout>` (the
harness executable and the staged chemistry files travel with the tree):

    python oracle/ref/make_ref_fixtures.py [--out DIR] [case ...]

Each fixture holds, for steps s = 0..S (s = 0 is the state after the
reference's initialisation and compute_cv_from_bv): cv[s] (n_var, N), the
pressure p[s] (N), sv[s] (n_scalar, N) for mixtures, reaction_timeScale[s]
(N) for reacting mixtures, dt[s] (s >= 1); the basic variables bv0 (6, N)
at s = 0; the reference's metric and Jacobian at
a strided sample of the padded nodes (grid_idx, metric, jac) and mul at the
interior; and the reference's derived scalars (param_* entries).
"""
from __future__ import annotations

import argparse
import dataclasses
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "corefl-cpc_b200"))

import cases  # noqa: E402
import mechanism  # noqa: E402

REF_BUILD = os.path.join(ROOT, "oracle", "_ref")
HARNESS = os.path.join(REF_BUILD, "refharness")
MECH_FILES = {"li2004": "2004-Li-IntJ.Chem.Kinet.inp", "premix_h2_ar": "H2_mech-PREMIX.inp"}
GRID_STRIDE = 3


@dataclasses.dataclass
class Spec:
    name: str
    case: cases.Case
    mode: str  # rk3 | wu | react
    steps: int
    react_dt: float = 0.0
    mech_name: str | None = None
    override_init: bool = True  # False: the reference initialises from setup.txt
    setup_extra: str = ""
    reference_state: str = ""  # setup.txt struct of the reference state
    block_shape: tuple | None = None  # (mx, my, mz) of the reference's block when it differs from the case's


def _struct(name: str, entries: dict) -> str:
    lines = [f"struct {name} {{"]
    for k, v in entries.items():
        if isinstance(v, str):
            lines.append(f"    string {k} = {v}")
        elif isinstance(v, (int, np.integer)) and not isinstance(v, bool):
            lines.append(f"    int {k} = {v}")
        else:
            lines.append(f"    real {k} = {float(v)!r}")
    lines.append("}")
    return "\n".join(lines) + "\n"


def setup_txt(spec: Spec) -> str:
    c = spec.case
    p = c.param
    temporal = {"rk3": 3, "wu": 4, "react": 4}[spec.mode]
    fixed = int(p.get("fixed_dt", 0))
    out = [
        "bool parallel = 0",
        "string canonical_problem = general",
        "int gridIsBinary = 0",
        "real gridScale = 1",
        "int initial = 0",
        "int total_step = 1000000",
        "int output_file = 1000000",
        "int output_screen = 1000000",
        "int output_time_series = 0",
        "bool steady = 0",
        f"int temporal_scheme = {temporal}",
        f"bool fixed_time_step = {fixed}",
        f"real dt = {float(p.get('dt', 0.0)) if fixed else 1e-8!r}",
        f"real cfl = {float(p['cfl'])!r}",
        "real total_simulation_time = 1e+30",
        f"int inviscid_scheme = {int(p['inviscid_scheme']) if p['inviscid_scheme'] else 52}",
        f"int reconstruction = {int(p['reconstruction'])}",
        f"int limiter = {int(p['limiter'])}",
        f"real entropy_fix_factor = {float(p['entropy_fix_factor'])!r}",
        f"int viscous_order = {int(p['viscous_order'])}",
        f"bool positive_preserving = {int(p['positive_preserving'])}",
        f"bool gradPInDiffusionFlux = {int(p['gradPInDiffusionFlux'])}",
        f"real prandtl_number = {float(p['Pr'])!r}",
        f"real schmidt_number = {float(p['Sc'])!r}",
        "bool turbulence = 0",
    ]
    if c.mech is not None:
        out += [
            "int species = 1",
            f"int reaction = {1 if c.mech.n_reac > 0 else 0}",
            "int hardCodedMech = 0",
            f"int chem_advance_method = {int(p.get('chem_advance_method', 1))}",
            f"string mechanism_file = chemistry/{MECH_FILES[spec.mech_name]}",
        ]
    else:
        out += ["int species = 0", "int reaction = 0"]
    if float(p.get("sensor_threshold", 0.0)) > 1e-10:
        out += [f"int shock_sensor = {int(p['shock_sensor'])}",
                f"real shockSensor_threshold = {float(p['sensor_threshold'])!r}",
                f"real shockSensor_epsilon = {float(p['sensor_eps'])!r}"]
    labels = sorted({lab for _, _, lab in c.faces})
    names = {6: "outflow", 8: "periodic", 2: "wall", 5: "inflow", 3: "symmetry"}
    bc_names = [names[lab] for lab in labels]
    if not bc_names:
        bc_names = ["outflow"]
        labels = [6]
    out.append("array string boundary_conditions {")
    out.append("    " + " ".join(bc_names))
    out.append("}")
    text = "\n".join(out) + "\n"
    for lab, n in zip(labels, bc_names):
        text += _struct(n, bc_entries(c, n, int(lab)))
    text += spec.reference_state
    text += spec.setup_extra
    return text


def bc_entries(c, name: str, label: int) -> dict:
    """The setup.txt struct of one boundary condition from the case settings
    (reference src/BoundCond.cpp:9-120 Inflow, :480-528 Wall, :597-618 Outflow)."""
    p = c.param
    e = {"type": name, "label": label}
    if name == "wall":
        e["thermal_type"] = "adiabatic" if int(p.get("wall_thermal_type", 0)) == 1 else "isothermal"
        e["temperature"] = float(p.get("wall_temperature", 300.0))
        if c.mech is not None and int(p.get("wall_catalytic_type", 0)) == 1:
            e["catalytic_type"] = 1
            for k, y in enumerate(p["wall_yk"]):
                e[c.mech.species[k]] = float(y)
    elif name == "inflow":
        u, v, w = (float(p[k]) for k in ("inflow_u", "inflow_v", "inflow_w"))
        if v != 0.0 or w != 0.0 or u <= 0.0:
            raise ValueError("inflow fixtures use a velocity along +x (the reference scales a direction by |V|)")
        e.update(density=float(p["inflow_density"]), velocity=u, pressure=float(p["inflow_pressure"]),
                 u=1.0, v=0.0, w=0.0, inflow_sub=int(p.get("inflow_subsonic", 0)))
        if c.mech is not None:
            for k, y in enumerate(p["inflow_sv"]):
                e[c.mech.species[k]] = float(y)
    elif name == "outflow" and int(p.get("outflow_back_pressure_on", 0)) == 1:
        e.update(if_backPressure=1, backPressure=float(p["outflow_back_pressure"]))
    return e


def write_grid(spec: Spec, d: str):
    c = spec.case
    mx, my, mz = spec.block_shape or (c.mx, c.my, c.mz)
    if c.xyz is None:
        raise ValueError(f"{spec.name}: the case carries no node coordinates")
    x, y, z = c.xyz
    with open(os.path.join(d, "input", "grid", "grid   0.grd"), "w") as f:
        f.write("1\n")
        f.write(f"{mx} {my} {mz}\n")
        for a in (x, y, z):
            f.write("\n".join(repr(float(v)) for v in a.reshape(-1)) + "\n")
    # boundary records: 0-based node ranges, one face per record
    recs = []
    for face, direction, lab in (spec.case.faces or [(0, -1, 6), (0, 1, 6), (1, -1, 6), (1, 1, 6)]):
        lo = [0, 0, 0]
        hi = [mx - 1, my - 1, mz - 1]
        v = 0 if direction < 0 else [mx, my, mz][face] - 1
        lo[face] = hi[face] = v
        recs.append(f"{lo[0]} {hi[0]} {lo[1]} {hi[1]} {lo[2]} {hi[2]} {lab}")
    with open(os.path.join(d, "input", "boundary_condition", "boundary   0.txt"), "w") as f:
        f.write(f"{len(recs)}\n" + "\n".join(recs) + "\n")
    with open(os.path.join(d, "input", "boundary_condition", "inner   0.txt"), "w") as f:
        f.write("1\n0\n\n")


def prepare_case(spec: Spec, workdir: str) -> str:
    """Writes the case directory of `spec` (setup.txt, grid, boundary files,
    chemistry files, initial-state override) under `workdir`; returns it."""
    c = spec.case
    d = os.path.join(workdir, spec.name)
    for sub in ("input/grid", "input/boundary_condition", "input/chemistry", "out", "output/message",
                "output/time_series"):
        os.makedirs(os.path.join(d, sub), exist_ok=True)
    with open(os.path.join(d, "input", "setup.txt"), "w") as f:
        f.write(setup_txt(spec))
    write_grid(spec, d)
    if spec.mech_name:
        src = os.path.join(REF_BUILD, "chem", spec.mech_name)
        for fn in os.listdir(src):
            shutil.copy(os.path.join(src, fn), os.path.join(d, "input", "chemistry", fn))
    if spec.override_init:
        c.bv.astype(np.float64).tofile(os.path.join(d, "input", "init_bv.bin"))
        if c.mech is not None:
            c.sv.astype(np.float64).tofile(os.path.join(d, "input", "init_sv.bin"))
    return d


def run_case(spec: Spec, workdir: str) -> dict:
    d = prepare_case(spec, workdir)
    cmd = [HARNESS, d, spec.mode, str(spec.steps)] + ([repr(spec.react_dt)] if spec.mode == "react" else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    with open(os.path.join(workdir, spec.name + ".log"), "w") as f:
        f.write(r.stdout + "\n--- stderr ---\n" + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"{spec.name}: refharness exited {r.returncode}\n{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
    return collect(spec, d)


def collect(spec: Spec, d: str) -> dict:
    c = spec.case
    out = os.path.join(d, "out")
    par = {}
    with open(os.path.join(out, "param.txt")) as f:
        for line in f:
            k, v = line.split()
            par[k] = float(v)
    ngg = int(par["ngg"])
    nv, nsc = int(par["n_var"]), int(par["n_scalar"])
    mx, my, mz = spec.block_shape or (c.mx, c.my, c.mz)
    shape = (mz + 2 * ngg, my + 2 * ngg, mx + 2 * ngg)
    P = shape[0] * shape[1] * shape[2]

    def interior(a, n):
        a = a.reshape(n, *shape)
        return a[:, ngg:ngg + mz, ngg:ngg + my, ngg:ngg + mx].reshape(n, -1)

    def load(name, n):
        a = np.fromfile(os.path.join(out, name), dtype=np.float64)
        assert a.size == n * P, (name, a.size, n * P)
        return a

    res = {f"param_{k}": np.float64(v) for k, v in par.items()}
    cv, bv, sv, ts, dts = [], [], [], [], []
    for s in range(spec.steps + 1):
        cv.append(interior(load(f"state_{s}_cv.bin", nv), nv))
        bv.append(interior(load(f"state_{s}_bv.bin", 6), 6))
        if nsc:
            sv.append(interior(load(f"state_{s}_sv.bin", nsc), nsc))
        if os.path.exists(os.path.join(out, f"state_{s}_reaction_timeScale.bin")):
            ts.append(interior(load(f"state_{s}_reaction_timeScale.bin", 1), 1)[0])
        if s:
            dts.append(np.fromfile(os.path.join(out, f"dt_{s}.bin"), dtype=np.float64)[0])
    res["cv"] = np.stack(cv)
    res["bv0"] = bv[0]
    res["p"] = np.stack([b[4] for b in bv])
    if sv:
        res["sv"] = np.stack(sv)
    if ts:
        res["reaction_timeScale"] = np.stack(ts)
    res["dt"] = np.array(dts)
    idx = np.arange(0, P, GRID_STRIDE)
    res["grid_idx"] = idx
    res["metric"] = load("metric.bin", 9).reshape(9, P)[:, idx]
    res["jac"] = load("jac.bin", 1)[idx]
    res["mul"] = interior(load("mul.bin", 1), 1)[0]
    res["shape"] = np.array([mx, my, mz, ngg])
    return res


def _air_state(name, rho, u, p):
    return _struct(name, {"type": "inflow", "label": 5, "density": rho, "velocity": abs(u), "pressure": p,
                          "u": 1.0 if u >= 0 else -1.0, "v": 0.0, "w": 0.0})


def _ref(name):
    return f"string default_init = {name}\nstring reference_state = {name}\n"


def _sod_ref():
    return (_struct("left", {"type": "inflow", "label": 5, "density": 1.0, "velocity": 0.0, "pressure": 1.0}) +
            _struct("right", {"type": "inflow", "label": 5, "density": 0.125, "velocity": 0.0, "pressure": 0.1}) +
            _ref("left") + "int groups_init = 2\n" +
            _struct("init_cond_0", {"x0": 0.5, "x1": 1.5, "y0": -10.0, "y1": 10.0, "z0": -2.0, "z1": 2.0,
                                    "name": "right"}))


def _sod():
    c = cases.sod(400, 7, scheme=52, cfl=0.5)
    return Spec("sod_400x7_weno5", c, "rk3", 20, override_init=False, reference_state=_sod_ref())


def _sod_scheme(scheme, recon, steps=10):
    c = cases.sod(200, 7, scheme=scheme, reconstruction=recon, cfl=0.5)
    return Spec(f"sod_200x7_s{scheme}_r{recon}", c, "rk3", steps, override_init=False, reference_state=_sod_ref())


def _sod_hybrid():
    c = cases.sod(200, 7, scheme=52, cfl=0.5)
    c.param.update(sensor_threshold=0.02, shock_sensor=1, sensor_eps=-1.0)
    return Spec("sod_200x7_hybrid_jameson", c, "rk3", 10, override_init=False, reference_state=_sod_ref())


def _sine_ref():
    return _air_state("freestream", 1.0, 1.0, 1.0 / cases.GAMMA_AIR) + _ref("freestream")


def _sine(n=21):
    c = cases.perturbed(cases.sine_wave(n=n, scheme=72, viscous=True), seed=7)
    return Spec(f"sine_{n}_weno7_visc", c, "rk3", 4, reference_state=_sine_ref())


def _sine_visc8():
    c = cases.perturbed(cases.sine_wave(n=15, ny=13, nz=11, scheme=72, viscous_order=8), seed=9, amp=1e-2)
    return Spec("sine_15x13x11_weno7_visc8", c, "rk3", 3, reference_state=_sine_ref())


def _channel_walls():
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=52, viscous=True), seed=5, amp=2e-2)
    c = cases.with_walls(base, thermal_type=0)
    return Spec("channel_17x13x9_walls_weno5_visc", c, "rk3", 3, reference_state=_sine_ref())


# The boundary-condition runs use a fixed step: the reference's grid minimum
# of the CFL step (global_time_step / min_of_arr, src/TimeAdvanceFunc.cu:102-152)
# lets blocks overwrite the partial minima other blocks are still reading and
# returns before the barrier in partly filled blocks; on these 576-node tubes
# its own run gave dt = 0 on the first step.
def _duct_inflow():
    base = cases.sod(64, 9, scheme=52, cfl=0.5)
    c = cases.with_inflow(base, rho=1.1, u=2.0, p=0.8, subsonic=0)
    c.param.update(fixed_dt=1, dt=2e-3)
    # the inflow boundary's own struct is the reference state
    return Spec("duct_64x9_supersonic_inflow_fixed_dt", c, "rk3", 10, reference_state=_ref("inflow"))


def _duct_subsonic_back_pressure():
    base = cases.sod(64, 9, scheme=52, cfl=0.5)
    c = cases.with_back_pressure(cases.with_inflow(base, rho=1.1, u=0.5, p=0.8, subsonic=1), 0.7)
    c.param.update(fixed_dt=1, dt=2e-3)
    return Spec("duct_64x9_subsonic_inflow_back_pressure_fixed_dt", c, "rk3", 10, reference_state=_ref("inflow"))


def _tube_back_pressure():
    c = cases.with_back_pressure(cases.sod(64, 9, scheme=52, cfl=0.5), 0.5)
    c.param.update(fixed_dt=1, dt=2e-3)
    return Spec("tube_64x9_back_pressure_fixed_dt", c, "rk3", 10, override_init=False, reference_state=_sod_ref())


TUBE_LEFT_Y = {"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433}


def _tube_ref():
    return (_struct("left", dict({"type": "inflow", "label": 5, "density": 0.18075, "velocity": 0.0,
                                  "pressure": 35594.0, "u": 1.0, "v": 0.0, "w": 0.0}, **TUBE_LEFT_Y)) + _ref("left"))


def _tube():
    c = cases.mix_tube(mechanism.load("premix_h2_ar"), 64, 7, scheme=52, reacting=True)
    return Spec("tube_h2o2ar_wu", c, "wu", 5, mech_name="premix_h2_ar", reference_state=_tube_ref())


def _mix_tube_roe():
    c = cases.mix_tube(mechanism.load("premix_h2_ar"), 64, 7, scheme=2, reconstruction=2)
    return Spec("mixtube_64x7_roe_muscl", c, "rk3", 8, mech_name="premix_h2_ar", reference_state=_tube_ref())


def _mix_wave(reacting):
    mech = mechanism.load("li2004")
    if reacting:
        c = cases.mix_wave(mech, 13, ny=11, nz=9, scheme=72, reacting=True, T0=1400.0)
        name = "mixwave_13x11x9_weno7_visc_reacting"
    else:
        c = cases.mix_wave(mech, 13, ny=11, nz=9, scheme=72)
        name = "mixwave_13x11x9_weno7_visc"
    Y = {mech.species[k]: float(c.sv[k, 0]) for k in range(mech.n_spec)}
    ref = _struct("stream", dict({"type": "inflow", "label": 5, "density": float(c.bv[0, 0]), "velocity": 50.0,
                                  "pressure": 101325.0, "u": 1.0, "v": 0.0, "w": 0.0}, **Y)) + _ref("stream")
    return Spec(name, c, "rk3", 2, mech_name="li2004", reference_state=ref)


def _reactors(n_side=32, steps=10, dt=1e-7, seed=2024):
    mech = mechanism.load("li2004")
    n = n_side * n_side
    base = cases.reactor_batch(mech, n, seed=seed)
    # the same reactors as an n_side x n_side 2-D block with the ghost layers
    # of the reference's WENO5 scheme
    ngg = cases.ghost_layers(52)
    shape = (1 + 2 * ngg, n_side + 2 * ngg, n_side + 2 * ngg)

    def pad(a):
        return np.pad(a.reshape(1, n_side, n_side), ((ngg, ngg), (ngg, ngg), (ngg, ngg)), mode="edge").reshape(-1)

    bv = np.stack([pad(base.bv[l]) for l in range(6)])
    sv = np.stack([pad(base.sv[l]) for l in range(mech.n_spec)])
    P = shape[0] * shape[1] * shape[2]
    metric = np.zeros((9, P))
    metric[0] = metric[4] = metric[8] = 1.0
    xs = np.arange(n_side, dtype=np.float64)
    x = np.broadcast_to(xs[None, None, :], (1, n_side, n_side)).copy()
    y = np.broadcast_to(xs[None, :, None], (1, n_side, n_side)).copy()
    c = dataclasses.replace(base, mx=n_side, my=n_side, mz=1, ngg=ngg, bv=bv, sv=sv, metric=metric,
                            jac=np.ones(P), faces=[(0, -1, 6), (0, 1, 6), (1, -1, 6), (1, 1, 6)],
                            xyz=(x, y, np.zeros_like(x)), param=dict(base.param, inviscid_scheme=52, fixed_dt=1,
                                                                     dt=dt))
    X = np.zeros(mech.n_spec)
    X[mech.index("H2")], X[mech.index("O2")], X[mech.index("N2")] = 2.0, 1.0, 3.76
    Yd = cases.mole_to_mass(mech, X / X.sum())
    st = {"type": "inflow", "label": 5, "density": 1.0, "velocity": 0.0, "pressure": 101325.0,
          "u": 1.0, "v": 0.0, "w": 0.0}
    st.update({mech.species[k]: float(Yd[k]) for k in range(mech.n_spec)})
    return Spec("reactors_li2004_1024", c, "react", steps, react_dt=dt, mech_name="li2004",
                reference_state=_struct("still", st) + _ref("still"))


SPECS = {
    "sod": _sod,
    "sine": _sine,
    "tube": _tube,
    "reactors": _reactors,
    "sod_roe": lambda: _sod_scheme(2, 2),
    "sod_ausm_nnd2": lambda: _sod_scheme(3, 3),
    "sod_hllc_first": lambda: _sod_scheme(4, 1),
    "sod_hybrid": _sod_hybrid,
    "sine_visc8": _sine_visc8,
    "channel_walls": _channel_walls,
    "duct_inflow": _duct_inflow,
    "back_pressure": _tube_back_pressure,
    "duct_subsonic": _duct_subsonic_back_pressure,
    "mixtube_roe": _mix_tube_roe,
    "mixwave": lambda: _mix_wave(False),
    "mixwave_reacting": lambda: _mix_wave(True),
}



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--work", default=None)
    ap.add_argument("cases", nargs="*", default=list(SPECS))
    a = ap.parse_args()
    if not os.path.exists(HARNESS):
        sys.exit(f"{HARNESS} not built (make -C oracle/ref REF=<reference checkout>)")
    os.makedirs(a.out, exist_ok=True)
    work = a.work or tempfile.mkdtemp(prefix="refharness_")
    failed = 0
    for name in a.cases:
        spec = SPECS[name]()
        try:
            res = run_case(spec, work)
        except Exception as e:  # keep going: one case's failure is reported, the others still run
            print(f"{spec.name}: FAILED: {e}")
            failed += 1
            continue
        path = os.path.join(a.out, f"ref_{spec.name}.npz")
        np.savez_compressed(path, **res)
        print(f"{spec.name}: {spec.steps} steps -> {path} ({os.path.getsize(path)} bytes)")
    sys.exit(1 if failed else 0)


if __name__ == "__main__":
    main()
