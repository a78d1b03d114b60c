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
        text += _struct(n, {"type": n, "label": int(lab)})
    text += spec.reference_state
    text += spec.setup_extra
    return text


def write_grid(spec: Spec, d: str):
    c = spec.case
    mx, my, mz = spec.block_shape or (c.mx, c.my, c.mz)
    # interior node coordinates [k, j, i], attached by the spec builders below
    xyz = spec.case.__dict__.get("_xyz")
    if xyz is None:
        raise ValueError(f"{spec.name}: interior coordinates not attached")
    x, y, z = xyz
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


def run_case(spec: Spec, workdir: str) -> dict:
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


def _attach_xyz(case, x, y, z):
    case.__dict__["_xyz"] = (x, y, z)
    return case


def _sod():
    c = cases.sod(400, 7, scheme=52, cfl=0.5)
    xs = np.linspace(0.0, 1.0, 400)
    ys = np.arange(7) * 0.01
    x = np.broadcast_to(xs[None, None, :], (1, 7, 400)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, 7, 400)).copy()
    _attach_xyz(c, x, y, np.zeros_like(x))
    ref = (_struct("left", {"type": "inflow", "label": 5, "density": 1.0, "velocity": 0.0, "pressure": 1.0}) +
           _struct("right", {"type": "inflow", "label": 5, "density": 0.125, "velocity": 0.0, "pressure": 0.1}) +
           "string default_init = left\nstring reference_state = left\nint groups_init = 2\n" +
           _struct("init_cond_0", {"x0": 0.5, "x1": 1.5, "y0": -10.0, "y1": 10.0, "z0": -2.0, "z1": 2.0,
                                   "name": "right"}))
    return Spec("sod_400x7_weno5", c, "rk3", 20, override_init=False, reference_state=ref)


def _sine(n=21):
    c = cases.perturbed(cases.sine_wave(n=n, scheme=72, viscous=True), seed=7)
    # the builder's coordinates, recomputed the same way
    p0 = 1.0 / cases.GAMMA_AIR
    T0 = p0 * cases.MW_AIR / (1.0 * cases.R_U)
    mu0 = 1.7894e-5 * (T0 / 288.16) ** 1.5 * (288.16 + 110) / (T0 + 110)
    L = 1000.0 * mu0
    g = np.linspace(0.0, 1.0, n)
    Z3, Y3, X3 = np.meshgrid(g, g, g, indexing="ij")
    x = (X3 + 0.05 * np.sin(2 * np.pi * Y3) * np.sin(2 * np.pi * Z3)) * L
    _attach_xyz(c, x, Y3 * L, Z3 * L)
    ref = (_struct("freestream", {"type": "inflow", "label": 5, "density": 1.0, "velocity": 1.0,
                                  "pressure": p0, "u": 1.0, "v": 0.0, "w": 0.0}) +
           "string default_init = freestream\nstring reference_state = freestream\n")
    return Spec(f"sine_{n}_weno7_visc", c, "rk3", 4, reference_state=ref)


def _tube():
    mech = mechanism.load("premix_h2_ar")
    nx, ny, length = 64, 7, 0.1
    c = cases.mix_tube(mech, nx, ny, scheme=52, reacting=True)
    xs = np.linspace(0.0, length, nx)
    ys = np.arange(ny) * length / 100.0
    x = np.broadcast_to(xs[None, None, :], (1, ny, nx)).copy()
    y = np.broadcast_to(ys[None, :, None], (1, ny, nx)).copy()
    _attach_xyz(c, x, y, np.zeros_like(x))
    Y = {"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433}
    ref = (_struct("left", dict({"type": "inflow", "label": 5, "density": 0.18075, "velocity": 0.0,
                                 "pressure": 35594.0, "u": 1.0, "v": 0.0, "w": 0.0}, **Y)) +
           "string default_init = left\nstring reference_state = left\n")
    return Spec("tube_h2o2ar_wu", c, "wu", 5, mech_name="premix_h2_ar", reference_state=ref)


def _reactors(n_side=32, steps=10, dt=1e-7):
    mech = mechanism.load("li2004")
    n = n_side * n_side
    base = cases.reactor_batch(mech, n, seed=2024)
    # the same reactors as an n_side x n_side 2-D block with the ghost layers
    # of the reference's default inviscid scheme for a reacting mixture run
    ngg = cases.ghost_layers(52)
    shape = (1 + 2 * ngg, n_side + 2 * ngg, n_side + 2 * ngg)

    def pad(a):
        return np.pad(a.reshape(1, n_side, n_side), ((ngg, ngg), (ngg, ngg), (ngg, ngg)), mode="edge").reshape(-1)

    bv = np.stack([pad(base.bv[l]) for l in range(6)])
    sv = np.stack([pad(base.sv[l]) for l in range(mech.n_spec)])
    P = shape[0] * shape[1] * shape[2]
    metric = np.zeros((9, P))
    metric[0] = metric[4] = metric[8] = 1.0
    c = dataclasses.replace(base, mx=n_side, my=n_side, mz=1, ngg=ngg, bv=bv, sv=sv, metric=metric,
                            jac=np.ones(P), faces=[(0, -1, 6), (0, 1, 6), (1, -1, 6), (1, 1, 6)])
    c.param.update(inviscid_scheme=52, fixed_dt=1, dt=dt)
    xs = np.arange(n_side, dtype=np.float64)
    x = np.broadcast_to(xs[None, None, :], (1, n_side, n_side)).copy()
    y = np.broadcast_to(xs[None, :, None], (1, n_side, n_side)).copy()
    _attach_xyz(c, x, y, np.zeros_like(x))
    X = np.zeros(mech.n_spec)
    X[mech.index("H2")], X[mech.index("O2")], X[mech.index("N2")] = 2.0, 1.0, 3.76
    Yd = cases.mole_to_mass(mech, X / X.sum())
    st = {"type": "inflow", "label": 5, "density": 1.0, "velocity": 0.0, "pressure": 101325.0,
          "u": 1.0, "v": 0.0, "w": 0.0}
    st.update({mech.species[k]: float(Yd[k]) for k in range(mech.n_spec)})
    ref = _struct("still", st) + "string default_init = still\nstring reference_state = still\n"
    return Spec("reactors_li2004_1024", c, "react", steps, react_dt=dt, mech_name="li2004", reference_state=ref)


SPECS = {"sod": _sod, "sine": _sine, "tube": _tube, "reactors": _reactors}


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
