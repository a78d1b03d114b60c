"""Tecplot V112 flowfield files (cfk_write_flowfield / cfk_read_flowfield;
reference src/FieldIO.h:83-420 and src/Initialize.cu:97-400), host only.

* The library's file is byte-identical to the oracle's restatement of the
  reference writer (oracle/plt.py) for air and mixture blocks, one and two
  zones, with and without ghost layers in the output.
* Its header parses to the reference's fields (magic number, byte order,
  title, variable names, zone records, end-of-header marker).
* Reading it back fills bv and sv exactly over the written nodes; names match
  case-insensitively with the reference's aliases, species by name in any
  order, and variables without a label are skipped.
* A run restarted from a file continues like the uninterrupted run (1e-13).
* Missing, foreign, truncated and mismatched files are reported."""
import dataclasses

import numpy as np
import pytest

import cases
import mechanism
import plt
import pyoracle
from gpuzone import interior_planes, rel_err

import corefl_b200 as cfk

AIR_NAMES = ["x", "y", "z", "density", "u", "v", "w", "pressure", "temperature"]


def _block(case, seed, n_other=1, bv=None, sv=None):
    rng = np.random.default_rng(seed)
    P = case.P
    b = {"mx": case.mx, "my": case.my, "mz": case.mz, "ngg": case.ngg,
         "x": np.ascontiguousarray(case.x), "y": rng.random(P), "z": rng.random(P),
         "bv": np.ascontiguousarray(case.bv if bv is None else bv),
         "ov": rng.random((n_other, P)) if n_other else None}
    s = case.sv if sv is None else sv
    b["sv"] = np.ascontiguousarray(s) if s.shape[0] else None
    return b


def _air_blocks():
    c1 = cases.perturbed(cases.sine_wave(n=13, ny=9, nz=7, scheme=52, viscous=False), seed=1, amp=0.02)
    c2 = cases.perturbed(cases.sine_wave(n=11, ny=9, nz=8, scheme=52, viscous=False), seed=2, amp=0.02)
    return [c1, c2], [_block(c1, 1), _block(c2, 2)]


@pytest.mark.parametrize("ngg_output", [0, 2])
@pytest.mark.parametrize("n_zone", [1, 2])
def test_air_file_is_byte_identical_to_the_oracle_writer(tmp_path, ngg_output, n_zone):
    _, blocks = _air_blocks()
    blocks = blocks[:n_zone]
    names = AIR_NAMES + ["mach"]
    path = tmp_path / "flowfield.plt"
    cfk.write_flowfield(path, blocks, names, ngg_output=ngg_output, n_other=1, solution_time=1.25e-3)
    data = path.read_bytes()
    assert data == plt.write(blocks, names, ngg_output=ngg_output, solution_time=1.25e-3)
    h = plt.parse(data)
    assert h["magic"] == "#!TDV112" and h["byte_order"] == 1 and h["file_type"] == 0
    assert h["title"] == "Solution file" and h["names"] == names and h["eoh"] == 357.0
    assert h["size"] == len(data)
    for b, z in enumerate(h["zones"]):
        B = blocks[b]
        assert z["name"] == f"zone {b}" and z["time"] == 1.25e-3 and (z["parent"], z["strand"]) == (-1, -2)
        assert z["dims"] == (B["mx"] + 2 * ngg_output, B["my"] + 2 * ngg_output, B["mz"] + 2 * ngg_output)
        assert z["formats"] == (2,) * len(names) and z["flags"] == (0, 0, -1)
        rho = plt._window(B["bv"][0], (B["mx"], B["my"], B["mz"]), B["ngg"], ngg_output)
        assert np.array_equal(z["data"][3], rho) and z["minmax"][3] == (rho.min(), rho.max())


def test_mixture_file_is_byte_identical_to_the_oracle_writer(tmp_path):
    mech = mechanism.load("li2004")
    c = cases.perturbed(cases.mix_wave(mech, 9, ny=7, nz=6, scheme=52), seed=4, amp=1e-2)
    blocks = [_block(c, 3)]
    names = AIR_NAMES + list(mech.species) + ["mach"]
    path = tmp_path / "mix.plt"
    cfk.write_flowfield(path, blocks, names, ngg_output=1, n_scalar=mech.n_spec, n_other=1)
    assert path.read_bytes() == plt.write(blocks, names, ngg_output=1)


def _empty_like(B):
    P = B["bv"].shape[1]
    out = {"mx": B["mx"], "my": B["my"], "mz": B["mz"], "ngg": B["ngg"], "bv": np.full((6, P), -7.0)}
    out["sv"] = np.full((B["sv"].shape[0], P), -7.0) if B.get("sv") is not None else None
    return out


def _check_window(got, want, B, g):
    dims = (B["mx"], B["my"], B["mz"])
    for l in range(want.shape[0]):
        assert np.array_equal(plt._window(got[l], dims, B["ngg"], g), plt._window(want[l], dims, B["ngg"], g))
    # nothing outside the written nodes was touched
    mask = np.ones(got.shape[1], dtype=bool)
    plt._window(mask, dims, B["ngg"], g)[...] = False
    assert np.all(got[:, mask] == -7.0)


@pytest.mark.parametrize("ngg_output", [0, 3])
def test_read_back_fills_basic_variables(tmp_path, ngg_output):
    _, blocks = _air_blocks()
    path = tmp_path / "f.plt"
    cfk.write_flowfield(path, blocks, AIR_NAMES + ["mach"], ngg_output=ngg_output, n_other=1, solution_time=2.5)
    targets = [_empty_like(B) for B in blocks]
    assert cfk.read_flowfield(path, targets) == 2.5
    for T, B in zip(targets, blocks):
        _check_window(T["bv"], B["bv"], B, ngg_output)


def test_read_matches_reference_aliases_and_species_by_name(tmp_path):
    mech = mechanism.load("li2004")
    c = cases.perturbed(cases.mix_wave(mech, 9, ny=7, nz=6, scheme=52), seed=5, amp=1e-2)
    B = _block(c, 6, n_other=2)
    species = list(mech.species)
    names = ["X", "Y", "Z", "RHO", "U", "v", "W", "P", "T"] + species + ["mach", "H2"]
    # the last plane is named like a species but comes after it: the later one wins, as in a sequential read
    path = tmp_path / "m.plt"
    cfk.write_flowfield(path, [B], names, n_scalar=len(species), n_other=2)
    T = _empty_like(B)
    cfk.read_flowfield(path, [T], species=species)
    _check_window(T["bv"], B["bv"], B, 0)
    want_sv = B["sv"].copy()
    want_sv[species.index("H2")] = B["ov"][1]
    _check_window(T["sv"], want_sv, B, 0)
    # species listed in another order land in the caller's order
    T2 = _empty_like(B)
    order = species[::-1]
    cfk.read_flowfield(path, [T2], species=order)
    for l, name in enumerate(order):
        src = B["ov"][1] if name == "H2" else B["sv"][species.index(name)]
        assert np.array_equal(plt._window(T2["sv"][l], (B["mx"], B["my"], B["mz"]), B["ngg"], 0),
                              plt._window(src, (B["mx"], B["my"], B["mz"]), B["ngg"], 0))


def test_restart_continues_like_the_uninterrupted_run(tmp_path):
    case = cases.perturbed(cases.sine_wave(n=17, ny=11, nz=9, scheme=52, viscous=True), seed=9, amp=0.02)
    ref = pyoracle.OracleZone(case)
    ref.initialize()
    for _ in range(3):
        ref.step()
    B = _block(case, 1, bv=ref["bv"].copy())
    path = tmp_path / "restart.plt"
    cfk.write_flowfield(path, [B], AIR_NAMES + ["mach"], n_other=1, solution_time=0.5)
    T = _empty_like(B)
    T["bv"][:] = case.bv          # ghosts keep the case's start values; the BCs refill them
    assert cfk.read_flowfield(path, [T]) == 0.5
    rz = pyoracle.OracleZone(dataclasses.replace(case, bv=T["bv"]))
    rz.initialize()
    for _ in range(2):
        ref.step()
        rz.step()
    assert rel_err(interior_planes(case, rz["cv"]), interior_planes(case, ref["cv"])) <= 1e-13


def test_bad_files_are_reported(tmp_path):
    _, blocks = _air_blocks()
    path = tmp_path / "f.plt"
    cfk.write_flowfield(path, blocks, AIR_NAMES + ["mach"], n_other=1)
    targets = [_empty_like(B) for B in blocks]
    with pytest.raises(cfk.CfkError, match="-5: cannot open"):
        cfk.read_flowfield(tmp_path / "missing.plt", targets)
    with pytest.raises(cfk.CfkError, match="2 zones, 1 blocks"):
        cfk.read_flowfield(path, targets[:1])
    with pytest.raises(cfk.CfkError, match="does not match block 0"):
        cfk.read_flowfield(path, targets[::-1])
    data = path.read_bytes()
    B1 = blocks[1]
    mach_plane = 8 * B1["mx"] * B1["my"] * B1["mz"]
    (tmp_path / "short.plt").write_bytes(data[:-(mach_plane + 100)])   # cut inside the temperature plane
    with pytest.raises(cfk.CfkError, match="-5: truncated data of zone 1"):
        cfk.read_flowfield(tmp_path / "short.plt", targets)
    # cut inside the last zone's trailing Mach plane, which the reader skips
    (tmp_path / "short2.plt").write_bytes(data[:-8])
    with pytest.raises(cfk.CfkError, match="-5: truncated data of zone 1"):
        cfk.read_flowfield(tmp_path / "short2.plt", targets)
    (tmp_path / "other.plt").write_bytes(b"hello world, not tecplot")
    with pytest.raises(cfk.CfkError, match="not a Tecplot"):
        cfk.read_flowfield(tmp_path / "other.plt", targets)
    with pytest.raises(cfk.CfkError, match="ngg below ngg_output"):
        cfk.write_flowfield(path, blocks, AIR_NAMES + ["mach"], ngg_output=4, n_other=1)
    with pytest.raises(cfk.CfkError, match="-5: cannot open"):
        cfk.write_flowfield(tmp_path / "no" / "dir.plt", blocks, AIR_NAMES + ["mach"], n_other=1)
