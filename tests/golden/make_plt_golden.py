"""Decodes a flowfield file written by this library's Tecplot writer
(cfk_write_flowfield) with the reference's own reader, read_tecplot_plt of
the reference's tools/TecplotUtilsGXL.py, and stores what it decoded in
plt_ref_reader.npz beside this script.  Usage:

    python make_plt_golden.py <reference root>

The file is built from seeded arrays by plt_blocks() (two zones, ghost
layers in the output, two scalars and one further variable) so that the test
(tests/test_flowfield_ref_reader_cpu.py) can rebuild it byte for byte: the
fixture holds the file's SHA-256 next to the decoded zones.
"""
import hashlib
import importlib.util
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "corefl-cpc_b200"))

import corefl_b200 as cfk  # noqa: E402

NAMES = ["x", "y", "z", "density", "u", "v", "w", "pressure", "temperature", "H2", "O2", "mach"]
NGG_OUTPUT = 1
SOLUTION_TIME = 3.75e-4


def plt_blocks():
    """Two blocks (ngg = 2) of seeded arrays in the reference's padded layout."""
    rng = np.random.default_rng(20261203)
    out = []
    for mx, my, mz in ((7, 5, 4), (6, 4, 3)):
        g = 2
        P = (mx + 2 * g) * (my + 2 * g) * (mz + 2 * g)
        out.append({"mx": mx, "my": my, "mz": mz, "ngg": g,
                    "x": rng.random(P), "y": rng.random(P), "z": rng.random(P),
                    "bv": rng.random((6, P)) + 0.5, "sv": rng.random((2, P)), "ov": rng.random((1, P))})
    return out


def write(path):
    cfk.write_flowfield(path, plt_blocks(), NAMES, ngg_output=NGG_OUTPUT, n_scalar=2, n_other=1,
                        solution_time=SOLUTION_TIME)
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


if __name__ == "__main__":
    if len(sys.argv) != 2 or not os.path.isdir(sys.argv[1]):
        sys.exit("usage: python make_plt_golden.py <reference root>")
    spec = importlib.util.spec_from_file_location("TecplotUtilsGXL",
                                                  os.path.join(sys.argv[1], "tools", "TecplotUtilsGXL.py"))
    tec = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(tec)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "flowfield.plt")
        digest = write(path)
        # the per-variable branch (variables given) decodes each variable in
        # the file's FORTRAN order
        r = tec.read_tecplot_plt(path, variables=NAMES)
    out = {"sha256": np.array(digest), "title": np.array(r["title"]), "variables": np.array(r["variables"]),
           "n_zone": np.array(len(r["zones"]))}
    for n, z in enumerate(r["zones"]):
        out[f"zone{n}_name"] = np.array(z["name"])
        out[f"zone{n}_time"] = np.array(z["solution_time"])
        out[f"zone{n}_dims"] = np.array(z["dimensions"])
        out[f"zone{n}_data"] = z["data"]
        out[f"zone{n}_min"] = z["variable_min"]
        out[f"zone{n}_max"] = z["variable_max"]
    np.savez_compressed(os.path.join(HERE, "plt_ref_reader.npz"), **out)
    print("wrote plt_ref_reader.npz", digest)
