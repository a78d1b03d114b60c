"""The library's flowfield file as the reference's own reader sees it.

tests/golden/plt_ref_reader.npz holds what read_tecplot_plt of the
reference's tools/TecplotUtilsGXL.py decoded from a file this library's
writer (cfk_write_flowfield) made from seeded arrays
(tests/golden/make_plt_golden.py, run against a reference checkout).  The
test writes the same file again, checks that it is the same file (SHA-256),
and that the reference's reader recovered every variable of every zone bit
for bit over the written nodes (the block plus one ghost layer), with the
variable names, zone dimensions, solution time and the min/max records."""
import hashlib
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _maker():
    spec = importlib.util.spec_from_file_location("make_plt_golden", os.path.join(HERE, "golden", "make_plt_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_reference_reader_recovers_every_variable(tmp_path):
    m = _maker()
    fx = np.load(os.path.join(HERE, "golden", "plt_ref_reader.npz"))
    path = tmp_path / "flowfield.plt"
    assert m.write(str(path)) == str(fx["sha256"]), "the writer no longer produces the recorded file"
    assert hashlib.sha256(path.read_bytes()).hexdigest() == str(fx["sha256"])
    assert list(fx["variables"]) == m.NAMES
    blocks = m.plt_blocks()
    assert int(fx["n_zone"]) == len(blocks)
    e = m.NGG_OUTPUT
    for n, b in enumerate(blocks):
        mx, my, mz, g = b["mx"], b["my"], b["mz"], b["ngg"]
        dims = (mx + 2 * e, my + 2 * e, mz + 2 * e)
        assert tuple(fx[f"zone{n}_dims"]) == dims
        assert float(fx[f"zone{n}_time"]) == m.SOLUTION_TIME
        shape = (mz + 2 * g, my + 2 * g, mx + 2 * g)
        sel = (slice(g - e, g + mz + e), slice(g - e, g + my + e), slice(g - e, g + mx + e))
        planes = [b["x"], b["y"], b["z"]] + list(b["bv"]) + list(b["sv"]) + list(b["ov"])
        data = fx[f"zone{n}_data"]
        for v, a in enumerate(planes):
            want = a.reshape(shape)[sel].transpose(2, 1, 0)  # [i, j, k] as the reader returns it
            assert np.array_equal(data[v], want), f"zone {n}, variable {m.NAMES[v]}"
            assert fx[f"zone{n}_min"][v] == want.min() and fx[f"zone{n}_max"][v] == want.max()
