"""Tecplot V112 binary flowfield files in plain Python.

TEST INFRASTRUCTURE ONLY: a restatement of the reference's flowfield.plt
writer (src/FieldIO.h:83-420, FieldIO::write_header and
write_common_data_section; strings as gxl::write_str, src/gxl_lib/MyString.cpp:151-163)
and a parser of the same layout, used by the tests to check the library's
writer byte for byte and its restart reader against an independent reading.

Layout: "#!TDV112", int32 1 (byte order), int32 0 (full file), the title
"Solution file", int32 n_var and the variable names; per zone the marker
299.0f, its name "zone <b>", parent -1, strand -2, the solution time
(double), colour -1, zone type 0, node location 0, two zero face-neighbour
counts, IMax JMax KMax (nodes widened by ngg_output on both sides) and a zero
auxiliary flag; the end-of-header marker 357.0f.  Then per zone the marker
299.0f, n_var int32 2 (double), int32 0 (passive), 0 (sharing), -1
(connectivity sharing), (min, max) doubles per variable and the variables'
node data, i fastest, in the order x, y, z, bv, sv, ov.
"""
from __future__ import annotations

import struct

import numpy as np


def _s(text: str) -> bytes:
    return b"".join(struct.pack("<i", ord(c)) for c in text) + struct.pack("<i", 0)


def _window(a: np.ndarray, dims, g_arr: int, g_out: int) -> np.ndarray:
    """The nodes of padded array `a` (ghost width g_arr) widened by g_out."""
    mx, my, mz = dims
    v = a.reshape(mz + 2 * g_arr, my + 2 * g_arr, mx + 2 * g_arr)
    o = g_arr - g_out
    return v[o:o + mz + 2 * g_out, o:o + my + 2 * g_out, o:o + mx + 2 * g_out]


def write(blocks, names, ngg_output=0, solution_time=0.0) -> bytes:
    """blocks: dicts with mx, my, mz, ngg and x, y, z, bv, sv, ov arrays
    (planes of the padded layout); names: all variable names in file order."""
    out = [b"#!TDV112", struct.pack("<ii", 1, 0), _s("Solution file"), struct.pack("<i", len(names))]
    out += [_s(n) for n in names]
    g = ngg_output
    for b, B in enumerate(blocks):
        out += [struct.pack("<f", 299.0), _s(f"zone {b}"), struct.pack("<ii", -1, -2),
                struct.pack("<d", solution_time), struct.pack("<iiiii", -1, 0, 0, 0, 0),
                struct.pack("<iii", B["mx"] + 2 * g, B["my"] + 2 * g, B["mz"] + 2 * g), struct.pack("<i", 0)]
    out.append(struct.pack("<f", 357.0))
    for B in blocks:
        dims = (B["mx"], B["my"], B["mz"])
        planes = [B["x"], B["y"], B["z"]] + list(B["bv"])
        for key in ("sv", "ov"):
            if B.get(key) is not None:
                planes += list(B[key])
        assert len(planes) == len(names)
        wins = [_window(np.asarray(p), dims, B["ngg"], g) for p in planes]
        out += [struct.pack("<f", 299.0), struct.pack(f"<{len(names)}i", *([2] * len(names))),
                struct.pack("<iii", 0, 0, -1)]
        out += [struct.pack("<dd", float(w.min()), float(w.max())) for w in wins]
        out += [np.ascontiguousarray(w, dtype="<f8").tobytes() for w in wins]
    return b"".join(out)


def parse(data: bytes) -> dict:
    """Header fields and per-zone min/max and node data of a file as write() lays it out."""
    at = 0

    def take(fmt):
        nonlocal at
        v = struct.unpack_from(fmt, data, at)
        at += struct.calcsize(fmt)
        return v

    def string():
        chars = []
        while True:
            (c,) = take("<i")
            if c == 0:
                return "".join(chars)
            chars.append(chr(c))

    magic = data[:8].decode()
    at = 8
    byte_order, file_type = take("<ii")
    title = string()
    (n_var,) = take("<i")
    names = [string() for _ in range(n_var)]
    zones = []
    while True:
        (marker,) = take("<f")
        if marker != 299.0:
            break
        z = {"name": string()}
        z["parent"], z["strand"] = take("<ii")
        (z["time"],) = take("<d")
        z["colour"], z["type"], z["location"], z["raw"], z["misc"] = take("<iiiii")
        z["dims"] = take("<iii")
        (z["aux"],) = take("<i")
        zones.append(z)
    eoh = marker
    for z in zones:
        (z["marker"],) = take("<f")
        z["formats"] = take(f"<{n_var}i")
        z["flags"] = take("<iii")
        z["minmax"] = [take("<dd") for _ in range(n_var)]
        n = z["dims"][0] * z["dims"][1] * z["dims"][2]
        z["data"] = []
        for _ in range(n_var):
            z["data"].append(np.frombuffer(data, dtype="<f8", count=n, offset=at).reshape(z["dims"][::-1]))
            at += 8 * n
    return {"magic": magic, "byte_order": byte_order, "file_type": file_type, "title": title, "names": names,
            "zones": zones, "eoh": eoh, "size": at}
