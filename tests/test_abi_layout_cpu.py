"""The ctypes mirrors in corefl_b200.py match the C ABI header byte for byte:
a small C program compiled against include/corefl_b200.h prints sizeof and
offsetof of every struct and field the Python binding declares, and they
must equal the ctypes layout (a drift would silently shift every field the
library reads behind it)."""
import os
import shutil
import subprocess

import pytest

import corefl_b200 as cfk
import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = ["cfk_face", "cfk_wall", "cfk_inflow", "cfk_outflow", "cfk_param", "cfk_zone", "cfk_mechanism",
           "cfk_inner_face", "cfk_plt_block", "cfk_plt_target", "cfk_surrogate_gate", "cfk_surrogate_stats"]


ORACLE_STRUCTS = ["orc_face", "orc_zone", "orc_mech", "orc_param", "orc_inner_face"]


def _ctypes_layout(module, name):
    t = getattr(module, name)
    return {"sizeof": __import__("ctypes").sizeof(t), **{f: getattr(t, f).offset for f, _ in t._fields_}}


def _c_layout(tmp_path, header, include_dir, module, names):
    lines = ["#include <stddef.h>", "#include <stdio.h>", f'#include "{header}"', "int main(void) {"]
    for name in names:
        lines.append(f'  printf("{name} sizeof %zu\\n", sizeof({name}));')
        for f, _ in getattr(module, name)._fields_:
            lines.append(f'  printf("{name} {f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / f"layout_{module.__name__}.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / f"layout_{module.__name__}"
    subprocess.run(["gcc", "-std=c99", "-I", include_dir, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        name, field, value = line.split()
        layout.setdefault(name, {})[field] = int(value)
    return layout


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    c_layout = _c_layout(tmp_path, "corefl_b200.h", os.path.join(ROOT, "include"), cfk, STRUCTS)
    for name in STRUCTS:
        assert c_layout[name] == _ctypes_layout(cfk, name), name


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs a C compiler")
def test_oracle_ctypes_structs_match_its_header(tmp_path):
    c_layout = _c_layout(tmp_path, "oracle.h", os.path.join(ROOT, "oracle"), pyoracle, ORACLE_STRUCTS)
    for name in ORACLE_STRUCTS:
        assert c_layout[name] == _ctypes_layout(pyoracle, name), name
