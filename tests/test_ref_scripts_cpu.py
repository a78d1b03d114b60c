"""The scripts that run the reference's own build against the library
(oracle/ref/time_ref_gpu.py, compare_flow_gpu.py, compare_reactors_gpu.py) write
their cases in the reference's input format; this checks, without a GPU or the
reference build, that the cases they write carry the settings of the
library's own workloads."""
import os
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle", "ref"))

import make_ref_fixtures as mrf  # noqa: E402
import time_ref_gpu as trg  # noqa: E402


def _setup(spec):
    d = mrf.prepare_case(spec, tempfile.mkdtemp(prefix="refscripts_"))
    with open(os.path.join(d, "input", "setup.txt")) as f:
        return d, f.read()


def test_wave_case_is_the_benchmark_block():
    spec = trg._wave_spec(9)
    d, text = _setup(spec)
    assert "int inviscid_scheme = 72" in text and "int viscous_order = 2" in text
    assert "bool fixed_time_step = 0" in text and "real cfl = 0.5" in text
    assert "int temporal_scheme = 3" in text
    with open(os.path.join(d, "input", "grid", "grid   0.grd")) as f:
        assert f.readline().strip() == "1" and f.readline().split() == ["9", "9", "9"]
    bv = np.fromfile(os.path.join(d, "input", "init_bv.bin"))
    assert bv.size == 6 * spec.case.P and np.allclose(bv.reshape(6, -1)[2:4], 0.0)


def test_reactor_case_is_the_benchmark_batch():
    if not os.path.isdir(os.path.join(mrf.REF_BUILD, "chem", "li2004")):
        pytest.skip("the reference build's staged chemistry files are not here")
    spec = trg._reactor_spec(4)
    d, text = _setup(spec)
    assert "int temporal_scheme = 4" in text and "int chem_advance_method = 1" in text
    assert "bool fixed_time_step = 1" in text and "real dt = 1e-07" in text
    sv = np.fromfile(os.path.join(d, "input", "init_sv.bin")).reshape(9, -1)
    assert np.allclose(sv.sum(axis=0), 1.0)


def test_tube_case_has_the_walls_and_the_shocked_reference_state():
    if not os.path.isdir(os.path.join(mrf.REF_BUILD, "chem", "premix_h2_ar")):
        pytest.skip("the reference build's staged chemistry files are not here")
    spec = trg._tube_spec(64, 16)
    _, text = _setup(spec)
    assert "string thermal_type = adiabatic" in text and "struct symmetry" in text
    assert "string reference_state = shocked" in text
    assert f"real density = {float(spec.case.param['rho_ref'])!r}" in text
    assert "int temporal_scheme = 4" in text and "int inviscid_scheme = 52" in text
