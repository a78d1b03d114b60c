"""The CPU oracle against the reference's own recorded runs.

tests/golden/ref_*.npz hold the reference solver's outputs, step by step,
recorded from its own sources built unmodified (oracle/ref/Makefile) and run
by oracle/ref/make_ref_fixtures.py, whose SPECS list the runs: the Sod tube of
the benchmark's small configuration (400 x 7, WENO5 characteristic, 20
steps) and of every primitive-variable scheme and the hybrid scheme; the
curvilinear periodic wave with WENO7 and the 2nd-order and 8th-order viscous
fluxes; no-slip walls, inflow and back-pressure boundaries; H2/O2/Ar and
H2/N2-air mixtures with Roe, WENO7, mixture-averaged transport and the
explicit source; Wu's splitting of a reacting tube; and 1024 Li-2004
reactors (10 point-implicit reaction steps of 1e-7 s).  The oracle replays
each from the same inputs.

Bar: the conserved variables agree to 1e-12 after every step, normwise
(max|a - b| / max|b| per variable) and pointwise (per node,
gpuzone.pointwise_rel_err); the time step to 1e-13; the builders' grid
metric and Jacobian to 1e-14 of the reference's.
"""
import numpy as np
import pytest

import cases
import reffix

TOL = 1e-12


@pytest.mark.parametrize("name", reffix.names())
def test_oracle_replays_reference_run(name):
    reports = reffix.replay(reffix.OracleReplay(name))
    for r in reports:
        print(f"{name} step {r.step}: dt {r.dt_rel:.2e}, cv normwise {r.cv_norm:.2e}, pointwise {r.cv_point:.2e}",
              r.extra)
    for r in reports:
        assert r.dt_rel <= 1e-13, f"step {r.step}: time step differs by {r.dt_rel:.3e}"
        assert r.cv_norm <= TOL, f"step {r.step}: normwise {r.cv_norm:.3e}"
        assert r.cv_point <= TOL, f"step {r.step}: pointwise {r.cv_point:.3e}"


@pytest.mark.parametrize("name", [n for n in reffix.names() if n != "reactors"])
def test_builder_grid_matches_reference(name):
    fx = reffix.load(name)
    _, case = reffix.spec_and_case(name, fx)
    e_m, e_j = reffix.grid_differences(case, fx)
    print(f"{name}: metric {e_m:.2e}, jacobian {e_j:.2e}")
    assert e_m <= 1e-14 and e_j <= 1e-14


def test_sod_builder_matches_reference_initial_state():
    """The reference initialised the Sod tube itself from setup.txt (two
    states split at x = 0.5 by its groups_init patch); the builder's interior
    basic variables equal its recorded ones."""
    fx = reffix.load("sod")
    _, case = reffix.spec_and_case("sod", fx)
    b = reffix.interior(case, case.bv)
    assert np.array_equal(b[:5], fx["bv0"][:5])
    assert np.allclose(b[5], fx["bv0"][5], rtol=1e-15, atol=0)


def test_fixture_shapes():
    for name in reffix.names():
        fx = reffix.load(name)
        mx, my, mz, g = (int(v) for v in fx["shape"])
        n = mx * my * mz
        assert fx["cv"].shape[2] == n and fx["bv0"].shape == (6, n) and fx["p"].shape == fx["cv"].shape[::2]
        assert fx["dt"].shape[0] == fx["cv"].shape[0] - 1
