"""CPU tests: the oracle against known answers and the reference's golden
data, and the C ABI's exports (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import cases
import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("order", [5, 7])
def test_weno_reproduces_linear_data(order):
    """With linear data every smoothness indicator is equal, the weights are
    the linear ones and f+ and f- both give the exact mid-face value."""
    L = pyoracle.lib()
    a, b = 0.7, -1.3
    r = 2 if order == 5 else 3
    n = 2 * r + 1
    vp = a + b * (np.arange(n) - r)          # points i-r .. i+r
    vm = a + b * (np.arange(n) - r + 1)      # points i-r+1 .. i+r+1
    fn = L.orc_weno5 if order == 5 else L.orc_weno7
    got = fn(_dp(vp), _dp(vm), 1e-40, 1)
    assert got == pytest.approx(2 * (a + 0.5 * b), rel=1e-14)
    got_lin = fn(_dp(vp), _dp(vm), 1e-40, 0)
    assert got_lin == pytest.approx(2 * (a + 0.5 * b), rel=1e-14)


@pytest.mark.parametrize("order", [5, 7])
def test_weno_picks_smooth_side_of_a_jump(order):
    """Across a jump the nonlinear weights suppress the stencils that cross it:
    the result stays within the data's range (no overshoot)."""
    L = pyoracle.lib()
    r = 2 if order == 5 else 3
    n = 2 * r + 1
    vp = np.where(np.arange(n) - r <= 0, 1.0, 0.0)
    vm = np.zeros(n)
    fn = L.orc_weno5 if order == 5 else L.orc_weno7
    got = fn(_dp(vp), _dp(vm), 1e-40, 1)
    assert -1e-6 <= got <= 1.0 + 1e-6


def test_sutherland_known_value():
    L = pyoracle.lib()
    assert L.orc_sutherland(288.16) == pytest.approx(1.7894e-5, rel=1e-15)


def test_oracle_sod_against_exact_solution():
    """Sod tube (400 x 7, WENO5 characteristic, CFL 0.5) to t = 0.2 against
    the exact solution shipped with the reference (golden fixture)."""
    golden = np.load(os.path.join(HERE, "golden", "sod_exact.npz"))
    c = cases.sod(400, 7, scheme=52, cfl=0.5)
    z = pyoracle.OracleZone(c)
    z.initialize()
    t, n = 0.0, 0
    while t < 0.2:
        t += z.step()
        n += 1
    xs = np.linspace(0, 1, 400)
    bv = z["bv"]
    for slot, key in ((0, "rho"), (1, "u"), (4, "p")):
        got = c.interior(bv[slot])[0, 3]
        ref = np.interp(xs, golden["x"], golden[key])
        assert np.abs(got - ref).mean() < 3.5e-3, key
    # the y rows of this 1-D problem stay identical up to round-off growth
    rho = c.interior(bv[0])[0]
    assert np.abs(rho - rho[3]).max() < 1e-6
    assert 300 < n < 400


def test_oracle_sine_wave_advects():
    """Inviscid density wave at u = 1 on the periodic curvilinear block moves
    with the flow: after t = 0.25 L the profile matches the shifted one."""
    n = 33
    c = cases.sine_wave(n=n, scheme=72, viscous=False, amp=0.0, dt=None, cfl=0.4)
    z = pyoracle.OracleZone(c)
    z.initialize()
    t = 0.0
    while t < 0.25 - 1e-12:
        z.p.fixed_dt = 1
        dt = min(0.25 - t, 0.4 / 32 / (1 + 1.0))
        z.p.dt = dt
        z.step()
        t += dt
    rho = c.interior(z["bv"][0])[n // 2, n // 2]
    x = np.linspace(0, 1, n)
    exact = 1 + 0.01 * np.sin(2 * np.pi * (x - 0.25))
    assert np.abs(rho - exact).max() < 2e-4


def test_c_abi_exports_every_declared_symbol():
    """libcorefl_b200.so loads without a GPU and exports each cfk_* function
    declared in include/corefl_b200.h."""
    import corefl_b200

    with open(os.path.join(ROOT, "include", "corefl_b200.h")) as f:
        decls = set(re.findall(r"\b(cfk_\w+)\s*\(", f.read()))
    assert len(decls) >= 20
    L = corefl_b200.lib()
    for name in sorted(decls):
        assert hasattr(L, name), name


def test_param_from_setup_reads_reference_keys(tmp_path):
    """setup.txt in the reference's syntax: typed scalars, structs, arrays,
    comments; the WENO scale comes from the reference state."""
    import corefl_b200

    setup = tmp_path / "setup.txt"
    setup.write_text(
        "// comment\n"
        "int inviscid_scheme = 52   // WENO5-ch\n"
        "real cfl = 0.5\n"
        "bool fixed_time_step = 0\n"
        "int viscous_order = 0\n"
        "int shock_sensor = 1\n"
        "real shockSensor_threshold = 0.02\n"
        "real shockSensor_epsilon = 1e-6\n"
        "array string boundary_conditions {\n  outflow wall\n}\n"
        "struct wall {\n    string type = wall\n    int label = 2\n    string  thermal_type    =   isothermal"
        "  // isothermal or adiabatic\n    real    temperature     =   322\n}\n"
        "string reference_state = left\n"
        "struct  left {\n    string type = inflow\n    int label = 5\n    real velocity = 0\n"
        "    real pressure = 1\n    real density = 1\n}\n")
    p = corefl_b200.cfk_param()
    err = ctypes.create_string_buffer(256)
    rc = corefl_b200.lib().cfk_param_from_setup(str(setup).encode(), ctypes.byref(p), err, 256)
    assert rc == 0, err.value
    assert p.inviscid_scheme == 52 and p.viscous_order == 0 and p.cfl == 0.5 and p.fixed_dt == 0
    assert p.n_var == 5 and p.Pr == 0.72
    assert p.shock_sensor == 1 and p.sensor_threshold == 0.02 and p.sensor_eps == 1e-6
    assert p.wall.thermal_type == 0 and p.wall.temperature == 322.0
    # |u| < 1, so v_ref is the speed of sound sqrt(gamma p / rho)
    assert p.v_ref == pytest.approx(np.sqrt(1.4), rel=1e-12)
    assert p.weno_eps_scale == pytest.approx(1.4, rel=1e-12)
    rc = corefl_b200.lib().cfk_param_from_setup(str(tmp_path / "missing.txt").encode(), ctypes.byref(p), err, 256)
    assert rc == -5 and b"cannot open" in err.value


def test_create_rejects_unsupported_settings():
    """Argument checks run before any device call."""
    import corefl_b200

    p = corefl_b200.make_param(dict(dim=3, n_var=5, inviscid_scheme=5), [])
    h = ctypes.c_void_p()
    assert corefl_b200.lib().cfk_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p = corefl_b200.make_param(dict(dim=3, n_var=6, inviscid_scheme=72), [])
    assert corefl_b200.lib().cfk_create(ctypes.byref(p), ctypes.byref(h)) == -1
    # the hybrid scheme exists for WENO5/7 only, with sensors 0..2
    p = corefl_b200.make_param(dict(dim=3, n_var=5, inviscid_scheme=4, reconstruction=2, sensor_threshold=0.1), [])
    assert corefl_b200.lib().cfk_create(ctypes.byref(p), ctypes.byref(h)) == -1
    p = corefl_b200.make_param(dict(dim=3, n_var=5, inviscid_scheme=72, weno_eps_scale=1.0, sensor_threshold=0.1,
                                    shock_sensor=3), [])
    assert corefl_b200.lib().cfk_create(ctypes.byref(p), ctypes.byref(h)) == -1
