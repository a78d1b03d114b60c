"""Constant inflow faces in the CPU oracle (apply_inflow, reference
src/BoundCond.cu:2190-2705, inflow_type 0 without fluctuations), the
setup.txt inflow struct (reference src/BoundCond.cpp:9-260) and the argument
checks.

The oracle's fill is checked against the reference's rules restated here in
numpy from the state before the boundary conditions: a supersonic inflow
puts the inflow state on the face and every ghost layer; a subsonic one
combines the inflow state with the inner node along the outward normal
(p = (p1 + p_in - rho1 c1 (V_in - V1).n) / 2, rho = rho_in + (p - p_in)/c1^2,
V = V_in - (p - p_in)/(rho1 c1) n) and reflects the inner nodes about the
face values in the ghosts, holding p and rho above 0.1 of the face values."""
import ctypes

import numpy as np
import pytest

import cases
import mechanism
import pyoracle

R_U, MW_AIR, GAMMA = 8314.462618, 28.9647, 1.4
R_AIR = R_U / MW_AIR


def _blocks(case, a):
    g = case.ngg
    return a.reshape(a.shape[0], case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)


def _fill(case):
    """State before and after the boundary conditions (properties first, so
    that mixtures carry their speed of sound)."""
    oz = pyoracle.OracleZone(case)
    oz.call("orc_update_physical_properties")
    before = oz["bv"].copy()
    c_before = oz["acoustic_speed"].copy() if case.mech is not None else None
    oz.call("orc_apply_boundary_conditions")
    return oz, before, c_before


def _tube(subsonic, u_in, p_in=0.8, rho_in=1.1):
    base = cases.sod(48, 9, scheme=52)
    return cases.with_inflow(base, rho=rho_in, u=u_in, p=p_in, subsonic=subsonic)


def test_supersonic_inflow_fills_face_and_ghosts_with_the_state():
    c_in = np.sqrt(GAMMA * 0.8 / 1.1)
    case = _tube(0, 2.5 * c_in)
    oz, _, _ = _fill(case)
    bv, g = _blocks(case, oz["bv"]), case.ngg
    T_in = case.param["inflow_temperature"]
    want = [1.1, 2.5 * c_in, 0.0, 0.0, 0.8, T_in]
    for l in range(6):
        assert np.all(bv[l, g, g:g + case.my, 0:g + 1] == want[l]), l


@pytest.mark.parametrize("u_scale", [0.3, -0.2, 1.4])
def test_subsonic_inflow_follows_the_characteristic_rule(u_scale):
    """Subsonic flag set: below Mach 1 (either direction) the characteristic
    combination; above it (normal Mach < -1) the inflow state itself."""
    c_in = np.sqrt(GAMMA * 0.8 / 1.1)
    case = _tube(1, u_scale * c_in)
    oz, before, _ = _fill(case)
    g = case.ngg
    B0, B = _blocks(case, before), _blocks(case, oz["bv"])
    jj = slice(g, g + case.my)
    u0 = B0[1, g, jj, g]                      # the face node's velocity before the fill
    c0 = np.sqrt(GAMMA * R_AIR * B0[5, g, jj, g])
    Mn = -u0 / c0                             # outward normal of the i-min face is -x
    rho1, p1, u1 = B0[0, g, jj, g + 1], B0[4, g, jj, g + 1], B0[1, g, jj, g + 1]
    c1 = np.sqrt(GAMMA * R_AIR * B0[5, g, jj, g + 1])
    p = 0.5 * (p1 + 0.8 - rho1 * c1 * ((u_scale * c_in - u1) * -1.0))
    rho = 1.1 + (p - 0.8) / (c1 * c1)
    u = u_scale * c_in - (p - 0.8) / (rho1 * c1) * -1.0
    sub = ~(Mn < -1.0)
    assert np.all(sub)                        # the tube starts at rest
    assert np.allclose(B[4, g, jj, g], p, rtol=1e-14, atol=0)
    assert np.allclose(B[0, g, jj, g], rho, rtol=1e-14, atol=0)
    assert np.allclose(B[1, g, jj, g], u, rtol=1e-14, atol=0)
    assert np.allclose(B[5, g, jj, g], p / (rho * R_AIR), rtol=1e-14, atol=0)
    for gg in range(1, g + 1):
        p2 = np.where(2 * p - B0[4, g, jj, g + gg] <= 0.1 * p, 0.1 * p, 2 * p - B0[4, g, jj, g + gg])
        r2 = np.where(2 * rho - B0[0, g, jj, g + gg] <= 0.1 * rho, 0.1 * rho, 2 * rho - B0[0, g, jj, g + gg])
        assert np.allclose(B[4, g, jj, g - gg], p2, rtol=1e-14, atol=0)
        assert np.allclose(B[0, g, jj, g - gg], r2, rtol=1e-14, atol=0)
        assert np.allclose(B[1, g, jj, g - gg], 2 * u - B0[1, g, jj, g + gg], rtol=1e-14, atol=1e-15)


def test_subsonic_ghost_pressure_clamp():
    """A high-pressure interior (the Sod left state, p = 1) behind a weak
    inflow (p_in = 0.2) whose velocity points out of the block: the face
    pressure p = (p1 + p_in + rho1 c1 u_in) / 2 leaves 2 p - p_i below 0.1 p
    in the ghosts."""
    case = _tube(1, -0.4, p_in=0.2, rho_in=0.3)
    oz, before, _ = _fill(case)
    g = case.ngg
    B0, B = _blocks(case, before), _blocks(case, oz["bv"])
    p = B[4, g, g:g + case.my, g]
    low = 2 * p - B0[4, g, g:g + case.my, g + 1] <= 0.1 * p
    assert np.any(low)
    assert np.all(B[4, g, g:g + case.my, g - 1][low] == 0.1 * p[low])


def test_mixture_subsonic_inflow_uses_the_mixture_state():
    mech = mechanism.load("premix_h2_ar")
    base = cases.mix_tube(mech, 40, 7)
    Y = np.zeros(mech.n_spec)
    Y[mech.index("O2")], Y[mech.index("AR")] = 0.2, 0.8
    case = cases.with_inflow(base, rho=0.1, u=50.0, p=1.2e4, Y=Y, subsonic=1)
    oz, before, c_before = _fill(case)
    g, ns = case.ngg, mech.n_spec
    B, S = _blocks(case, oz["bv"]), _blocks(case, oz["sv"])
    jj = slice(g, g + case.my)
    mw = 1.0 / np.sum(Y / mech.mw)
    assert np.allclose(B[5, g, jj, g], B[4, g, jj, g] * mw / (B[0, g, jj, g] * R_U), rtol=1e-14, atol=0)
    for gg in range(0, g + 1):
        assert np.all(S[:ns, g, jj, g - gg] == Y[:, None])
    c1 = _blocks(case, c_before[None])[0, g, jj, g + 1]
    B0 = _blocks(case, before)
    p = 0.5 * (B0[4, g, jj, g + 1] + 1.2e4 - B0[0, g, jj, g + 1] * c1 * ((50.0 - B0[1, g, jj, g + 1]) * -1.0))
    assert np.allclose(B[4, g, jj, g], p, rtol=1e-14, atol=0)


def test_inflow_tube_steps_stay_finite():
    c_in = np.sqrt(GAMMA * 0.8 / 1.1)
    for sub, us in ((0, 2.0), (1, 0.4)):
        oz = pyoracle.OracleZone(_tube(sub, us * c_in))
        oz.initialize()
        for _ in range(5):
            oz.step()
        assert np.all(np.isfinite(oz["cv"]))


def test_setup_inflow_struct_and_checks(tmp_path):
    import corefl_b200

    def param_of(text):
        f = tmp_path / "setup.txt"
        f.write_text(text)
        p = corefl_b200.cfk_param()
        err = ctypes.create_string_buffer(256)
        rc = corefl_b200.lib().cfk_param_from_setup(str(f).encode(), ctypes.byref(p), err, 256)
        return rc, p, err.value.decode()

    head = "int inviscid_scheme = 52\narray string boundary_conditions {\n  farfield outflow\n}\n"
    rc, p, _ = param_of(head + "struct farfield {\n string type = inflow\n int label = 5\n real mach = 2.0\n"
                        " real pressure = 101325\n real temperature = 300\n real aoa = 30\n int inflow_sub = 1\n}\n")
    assert rc == 0 and p.inflow.subsonic == 1
    c = np.sqrt(1.4 * R_U / MW_AIR * 300.0)
    assert p.inflow.u == pytest.approx(np.cos(np.pi / 6) * 2 * c, rel=1e-14)
    assert p.inflow.v == pytest.approx(np.sin(np.pi / 6) * 2 * c, rel=1e-14)
    assert p.inflow.density == pytest.approx(101325 * MW_AIR / (R_U * 300.0), rel=1e-14)
    rc, p, _ = param_of(head + "struct farfield {\n string type = inflow\n real density = 1.2\n real velocity = 100\n"
                        " real pressure = 1e5\n}\n")
    assert rc == 0 and p.inflow.temperature == pytest.approx(1e5 * MW_AIR / (1.2 * R_U), rel=1e-14)
    assert p.inflow.u == 100.0 and p.inflow.v == 0.0
    rc, p, _ = param_of(head + "struct farfield {\n string type = inflow\n real mach = 0.5\n real temperature = 288.16\n"
                        " real reynolds = 1e6\n}\n")
    mu = 1.7894e-5
    assert rc == 0 and p.inflow.density == pytest.approx(mu * 1e6 / (0.5 * np.sqrt(1.4 * R_U / MW_AIR * 288.16)),
                                                         rel=1e-13)
    rc, _, err = param_of(head + "struct farfield {\n string type = inflow\n int inflow_type = 1\n}\n")
    assert rc == -5 and "not supported" in err
    # the C ABI checks the inflow state before any device call
    h = ctypes.c_void_p()
    bad = corefl_b200.make_param(dict(dim=3, n_var=5, inviscid_scheme=52, weno_eps_scale=1.0, inflow_density=-1.0,
                                      inflow_pressure=1.0, inflow_temperature=1.0), [(0, -1, 5)])
    assert corefl_b200.lib().cfk_create(ctypes.byref(bad), ctypes.byref(h)) == -1


def test_setup_mixing_layer_and_white_noise(tmp_path):
    """problem_type 1 makes the inflow the mixing-layer inflow with the air
    streams of get_mixing_layer_info (src/MixingLayer.cu:9-119); the white
    noise takes its intensity and the seed; other fluctuation forms and
    profile inflows are reported."""
    import corefl_b200

    def param_of(text):
        f = tmp_path / "setup.txt"
        f.write_text(text)
        p = corefl_b200.cfk_param()
        err = ctypes.create_string_buffer(256)
        rc = corefl_b200.lib().cfk_param_from_setup(str(f).encode(), ctypes.byref(p), err, 256)
        return rc, p, err.value.decode()

    head = "int inviscid_scheme = 52\narray string boundary_conditions {\n  farfield outflow\n}\n"
    inflow = ("struct farfield {\n string type = inflow\n int label = 5\n int fluctuation_type = 1\n"
              " real fluctuation_intensity = 0.01\n}\n")
    streams = ("int problem_type = 1\nreal ma_c = 0.3\nreal velocity_ratio = 1.5\nbool upper_faster = 1\n"
               "real delta_omega = 1e-3\nint random_seed = 42\n"
               "struct upper_stream {\n real temperature = 600\n real pressure = 101325\n}\n"
               "struct lower_stream {\n real temperature = 400\n real pressure = 101325\n}\n")
    rc, p, err = param_of(head + streams + inflow)
    assert rc == 0, err
    q = p.inflow
    c_up, c_lo = np.sqrt(1.4 * R_U / MW_AIR * 600.0), np.sqrt(1.4 * R_U / MW_AIR * 400.0)
    u_slow = 0.3 * (c_up + c_lo) / 0.5
    assert q.inflow_type == 2 and q.u == pytest.approx(1.5 * u_slow, rel=1e-14)
    assert q.u_lower == pytest.approx(u_slow, rel=1e-14)
    assert q.density_lower == pytest.approx(101325 * MW_AIR / (R_U * 400.0), rel=1e-14)
    assert q.delta_omega == 1e-3 and q.fluctuation_type == 1 and q.fluctuation_intensity == 0.01 and q.seed == 42
    rc, _, err = param_of(head + "int problem_type = 1\n" + inflow)
    assert rc == -5 and "upper_stream" in err
    rc, _, err = param_of(head + "struct farfield {\n string type = inflow\n int fluctuation_type = 2\n"
                          " real mach = 2\n real pressure = 1e5\n real temperature = 300\n}\n")
    assert rc == -5 and "white-noise" in err
    rc, p, err = param_of(head + "struct farfield {\n string type = inflow\n int fluctuation_type = 1\n"
                          " real fluctuation_intensity = 0.02\n real mach = 2\n real pressure = 1e5\n"
                          " real temperature = 300\n}\n")
    assert rc == 0 and p.inflow.inflow_type == 0 and p.inflow.fluctuation_intensity == 0.02
