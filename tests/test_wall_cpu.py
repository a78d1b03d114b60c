"""No-slip wall faces in the CPU oracle (apply_wall, reference
src/BoundCond.cu:2761-3031) and the argument checks of the wall description.

The oracle's wall fill is checked against the reference's rules directly on
the padded arrays: the boundary node takes zero velocity, its inner
neighbour's pressure, the wall temperature (isothermal) or the inner
temperature (adiabatic) and rho = p / (R T); ghost layer g mirrors inner node
g with the velocity reversed, the pressure copied and the temperature
reflected about the wall temperature (isothermal, clamped to T_w at or below
0.1 T_w) or copied (adiabatic); mixtures carry the inner (non-catalytic) or
the wall's (catalytic) mass fractions.  The GPU kernels are compared with
this oracle in test_wall_gpu.py."""
import ctypes

import numpy as np
import pytest

import cases
import mechanism
import pyoracle

R_AIR = 8314.462618 / 28.9647


def _blocks(case, oz, key):
    g = case.ngg
    a = oz[key]
    return a.reshape(a.shape[0], case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)


def _air_channel(thermal_type, temperature=None, scheme=52):
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=scheme, viscous=True), seed=5, amp=2e-2)
    return cases.with_walls(base, thermal_type=thermal_type, temperature=temperature)


def _check_wall_rows(case, oz, R_of, T_wall=None):
    """Checks both j walls over the nodes the periodic i and k faces leave
    alone (interior i, k); R_of(j_node, j_source, j_face) gives the gas
    constants of a node in row j_node and of the ghost filled from row
    j_source.  Returns how many ghosts took the 0.1 T_w clamp."""
    g = case.ngg
    bv = _blocks(case, oz, "bv")
    ii = slice(g + 1, g + case.mx - 1)
    kk = slice(g + 1, g + case.mz - 1)
    clamped = 0
    for jf, sgn in ((g, -1), (g + case.my - 1, 1)):
        jin = jf - sgn
        T_face = bv[5, kk, jf, ii]
        assert np.all(bv[1:4, kk, jf, ii] == 0.0)
        assert np.array_equal(bv[4, kk, jf, ii], bv[4, kk, jin, ii])
        if T_wall is None:
            assert np.array_equal(T_face, bv[5, kk, jin, ii])
        else:
            assert np.all(T_face == T_wall)
        R_face, _ = R_of(jf, jin, jf)
        assert np.allclose(bv[0, kk, jf, ii], bv[4, kk, jf, ii] / (T_face * R_face), rtol=1e-15, atol=0)
        for gg in range(1, g + 1):
            jg, ji = jf + sgn * gg, jf - sgn * gg
            assert np.array_equal(bv[1, kk, jg, ii], -bv[1, kk, ji, ii])
            assert np.array_equal(bv[2, kk, jg, ii], -bv[2, kk, ji, ii])
            assert np.array_equal(bv[3, kk, jg, ii], -bv[3, kk, ji, ii])
            assert np.array_equal(bv[4, kk, jg, ii], bv[4, kk, ji, ii])
            Ti = bv[5, kk, ji, ii]
            if T_wall is None:
                expect = Ti
            else:
                expect = 2 * T_wall - Ti
                low = expect <= 0.1 * T_wall
                clamped += int(low.sum())
                expect = np.where(low, T_wall, expect)
            assert np.array_equal(bv[5, kk, jg, ii], expect)
            _, R_ghost = R_of(jg, ji, jf)
            assert np.allclose(bv[0, kk, jg, ii], bv[4, kk, jg, ii] / (bv[5, kk, jg, ii] * R_ghost), rtol=1e-15,
                               atol=0)
    return clamped


@pytest.mark.parametrize("thermal_type", [0, 1])
def test_air_wall_fill(thermal_type):
    case = _air_channel(thermal_type)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    Tw = case.param["wall_temperature"] if thermal_type == 0 else None
    _check_wall_rows(case, oz, lambda *_: (R_AIR, R_AIR), T_wall=Tw)
    # the ghosts' cv follow from their bv
    g = case.ngg
    cv, bv = _blocks(case, oz, "cv"), _blocks(case, oz, "bv")
    j = g - 1
    assert np.allclose(cv[1, :, j], bv[0, :, j] * bv[1, :, j], rtol=1e-15, atol=0)


def test_isothermal_ghost_temperature_clamp():
    """A cold wall (0.5 of the mean temperature) drives 2 T_w - T_i below
    0.1 T_w, where the ghost takes T_w."""
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=52, viscous=True), seed=5, amp=2e-2)
    Tw = 0.5 * float(np.mean(base.bv[5]))
    case = cases.with_walls(base, thermal_type=0, temperature=Tw)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    assert _check_wall_rows(case, oz, lambda *_: (R_AIR, R_AIR), T_wall=Tw) > 0


def _li_wall_case(catalytic):
    mech = mechanism.load("li2004")
    base = cases.perturbed(cases.mix_wave(mech, 13, ny=11, nz=9, scheme=52, viscous=True), seed=2, amp=1e-2)
    yk = np.zeros(mech.n_spec)
    yk[list(mech.species).index("N2")] = 0.7
    yk[list(mech.species).index("O2")] = 0.3
    return mech, yk, cases.with_walls(base, thermal_type=0, catalytic_type=catalytic, yk=yk if catalytic else None)


@pytest.mark.parametrize("catalytic", [0, 1])
def test_mixture_wall_fill(catalytic):
    mech, yk, case = _li_wall_case(catalytic)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    g, ns = case.ngg, mech.n_spec
    sv = _blocks(case, oz, "sv")
    Rk = 8314.462618 / np.asarray(mech.mw)
    ii = slice(g + 1, g + case.mx - 1)
    kk = slice(g + 1, g + case.mz - 1)

    def R_of(j_node, j_src, j_face):
        Rn = np.tensordot(Rk, sv[:ns, kk, j_node, ii], axes=1)
        Rg = np.tensordot(Rk, sv[:ns, kk, j_face if catalytic else j_src, ii], axes=1)
        return Rn, Rg

    _check_wall_rows(case, oz, R_of, T_wall=case.param["wall_temperature"])
    wall_y = np.broadcast_to(yk[:, None, None], sv[:ns, kk, g, ii].shape)
    for jf, sgn in ((g, -1), (g + case.my - 1, 1)):
        assert np.array_equal(sv[:ns, kk, jf, ii], wall_y if catalytic else sv[:ns, kk, jf - sgn, ii])
        for gg in range(1, g + 1):
            src = wall_y if catalytic else sv[:ns, kk, jf - sgn * gg, ii]
            assert np.array_equal(sv[:ns, kk, jf + sgn * gg, ii], src)


def test_wall_channel_steps_stay_no_slip():
    """A few RK3 steps of the viscous channel: the state stays finite, the
    wall rows keep zero velocity and the isothermal wall temperature, and
    the wall shear takes streamwise momentum out of the channel."""
    case = _air_channel(0)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    g = case.ngg
    inner = lambda: _blocks(case, oz, "cv")[1, g:g + case.mz, g + 1:g + case.my - 1, g:g + case.mx].sum()
    m0 = inner()
    for _ in range(4):
        oz.step()
    assert np.all(np.isfinite(oz["cv"]))
    bv = _blocks(case, oz, "bv")
    ii = slice(g + 1, g + case.mx - 1)
    kk = slice(g + 1, g + case.mz - 1)
    assert np.all(bv[1:4, kk, g, ii] == 0.0)
    assert np.all(bv[5, kk, g, ii] == case.param["wall_temperature"])
    assert inner() < m0


def test_wall_description_checked_before_device_use():
    import corefl_b200

    h = ctypes.c_void_p()
    faces = [(1, -1, 2), (1, 1, 2)]
    base = dict(dim=3, n_var=5, inviscid_scheme=72, weno_eps_scale=1.0)
    for bad in (dict(wall_thermal_type=2, wall_temperature=300.0), dict(wall_thermal_type=0, wall_temperature=0.0),
                dict(wall_thermal_type=-1, wall_temperature=300.0)):
        p = corefl_b200.make_param({**base, **bad}, faces)
        assert corefl_b200.lib().cfk_create(ctypes.byref(p), ctypes.byref(h)) == -1, bad
    ok = corefl_b200.make_param({**base, "wall_thermal_type": 1, "wall_yk": [0.5, 0.5]}, faces)
    assert ok.wall.thermal_type == 1 and ok.faces[0].label == 2 and list(ok.wall.yk[:3]) == [0.5, 0.5, 0.0]


def test_setup_wall_struct(tmp_path):
    """The wall struct of setup.txt: thermal type and temperature are read;
    wall fluctuations (a problem set-up outside this path) are reported
    instead of being dropped silently."""
    import corefl_b200

    def param_of(text):
        f = tmp_path / "setup.txt"
        f.write_text(text)
        p = corefl_b200.cfk_param()
        err = ctypes.create_string_buffer(256)
        rc = corefl_b200.lib().cfk_param_from_setup(str(f).encode(), ctypes.byref(p), err, 256)
        return rc, p, err.value.decode()

    head = "int inviscid_scheme = 72\narray string boundary_conditions {\n  wall\n}\n"
    rc, p, _ = param_of(head + "struct wall {\n string type = wall\n int label = 2\n string thermal_type = adiabatic\n}\n")
    assert rc == 0 and p.wall.thermal_type == 1
    rc, p, _ = param_of(head + "struct wall {\n string type = wall\n string thermal_type = isothermal\n"
                        " real temperature = 322\n}\n")
    assert rc == 0 and p.wall.thermal_type == 0 and p.wall.temperature == 322.0
    rc, _, err = param_of(head + "struct wall {\n string type = wall\n real temperature = 322\n"
                          " int fluctuation_type = 1\n real fluctuation_intensity = 0.04\n}\n")
    assert rc == -5 and "fluctuations" in err
