"""Outflow faces with a back pressure in the CPU oracle (apply_outflow's
if_backPressure branch, reference src/BoundCond.cu:2082-2171), the setup.txt
outflow struct (reference src/BoundCond.cpp:597-618) and the argument checks.

Checked against the reference's rules restated in numpy from the state
before the boundary conditions: below a normal Mach number of 1 the face
state is the characteristic one at the back pressure, rho_b = rho1 +
(p_b - p1)/c1^2, u_b = u1 - (p_b - p1)/(rho1 c1) n_x, with c1 from the inner
node's gamma (the mixture's cp/(cp - R) for mixtures), and the ghosts
reflect the inner nodes about it (mass fractions about the face node's);
at or above Mach 1 the ghosts copy the face state.  The face node itself is
not changed."""
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
    oz = pyoracle.OracleZone(case)
    oz.call("orc_update_physical_properties")
    before = {k: oz[k].copy() for k in ("bv", "sv")}
    gam = oz["gamma"].copy() if case.mech is not None else None
    oz.call("orc_apply_boundary_conditions")
    return oz, before, gam


def test_subsonic_outflow_takes_the_back_pressure():
    case = cases.with_back_pressure(cases.sod(48, 9, scheme=52), 0.05)
    oz, before, _ = _fill(case)
    g, m = case.ngg, case.mx
    B0, B = _blocks(case, before["bv"]), _blocks(case, oz["bv"])
    jj, f, i1 = slice(g, g + case.my), g + m - 1, g + m - 2
    assert np.array_equal(B[:, g, jj, f], B0[:, g, jj, f])          # the face node is left alone
    d1, u1, p1 = B0[0, g, jj, i1], B0[1, g, jj, i1], B0[4, g, jj, i1]
    c1 = np.sqrt(GAMMA * p1 / d1)
    temp = (0.05 - p1) / c1
    rho_b, u_b = d1 + temp / c1, u1 - 1.0 * temp / d1
    for gg in range(1, g + 1):
        ii, gi = f - gg, f + gg
        assert np.allclose(B[4, g, jj, gi], 2 * 0.05 - B0[4, g, jj, ii], rtol=1e-14, atol=0)
        assert np.allclose(B[0, g, jj, gi], 2 * rho_b - B0[0, g, jj, ii], rtol=1e-14, atol=0)
        assert np.allclose(B[1, g, jj, gi], 2 * u_b - B0[1, g, jj, ii], rtol=1e-14, atol=1e-15)
        assert np.allclose(B[5, g, jj, gi], B[4, g, jj, gi] / (B[0, g, jj, gi] * R_AIR), rtol=1e-14, atol=0)


def test_supersonic_outflow_copies_the_face():
    base = cases.sod(48, 9, scheme=52)
    bv = base.bv.copy()
    bv[1] = 3.0 * np.sqrt(GAMMA * bv[4] / bv[0])   # Mach 3 everywhere
    case = cases.with_back_pressure(base.__class__(**{**base.__dict__, "bv": bv}), 0.05)
    oz, before, _ = _fill(case)
    g, m = case.ngg, case.mx
    B = _blocks(case, oz["bv"])
    jj, f = slice(g, g + case.my), g + m - 1
    for gg in range(1, g + 1):
        assert np.array_equal(B[:, g, jj, f + gg], B[:, g, jj, f])


def test_mixture_back_pressure_uses_the_mixture_gamma():
    mech = mechanism.load("premix_h2_ar")
    case = cases.with_back_pressure(cases.mix_tube(mech, 40, 7), 5000.0)
    oz, before, gam = _fill(case)
    g, m, ns = case.ngg, case.mx, mech.n_spec
    B0, B = _blocks(case, before["bv"]), _blocks(case, oz["bv"])
    S0, S = _blocks(case, before["sv"]), _blocks(case, oz["sv"])
    G = _blocks(case, gam[None])[0]
    jj, f, i1 = slice(g, g + case.my), g + m - 1, g + m - 2
    d1, p1 = B0[0, g, jj, i1], B0[4, g, jj, i1]
    c1 = np.sqrt(G[g, jj, i1] * p1 / d1)
    rho_b = d1 + (5000.0 - p1) / c1 / c1
    Rk = R_U / np.asarray(mech.mw)
    for gg in range(1, g + 1):
        ii, gi = f - gg, f + gg
        assert np.allclose(B[4, g, jj, gi], 2 * 5000.0 - B0[4, g, jj, ii], rtol=1e-14, atol=0)
        assert np.allclose(B[0, g, jj, gi], 2 * rho_b - B0[0, g, jj, ii], rtol=1e-13, atol=0)
        assert np.allclose(S[:ns, g, jj, gi], 2 * S0[:ns, g, jj, f] - S0[:ns, g, jj, ii], rtol=1e-14, atol=1e-16)
        R = np.tensordot(Rk, S[:ns, g, jj, gi], axes=1)
        assert np.allclose(B[5, g, jj, gi], B[4, g, jj, gi] / (B[0, g, jj, gi] * R), rtol=1e-14, atol=0)


def nozzle(scheme=52, p_back=0.3, reconstruction=2):
    """The Sod tube as a duct: subsonic inflow at i-min, back-pressure outflow
    at i-max, symmetry planes on the j faces (the back pressure applies to
    every outflow face, so the lateral faces must not be outflows)."""
    base = cases.sod(48, 9, scheme=scheme, reconstruction=reconstruction)
    base = base.__class__(**{**base.__dict__, "faces": [(f, d, 3 if f == 1 else lab) for f, d, lab in base.faces]})
    c_in = np.sqrt(GAMMA * 0.8 / 1.1)
    return cases.with_back_pressure(cases.with_inflow(base, rho=1.1, u=0.5 * c_in, p=0.8, subsonic=1), p_back)


def test_tube_with_inflow_and_back_pressure_steps():
    case = nozzle()
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    for _ in range(8):
        oz.step()
    assert np.all(np.isfinite(oz["cv"]))


def test_setup_outflow_struct_and_checks(tmp_path):
    import corefl_b200

    def param_of(text):
        f = tmp_path / "setup.txt"
        f.write_text(text)
        p = corefl_b200.cfk_param()
        err = ctypes.create_string_buffer(256)
        rc = corefl_b200.lib().cfk_param_from_setup(str(f).encode(), ctypes.byref(p), err, 256)
        return rc, p, err.value.decode()

    head = "int inviscid_scheme = 52\narray string boundary_conditions {\n  exit exit2\n}\n"
    rc, p, _ = param_of(head + "struct exit {\n string type = outflow\n int label = 6\n int if_backPressure = 1\n"
                        " real backPressure = 5e4\n}\n")
    assert rc == 0 and p.outflow.back_pressure_on == 1 and p.outflow.back_pressure == 5e4
    rc, _, err = param_of(head + "struct exit {\n string type = outflow\n int nonReflecting = 1\n}\n")
    assert rc == -5 and "non-reflecting" in err
    rc, _, err = param_of(head + "struct exit {\n string type = outflow\n int if_backPressure = 1\n"
                          " real backPressure = 5e4\n}\nstruct exit2 {\n string type = outflow\n}\n")
    assert rc == -5 and "differ" in err
    h = ctypes.c_void_p()
    bad = corefl_b200.make_param(dict(dim=3, n_var=5, inviscid_scheme=52, weno_eps_scale=1.0, outflow_back_pressure_on=1,
                                      outflow_back_pressure=0.0), [(0, 1, 6)])
    assert corefl_b200.lib().cfk_create(ctypes.byref(bad), ctypes.byref(h)) == -1
