"""Shock sensor and hybrid UD/WENO scheme in the CPU oracle (reference
src/FieldOperation.cu:74-179, src/WENO.cu:839-849 and 3059-3222).

The oracle's sensors are checked against an independent numpy restatement of
the three formulas on a curvilinear block; the linear branches of its WENO5 /
WENO7 against the closed-form upwind-biased stencils; the hybrid Sod run for
the expected switching pattern."""
import ctypes

import numpy as np
import pytest

import cases
import pyoracle


def _grid(case, a, n):
    g = case.ngg
    return a.reshape(n, case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)


def _d4(f, axis):
    """4th-order central difference along an array axis (node spacing 1)."""
    r = lambda s: np.roll(f, -s, axis=axis)
    return r(-2) / 12 - 2 * r(-1) / 3 + 2 * r(1) / 3 - r(2) / 12


def _sensors_numpy(case, bv, metric, eps):
    g = case.ngg
    B = _grid(case, bv, 6)
    M = _grid(case, metric, 9)
    u, v, w = B[1], B[2], B[3]
    rho, p = B[0], B[4]
    # axes of the padded array: (k, j, i) -> xi is axis 2, eta 1, zeta 0
    du = [_d4(u, 2), _d4(u, 1), _d4(u, 0)]
    dv = [_d4(v, 2), _d4(v, 1), _d4(v, 0)]
    dw = [_d4(w, 2), _d4(w, 1), _d4(w, 0)]
    grad = lambda d, c: d[0] * M[c] + d[1] * M[3 + c] + d[2] * M[6 + c]
    div = grad(du, 0) + grad(dv, 1) + grad(dw, 2)
    cx = grad(dw, 1) - grad(dv, 2)
    cy = grad(du, 2) - grad(dw, 0)
    cz = grad(dv, 0) - grad(du, 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        ducros = np.where(div > 0, 0.0, div * div / (div * div + cx * cx + cy * cy + cz * cz + eps))
    jam = 0.0
    for ax in (2, 1, 0):
        s = np.roll(p, -1, axis=ax) + np.roll(p, 1, axis=ax)
        jam = jam + np.abs(s - 2 * p) / (s + 2 * p)
    jump = np.zeros_like(p)
    for f in (rho, p):
        for ax in (2, 1, 0):
            jump = np.maximum(jump, np.abs(np.roll(f, -1, axis=ax) - f) / f)
    inner = (slice(g, g + case.mz), slice(g, g + case.my), slice(g, g + case.mx))
    return [s[inner] for s in (ducros, jam, jump)]


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_oracle_sensor_matches_numpy_restatement(kind):
    case = cases.perturbed(cases.sine_wave(n=13, ny=11, nz=9, scheme=72, viscous=False, amp=0.05), seed=2,
                           amp=0.05)
    case.param.update(sensor_threshold=0.1, shock_sensor=kind, sensor_eps=1e-3)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_shock_sensor")
    ref = _sensors_numpy(case, oz["bv"], oz["metric"], 1e-3)[kind]
    got = _grid(case, oz["shock_sensor"], 1)[0]
    g = case.ngg
    inner = got[g:g + case.mz, g:g + case.my, g:g + case.mx]
    assert np.allclose(inner, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
    # ghost layers keep their zero initialisation
    ghost = np.ones(got.shape, bool)
    ghost[g:g + case.mz, g:g + case.my, g:g + case.mx] = False
    assert not got[ghost].any()
    if kind == 0:
        assert 0.0 <= inner.min() and inner.max() <= 1.0 and (inner == 0).any() and (inner > 0).any()


def _weno(L, name):
    f = getattr(L, name)
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int]
    return f


def _arr(x):
    return (ctypes.c_double * len(x))(*x)


def test_oracle_linear_branches_are_upwind_stencils():
    """if_shock = 0: WENO5 -> UD5 (2,-13,47,27,-3)/60, WENO7 -> UD7
    (-3,25,-101,319,214,-38,4)/420, minus side mirrored; on a quartic
    (resp. sextic) the nonlinear weights reproduce the linear result."""
    L = pyoracle.lib()
    w5, w7 = _weno(L, "orc_weno5"), _weno(L, "orc_weno7")
    rng = np.random.default_rng(4)
    ud5 = np.array([2, -13, 47, 27, -3]) / 60
    ud7 = np.array([-3, 25, -101, 319, 214, -38, 4]) / 420
    for _ in range(20):
        vp, vm = rng.normal(size=5), rng.normal(size=5)
        ref = ud5 @ vp + ud5 @ vm[::-1]
        assert w5(_arr(vp), _arr(vm), 1e-40, 0) == pytest.approx(ref, rel=1e-13, abs=1e-15)
        vp, vm = rng.normal(size=7), rng.normal(size=7)
        ref = ud7 @ vp + ud7 @ vm[::-1]
        assert w7(_arr(vp), _arr(vm), 1e-40, 0) == pytest.approx(ref, rel=1e-13, abs=1e-15)
    x = np.arange(7) * 1e-2
    smooth = 1 + x + 0.3 * x ** 2
    lin = w7(_arr(smooth), _arr(smooth), 1e-40, 0)
    non = w7(_arr(smooth), _arr(smooth), 1e-40, 1)
    assert non == pytest.approx(lin, rel=1e-9)


def test_oracle_hybrid_sod_switches_at_the_shock():
    """Sod tube with the density/pressure jump sensor: faces near the
    discontinuities take WENO, the plateaus the linear scheme.  The run stays
    positive and its solution differs from pure WENO5 only in a few nodes
    around the waves."""
    weno = cases.sod(200, 7, scheme=52)
    hyb = cases.sod(200, 7, scheme=52)
    hyb.param.update(sensor_threshold=0.05, shock_sensor=2)
    ow, oh = pyoracle.OracleZone(weno), pyoracle.OracleZone(hyb)
    ow.initialize()
    oh.initialize()
    for _ in range(30):
        ow.step()
        oh.step()
    g = hyb.ngg
    s = _grid(hyb, oh["shock_sensor"], 1)[0][g + 0, g + 3, g:g + hyb.mx]
    shocked = s > 0.05
    assert 0 < shocked.sum() < 40
    rho_h = _grid(hyb, oh["cv"], hyb.param["n_var"])[0][g, g + 3, g:g + hyb.mx]
    rho_w = _grid(weno, ow["cv"], weno.param["n_var"])[0][g, g + 3, g:g + weno.mx]
    assert np.all(np.isfinite(rho_h)) and rho_h.min() > 0.1
    diff = np.abs(rho_h - rho_w)
    assert diff.max() < 0.05
    assert diff.max() > 1e-8  # the linear branch was taken somewhere


def _pp_tube(scheme, pp, left, right, cfl=0.5):
    import mechanism

    case = cases.mix_tube(mechanism.load("premix_h2_ar"), 120, 7, scheme=scheme, left=left, right=right)
    case.param.update(positive_preserving=pp, cfl=cfl)
    return case


PP_STATES = [
    (dict(rho=0.8, p=1e6, Y={"H2": 1.0}), dict(rho=0.16, p=1e4, Y={"O2": 0.3, "AR": 0.7})),
    (dict(rho=1.6, p=1e6, Y={"AR": 1.0}), dict(rho=0.008, p=1e3, Y={"H2": 1.0})),
]


@pytest.mark.parametrize("states", PP_STATES)
def test_oracle_positive_preserving_limiter_acts(states):
    """Strong pressure jump across a contact between disjoint species sets:
    the limiter of the x-face species fluxes (reference src/WENO.cu:1471-1540)
    changes the solution and the run stays finite."""
    out = []
    for pp in (0, 1):
        oz = pyoracle.OracleZone(_pp_tube(52, pp, *states))
        oz.initialize()
        for _ in range(20):
            oz.step()
        out.append(oz["cv"].copy())
    assert np.all(np.isfinite(out[1]))
    assert np.abs(out[1] - out[0]).max() > 1e-6 * np.abs(out[0]).max()
