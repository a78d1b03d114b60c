"""The mixing-layer inflow and its white noise on the CPU oracle: the
reference's apply_inflow branches (src/BoundCond.cu:2455-2506 for the
mixing layer, :2573-2596 for a constant inflow) with this library's seeded
deviates in place of curand's, and the stream set-up of
get_mixing_layer_info (src/MixingLayer.cu:9-119)."""
import ctypes
import dataclasses

import numpy as np
import pytest

import cases
import mechanism
import pyoracle


@pytest.fixture(scope="module")
def mech():
    return mechanism.load("li2004")


def test_uniform_deviates_are_in_range_and_distinct():
    L = pyoracle.lib()
    u = np.array([L.orc_noise_uniform(7, c, node, n) for c in range(3) for node in range(200) for n in range(4)])
    assert np.all(u > 0) and np.all(u <= 1)
    assert len(np.unique(u)) == u.size
    assert abs(u.mean() - 0.5) < 0.03 and abs(u.var() - 1 / 12) < 0.01
    assert L.orc_noise_uniform(7, 1, 5, 2) == L.orc_noise_uniform(7, 1, 5, 2)
    assert L.orc_noise_uniform(7, 1, 5, 2) != L.orc_noise_uniform(8, 1, 5, 2)


def test_streams_follow_the_convective_mach_number(mech):
    c = cases.mixing_layer(mech, 9, 9, 7)
    up, lo = cases.mixing_layer_streams(mech, dict(T=600.0, p=101325.0, Y={"O2": 0.233, "N2": 0.767}),
                                        dict(T=600.0, p=101325.0, Y={"H2": 0.067, "N2": 0.933}), 0.2, 1.5)
    assert up["u"] == pytest.approx(1.5 * lo["u"], rel=1e-14)
    assert (up["u"] - lo["u"]) / (up["c"] + lo["c"]) == pytest.approx(0.2, rel=1e-12)
    assert c.param["inflow_u"] == pytest.approx(1.5 * c.param["inflow_u_lower"], rel=1e-14)


def _face0(c, arr):
    g = c.ngg
    return arr.reshape((arr.shape[0],) + c.shape())[:, g:g + c.mz, :, g]


def _apply(case):
    oz = pyoracle.OracleZone(case)
    oz.call("orc_update_physical_properties")
    oz.call("orc_apply_boundary_conditions")
    return oz


def test_mixing_layer_inflow_without_noise(mech):
    c = cases.mixing_layer(mech, 9, 17, 7, fluctuation=0.0)
    oz = _apply(c)
    g = c.ngg
    bv = oz["bv"].reshape((6,) + c.shape())
    y = c.y.reshape(c.shape())[g:g + c.mz, :, g]
    p = c.param
    u = 0.5 * (p["inflow_u"] + p["inflow_u_lower"]) + 0.5 * (p["inflow_u"] - p["inflow_u_lower"]) * np.tanh(
        2 * y / p["inflow_delta_omega"])
    face = bv[:, g:g + c.mz, :, g]
    assert np.array_equal(face[1], u)
    above = y >= 0
    assert np.array_equal(face[0], np.where(above, p["inflow_density"], p["inflow_density_lower"]))
    assert np.array_equal(face[5], np.where(above, p["inflow_temperature"], p["inflow_t_lower"]))
    assert np.all(face[2] == 0) and np.all(face[3] == 0)
    for gg in range(1, g + 1):
        assert np.array_equal(bv[:, g:g + c.mz, :, g - gg], face)
    sv = oz["sv"].reshape((-1,) + c.shape())[:, g:g + c.mz, :, g]
    assert np.array_equal(sv[:, above], np.repeat(np.array(p["inflow_sv"])[:, None], above.sum(), axis=1))
    assert oz.z.inflow_draws == 0


def test_white_noise_has_the_stated_rms_and_moves_on(mech):
    c = cases.mixing_layer(mech, 9, 129, 65, fluctuation=0.01, seed=11)
    g = c.ngg
    p = c.param
    oz = _apply(c)
    base = _apply(dataclasses.replace(c, param=dict(c.param, inflow_fluctuation_type=0)))
    y = c.y.reshape(c.shape())[g:g + c.mz, :, g]
    u0 = _face0(c, base["bv"])[1]
    rms = p["inflow_fluctuation_intensity"] * u0 * np.exp(-y * y)
    for l in (1, 2, 3):
        dev = (_face0(c, oz["bv"])[l] - _face0(c, base["bv"])[l]) / rms
        assert abs(dev.mean()) < 0.03 and abs(dev.std() - 1.0) < 0.03
    assert oz.z.inflow_draws == 1
    first = oz["bv"].copy()
    oz.call("orc_apply_boundary_conditions")
    assert oz.z.inflow_draws == 2 and not np.array_equal(_face0(c, oz["bv"])[1], _face0(c, first)[1])
    again = _apply(c)
    assert np.array_equal(again["bv"], first)


def test_constant_inflow_noise_on_u_only():
    c = cases.with_inflow(cases.sod(16, 9), rho=1.0, u=2.0, p=1.0)
    c = dataclasses.replace(c, param=dict(c.param, inflow_fluctuation_type=1, inflow_fluctuation_intensity=0.05,
                                          inflow_seed=3))
    oz = _apply(c)
    g = c.ngg
    inflow_face = [f for f in c.faces if f[2] == 5][0]
    assert inflow_face[0] == 0
    bv = oz["bv"].reshape((6,) + c.shape())
    side = g if inflow_face[1] < 0 else g + c.mx - 1
    face = bv[:, g, g:g + c.my, side]
    assert np.all(face[2] == 0) and np.all(face[0] == 1.0)
    dev = (face[1] - 2.0) / (0.05 * 2.0)
    assert np.all(np.abs(dev) < 6) and dev.std() > 0.3


def test_mixing_layer_steps_stay_finite(mech):
    c = cases.mixing_layer(mech, 17, 17, 9, reacting=True)
    oz = pyoracle.OracleZone(c)
    oz.initialize()
    for _ in range(3):
        dt = oz.step()
        assert dt > 0
    assert np.all(np.isfinite(oz["cv"])) and np.all(np.isfinite(oz["bv"]))
    assert oz.z.inflow_draws == 1 + 3 * 3
