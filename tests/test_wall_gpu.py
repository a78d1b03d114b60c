"""No-slip wall faces on the GPU (bc_wall_kernel, reference
src/BoundCond.cu:2761-3031) against the CPU oracle.

The wall fill itself: copies and sign flips (velocity, pressure, wall
temperature, mass fractions) are bitwise equal to the oracle's; the densities
and conserved variables built from them agree to 1e-14.  Whole RK3 steps of
walled blocks (air isothermal and adiabatic, WENO5/7, second- and
eighth-order viscous terms, a 2-D tube, mixtures with non-catalytic and
catalytic walls) meet the per-step bar of 1e-12 with bounded free-running
drift, as the other parity tests."""
import numpy as np
import pytest

import cases
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix
from test_parity_gpu import _lockstep
from test_wall_cpu import _li_wall_case

pytestmark = pytest.mark.gpu


def _channel(thermal_type, scheme=52, viscous_order=2, seed=5):
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=scheme, viscous=True,
                                           viscous_order=viscous_order), seed=seed, amp=2e-2)
    return cases.with_walls(base, thermal_type=thermal_type)


def _fill_parity(case):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    bo, bg = oz["bv"], gz.get("bv")
    for l in (1, 2, 3, 4, 5):
        assert np.array_equal(bg[l], bo[l]), f"bv plane {l}"
    assert rel_err(bg[:1], bo[:1], momentum=()) <= 1e-14
    assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-14
    if case.param["n_spec"]:
        assert np.array_equal(gz.get("sv"), oz["sv"])


@pytest.mark.parametrize("thermal_type,temp_scale", [(0, 0.95), (1, None), (0, 0.5)])
def test_air_wall_fill_matches_oracle(thermal_type, temp_scale):
    """Isothermal, adiabatic and a cold isothermal wall whose ghosts take the
    0.1 T_w clamp."""
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=52, viscous=True), seed=5, amp=2e-2)
    T = None if temp_scale is None else temp_scale * float(np.mean(base.bv[5]))
    _fill_parity(cases.with_walls(base, thermal_type=thermal_type, temperature=T))


@pytest.mark.parametrize("catalytic", [0, 1])
def test_mixture_wall_fill_matches_oracle(catalytic):
    _fill_parity(_li_wall_case(catalytic)[2])


@pytest.mark.parametrize("thermal_type,scheme", [(0, 52), (1, 72)])
def test_air_channel_steps(thermal_type, scheme):
    _lockstep(_channel(thermal_type, scheme=scheme), 4)


def test_air_block_walls_on_i_and_k_faces():
    """Walls on i and k faces too (the i-face kernel splits a node's ghost
    layers over threads)."""
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=52, viscous=True), seed=8, amp=2e-2)
    _lockstep(cases.with_walls(base, thermal_type=0, faces=((0, -1), (0, 1), (2, -1), (1, 1))), 3)


def test_air_channel_eighth_order_viscous():
    _lockstep(_channel(0, scheme=72, viscous_order=8), 3)


def test_sod_tube_between_walls_2d():
    _lockstep(cases.with_walls(cases.sod(96, 9, scheme=52), thermal_type=1), 10)


@pytest.mark.parametrize("catalytic", [0, 1])
def test_mixture_channel_steps(catalytic):
    _lockstep_mix(_li_wall_case(catalytic)[2], 3)
