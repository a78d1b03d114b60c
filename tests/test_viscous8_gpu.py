"""Parity of the collocated viscous schemes against the CPU oracle: the
reference's 8th-order scheme (viscous_order = 8: node fluxes, periodic
exchange in face order, derivative; reference src/ViscousScheme.cu:41-70,
129-612) and its 4th-order variant (viscous_order = 4).  Bar: single viscous
calls 1e-11, RK3 / Wu steps 1e-12 per step."""
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix, _lockstep_wu
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


def _single_viscous(case):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    oz["dq"][:] = 0
    gz.t["dq"].zero_()
    gz.ctx.viscous()
    oz.call("orc_compute_viscous_flux")
    # mass slot stays zero; the other rows share the momentum scale
    return rel_err(gz.get("dq")[1:], oz["dq"][1:], momentum=(0, 1, 2))


ORDERS = pytest.mark.parametrize("order", [8, 4])


@ORDERS
def test_air_periodic_3d_single_call(order):
    case = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=72, viscous_order=order), seed=7, amp=1e-2)
    assert _single_viscous(case) <= 1e-11


@ORDERS
def test_air_walls_2d_single_call(order):
    """Physical faces on every side: the one-sided boundary stencils."""
    case = cases.perturbed(cases.sod(64, 13, scheme=4, viscous_order=order), seed=2, amp=1e-2)
    assert _single_viscous(case) <= 1e-11


@ORDERS
def test_mixture_periodic_3d_single_call(order):
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 13, ny=17, nz=19, scheme=72, viscous_order=order),
                           seed=4, amp=1e-2)
    assert _single_viscous(case) <= 1e-11


@pytest.mark.parametrize("scheme", [72, 52, 4])
def test_air_rk3_steps(scheme):
    case = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=scheme, viscous_order=8), seed=7)
    _lockstep(case, 3)


@ORDERS
def test_air_sod_viscous_collocated_steps(order):
    _lockstep(cases.sod(200, 9, scheme=52, viscous_order=order), 10)


def test_air_rk3_steps_fourth_order():
    case = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=72, viscous_order=4), seed=7)
    _lockstep(case, 3)


def test_mixture_rk3_steps():
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 13, ny=17, nz=19, scheme=72, viscous_order=8),
                           seed=4, amp=1e-2)
    _lockstep_mix(case, 3)


def test_mixture_tube_hllc_viscous8_steps():
    case = cases.mix_tube(mechanism.load("premix_h2_ar"), 120, 9, scheme=4, viscous_order=8)
    _lockstep_mix(case, 6)


def test_wu_splitting_viscous8():
    case = cases.mix_wave(mechanism.load("li2004"), 11, ny=13, nz=9, scheme=52, reacting=True, T0=1100.0,
                          viscous_order=8)
    _lockstep_wu(case, 2)
