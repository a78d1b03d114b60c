"""The pressure-gradient term of the mixture diffusion flux
(gradPInDiffusionFlux; reference src/ViscousScheme.cu:495-520, 742-766,
931-955, 1115-1139) on the GPU against the CPU oracle: single viscous calls
of the second-order and collocated 8th-order schemes to 1e-11, and RK3 steps
to the per-step bar of 1e-12, as the other mixture parity tests."""
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix

pytestmark = pytest.mark.gpu


def _case(order):
    mech = mechanism.load("li2004")
    base = cases.perturbed(cases.mix_wave(mech, 13, ny=11, nz=9, scheme=52, viscous=True, viscous_order=order), seed=6,
                           amp=2e-2)
    return base.__class__(**{**base.__dict__, "param": {**base.param, "gradPInDiffusionFlux": 1}})


@pytest.mark.parametrize("order", [2, 8])
def test_single_viscous_call_with_gradp(order):
    case = _case(order)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    oz["dq"][:] = 0
    gz.t["dq"].zero_()
    gz.ctx.viscous()
    oz.call("orc_compute_viscous_flux")
    assert rel_err(gz.get("dq")[1:], oz["dq"][1:], momentum=(0, 1, 2)) <= 1e-11


@pytest.mark.parametrize("order", [2, 8])
def test_rk3_steps_with_gradp(order):
    _lockstep_mix(_case(order), 2)
