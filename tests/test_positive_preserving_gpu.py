"""Parity of the positive-preserving limiter of the species face fluxes
(reference src/WENO.cu:1471-1540: characteristic WENO, x sweep) against the
CPU oracle, in RK3 steps with the CFL dt read on the device and in Wu's
splitting step with the host dt.  Bar: 1e-12 per step."""
import pytest

import cases
import mechanism
from test_mixture_gpu import _lockstep_mix, _lockstep_wu
from test_shock_sensor_cpu import PP_STATES, _pp_tube

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme", [52, 72])
@pytest.mark.parametrize("states", PP_STATES)
def test_positive_preserving_tube_steps(scheme, states):
    _lockstep_mix(_pp_tube(scheme, 1, *states), 10)


def test_positive_preserving_hybrid_tube():
    case = _pp_tube(72, 1, *PP_STATES[0])
    case.param.update(sensor_threshold=0.05, shock_sensor=2)
    _lockstep_mix(case, 6)


def test_positive_preserving_wu_splitting_fixed_step():
    left, right = PP_STATES[0]
    case = cases.mix_tube(mechanism.load("premix_h2_ar"), 96, 7, scheme=52, reacting=True, left=left, right=right)
    case.param.update(positive_preserving=1, fixed_dt=1, dt=2e-8)
    _lockstep_wu(case, 3)
