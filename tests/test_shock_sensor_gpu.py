"""Parity of the shock sensor and the hybrid UD5/UD7 + WENO5/WENO7 schemes
(shockSensor_threshold > 0; reference src/FieldOperation.cu:74-179,
src/WENO.cu:839-849, src/RK.cuh:112-117, src/StrangSplitting.cu:19-24)
against the CPU oracle.  Bar as for the WENO path: per RK3 step from identical
inputs max|gpu - oracle| / max|oracle| <= 1e-12 per conserved variable; the
sensor itself to 1e-12 relative."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix, _lockstep_wu
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


def _hybrid(case, kind, threshold, eps=-1.0):
    case.param.update(sensor_threshold=threshold, shock_sensor=kind, sensor_eps=eps)
    return case


def _median_threshold(case, kind, eps):
    """A threshold near the median sensor value of the block, so that both the
    linear and the WENO branch are exercised.  It is placed in the middle of
    a gap between two sorted sensor values: a threshold equal to a node's
    value would let last-bit differences of the sensor flip that node's
    branch."""
    _hybrid(case, kind, 1.0, eps)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_shock_sensor")
    s = np.sort(oz["shock_sensor"][oz["shock_sensor"] != 0])
    m = len(s) // 2
    gaps = (s[m + 1:m + 200] - s[m:m + 199]) / s[m:m + 199]
    n = m + int(np.argmax(gaps))
    assert gaps.max() > 1e-6
    return float(0.5 * (s[n] + s[n + 1]))


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_sensor_values_3d_curvilinear(kind):
    case = _hybrid(cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=72, viscous=False, amp=0.05),
                                   seed=5, amp=0.05), kind, 0.1, 1e-3)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_shock_sensor")
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.shock_sensor()
    assert rel_err(gz.get("shock_sensor"), oz["shock_sensor"], momentum=()) <= 1e-12


@pytest.mark.parametrize("kind,threshold", [(0, 0.5), (1, 0.02), (2, 0.05)])
@pytest.mark.parametrize("scheme", [52, 72])
def test_hybrid_sod_steps(scheme, kind, threshold):
    _lockstep(_hybrid(cases.sod(200, 7, scheme=scheme), kind, threshold), 10)


@pytest.mark.parametrize("scheme,kind", [(72, 0), (52, 1), (72, 2)])
def test_hybrid_3d_viscous_ragged(scheme, kind):
    """Curvilinear periodic block, extents that are not tile multiples, a
    threshold at the median sensor value: about half the faces linear."""
    case = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=scheme, viscous=True), seed=7, amp=1e-2)
    th = _median_threshold(case, kind, 1e-3)
    _lockstep(_hybrid(case, kind, th, 1e-3), 3)


def test_hybrid_context_owned_sensor_and_graph():
    """A zone bound without a sensor array: the context allocates a zeroed
    one; the graph-replayed step gives the plain step's result."""
    case = _hybrid(cases.sod(120, 7, scheme=72), 2, 0.05)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case, sensor_array=False)
    gz.initialize()
    assert "shock_sensor" not in gz.t
    for _ in range(5):
        oz.step()
        gz.ctx.rk3_step(graph=True)
    assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-10


@pytest.mark.parametrize("scheme", [52, 72])
def test_hybrid_mixture_tube(scheme):
    case = _hybrid(cases.mix_tube(mechanism.load("premix_h2_ar"), 120, 7, scheme=scheme), 2, 0.05)
    _lockstep_mix(case, 6)


def test_hybrid_mixture_3d_viscous():
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 13, ny=17, nz=19, scheme=72), seed=4, amp=1e-2)
    th = _median_threshold(case, 1, 1.0)
    _lockstep_mix(_hybrid(case, 1, th, 1.0), 3)


def test_hybrid_wu_splitting_tube():
    """Wu's splitting with the sensor computed in compute_cn."""
    mech = mechanism.load("premix_h2_ar")
    left = dict(rho=0.18075, p=35594.0 * 4, Y={"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433})
    right = dict(rho=0.072, p=7173.0 * 4, Y={"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433})
    case = _hybrid(cases.mix_tube(mech, 96, 7, scheme=72, reacting=True, left=left, right=right), 2, 0.05)
    case.param["fixed_dt"] = 1
    case.param["dt"] = 1e-8
    _lockstep_wu(case, 3)
