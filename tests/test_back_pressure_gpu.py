"""Outflow faces with a back pressure on the GPU (bc_outflow_kernel's
back-pressure branch, reference src/BoundCond.cu:2082-2171) against the CPU
oracle: the fill to 1e-14 (air and mixture, subsonic and supersonic faces)
and whole RK3 steps of a duct with a subsonic inflow and a back-pressure
exit to the per-step bar of 1e-12 with bounded drift."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_back_pressure_cpu import GAMMA, nozzle
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


def _fill_parity(case, tol=1e-14):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    assert rel_err(gz.get("bv"), oz["bv"]) <= tol
    assert rel_err(gz.get("cv"), oz["cv"]) <= tol
    if case.mech is not None:
        assert rel_err(gz.get("sv"), oz["sv"], momentum=()) <= tol


def test_air_fill_subsonic_and_supersonic():
    base = cases.sod(48, 9, scheme=52)
    _fill_parity(cases.with_back_pressure(base, 0.05))
    bv = base.bv.copy()
    bv[1] = 3.0 * np.sqrt(GAMMA * bv[4] / bv[0])
    _fill_parity(cases.with_back_pressure(base.__class__(**{**base.__dict__, "bv": bv}), 0.05))


def test_mixture_fill():
    mech = mechanism.load("premix_h2_ar")
    _fill_parity(cases.with_back_pressure(cases.mix_tube(mech, 40, 7), 5000.0), tol=1e-13)


@pytest.mark.parametrize("scheme,recon", [(52, 2), (4, 2)])
def test_duct_with_back_pressure_steps(scheme, recon):
    _lockstep(nozzle(scheme=scheme, reconstruction=recon), 10)
