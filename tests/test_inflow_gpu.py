"""Constant inflow faces on the GPU (bc_inflow_kernel, reference
src/BoundCond.cu:2190-2705) against the CPU oracle.

The fill itself: a supersonic inflow copies the state, bitwise equal to the
oracle; the subsonic characteristic combination agrees to 1e-14 (fused
multiply-adds on the GPU).  Whole RK3 steps of a 2-D tube (supersonic and
subsonic inflow, WENO5 and HLLC), a curvilinear 3-D block with an inflow
face and a mixture tube meet the per-step bar of 1e-12 with bounded
free-running drift, as the other parity tests."""
import dataclasses

import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu

C_IN = np.sqrt(1.4 * 0.8 / 1.1)


def _tube(subsonic, u_in, scheme=52, reconstruction=2):
    return cases.with_inflow(cases.sod(64, 9, scheme=scheme, reconstruction=reconstruction), rho=1.1, u=u_in, p=0.8,
                             subsonic=subsonic)


def _fill(case):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    return oz, gz


def test_supersonic_fill_is_bitwise():
    oz, gz = _fill(_tube(0, 2.5 * C_IN))
    assert np.array_equal(gz.get("bv"), oz["bv"])


@pytest.mark.parametrize("u_scale", [0.3, -0.4])
def test_subsonic_fill_matches_oracle(u_scale):
    oz, gz = _fill(_tube(1, u_scale * C_IN))
    assert rel_err(gz.get("bv"), oz["bv"]) <= 1e-14
    assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-14


@pytest.mark.parametrize("sub,u_scale,scheme,recon", [(0, 2.0, 52, 2), (1, 0.4, 52, 2), (1, 0.4, 4, 2)])
def test_tube_with_inflow_steps(sub, u_scale, scheme, recon):
    _lockstep(_tube(sub, u_scale * C_IN, scheme, recon), 10)


def test_curvilinear_block_with_inflow_face_steps():
    base = cases.perturbed(cases.sine_wave(n=21, ny=11, nz=9, scheme=72, viscous=True), seed=4, amp=1e-2)
    base = dataclasses.replace(base, faces=[(f, d, 6 if f == 0 else lab) for f, d, lab in base.faces])
    p0 = float(np.mean(base.bv[4]))
    case = cases.with_inflow(base, rho=1.0, u=1.0, p=p0, v=0.05, subsonic=1)
    _lockstep(case, 3)


def test_mixture_tube_with_subsonic_inflow_steps():
    mech = mechanism.load("premix_h2_ar")
    base = cases.mix_tube(mech, 64, 7)
    Y = np.zeros(mech.n_spec)
    Y[mech.index("O2")], Y[mech.index("AR")] = 0.2, 0.8
    case = cases.with_inflow(base, rho=0.1, u=50.0, p=1.2e4, Y=Y, subsonic=1)
    oz, gz = _fill(case)
    assert rel_err(gz.get("bv"), oz["bv"]) <= 1e-13
    _lockstep_mix(case, 5)
