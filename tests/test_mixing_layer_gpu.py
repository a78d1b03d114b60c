"""The mixing-layer inflow with white noise on the GPU against the oracle:
boundary applications (the seeded deviates advance with every application),
RK3 steps and Wu-splitting steps of a small reacting H2/air mixing layer
(WENO7 characteristic, mixture-averaged viscous fluxes, periodic span)."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, interior_planes, rel_err

pytestmark = pytest.mark.gpu

MIX_KEYS = ("cv", "bv", "mul", "qn", "acoustic_speed", "gamma", "thermal_conductivity", "rho_D",
            "reaction_timeScale")


@pytest.fixture(scope="module")
def mech():
    return mechanism.load("li2004")


def test_noisy_inflow_applications_match(mech):
    """Three boundary applications: the face velocity deviates agree to the
    rounding of log and sincospi; everything else bit for bit."""
    case = cases.mixing_layer(mech, 13, 33, 17, fluctuation=0.01, seed=5)
    oz = pyoracle.OracleZone(case)
    oz.call("orc_update_physical_properties")
    gz = GpuZone(case)
    gz.ctx.properties()
    for _ in range(3):
        oz.call("orc_apply_boundary_conditions")
        gz.ctx.boundary_conditions()
        assert rel_err(gz.get("bv"), oz["bv"]) <= 1e-14
        assert np.array_equal(gz.get("sv"), oz["sv"])
        assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-14
    assert oz.z.inflow_draws == 3


def test_mixing_layer_rk3_steps_match(mech):
    case = cases.mixing_layer(mech, 17, 17, 9, fluctuation=0.01)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for s in range(3):
        gz.load_from(oz, keys=MIX_KEYS)
        dt_o = oz.step()
        dt_g = gz.ctx.rk3_step()
        assert dt_g == pytest.approx(dt_o, rel=1e-12)
        e = rel_err(interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"]))
        assert e <= 1e-12, f"step {s}: {e:.3e}"


def test_mixing_layer_wu_steps_match(mech):
    case = cases.mixing_layer(mech, 17, 17, 9, fluctuation=0.01)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for s in range(2):
        gz.load_from(oz, keys=MIX_KEYS)
        dt_o = oz.wu_splitting_step()
        dt_g = gz.ctx.wu_splitting_step(schedule=1)
        assert dt_g == pytest.approx(dt_o, rel=1e-12)
        e = rel_err(interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"]))
        assert e <= 1e-12, f"step {s}: {e:.3e}"
