"""Parity at the benchmark configurations' own sizes, with both metrics.

* One SSP-RK3 step of the 257^3 curvilinear periodic block (WENO7
  characteristic + 2nd-order viscous, Sutherland at Re = 1000, CFL 0.5): the
  benchmark's headline workload, against the CPU oracle from identical inputs.
* Point-implicit Wu reaction steps of 65536 seeded H2/air reactors (Li-2004;
  T ~ U[1000, 1600] K, p log-uniform in [1, 10] atm, phi ~ U[0.5, 2]; 1e-7 s
  per step) through the work-queue schedule, against the oracle.

Both the normwise difference (max|gpu - oracle| / max|oracle| per variable)
and the pointwise one (per node, see gpuzone.pointwise_rel_err) must stay
within 1e-12.  The oracle step of the 257^3 block takes a few seconds on the
host's cores.
"""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, interior_planes, pointwise_rel_err, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def test_headline_block_257_one_rk3_step():
    case = cases.sine_wave(n=257, scheme=72, viscous=True)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.load_from(oz)
    dt_o = oz.step()
    dt_g = gz.ctx.rk3_step()
    assert dt_g == pytest.approx(dt_o, rel=1e-13)
    g = interior_planes(case, gz.get("cv"))
    o = interior_planes(case, oz["cv"])
    e_norm = rel_err(g, o)
    e_point = pointwise_rel_err(g, o)
    print(f"257^3 RK3 step: normwise {e_norm:.3e}, pointwise {e_point:.3e}")
    assert e_norm <= TOL
    assert e_point <= TOL


def test_reactor_batch_65536_point_implicit_steps():
    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, 65536, seed=2024)
    oz = pyoracle.OracleZone(case)
    oz.call("orc_compute_cv_from_bv")
    gz = GpuZone(case)
    import torch
    nsub = torch.zeros(case.N, dtype=torch.int32, device="cuda:0")
    for s in range(2):
        gz.load_from(oz, keys=("cv", "bv", "sv", "reaction_timeScale"))
        ns_o = oz.reaction_step(1e-7, want_nsub=True)
        gz.ctx.wu_reaction_step(1e-7, schedule=1, nsub_ptr=nsub.data_ptr())
        gz.ctx.sync()
        assert np.array_equal(nsub.cpu().numpy(), ns_o), f"substep counts differ at step {s}"
        g, o = gz.get("cv"), oz["cv"]
        e_norm = rel_err(g, o)
        e_point = pointwise_rel_err(g, o, n_spec=mech.n_spec)
        print(f"65536 reactors, step {s}: normwise {e_norm:.3e}, pointwise {e_point:.3e}")
        assert e_norm <= TOL
        assert e_point <= TOL
