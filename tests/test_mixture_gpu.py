"""Parity of the mixture flow path on the GPU against the CPU oracle:
characteristic WENO5/WENO7 with species, second-order viscous flux with
mixture-averaged diffusion, mixture properties and transport, the
temperature Newton iteration in the stage update, boundary faces, and (for a
reacting mixture) the explicit chemical source inside RK3.  Bar as for air:
per RK3 step from identical inputs max|gpu - oracle| / max|oracle| <= 1e-12
per conserved variable (species included); bounded free-running drift."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, interior_planes, rel_err

pytestmark = pytest.mark.gpu

MIX_KEYS = ("cv", "bv", "mul", "qn", "acoustic_speed", "gamma", "thermal_conductivity", "rho_D",
            "reaction_timeScale")


def _lockstep_mix(case, n_steps, tol=1e-12, drift_tol=1e-10):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for s in range(n_steps):
        gz.load_from(oz, keys=MIX_KEYS)
        dt_o = oz.step()
        dt_g = gz.ctx.rk3_step()
        assert dt_g == pytest.approx(dt_o, rel=1e-12), f"dt differs at step {s}"
        e = rel_err(interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"]))
        assert e <= tol, f"step {s}: conserved-variable relative difference {e:.3e}"
    assert rel_err(gz.get("bv"), oz["bv"]) <= tol
    assert rel_err(gz.get("sv"), oz["sv"], momentum=()) <= tol
    oz2 = pyoracle.OracleZone(case)
    oz2.initialize()
    gz2 = GpuZone(case)
    gz2.initialize()
    for _ in range(n_steps):
        oz2.step()
        gz2.ctx.rk3_step()
    e = rel_err(interior_planes(case, gz2.get("cv")), interior_planes(case, oz2["cv"]))
    assert e <= drift_tol, f"free-running difference {e:.3e}"


def test_initial_mixture_properties_match():
    mech = mechanism.load("li2004")
    case = cases.mix_wave(mech, 11)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for k in ("acoustic_speed", "gamma", "mul", "thermal_conductivity"):
        assert rel_err(gz.get(k)[None], oz[k][None], momentum=()) <= 1e-13, k
    assert rel_err(gz.get("rho_D"), oz["rho_D"], momentum=()) <= 1e-13
    assert rel_err(gz.get("cv"), oz["cv"]) <= 1e-14


@pytest.mark.parametrize("scheme", [52, 72])
def test_mixture_shock_tube_steps(scheme):
    """H2/O2/Ar tube (composition jump at the contact), outflow faces."""
    _lockstep_mix(cases.mix_tube(mechanism.load("premix_h2_ar"), 120, 7, scheme=scheme), 8)


def test_mixture_3d_viscous_weno7_ragged():
    """Curvilinear periodic 3-D block, non-uniform H2/N2-air mixture: WENO7 with
    species, viscous stress, conduction, species diffusion; extents that are
    not tile multiples."""
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 13, ny=17, nz=19, scheme=72), seed=4)
    _lockstep_mix(case, 3)


def test_mixture_3d_viscous_weno5_reacting():
    """The same block at 1100 K with the Li-2004 reactions: RK3 with the
    explicit finite-rate source (fixed step)."""
    case = cases.mix_wave(mechanism.load("li2004"), 11, ny=13, nz=9, scheme=52, reacting=True, T0=1100.0, dt=2e-9)
    _lockstep_mix(case, 3)


@pytest.mark.parametrize("scheme", [52, 72])
def test_mixture_flux_single_calls(scheme):
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 15, scheme=scheme), seed=9, amp=2e-2)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.inviscid()
    oz.call("orc_compute_inviscid_flux")
    assert rel_err(gz.get("dq"), oz["dq"]) <= 1e-11
    gz.t["dq"].zero_()
    oz["dq"][:] = 0
    gz.ctx.viscous()
    oz.call("orc_compute_viscous_flux")
    assert rel_err(gz.get("dq")[1:], oz["dq"][1:], momentum=(0, 1, 2)) <= 1e-11


def _lockstep_wu(case, n_steps, tol=1e-12):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for s in range(n_steps):
        gz.load_from(oz, keys=MIX_KEYS)
        dt_o = oz.wu_splitting_step()
        dt_g = gz.ctx.wu_splitting_step(schedule=1)
        assert dt_g == pytest.approx(dt_o, rel=1e-12), f"dt differs at step {s}"
        e = rel_err(interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"]))
        assert e <= tol, f"step {s}: conserved-variable relative difference {e:.3e}"
        assert rel_err(gz.get("Cn"), oz["Cn"]) <= 1e-11
    assert rel_err(gz.get("sv"), oz["sv"], momentum=()) <= tol


def test_wu_splitting_reacting_3d_viscous_cfl_step():
    """Wu's splitting on the reacting 3-D block (1100 K, Li-2004): CFL step
    without the reaction limit, Cn from the viscous + WENO5 right-hand side,
    point-implicit reaction step with the frozen Cn, half-step RK3 on dq - Cn."""
    case = cases.mix_wave(mechanism.load("li2004"), 11, ny=13, nz=9, scheme=52, reacting=True, T0=1100.0)
    _lockstep_wu(case, 3)


def test_wu_splitting_reacting_tube_fixed_step():
    """Reacting H2/O2/Ar tube (WENO7, 2-D), fixed step of 1e-8 s."""
    mech = mechanism.load("premix_h2_ar")
    left = dict(rho=0.18075, p=35594.0 * 4, Y={"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433})
    right = dict(rho=0.072, p=7173.0 * 4, Y={"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433})
    case = cases.mix_tube(mech, 96, 7, scheme=72, reacting=True, left=left, right=right)
    case.param["fixed_dt"] = 1
    case.param["dt"] = 1e-8
    _lockstep_wu(case, 3)
