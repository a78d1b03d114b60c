"""Parity of the primitive-variable schemes for mixtures (Roe with the species
terms, AUSM+, HLLC; first-order, MUSCL and NND2 reconstruction of the flow
variables and mass fractions) against the CPU oracle.  Bar as for the other
flux paths: per RK3 step from identical inputs max|gpu - oracle| /
max|oracle| <= 1e-12 per conserved variable; single flux calls 1e-11."""
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_mixture_gpu import _lockstep_mix, _lockstep_wu

pytestmark = pytest.mark.gpu

H2_O2_AR = {"H2": 0.012772428, "O2": 0.101362139, "AR": 0.885865433}


@pytest.mark.parametrize("recon", [1, 2, 3])
@pytest.mark.parametrize("scheme", [2, 3, 4])
def test_mixture_tube_pv_scheme_steps(scheme, recon):
    """Composition and pressure jump (H2/O2/Ar against pure Ar)."""
    left = dict(rho=0.18075, p=35594.0 * 4, Y=H2_O2_AR)
    right = dict(rho=0.072, p=7173.0, Y={"AR": 1.0})
    case = cases.mix_tube(mechanism.load("premix_h2_ar"), 120, 7, scheme=scheme, left=left, right=right,
                          reconstruction=recon)
    _lockstep_mix(case, 6)


@pytest.mark.parametrize("scheme,recon", [(2, 2), (4, 3), (3, 1)])
def test_mixture_3d_viscous_pv_scheme_ragged(scheme, recon):
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 13, ny=17, nz=19, scheme=scheme,
                                          reconstruction=recon), seed=4, amp=1e-2)
    _lockstep_mix(case, 3)


@pytest.mark.parametrize("scheme", [2, 3, 4])
def test_mixture_pv_flux_perturbed_single_call(scheme):
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 15, scheme=scheme, viscous=False), seed=9,
                           amp=2e-2)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.inviscid()
    oz.call("orc_compute_inviscid_flux")
    assert rel_err(gz.get("dq"), oz["dq"]) <= 1e-11


def test_mixture_reacting_rk3_roe():
    case = cases.mix_wave(mechanism.load("li2004"), 11, ny=13, nz=9, scheme=2, reacting=True, T0=1100.0, dt=2e-9)
    _lockstep_mix(case, 3)


def test_wu_splitting_hllc_tube():
    left = dict(rho=0.18075, p=35594.0 * 4, Y=H2_O2_AR)
    right = dict(rho=0.072, p=7173.0 * 4, Y=H2_O2_AR)
    case = cases.mix_tube(mechanism.load("premix_h2_ar"), 96, 7, scheme=4, reacting=True, left=left, right=right)
    case.param.update(fixed_dt=1, dt=1e-8)
    _lockstep_wu(case, 3)
