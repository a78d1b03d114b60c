"""Parity of the primitive-variable schemes (Lax-Friedrichs, Roe with the
entropy fix, AUSM+, HLLC; first-order, MUSCL and NND2 reconstruction)
against the CPU oracle.  Bar as for the WENO path: per RK3 step from
identical inputs max|gpu - oracle| / max|oracle| <= 1e-12 per conserved
variable; bounded free-running drift."""
import numpy as np
import pytest

import cases
import pyoracle
from gpuzone import GpuZone, rel_err
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("recon", [1, 2, 3])
@pytest.mark.parametrize("scheme", [1, 2, 3, 4])
def test_sod_pv_scheme_steps(scheme, recon):
    _lockstep(cases.sod(400, 7, scheme=scheme, reconstruction=recon), 10)


@pytest.mark.parametrize("scheme,recon", [(2, 2), (4, 3), (3, 1), (1, 2)])
def test_sine_wave_3d_pv_scheme_ragged_tiles(scheme, recon):
    """Curvilinear periodic 3-D block with viscous flux, extents that are not
    tile multiples; Roe uses the 3-D entropy-fix width."""
    case = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=scheme, reconstruction=recon, viscous=True),
                           seed=7)
    _lockstep(case, 4)


@pytest.mark.parametrize("scheme", [1, 2, 3, 4])
def test_pv_inviscid_flux_perturbed_single_call(scheme):
    """One cfk_compute_inviscid_flux on a strongly perturbed 3-D state
    (supersonic and subsonic faces, both HLLC star regions)."""
    case = cases.perturbed(cases.sine_wave(n=21, scheme=scheme, viscous=False, amp=0.2), seed=3, amp=0.3)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.inviscid()
    oz.call("orc_compute_inviscid_flux")
    assert rel_err(gz.get("dq"), oz["dq"]) <= 1e-11
