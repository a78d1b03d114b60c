"""Parity of the sm_100a path against the CPU oracle (FP64, air model).

Bar: per-variable relative difference max|gpu - oracle| / max|oracle| of the
conserved variables <= 1e-12 after every RK3 step (the three momentum planes
share the largest momentum magnitude as their scale), and the pointwise
relative difference (per node; gpuzone.pointwise_rel_err) <= 1e-12 as well;
the CFL time step agrees to 1e-13.  Inputs are seeded; sizes are small enough for the oracle to
finish in seconds.
"""
import numpy as np
import pytest

import cases
import pyoracle
from gpuzone import GpuZone, interior_planes, pointwise_rel_err, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _lockstep(case, n_steps, graph=False, tol=TOL, drift_tol=1e-10, tiles=None):
    """Per-step parity: before every step the device state is reset to the
    oracle's, so each comparison covers exactly one RK3 step from identical
    inputs (tolerance `tol`).  A second, free-running pair checks that the
    round-off difference stays bounded over n_steps (tolerance `drift_tol`)."""
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    if tiles is not None:
        gz.ctx.set_tile_variants(tiles)
    worst = 0.0
    for s in range(n_steps):
        gz.load_from(oz)
        dt_o = oz.step()
        dt_g = gz.ctx.rk3_step(graph=graph)
        assert dt_g == pytest.approx(dt_o, rel=1e-13), f"dt differs at step {s}"
        g, o = interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"])
        e = rel_err(g, o)
        worst = max(worst, e)
        assert e <= tol, f"step {s}: conserved-variable relative difference {e:.3e} > {tol:g}"
        ep = pointwise_rel_err(g, o)
        assert ep <= tol, f"step {s}: pointwise relative difference {ep:.3e} > {tol:g}"
    # the padded arrays (ghosts filled by the BCs) agree as well
    assert rel_err(gz.get("cv"), oz["cv"]) <= tol
    assert rel_err(gz.get("bv"), oz["bv"]) <= tol
    # free-running drift
    oz2 = pyoracle.OracleZone(case)
    oz2.initialize()
    gz2 = GpuZone(case)
    gz2.initialize()
    if tiles is not None:
        gz2.ctx.set_tile_variants(tiles)
    for s in range(n_steps):
        oz2.step()
        gz2.ctx.rk3_step(graph=graph)
    e = rel_err(interior_planes(case, gz2.get("cv")), interior_planes(case, oz2["cv"]))
    assert e <= drift_tol, f"after {n_steps} free-running steps the difference is {e:.3e}"
    return worst


def test_sod_weno5_char_steps():
    """Sod tube, WENO5 characteristic (scheme 52), CFL 0.5, outflow faces."""
    _lockstep(cases.sod(400, 7, scheme=52), 20)


def test_sod_weno7_char_steps():
    _lockstep(cases.sod(200, 7, scheme=72), 20)


def test_sine_wave_3d_viscous_weno7():
    """Curvilinear periodic block, WENO7 characteristic + 2nd-order viscous."""
    case = cases.perturbed(cases.sine_wave(n=25, scheme=72, viscous=True), seed=1)
    _lockstep(case, 5)


def test_sine_wave_3d_weno5_ragged_tiles():
    """Extents that are not multiples of the CTA tiles in any direction."""
    case = cases.perturbed(cases.sine_wave(n=19, ny=23, nz=17, scheme=52, viscous=True), seed=2)
    _lockstep(case, 4)


def test_graph_step_matches_plain_step():
    case = cases.sine_wave(n=17, scheme=72, viscous=True)
    a = GpuZone(case)
    a.initialize()
    b = GpuZone(case)
    b.initialize()
    for _ in range(3):
        a.ctx.rk3_step(graph=False)
        b.ctx.rk3_step(graph=True)
    assert np.array_equal(a.get("cv"), b.get("cv"))


def test_inviscid_flux_perturbed_single_call():
    """One cfk_compute_inviscid_flux on a strongly perturbed state (all
    characteristic fields active, |kx| > 0.8 and <= 0.8 branches)."""
    case = cases.perturbed(cases.sine_wave(n=21, scheme=72, viscous=False, amp=0.2), seed=3, amp=5e-2)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.inviscid()
    oz.call("orc_compute_inviscid_flux")
    assert rel_err(gz.get("dq"), oz["dq"]) <= 1e-11


def test_viscous_flux_single_call():
    case = cases.perturbed(cases.sine_wave(n=21, scheme=72, viscous=True, amp=0.2), seed=4, amp=5e-2)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.viscous()
    oz.call("orc_compute_viscous_flux")
    assert rel_err(gz.get("dq")[1:], oz["dq"][1:], momentum=(0, 1, 2)) <= 1e-12


def test_local_time_step_matches():
    case = cases.perturbed(cases.sine_wave(n=21, scheme=72, viscous=True), seed=5)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    dt_g = gz.ctx.local_time_step()
    oz.call("orc_local_time_step")
    dt_o = oz.L.orc_global_time_step(__import__("ctypes").byref(oz.z))
    assert dt_g == pytest.approx(dt_o, rel=1e-14)
    assert rel_err(gz.get("dt_local"), oz["dt_local"], momentum=()) <= 1e-14


def test_sod_long_run_against_exact_solution():
    """Sod to t = 0.2 on the GPU; L1 errors against the exact Riemann solution
    (golden fixture from the reference's example) stay at the oracle's level."""
    import os
    golden = np.load(os.path.join(os.path.dirname(__file__), "golden", "sod_exact.npz"))
    case = cases.sod(400, 7, scheme=52)
    gz = GpuZone(case)
    gz.initialize()
    t = 0.0
    while t < 0.2:
        t += gz.ctx.rk3_step(graph=True)
    bv = gz.get("bv")
    xs = np.linspace(0, 1, 400)
    rho = case.interior(bv[0])[0, 3]
    p = case.interior(bv[4])[0, 3]
    rho_ex = np.interp(xs, golden["x"], golden["rho"])
    p_ex = np.interp(xs, golden["x"], golden["p"])
    assert np.abs(rho - rho_ex).mean() < 3e-3
    assert np.abs(p - p_ex).mean() < 3e-3
