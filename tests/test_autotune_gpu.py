"""Tile variants of the WENO flux kernels and the tile autotuner.

Every tile shape computes each face with the same arithmetic, so the flux
differences of all variants are bitwise identical and each matches the CPU
oracle at the single-call bar (1e-11, as for the other single-call tests).
The autotuner leaves the zone's arrays untouched and the tuned context still
steps in parity with the oracle (1e-12)."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, rel_err
from test_parity_gpu import _lockstep

pytestmark = pytest.mark.gpu


def _flux_per_variant(case, keys=("cv", "bv", "mul", "qn")):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_inviscid_flux")
    gz = GpuZone(case)
    gz.initialize()
    out = []
    for v in range(3):
        gz.t["dq"].zero_()
        gz.ctx.set_tile_variants([v, v, v])
        gz.ctx.inviscid()
        out.append(gz.get("dq"))
    return oz["dq"], out


@pytest.mark.parametrize("scheme", [52, 72])
def test_air_tile_variants_identical_and_in_parity(scheme):
    case = cases.perturbed(cases.sine_wave(n=41, ny=37, nz=30, scheme=scheme, viscous=False, amp=0.2), seed=3,
                           amp=0.3)
    ref, out = _flux_per_variant(case)
    for v in range(3):
        assert rel_err(out[v], ref) <= 1e-11, f"variant {v}"
        assert np.array_equal(out[v], out[0]), f"variant {v} differs from variant 0"


def test_air_tile_variants_hybrid():
    case = cases.perturbed(cases.sine_wave(n=41, ny=37, nz=30, scheme=72, viscous=False, amp=0.2), seed=3,
                           amp=0.3)
    case.param.update(sensor_threshold=0.02, shock_sensor=1, sensor_eps=1e-3)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_shock_sensor")
    oz.call("orc_compute_inviscid_flux")
    gz = GpuZone(case)
    gz.initialize()
    gz.ctx.shock_sensor()
    out = []
    for v in range(3):
        gz.t["dq"].zero_()
        gz.ctx.set_tile_variants([v, v, v])
        gz.ctx.inviscid()
        out.append(gz.get("dq"))
        assert rel_err(out[v], oz["dq"]) <= 1e-11
    assert all(np.array_equal(o, out[0]) for o in out)


@pytest.mark.parametrize("scheme", [52, 72])
def test_mixture_tile_variants_identical_and_in_parity(scheme):
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 35, ny=19, nz=17, scheme=scheme), seed=9,
                           amp=2e-2)
    ref, out = _flux_per_variant(case)
    for v in range(3):
        assert rel_err(out[v], ref) <= 1e-11, f"variant {v}"
        assert np.array_equal(out[v], out[0]), f"variant {v} differs from variant 0"


def test_autotune_keeps_arrays_and_parity():
    case = cases.perturbed(cases.sine_wave(n=65, ny=67, nz=33, scheme=72, viscous=True), seed=7, amp=1e-2)
    gz = GpuZone(case)
    gz.initialize()
    before = {k: gz.get(k).copy() for k in ("cv", "bv", "dq")}
    choice, ms = gz.ctx.autotune_tiles(reps=3)
    assert all(0 <= c < 3 for c in choice)
    assert all(t > 0 for row in ms for t in row)
    for d in range(3):
        assert ms[d][choice[d]] == min(ms[d])
    for k, v in before.items():
        assert np.array_equal(gz.get(k), v), f"{k} changed by the autotuner"
    # a tuned context steps in parity (the chosen tiles feed every later call)
    small = cases.perturbed(cases.sine_wave(n=19, ny=37, nz=30, scheme=72, viscous=True), seed=7)
    _lockstep(small, 2, tiles=choice)


def test_autotune_mixture_and_pv_noop():
    case = cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 35, ny=19, nz=17, scheme=72), seed=4)
    gz = GpuZone(case)
    gz.initialize()
    choice, ms = gz.ctx.autotune_tiles(reps=2)
    assert all(0 <= c < 3 for c in choice) and all(t > 0 for row in ms for t in row)
    pv = GpuZone(cases.sod(64, 7, scheme=4))
    choice, ms = pv.ctx.autotune_tiles(reps=2)
    # a no-op keeps the context's starting shapes (air: x 31x8, y/z 31x16)
    assert choice == [2, 1, 1] and all(t == 0 for row in ms for t in row)


@pytest.mark.parametrize("name", ["wave_3d", "walls_3d", "tube_2d"])
def test_viscous_forms_identical_and_in_parity(name):
    """The staged and the two cp.async-ring forms (the second with the L2
    prefetch of the metric) of the fused air viscous kernel
    agree to the last bits (blocks not a multiple of the 32 x 8 x 32 tile, 2-D
    and 3-D, walls widening the boundary ranges) and each matches the oracle's
    viscous flux at the single-call bar."""
    if name == "wave_3d":
        case = cases.perturbed(cases.sine_wave(n=41, ny=37, nz=35, scheme=52, amp=0.2), seed=5, amp=0.3)
    elif name == "walls_3d":
        case = cases.with_walls(cases.perturbed(cases.sine_wave(n=33, ny=19, nz=13, scheme=72), seed=6, amp=0.1))
    else:
        case = cases.sod(70, 11, scheme=52, viscous_order=2)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    oz.call("orc_compute_viscous_flux")
    gz = GpuZone(case)
    gz.initialize()
    out = []
    for v in (0, 1, 2):
        gz.t["dq"].zero_()
        gz.ctx.viscous_variant(v)
        gz.ctx.viscous()
        out.append(gz.get("dq"))
    # the kernels may contract products into FMAs differently: the same
    # arithmetic to the last bits, not bit for bit
    for v in (1, 2):
        assert rel_err(out[v][1:], out[0][1:], momentum=(0, 1, 2)) <= 1e-14, f"form {v}"
    for v in (0, 1, 2):
        assert rel_err(out[v][1:], oz["dq"][1:], momentum=(0, 1, 2)) <= 1e-11, f"form {v}"
    var, ms = gz.ctx.viscous_variant()
    assert var == 2
