"""limit_flow on the GPU (cfk_limit_flow; reference
src/TimeAdvanceFunc.cuh:117-220) against the CPU oracle's orc_limit_flow,
which judges every node on the state before the call, and the RK3 step with
limit_flow after each stage update (reference src/RK.cuh:163-164) against
the oracle's.

Bar: in a single call the repaired rho, u, v, w, p agree bit for bit (the
same sums in the same order) and T and cv to 1e-14; the RK3 steps to 1e-12
as the other parity tests; the number of repaired nodes agrees."""
import math

import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, interior_planes, rel_err

pytestmark = pytest.mark.gpu


def _bounds(case, rho_inf=1.0, p_inf=1.0):
    v = case.param["v_ref"]
    return dict(limit_ll=[1e-6 * rho_inf, -1000 * v, -1000 * v, -1000 * v, 1e-6 * p_inf],
                limit_ul=[1e3 * rho_inf, 1000 * v, 1000 * v, 1000 * v, 1e3 * p_inf])


def _plant(case, nodes):
    """Copy of the case with bad values planted at interior nodes:
    nodes = [(i, j, k, var, value)]."""
    bv = case.bv.copy()
    g = case.ngg
    B = bv.reshape(6, case.mz + 2 * g, case.my + 2 * g, case.mx + 2 * g)
    for i, j, k, l, v in nodes:
        B[l, k + g, j + g, i + g] = v
    return case.__class__(**{**case.__dict__, "bv": bv})


def _single_call(case, nodes, expect):
    case = _plant(case, nodes)
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.load_from(oz, keys=("cv", "bv", "mul"))
    n_o = oz.limit_flow(case.param["limit_ll"], case.param["limit_ul"])
    n_g = gz.ctx.limit_flow()
    assert n_o == n_g == expect
    bg, bo = gz.get("bv"), oz["bv"]
    assert np.array_equal(bg[:5], bo[:5], equal_nan=True)  # the same sums in the same order
    # T and cv from the repaired state: the same formulas, compiled with different contractions
    assert np.allclose(bg[5], bo[5], rtol=1e-14, atol=0, equal_nan=True)
    assert np.allclose(gz.get("cv"), oz["cv"], rtol=1e-14, atol=0, equal_nan=True)


def test_air_repairs_match_oracle_bitwise():
    base = cases.perturbed(cases.sine_wave(n=17, ny=13, nz=9, scheme=72, viscous=True), seed=3, amp=1e-2)
    base.param.update(limit_flow=1, **_bounds(base, rho_inf=1.0, p_inf=1.0 / 1.4))
    nodes = [(4, 5, 3, 0, math.nan),            # NaN density: neighbour mean
             (10, 2, 6, 4, -1.0),               # negative pressure
             (7, 7, 7, 1, 5000.0),              # velocity beyond 1000 v_ref
             # a cluster whose centre has no good neighbour (26 of them bad): clamped
             ] + [(13 + a, 6 + b, 4 + c, 0, 1e5) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    _single_call(base, nodes, expect=3 + 27)


def test_air_2d_edges_and_corners():
    base = cases.sod(40, 9, scheme=52)
    base.param.update(limit_flow=1, **_bounds(base))
    nodes = [(0, 0, 0, 0, -1.0), (39, 8, 0, 4, math.nan), (20, 0, 0, 2, 1e9), (21, 0, 0, 4, 1e9)]
    _single_call(base, nodes, expect=4)


def test_mixture_repairs_take_temperature_from_mixture_gas_constant():
    mech = mechanism.load("li2004")
    base = cases.mix_wave(mech, 13, ny=11, nz=9, scheme=72)
    base.param.update(limit_flow=1, **_bounds(base, rho_inf=float(base.bv[0].mean()), p_inf=101325.0))
    nodes = [(3, 3, 3, 0, -0.5), (6, 5, 4, 4, math.inf), (9, 8, 2, 3, math.nan)]
    _single_call(base, nodes, expect=3)


@pytest.mark.parametrize("scheme", [52, 2])
def test_rk3_steps_with_limit_flow(scheme):
    """Density spikes above the upper bound survive each stage update and are
    repaired inside every stage; the GPU step matches the oracle's."""
    base = cases.sod(96, 7, scheme=scheme)
    b = _bounds(base)
    b["limit_ul"][0] = 2.0
    base.param.update(limit_flow=1, **b)
    case = _plant(base, [(20, 3, 0, 0, 4.0), (70, 2, 0, 0, 3.0), (71, 2, 0, 0, 3.5)])
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    gz = GpuZone(case)
    gz.initialize()
    for s in range(4):
        gz.load_from(oz)
        dt_o = oz.step()
        dt_g = gz.ctx.rk3_step()
        assert dt_g == pytest.approx(dt_o, rel=1e-13)
        e = rel_err(interior_planes(case, gz.get("cv")), interior_planes(case, oz["cv"]))
        assert e <= 1e-12, f"step {s}: {e:.3e}"
