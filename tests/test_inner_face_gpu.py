"""Inner faces of multi-block meshes on the GPU (cfk_inner_communication,
reference src/DataCommunication.cu:6-102) against the CPU oracle.

* One communication over faces with every normal axis and side and reversed
  or permuted tangential axes: bv bitwise equal to the oracle's (copies and
  averages), cv to 1e-14.
* Two-block runs stepped in lockstep with the oracle's two-block runs (the
  device state reset to the oracle's before each step): a periodic viscous
  WENO7 wave cut in two with its periodic seam also an inner face, a 2-D
  tube (with the k-ghost copy after the communication) and a viscous
  mixture, each step to 1e-12 as the single-block parity tests.
* A block cut in two on the GPU steps like the whole block on the GPU.
* Faces that leave a block's padded range, blocks that do not match, and a
  k-ghost copy asked of a 3-D block are rejected before any launch."""
import numpy as np
import pytest

import cases
import mechanism
import pyoracle
from gpuzone import GpuZone, interior_planes, rel_err
from multiblock import GpuBlocks, OracleBlocks, split_difference
from test_inner_face_cpu import _outflow_i, _random_zone_case, _records_3d
from test_mixture_gpu import MIX_KEYS

import corefl_b200 as cfk

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", range(0, 96, 11))
def test_communication_matches_oracle(k):
    m, t, g = (7, 6, 5), (6, 5, 7), 3
    recs = _records_3d(m, t)
    src, tar = recs[k % len(recs)]
    ca, cb = _random_zone_case(m, g, 5), _random_zone_case(t, g, 6)
    za, zb = pyoracle.OracleZone(ca), pyoracle.OracleZone(cb)
    ga, gb = GpuZone(ca), GpuZone(cb)
    for z in (za, zb):
        z.call("orc_compute_cv_from_bv")
    for z in (ga, gb):
        z.ctx.cv_from_bv()
    za.inner_communication(zb, pyoracle.register_inner_face(3, g, src, tar, 2))
    ga.ctx.inner_communication(gb.ctx, cfk.register_inner_face(3, g, src, tar, 2))
    assert np.array_equal(ga.get("bv"), za["bv"]) and np.array_equal(gb.get("bv"), zb["bv"])
    assert rel_err(ga.get("cv"), za["cv"]) <= 1e-14 and rel_err(gb.get("cv"), zb["cv"]) <= 1e-14


def _lockstep_blocks(cases_, links, steps, keys=("cv", "bv", "mul", "qn"), tol=1e-12):
    ob = OracleBlocks(cases_, links)
    ob.initialize()
    gb = GpuBlocks(cases_, links)
    gb.initialize()
    for b, c in enumerate(cases_):
        assert rel_err(gb.g[b].get("cv"), ob.z[b]["cv"]) <= 1e-13, f"block {b} after the start-up"
    for s in range(steps):
        for b in range(len(cases_)):
            gb.g[b].load_from(ob.z[b], keys=keys)
        dt_o, dt_g = ob.step(), gb.step()
        assert dt_g == pytest.approx(dt_o, rel=1e-13)
        for b, c in enumerate(cases_):
            e = rel_err(interior_planes(c, gb.g[b].get("cv")), interior_planes(c, ob.z[b]["cv"]))
            assert e <= tol, f"step {s}, block {b}: {e:.3e}"
            assert rel_err(gb.g[b].get("bv"), ob.z[b]["bv"]) <= tol


def test_periodic_viscous_wave_in_two_blocks():
    whole = cases.perturbed(cases.sine_wave(n=25, ny=11, nz=9, scheme=72, viscous=True), seed=3, amp=0.02)
    A, B, links = cases.split_i(whole, 12)
    _lockstep_blocks([A, B], links, 3)


def test_2d_tube_in_two_blocks():
    A, B, links = cases.split_i(cases.sod(64, 9, scheme=52), 30)
    _lockstep_blocks([A, B], links, 6)


def test_viscous_mixture_in_two_blocks():
    mech = mechanism.load("li2004")
    whole = cases.perturbed(cases.mix_wave(mech, 15, ny=9, nz=7, scheme=52, viscous=True), seed=2, amp=1e-2)
    A, B, links = cases.split_i(whole, 7)
    _lockstep_blocks([A, B], links, 2, keys=MIX_KEYS)


def test_split_block_on_gpu_steps_like_whole_block():
    whole = _outflow_i(cases.perturbed(cases.sine_wave(n=25, ny=11, nz=9, scheme=72, viscous=False), seed=3,
                                       amp=0.05))
    A, B, links = cases.split_i(whole, 9, periodic_i=False)
    gw = GpuZone(whole)
    gw.initialize()
    gb = GpuBlocks([A, B], links)
    gb.initialize()
    for _ in range(4):
        assert gw.ctx.rk3_step() == pytest.approx(gb.step(), rel=1e-13)
    assert split_difference(whole, gw.get("cv"), A, B, [gb.g[0].get("cv"), gb.g[1].get("cv")], 9) <= 1e-14


def test_bad_faces_and_blocks_are_rejected():
    m, g = (7, 6, 5), 3
    ga, gb = GpuZone(_random_zone_case(m, g, 1)), GpuZone(_random_zone_case(m, g, 2))
    f = cfk.register_inner_face(3, g, [7, 7, -1, -6, 1, 5], [1, 1, -1, -6, 1, 5], 2)
    ga.ctx.inner_communication(gb.ctx, f)
    bad = cfk.cfk_inner_face.from_buffer_copy(f)
    bad.n_point[1] = 10  # rows 0..9: past the 6 nodes and 3 ghost layers of j
    with pytest.raises(cfk.CfkError, match="padded range"):
        ga.ctx.inner_communication(gb.ctx, bad)
    bad = cfk.cfk_inner_face.from_buffer_copy(f)
    bad.target_start[0] = -4
    with pytest.raises(cfk.CfkError, match="target block"):
        ga.ctx.inner_communication(gb.ctx, bad)
    bad = cfk.cfk_inner_face.from_buffer_copy(f)
    bad.src_tar[2] = 1
    with pytest.raises(cfk.CfkError, match="permutation"):
        ga.ctx.inner_communication(gb.ctx, bad)
    other = GpuZone(cases.sine_wave(n=9, ny=9, nz=9, scheme=72, viscous=False))  # ngg 4
    with pytest.raises(cfk.CfkError, match="differ"):
        ga.ctx.inner_communication(other.ctx, f)
    thin = GpuZone(cases.split_i(_random_zone_case((9, 6, 5), g, 3), 2, periodic_i=False)[0])  # 3 nodes in i
    with pytest.raises(cfk.CfkError, match="thicker"):
        thin.ctx.inner_communication(gb.ctx, cfk.register_inner_face(3, g, [3, 3, -1, -6, 1, 5],
                                                                      [1, 1, -1, -6, 1, 5], 2))
    with pytest.raises(cfk.CfkError, match="2-D"):
        ga.ctx.eliminate_k_gradient()
