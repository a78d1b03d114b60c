"""Slab decomposition on the GPU through the C ABI: cfk_halo_pack /
cfk_halo_assign against the oracle's restatement of the reference's parallel
faces (src/DataCommunication.cu:210-307), and a block cut into slabs stepped
by slabs.SlabRun with LibraryZone against the same decomposition on the
oracle and against the whole block."""
import dataclasses

import numpy as np
import pytest

import cases
import mechanism
import slabs as sl
from gpuzone import GpuZone
from slabzone import OracleSlabZone, assemble, plane_scale, rel_diff

pytestmark = pytest.mark.gpu


def _outflow(case, axis):
    return dataclasses.replace(case, faces=[(f, d, 6 if f == axis else lab) for f, d, lab in case.faces])


def _randomised(case, seed):
    rng = np.random.default_rng(seed)
    bv = case.bv.copy()
    bv[0] *= rng.uniform(0.8, 1.2, bv.shape[1])
    bv[1:4] = rng.uniform(-0.5, 0.5, bv[1:4].shape)
    bv[4] *= rng.uniform(0.8, 1.2, bv.shape[1])
    return dataclasses.replace(case, bv=bv)


@pytest.mark.parametrize("mix", [False, True])
def test_halo_pack_and_assign_match_the_oracle(mix):
    torch = pytest.importorskip("torch")
    if mix:
        base = cases.mix_wave(mechanism.load("li2004"), 9, ny=8, nz=7, scheme=52, viscous=False)
    else:
        base = cases.sine_wave(n=9, ny=8, nz=7, scheme=72, viscous=False)
    case = _randomised(base, 3)
    for face in range(3):
        for d in (-1, 1):
            gz = GpuZone(case)
            oz = OracleSlabZone(case)
            gz.initialize()
            oz.oz.initialize()
            got = sl.LibraryZone(gz.ctx, gz.t, gz.param).halo_pack(face, d).cpu().numpy()
            want = oz.halo_pack(face, d).numpy()
            assert np.array_equal(got, want)
            # a neighbour's buffer: the pack scaled, one face node at rest
            buf = want.copy() * 1.25
            nt = 6 + case.param["n_scalar"]
            buf[1 * (case.ngg + 1) * nt + 1: 1 * (case.ngg + 1) * nt + 4] = 0.0
            dbuf = torch.from_numpy(buf).cuda()
            gz.ctx.halo_assign(face, d, dbuf.data_ptr())
            oz.halo_assign(face, d, torch.from_numpy(buf))
            assert np.array_equal(gz.get("bv"), oz["bv"])
            if mix:
                assert np.array_equal(gz.get("sv"), oz["sv"])
            assert rel_diff(gz.get("cv"), oz["cv"]) <= 1e-14


def _sod():
    return cases.sod(96, 9, scheme=52)


def _wave():
    return _outflow(cases.perturbed(cases.sine_wave(n=17, ny=19, nz=13, scheme=72, viscous=False), seed=4,
                                    amp=0.05), 1)


def _mix():
    return _outflow(cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 15, ny=9, nz=7, scheme=52,
                                                   viscous=False), seed=2, amp=1e-2), 0)


@pytest.mark.parametrize("case_fn,n,axis,periodic,tol", [
    (_sod, 3, 0, False, 1e-13), (_wave, 2, 1, False, 1e-13), (_mix, 2, 0, False, 1e-9),
    (lambda: cases.sine_wave(n=13, ny=14, nz=10, scheme=52, viscous=False), 3, 2, True, 1e-13)])
def test_slab_run_on_the_gpu_matches_the_oracle_and_the_whole_block(case_fn, n, axis, periodic, tol):
    torch = pytest.importorskip("torch")
    whole = case_fn()
    parts = sl.split_slabs(whole, n, axis, periodic=periodic)
    gz = [GpuZone(p) for p in parts]
    run = sl.SlabRun([sl.LibraryZone(g.ctx, g.t, g.param) for g in gz], range(n), n, axis, sl.LocalTransport(),
                     two_d=whole.mz == 1, periodic=periodic)
    oz = [OracleSlabZone(p) for p in parts]
    ref = sl.SlabRun(oz, range(n), n, axis, sl.LocalTransport(), two_d=whole.mz == 1, periodic=periodic)
    run.initialize()
    ref.initialize()
    for _ in range(3):
        assert run.step() == pytest.approx(ref.step(), rel=1e-13)
    torch.cuda.synchronize()
    # every slab against the decomposition's scale: the Sod tube's outer slabs
    # are gas at rest, whose momenta are round-off on both sides
    scale = plane_scale(*[o["cv"] for o in oz])
    for g, o in zip(gz, oz):
        assert rel_diff(g.get("cv"), o["cv"], scale) <= tol
    cv, seam = assemble(whole, parts, [g.get("cv") for g in gz], axis)
    assert seam <= 1e-13 * np.abs(cv).max()
    whole_gz = GpuZone(whole)
    whole_gz.initialize()
    for _ in range(3):
        whole_gz.ctx.rk3_step()
    g = whole.ngg
    W = whole_gz.get("cv").reshape((-1,) + whole.shape())[:, g:g + whole.mz, g:g + whole.my, g:g + whole.mx]
    assert rel_diff(cv, W) <= tol
