"""Slab decomposition (slabs.py) on the CPU oracle: a block cut into slabs
that exchange halos every stage steps like the whole block, in one process
and as gloo ranks; the halo pack/assign rules of the reference's parallel
faces (src/DataCommunication.cu:210-307) on hand-made values."""
import dataclasses
import socket

import numpy as np
import pytest

import cases
import mechanism
import slabs as sl
from slabzone import OracleSlabZone, assemble, rel_diff, run_rank
import pyoracle


def _outflow(case, axis):
    return dataclasses.replace(case, faces=[(f, d, 6 if f == axis else lab) for f, d, lab in case.faces])


def sod_2d():
    return cases.sod(64, 9, scheme=52)


def wave_3d():
    return _outflow(cases.perturbed(cases.sine_wave(n=13, ny=14, nz=10, scheme=72, viscous=False), seed=4,
                                    amp=0.05), 1)


def wave_3d_periodic():
    return cases.sine_wave(n=13, ny=14, nz=10, scheme=52, viscous=False)


def mix_3d():
    return _outflow(cases.perturbed(cases.mix_wave(mechanism.load("li2004"), 15, ny=9, nz=7, scheme=52,
                                                   viscous=False), seed=2, amp=1e-2), 0)


def _whole(case, steps):
    oz = pyoracle.OracleZone(case)
    oz.initialize()
    dts = [oz.step() for _ in range(steps)]
    return oz, dts


def test_slab_bounds_share_cut_planes():
    assert sl.slab_bounds(64, 2) == [(0, 32), (32, 63)]
    b = sl.slab_bounds(100, 7)
    assert b[0][0] == 0 and b[-1][1] == 99 and all(b[r][1] == b[r + 1][0] for r in range(6))
    with pytest.raises(ValueError):
        sl.split_slabs(sod_2d(), 2, 2)


def test_split_slabs_keeps_outer_faces_and_arrays():
    whole = sod_2d()
    parts = sl.split_slabs(whole, 3, 0)
    assert [p.mx for p in parts] == [22, 22, 22] and all(p.my == 9 for p in parts)
    assert (0, -1, 6) in parts[0].faces and (0, 1, 6) not in parts[0].faces
    assert (0, 1, 6) in parts[2].faces and not any(f == 0 for f, _, _ in parts[1].faces)
    g = whole.ngg
    W = whole.bv.reshape((6,) + whole.shape())
    P1 = parts[1].bv.reshape((6,) + parts[1].shape())
    assert np.array_equal(P1, W[..., 21:21 + 22 + 2 * g])
    assert sl.split_slabs(whole, 2, 0, periodic=True)[0].faces == [(1, -1, 6), (1, 1, 6)]


@pytest.mark.parametrize("case_fn,n,axis,steps,tol", [
    (sod_2d, 2, 0, 4, 1e-14), (sod_2d, 3, 0, 3, 1e-14), (sod_2d, 2, 1, 3, 1e-14),
    (wave_3d, 3, 1, 2, 1e-14), (mix_3d, 2, 0, 2, 1e-10)])
def test_slabs_in_one_process_step_like_the_whole_block(case_fn, n, axis, steps, tol):
    """The halo carries every node a stencil reads across a cut, and the
    shared cut plane is computed identically on both sides (its average is the
    value itself), so the decomposed run reproduces the whole block up to the
    rounding of the cut plane's cv, which the assignment recomputes from bv
    as the reference's does."""
    whole = case_fn()
    oz, dts = _whole(whole, steps)
    parts = sl.split_slabs(whole, n, axis)
    zones = [OracleSlabZone(p) for p in parts]
    run = sl.SlabRun(zones, range(n), n, axis, sl.LocalTransport(), two_d=whole.mz == 1)
    run.initialize()
    got = [run.step() for _ in range(steps)]
    assert np.allclose(got, dts, rtol=1e-14, atol=0)
    cv, seam = assemble(whole, parts, [z["cv"] for z in zones], axis)
    assert seam <= 1e-14 * np.abs(cv).max()
    assert rel_diff(cv, _interior(whole, oz["cv"])) <= tol


def _interior(case, a):
    g = case.ngg
    return a.reshape((a.shape[0],) + case.shape())[:, g:g + case.mz, g:g + case.my, g:g + case.mx]


def test_periodic_seam_between_first_and_last_slab():
    """A periodic block (the curvilinear wave, whose first and last node
    planes coincide) cut in three along each axis with its seam exchanged
    between the first and last slab: the periodic planes agree after the
    steps and the run reproduces the whole block's periodic boundary
    condition to rounding."""
    whole = wave_3d_periodic()
    oz, _ = _whole(whole, 2)
    for axis in range(3):
        parts = sl.split_slabs(whole, 3, axis, periodic=True)
        zones = [OracleSlabZone(p) for p in parts]
        run = sl.SlabRun(zones, range(3), 3, axis, sl.LocalTransport(), two_d=False, periodic=True)
        run.initialize()
        for _ in range(2):
            run.step()
        cv, seam = assemble(whole, parts, [z["cv"] for z in zones], axis)
        assert seam <= 1e-14 * np.abs(cv).max()
        first, last = np.take(cv, [0], axis=3 - axis), np.take(cv, [-1], axis=3 - axis)
        assert np.abs(first - last).max() <= 1e-14 * np.abs(cv).max()
        assert rel_diff(cv, _interior(whole, oz["cv"])) <= 1e-14
    with pytest.raises(ValueError):
        sl.SlabRun(zones[:1], [0], 1, 1, sl.LocalTransport(), two_d=False, periodic=True)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


@pytest.mark.parametrize("case_fn,n,axis,rank_of,periodic", [
    (sod_2d, 2, 0, [0, 1], False), (wave_3d, 3, 1, [0, 1, 1], False), (wave_3d_periodic, 2, 1, [0, 1], True)])
def test_two_gloo_ranks_step_like_one_process(case_fn, n, axis, rank_of, periodic):
    """The same decomposition with its slabs on two gloo ranks: the halo
    buffers cross ranks by send/receive and dt is the all-reduce minimum;
    the result is bit-identical to the in-process run."""
    import torch.multiprocessing as mp

    steps = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(run_rank, args=(2, _free_port(), (case_fn, n, axis, steps, rank_of, periodic), out), nprocs=2,
             join=True)
    got = {}
    for r in range(2):
        got.update(out[r])
    whole = case_fn()
    parts = sl.split_slabs(whole, n, axis, periodic=periodic)
    zones = [OracleSlabZone(p) for p in parts]
    run = sl.SlabRun(zones, range(n), n, axis, sl.LocalTransport(), two_d=whole.mz == 1, periodic=periodic)
    run.initialize()
    dts = [run.step() for _ in range(steps)]
    for s in range(n):
        cv, bv, dd = got[s]
        assert dd == dts
        assert np.array_equal(cv, zones[s]["cv"]) and np.array_equal(bv, zones[s]["bv"])


def _hand_zone():
    c = cases.sod(8, 6, scheme=52)
    z = OracleSlabZone(c)
    rng = np.random.default_rng(0)
    z.oz["bv"][:] = rng.uniform(0.5, 2.0, z.oz["bv"].shape)
    return c, z


def test_halo_pack_layout():
    """Buffer order: face node t (first tangential axis fastest), layer q
    (0 the face node, q inwards), variable l."""
    c, z = _hand_zone()
    g = c.ngg
    bv = z.oz["bv"].reshape((6,) + c.shape())
    buf = z.halo_pack(0, 1).numpy().reshape(c.mz, c.my, g + 1, 6)
    for q in range(g + 1):
        assert np.array_equal(buf[:, :, q, :], np.moveaxis(bv[:, g:g + 1, g:g + c.my, g + c.mx - 1 - q], 0, -1))
    buf = z.halo_pack(1, -1).numpy().reshape(c.mz, c.mx, g + 1, 6)
    for q in range(g + 1):
        assert np.array_equal(buf[:, :, q, :], np.moveaxis(bv[:, g:g + 1, g + q, g:g + c.mx], 0, -1))


def test_halo_assign_averages_copies_or_keeps_the_face():
    """Face node: kept where this node is at rest, copied where only the
    neighbour's is at rest, averaged otherwise (src/DataCommunication.cu:
    226-252); ghost layers from the neighbour's inner layers; cv recomputed."""
    c, z = _hand_zone()
    g = c.ngg
    bv = z.oz["bv"].reshape((6,) + c.shape())
    bv[1:4, g, g + 1, g] = 0.0          # this face node at rest
    other = z.halo_pack(0, -1).numpy().reshape(c.my, g + 1, 6).copy()
    other[:, :, :] *= 1.5
    other[2, 0, 1:4] = 0.0              # neighbour's face node at rest
    before = bv.copy()
    z.halo_assign(0, -1, __import__("torch").from_numpy(other.reshape(-1).copy()))
    face = bv[:, g, g:g + c.my, g]
    for t in range(c.my):
        if t == 1:
            assert np.array_equal(face[:, t], before[:, g, g + t, g])
        elif t == 2:
            assert np.array_equal(face[:, t], other[t, 0])
        else:
            assert np.array_equal(face[:, t], 0.5 * (before[:, g, g + t, g] + other[t, 0]))
    for q in range(1, g + 1):
        assert np.array_equal(bv[:, g, g:g + c.my, g - q].T, other[:, q])
    cv = z.oz["cv"].reshape((-1,) + c.shape())
    assert np.allclose(cv[0, g, g:g + c.my, g - 1], other[:, 1, 0], rtol=0, atol=0)
